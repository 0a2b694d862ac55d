"""CPU checks of the polynomial coefficients compiled into the MCMC kernel (bpx_device.cuh).

The header's generated block is parsed and evaluated in FP32 the way the kernel evaluates it
(FMA Horner steps); the error bounds are those the kernel's comments state."""
import os
import re

import numpy as np
import pytest
from scipy.special import i0e

from fdt_b200 import polyfit

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "fdt_b200", "csrc", "bpx_device.cuh")


def header_coefficients() -> dict:
    txt = open(HEADER).read()
    block = txt[txt.index("// BEGIN generated"):txt.index("// END generated")]
    out = {"split": float(re.search(r"kI0Split = ([0-9.e+-]+)f;", block).group(1))}
    for name in ["kI0Small", "kI0Large", "kSinQ", "kCosQ"]:
        body = re.search(name + r"\(int i\) \{ return (.*?); \}", block).group(1)
        vals = [float(v) for v in re.findall(r"\? ([-0-9.e+]+)f", body)] + [float(re.findall(r": ([-0-9.e+]+)f$", body)[0])]
        out[name] = np.array(vals, np.float32)
    return out


def test_header_matches_a_fresh_fit():
    h = header_coefficients()
    a, b = polyfit.fit_i0()
    s, c = polyfit.fit_sincos()
    assert h["split"] == polyfit.I0_SPLIT
    for got, want in [(h["kI0Small"], a), (h["kI0Large"], b), (h["kSinQ"], s), (h["kCosQ"], c)]:
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want.astype(np.float32), rtol=1e-5)


def test_log_i0_error_bound_in_fp32():
    h = header_coefficients()
    assert h["kI0Small"][0] == 1.0  # z = 0 (padding) contributes exactly log 1
    z = np.concatenate([np.linspace(0, 20, 200001), np.logspace(-6, 10, 200001)]).astype(np.float32)
    got = polyfit.log_i0e_f32(z, h["split"], h["kI0Small"], h["kI0Large"])
    err = np.abs(got - np.log(i0e(z.astype(np.float64))))
    assert err.max() < 6e-7, (err.max(), z[np.argmax(err)])
    assert polyfit.log_i0e_f32(np.zeros(4, np.float32), h["split"], h["kI0Small"], h["kI0Large"]).max() == 0.0


def _sincos_f32(x: np.ndarray, s: np.ndarray, c: np.ndarray):
    """sincos_fast of bpx_device.cuh in numpy FP32 (FMA steps rounded once)."""
    f = np.float32

    def fma(a, b, cc):
        return (a.astype(np.float64) * b.astype(np.float64) + cc.astype(np.float64)).astype(np.float32)

    x = x.astype(np.float32)
    k = np.rint((x * f(0.636619772)).astype(np.float32)).astype(np.float32)
    one = np.ones_like(x)
    r = fma(-k, one * f(1.57079637), x)
    r = fma(-k, one * f(-4.37113883e-08), r)
    r = fma(-k, one * f(-1.71512451e-15), r)
    u = (r * r).astype(np.float32)
    p = fma(u, one * s[2], one * s[1])
    p = fma(u, p, one * s[0])
    sn = fma((r * u).astype(np.float32), p, r)
    q = fma(u, one * c[2], one * c[1])
    q = fma(u, q, one * c[0])
    q = fma(u, q, one * f(-0.5))
    cs = fma(u, q, one)
    qi = k.astype(np.int64) & 3
    sw = (qi & 1) == 1
    a, b = np.where(sw, cs, sn), np.where(sw, sn, cs)
    return np.where((qi & 2) != 0, -a, a), np.where(((qi + 1) & 2) != 0, -b, b)


@pytest.mark.parametrize("lim", [4.0, 100.0, 1e5])
def test_sincos_within_two_ulp(lim):
    h = header_coefficients()
    x = np.random.default_rng(3).uniform(-lim, lim, 1_000_000).astype(np.float32)
    sn, cs = _sincos_f32(x, h["kSinQ"], h["kCosQ"])
    xs = x.astype(np.float64)
    assert np.abs(sn - np.sin(xs)).max() < 1.2e-7
    assert np.abs(cs - np.cos(xs)).max() < 1.2e-7
