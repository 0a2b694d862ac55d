"""Polynomial coefficients of the MCMC kernel's FP32 special functions (bpx_device.cuh).

    python -m fdt_b200.polyfit        # prints the constexpr block between the GENERATED markers

Fitted here, by iteratively reweighted least squares towards the minimax (equal-ripple) error, to
the exact functions (scipy's i0/i0e, numpy's sin/cos), not taken from any library:

* ``kI0Small(i)``: I0(z) = sum_i a_i (z^2)^i for 0 <= z < ``kI0Split``, a_0 = 1 exactly (so padding
  measurements with z = 0 contribute log 1 = 0), relative error;
* ``kI0Large(i)``: e^-z I0(z) sqrt(z) = sum_i b_i z^-i for z >= ``kI0Split`` (evaluated in v = 1/z, which
  the kernel forms as rsqrt(z)^2), relative error;
* ``kSinQ(i)``/``kCosQ(i)``: sin r = r + r^3 sum_i s_i r^(2i), cos r = 1 - r^2/2 + r^4 sum_i c_i r^(2i)
  on |r| <= pi/4 (plus a margin for the reduction's rounding).

These replace the reference's Abramowitz & Stegun 9.8.1/9.8.2 forms of log I0 (fibre.h:31-51,
CUDA/runmcmc_kernels.cu:126-145), which split at 3.75 with degrees 6 and 8: the split at 4.75 needs
degrees 6 and 5 for a log I0 error below 6e-7 after FP32 rounding (A&S: 1.6e-7 and 1.9e-7 before
rounding).  tests/test_polyfit.py checks the literals in the header against these bounds.
"""
from __future__ import annotations

import numpy as np

I0_SPLIT = 4.75
I0_SMALL_DEG = 6
I0_LARGE_DEG = 5


def _irls(x: np.ndarray, y: np.ndarray, basis: np.ndarray, weight: np.ndarray, iters: int = 300) -> np.ndarray:
    """Weighted least squares re-weighted towards equal ripple of weight * (basis @ c - y)."""
    w = np.ones_like(x)
    best, best_err = None, np.inf
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(basis * (w * weight)[:, None], y * w * weight, rcond=None)
        e = (basis @ c - y) * weight
        m = np.abs(e).max()
        if m < best_err:
            best, best_err = c, m
        w = w * (1.0 + np.abs(e) / m) ** 1.5
        w /= w.max()
    return best


def _cheb_nodes(n: int) -> np.ndarray:
    return 0.5 * (np.cos(np.pi * (np.arange(n) + 0.5) / n) + 1.0)  # (0, 1)


def fit_i0() -> tuple[np.ndarray, np.ndarray]:
    """(a_i for powers of z^2, b_i for powers of 1/z), both as float64."""
    from scipy.special import i0, i0e

    u = _cheb_nodes(40000)                      # (z / split)^2
    z = I0_SPLIT * np.sqrt(u)
    y = i0(z)
    # a_0 = 1: fit (I0 - 1) / u with a polynomial of degree deg-1 in u
    V = np.vander(u, I0_SMALL_DEG, increasing=True) * u[:, None]
    a_rest = _irls(u, y - 1.0, V, 1.0 / y)
    a = np.concatenate([[1.0], a_rest]) / np.array([I0_SPLIT ** (2 * i) for i in range(I0_SMALL_DEG + 1)])
    c = np.clip(_cheb_nodes(40000), 1e-12, 1.0)  # split / z
    zl = I0_SPLIT / c
    g = i0e(zl) * np.sqrt(zl)
    b = _irls(c, g, np.vander(c, I0_LARGE_DEG + 1, increasing=True), 1.0 / g)
    b = b * np.array([I0_SPLIT ** i for i in range(I0_LARGE_DEG + 1)])
    return a, b


def fit_sincos() -> tuple[np.ndarray, np.ndarray]:
    r = np.pi / 4 * 1.001 * _cheb_nodes(4000)
    u = r * r
    s = _irls(u, (np.sin(r) - r) / r**3, np.vander(u, 3, increasing=True), r**3 / np.sin(r))
    c = _irls(u, (np.cos(r) - 1.0 + u / 2) / u**2, np.vander(u, 3, increasing=True), u**2)
    return s, c


def _lit(x: float) -> str:
    return repr(np.float32(x)).replace("np.float32(", "").replace(")", "") + "f"


def _fmt(name: str, v: np.ndarray) -> str:
    """A constexpr function of the coefficient index (folds to immediates in unrolled loops)."""
    chain = " : ".join(f"i == {i} ? {_lit(x)}" for i, x in enumerate(v[:-1])) + f" : {_lit(v[-1])}"
    return f"__host__ __device__ constexpr float {name}(int i) {{ return {chain}; }}"


def generated_block() -> str:
    a, b = fit_i0()
    s, c = fit_sincos()
    return "\n".join([
        f"constexpr float kI0Split = {I0_SPLIT}f;",
        _fmt("kI0Small", a),
        _fmt("kI0Large", b),
        _fmt("kSinQ", s),
        _fmt("kCosQ", c),
    ])


# ---- FP32 evaluation exactly as the kernel does it (used by the tests) ----

def _f32_horner(coef: np.ndarray, x: np.ndarray) -> np.ndarray:
    acc = np.full_like(x, np.float32(coef[-1]))
    with np.errstate(over="ignore", invalid="ignore"):
        for cf in coef[-2::-1]:
            acc = (acc.astype(np.float64) * x + np.float64(np.float32(cf))).astype(np.float32)  # one FMA rounding
    return acc


def log_i0e_f32(z: np.ndarray, split: float, small: np.ndarray, large: np.ndarray) -> np.ndarray:
    """log(e^-z I0(z)) from the two polynomials in FP32 (FMA Horner), as rician_acc forms it."""
    z = np.asarray(z, np.float32)
    u = (z * z).astype(np.float32)
    q = _f32_horner(small, u)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        rs = (1.0 / np.sqrt(z.astype(np.float64))).astype(np.float32)
        v = (rs * rs).astype(np.float32)
        p = _f32_horner(large, v)
        pr = (p * rs).astype(np.float32)
        return np.where(z < np.float32(split), np.log(q.astype(np.float64)) - z, np.log(pr.astype(np.float64)))


def main() -> None:
    print("// BEGIN generated by python -m fdt_b200.polyfit")
    print(generated_block())
    print("// END generated")


if __name__ == "__main__":
    main()
