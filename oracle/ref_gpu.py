"""ctypes wrapper of the reference's own CUDA kernels (oracle/_ref/librefgpu.so).  TEST INFRASTRUCTURE ONLY.

The library is built by ``make -C oracle ref`` from the reference tree's CUDA/PVM_single.cu,
CUDA/PVM_single_c.cu, CUDA/PVM_multi.cu and CUDA/runmcmc_kernels.cu (compiled where they lie, with
the harness oracle/refgpu_harness.cu); the built file travels with the repository to a GPU machine,
the reference tree does not.  Loaded only by tests/ to check the oracle (and through it the product)
against the reference's arithmetic: its LM cost/gradient/Hessian and fits, its initial MCMC energies
and its chains.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from fdt_b200.abi import Options, nrec

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "librefgpu.so")
REF_TREE = os.environ.get("BPX_REFERENCE_TREE", "/root/reference")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class McmcOpts(C.Structure):
    """refgpu_mcmc_opts: the xfibresOptions fields CUDA/runmcmc.cu passes to its kernels."""

    _fields_ = [("model", C.c_int), ("nfib", C.c_int), ("f0", C.c_int), ("rician", C.c_int),
                ("ardf0", C.c_int), ("all_ard", C.c_int), ("no_ard", C.c_int), ("fudge", C.c_float),
                ("R_mean", C.c_float), ("R_std", C.c_float), ("R_fudge", C.c_float), ("nburn", C.c_int),
                ("njumps", C.c_int), ("sampleevery", C.c_int), ("upe", C.c_int), ("seed", C.c_double)]

    @classmethod
    def from_options(cls, o: Options, seed: float) -> "McmcOpts":
        return cls(o.model, o.nfibres, o.f0, o.rician, o.ardf0, o.all_ard, o.no_ard, o.fudge, o.R_prior_mean,
                   o.R_prior_std, o.R_prior_fudge, o.nburn, o.njumps, o.sampleevery, o.updateproposalevery, seed)


def build() -> str | None:
    """Compile the reference kernels with the harness if the reference tree is present (else keep
    whatever was built before).  Returns the library path, or None if there is none."""
    if os.path.isdir(os.path.join(REF_TREE, "CUDA")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REF_TREE}"], check=True)
    return LIB if os.path.exists(LIB) else None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        L.refgpu_last_error.restype = C.c_char_p
        L.refgpu_last_times.argtypes = [_f32p]
        L.refgpu_lm_eval.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, _f32p, _f32p,
                                     _f32p, _f32p, _f64p, _f32p, _f32p]
        L.refgpu_fit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, _f32p, _f32p, _f32p,
                                 _f32p, _f32p]
        L.refgpu_mcmc.argtypes = [C.POINTER(McmcOpts), C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p, _f32p,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().refgpu_last_error().decode()}")


def nparams(kind: int, nfib: int, f0: bool) -> int:
    return 3 * nfib + 2 + (1 if kind == 2 else 0) + (1 if f0 else 0)


def lm_eval(kind: int, nfib: int, f0: bool, gbo: int, R: float, data, bvecs, bvals, params):
    """cf_/grad_/hess_PVM_{single,single_c,multi} at raw parameters [nvox][np]: (cf, grad, hess)."""
    data = _f32(data)
    nvox, ndir = data.shape
    np_ = nparams(kind, nfib, f0)
    p = _f32(params).reshape(nvox, np_)
    cf = np.zeros(nvox)
    g = np.zeros((nvox, np_), np.float32)
    H = np.zeros((nvox, np_, np_), np.float32)
    _check(lib().refgpu_lm_eval(kind, nfib, int(f0), gbo, R, nvox, ndir, data, _f32(bvecs), _f32(bvals), p, cf, g,
                                H), "refgpu_lm_eval")
    return cf, g, H


def fit(kind: int, nfib: int, f0: bool, gbo: int, R: float, data, bvecs, bvals, start) -> np.ndarray:
    """fit_PVM_{single,single_c,multi}_kernel from start values; finalised parameters [nvox][np]."""
    data = _f32(data)
    nvox, ndir = data.shape
    np_ = nparams(kind, nfib, f0)
    out = np.zeros((nvox, np_), np.float32)
    _check(lib().refgpu_fit(kind, nfib, int(f0), gbo, R, nvox, ndir, data, _f32(bvecs), _f32(bvals), _f32(start),
                            out), "refgpu_fit")
    return out


def init_energies(opts: Options, data, bvecs, bvals, params, tau=None):
    """Likelihood and prior energies init_Fibres_Multifibres_kernel computes from fit-layout params."""
    data = _f32(data)
    nvox, ndir = data.shape
    lik = np.zeros(nvox, np.float32)
    prior = np.zeros(nvox, np.float32)
    t = _f32(tau if tau is not None else np.zeros(nvox))
    o = McmcOpts.from_options(opts, 0.0)
    _check(lib().refgpu_mcmc(C.byref(o), nvox, ndir, data, _f32(bvecs), _f32(bvals), _f32(params), t,
                             lik.ctypes.data, prior.ctypes.data, None), "refgpu_mcmc")
    return lik, prior


def mcmc(opts: Options, data, bvecs, bvals, params, tau=None, seed: float = 8665904.0) -> np.ndarray:
    """The reference's chain (cuRAND XORWOW seeded by `seed`, FP64 likelihoods): records
    [6+3K][nsamples][nvox] in the record-row order of this library."""
    data = _f32(data)
    nvox, ndir = data.shape
    rec = np.zeros((nrec(opts.nfibres), opts.nsamples, nvox), np.float32)
    t = _f32(tau if tau is not None else np.zeros(nvox))
    o = McmcOpts.from_options(opts, seed)
    _check(lib().refgpu_mcmc(C.byref(o), nvox, ndir, data, _f32(bvecs), _f32(bvals), _f32(params), t, None, None,
                             rec.ctypes.data), "refgpu_mcmc")
    return rec


def last_times() -> tuple[float, float, float]:
    """Device milliseconds of the last fit (fit kernels) and chain (init + randoms + burn-in;
    recording) calls, CUDA events around the kernels only."""
    ms = np.zeros(3, np.float32)
    lib().refgpu_last_times(ms)
    return float(ms[0]), float(ms[1]), float(ms[2])
