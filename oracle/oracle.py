"""ctypes wrapper of the CPU oracle (oracle/libbpx_oracle.so).  TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm, as the checker
or the timed CPU baseline.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from fdt_b200.abi import BPX_NSTATE, Options, TrackOptions, TrackVolume, nrec

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libbpx_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_rng_slot.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_logI0.restype = C.c_double
        L.orc_logI0.argtypes = [C.c_double]
        L.orc_dti.argtypes = [C.c_int, _f32p, _f32p, _f32p, _f64p]
        L.orc_prepare_data.argtypes = [C.c_int, C.c_int, _f32p]
        L.orc_fit.argtypes = [C.POINTER(Options), C.c_int, C.c_int, _f32p, _f32p, _f32p, _f64p,
                              C.c_void_p, C.c_void_p, C.c_int]
        L.orc_lm_start.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f64p]
        L.orc_lm_starts.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f64p,
                                    C.c_int]
        L.orc_lm_fit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, _f32p,
                                 _f32p, _f32p, _f64p, _f64p]
        L.orc_lm_eval.restype = C.c_double
        L.orc_lm_eval.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, _f32p,
                                  _f32p, _f32p, _f64p, C.c_void_p, C.c_void_p]
        L.orc_mcmc.argtypes = [C.POINTER(Options), C.c_int, C.c_int, _f32p, _f32p, _f32p, _f64p,
                               C.c_void_p, C.c_uint64, _f64p, C.c_int]
        L.orc_finish.argtypes = [C.POINTER(Options), C.c_int, _f64p] + [C.c_void_p] * 11
        L.orc_energy.argtypes = [C.POINTER(Options), C.c_int, C.c_int, _f32p, _f32p, _f32p, _f64p,
                                 C.c_void_p, C.c_void_p]
        L.orc_probtrack.argtypes = [C.POINTER(TrackOptions), C.POINTER(TrackVolume), C.c_int, _f32p,
                                    np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS"), C.POINTER(C.c_int64)]
        L.orc_track_uniforms.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_uint32, _f32p]
        L.orc_sincos_fast.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def nthreads_default() -> int:
    return os.cpu_count() or 1


def philox(ctr, key) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def rng_slot(seed: int, vox: int, it: int, slot: int) -> tuple[float, float]:
    n, lu = C.c_double(), C.c_double()
    lib().orc_rng_slot(seed, vox, it, slot, C.byref(n), C.byref(lu))
    return n.value, lu.value


def logI0(x: float) -> float:
    return lib().orc_logI0(x)


def dti(y, bvecs, bvals) -> dict:
    out = np.zeros(16)
    rc = lib().orc_dti(len(y), np.ascontiguousarray(y, np.float32),
                       np.ascontiguousarray(bvecs, np.float32),
                       np.ascontiguousarray(bvals, np.float32), out)
    assert rc == 0
    return dict(s0=out[0], md=out[1], fa=out[2], l=out[3:6], v1=out[6:9], v2=out[9:12],
                v3=out[12:15], sse=out[15])


def prepare_data(data: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(data, np.float32).copy()
    lib().orc_prepare_data(d.shape[0], d.shape[1], d)
    return d


def fit(opts: Options, data, bvecs, bvals, nthreads: int | None = None):
    data = np.ascontiguousarray(data, np.float32)
    nvox, ndir = data.shape
    params = np.zeros((nvox, opts.nparams_fit))
    tau = np.zeros(nvox)
    status = np.zeros(nvox, np.uint32)
    rc = lib().orc_fit(C.byref(opts), nvox, ndir, data, np.ascontiguousarray(bvecs, np.float32),
                       np.ascontiguousarray(bvals, np.float32), params, _ptr(tau), _ptr(status),
                       nthreads or nthreads_default())
    assert rc == 0, "orc_fit failed"
    return params, tau, status


def lm_start(kind: int, nfib: int, f0: bool, y, bvecs, bvals) -> np.ndarray:
    np_ = 3 * nfib + 2 + (1 if f0 else 0)
    p = np.zeros(np_)
    lib().orc_lm_start(kind, nfib, int(f0), len(y), np.ascontiguousarray(y, np.float32),
                       np.ascontiguousarray(bvecs, np.float32),
                       np.ascontiguousarray(bvals, np.float32), p)
    return p


def lm_starts(kind: int, nfib: int, f0: bool, data, bvecs, bvals, nthreads: int | None = None) -> np.ndarray:
    """Start parameters of every voxel of data [nvox][ndir] (DTI + the model's start rule)."""
    data = np.ascontiguousarray(data, np.float32)
    nvox, ndir = data.shape
    p = np.zeros((nvox, 3 * nfib + 2 + (1 if f0 else 0)))
    lib().orc_lm_starts(kind, nfib, int(f0), nvox, ndir, data, np.ascontiguousarray(bvecs, np.float32),
                        np.ascontiguousarray(bvals, np.float32), p, nthreads or nthreads_default())
    return p


def lm_fit(kind: int, nfib: int, f0: bool, gbo: int, R: float, y, bvecs, bvals, start):
    np_ = 3 * nfib + 2 + (1 if kind == 2 else 0) + (1 if f0 else 0)
    out = np.zeros(np_)
    it = lib().orc_lm_fit(kind, nfib, int(f0), gbo, R, len(y), np.ascontiguousarray(y, np.float32),
                          np.ascontiguousarray(bvecs, np.float32),
                          np.ascontiguousarray(bvals, np.float32),
                          np.ascontiguousarray(start, np.float64), out)
    return out, it


def lm_eval(kind: int, nfib: int, f0: bool, gbo: int, R: float, y, bvecs, bvals, p):
    np_ = len(p)
    g = np.zeros(np_)
    H = np.zeros((np_, np_))
    cf = lib().orc_lm_eval(kind, nfib, int(f0), gbo, R, len(y), np.ascontiguousarray(y, np.float32),
                           np.ascontiguousarray(bvecs, np.float32),
                           np.ascontiguousarray(bvals, np.float32),
                           np.ascontiguousarray(p, np.float64), g.ctypes.data, H.ctypes.data)
    return cf, g, H


def mcmc(opts: Options, data, bvecs, bvals, params, tau=None, voxel_offset: int = 0,
         nthreads: int | None = None) -> np.ndarray:
    data = np.ascontiguousarray(data, np.float32)
    nvox, ndir = data.shape
    rec = np.zeros((nrec(opts.nfibres), opts.nsamples, nvox))
    tau_a = None if tau is None else np.ascontiguousarray(tau, np.float64)
    rc = lib().orc_mcmc(C.byref(opts), nvox, ndir, data, np.ascontiguousarray(bvecs, np.float32),
                        np.ascontiguousarray(bvals, np.float32),
                        np.ascontiguousarray(params, np.float64), _ptr(tau_a), voxel_offset, rec,
                        nthreads or nthreads_default())
    assert rc == 0
    return rec


def finish(opts: Options, records: np.ndarray) -> dict:
    K, ns, nvox = opts.nfibres, opts.nsamples, records.shape[2]
    out = dict(
        th=np.zeros((K, ns, nvox)), ph=np.zeros((K, ns, nvox)), f=np.zeros((K, ns, nvox)),
        mean_d=np.zeros(nvox), mean_dstd=np.zeros(nvox), mean_R=np.zeros(nvox),
        mean_f0=np.zeros(nvox), mean_tau=np.zeros(nvox), mean_S0=np.zeros(nvox),
        mean_f=np.zeros((K, nvox)), dyads=np.zeros((K, 3, nvox)),
    )
    keys = ["th", "ph", "f", "mean_d", "mean_dstd", "mean_R", "mean_f0", "mean_tau", "mean_S0",
            "mean_f", "dyads"]
    lib().orc_finish(C.byref(opts), nvox, np.ascontiguousarray(records, np.float64),
                     *[out[k].ctypes.data for k in keys])
    return out


def energy(opts: Options, data, bvecs, bvals, states):
    data = np.ascontiguousarray(data, np.float32)
    nvox, ndir = data.shape
    lik = np.zeros(nvox)
    prior = np.zeros(nvox)
    st = np.ascontiguousarray(states, np.float64).reshape(nvox, BPX_NSTATE)
    lib().orc_energy(C.byref(opts), nvox, ndir, data, np.ascontiguousarray(bvecs, np.float32),
                     np.ascontiguousarray(bvals, np.float32), st, lik.ctypes.data,
                     prior.ctypes.data)
    return lik, prior


def probtrack(topts: TrackOptions, th, ph, f, mask, seeds, voxel_size=(2.0, 2.0, 2.0), avoid=None, stop=None,
              waypoints=None, targets=None, matrix2=None, matrix1=None, prefdir=None):
    """probtrackx simple mode on host arrays (th/ph/f [nfib][nsamples][nz][ny][nx], mask [nz][ny][nx],
    seeds [nseeds][3] voxel coordinates; optional avoid and stop masks and a list of waypoint masks,
    each [nz][ny][nx]; target masks, each [nz][ny][nx]; matrix2 = (tract-space mask [lz][ly][lx], its
    voxel size); matrix1 = the seed mask [nz][ny][nx]): (paths [nz][ny][nx] int32, or
    [nseeds][nz][ny][nx] with topts.per_seed, waytotal[, seeds_to_targets [ntargets][nseeds] int32
    when targets are given][, fdt_matrix2 [nseeds][columns] int32 when matrix2 is given][,
    fdt_matrix1 [nseeds][seed-mask voxels] int32 when matrix1 is given]); prefdir: a preferred
    direction volume [3][nz][ny][nx] (--prefdir)."""
    th, ph, f, mask = (np.ascontiguousarray(a, np.float32) for a in (th, ph, f, mask))
    v = TrackVolume()
    v.nfib, v.nsamples, v.nz, v.ny, v.nx = th.shape
    v.dx, v.dy, v.dz = voxel_size
    v.th, v.ph, v.f, v.mask = th.ctypes.data, ph.ctypes.data, f.ctypes.data, mask.ctypes.data
    keep = []
    if avoid is not None:
        keep.append(np.ascontiguousarray(avoid, np.float32))
        v.avoid = keep[-1].ctypes.data
    if stop is not None:
        keep.append(np.ascontiguousarray(stop, np.float32))
        v.stop = keep[-1].ctypes.data
    if waypoints is not None:
        bits = np.zeros(mask.shape, np.uint32)
        for w, m in enumerate(waypoints):
            bits |= (np.asarray(m) != 0).astype(np.uint32) << np.uint32(w)
        keep.append(bits)
        v.waypoints, v.nwaypoints = bits.ctypes.data, len(waypoints)
    sd = np.ascontiguousarray(seeds, np.float32).reshape(-1, 3)
    s2t = None
    if targets is not None:
        tb = np.zeros(mask.shape, np.uint32)
        for t, m in enumerate(targets):
            tb |= (np.asarray(m) != 0).astype(np.uint32) << np.uint32(t)
        s2t = np.zeros((len(targets), sd.shape[0]), np.int32)
        keep += [tb, s2t]
        v.ntargets, v.targets, v.seeds_to_targets = len(targets), tb.ctypes.data, s2t.ctypes.data
    m2 = None
    if matrix2 is not None:
        lrmask, lr_size = matrix2
        inside = np.asarray(lrmask) != 0
        lut = np.full(inside.shape, -1, np.int32)  # columns in z, y, x order (Counter::initialise_matrix2)
        lut[inside] = np.arange(int(inside.sum()), dtype=np.int32)
        m2 = np.zeros((sd.shape[0], int(inside.sum())), np.int32)
        keep += [lut, m2]
        v.m2_ncols = m2.shape[1]
        v.lr_nz, v.lr_ny, v.lr_nx = lut.shape
        v.lr_dx, v.lr_dy, v.lr_dz = lr_size
        v.m2_lookup, v.matrix2 = lut.ctypes.data, m2.ctypes.data
    m1 = None
    if matrix1 is not None:
        inside1 = np.asarray(matrix1) != 0
        assert inside1.shape == mask.shape
        lut1 = np.full(inside1.shape, -1, np.int32)  # columns in z, y, x order (Counter::initialise_matrix1)
        lut1[inside1] = np.arange(int(inside1.sum()), dtype=np.int32)
        m1 = np.zeros((sd.shape[0], int(inside1.sum())), np.int32)
        keep += [lut1, m1]
        v.m1_ncols = m1.shape[1]
        v.m1_lookup, v.matrix1 = lut1.ctypes.data, m1.ctypes.data
    if prefdir is not None:
        pd = np.ascontiguousarray(prefdir, np.float32)
        assert pd.shape == (3,) + mask.shape
        keep.append(pd)
        v.prefdir = pd.ctypes.data
    paths = np.zeros(((sd.shape[0],) if topts.per_seed else ()) + tuple(mask.shape), np.int32)
    way = C.c_int64(0)
    rc = lib().orc_probtrack(C.byref(topts), C.byref(v), sd.shape[0], sd, paths, C.byref(way))
    assert rc == 0
    out = (paths, int(way.value))
    if targets is not None:
        out += (s2t,)
    if matrix2 is not None:
        out += (m2,)
    if matrix1 is not None:
        out += (m1,)
    return out


def sincos_fast(x: float) -> tuple[float, float]:
    s, c = C.c_float(), C.c_float()
    lib().orc_sincos_fast(x, C.byref(s), C.byref(c))
    return s.value, c.value
