"""Python binding of libbpx.so (the sm_100a CUDA library) through its C-ABI.

Host-side mirror of the xfibres_gpu interface for tests, benchmarks and Python users.  Device
memory comes from torch (plumbing only); every computation runs in the library's CUDA kernels.
There is no CPU fallback: if the library is missing or the device is not sm_100, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import BPX_NSTATE, Item, Options, Outputs, PostProc, TrackOptions, TrackVolume, Volume, nrec

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbpx.so")

# exported functions: name -> (restype, argtypes)
_SIGS = {
    "bpx_abi_version": (C.c_int32, []),
    "bpx_options_default": (None, [C.POINTER(Options)]),
    "bpx_nparams_fit": (C.c_int32, [C.POINTER(Options)]),
    "bpx_nsamples": (C.c_int32, [C.POINTER(Options)]),
    "bpx_max_ndir": (C.c_int32, []),
    "bpx_last_error": (C.c_char_p, []),
    "bpx_fit_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_prepare_data_dev": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "bpx_mcmc_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "bpx_finish_dev": (C.c_int, [C.POINTER(Options), C.c_int32, C.c_void_p, C.POINTER(Outputs), C.c_void_p]),
    "bpx_xfibres_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.POINTER(Outputs), C.c_void_p]),
    "bpx_xfibres_host": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.POINTER(Outputs)]),
    "bpx_energy_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "bpx_gradnonlin_dev": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "bpx_mcmc_layouts": (C.c_int32, [C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32]),
    "bpx_release_workspace": (C.c_int, []),
    "bpx_track_options_default": (None, [C.POINTER(TrackOptions)]),
    "bpx_probtrack_dev": (C.c_int, [C.POINTER(TrackOptions), C.POINTER(TrackVolume), C.c_int32, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_handle_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "bpx_handle_bind": (C.c_int, [C.c_void_p]),
    "bpx_handle_destroy": (C.c_int, [C.c_void_p]),
    "bpx_measure_pipes": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "bpx_xfibres_noalloc_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.POINTER(Outputs), C.c_void_p]),
    "bpx_mcmc_ex_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mcmc_stretch_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mlp_nin": (C.c_int32, [C.c_int32]),
    "bpx_mlp_nparams": (C.c_int64, [C.c_int32]),
    "bpx_mlp_features_dev": (C.c_int, [C.POINTER(Volume), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mlp_forward_dev": (C.c_int, [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mlp_train_step_dev": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mlp_adam_dev": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                   C.c_float, C.c_float, C.c_int32, C.c_void_p]),
    "bpx_mlp_targets_dev": (C.c_int, [C.POINTER(Options), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_mlp_decode_dev": (C.c_int, [C.POINTER(Options), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "bpx_xfibres_learned_dev": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_int32,
                                          C.POINTER(Outputs), C.c_void_p]),
    "bpx_xfibres_learned_host": (C.c_int, [C.POINTER(Options), C.POINTER(Volume), C.c_void_p, C.c_int32,
                                           C.POINTER(Outputs)]),
    "bpx_gemm_bf16_dev": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                    C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p]),
    "bpx_mlp_poll_error": (C.c_int, [C.POINTER(C.c_int32)]),
    "bpx_batch_create": (C.c_int, [C.POINTER(Options), C.POINTER(Item), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "bpx_batch_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bpx_batch_buckets": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32), C.c_int32]),
    "bpx_batch_destroy": (C.c_int, [C.c_void_p]),
    "bpx_autotune_layout": (C.c_int, [C.POINTER(Options), C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_float), C.c_void_p]),
    "bpx_postproc_dev": (C.c_int, [C.POINTER(Options), C.c_int32, C.POINTER(Outputs), C.c_float, C.POINTER(PostProc),
                                   C.c_void_p]),
    "bpx_synth_dev": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64, C.c_float,
                                C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


class BpxError(RuntimeError):
    pass


def load(path: str | None = None):
    """Load libbpx.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise BpxError(f"{p} not found: build it with `python -m fdt_b200.build`")
    L = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().bpx_last_error().decode(errors="replace")
        raise BpxError(f"{what} failed with status {rc}: {msg}")


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise BpxError("CUDA device required")
    return torch


def _stream(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def make_volume(data, bvecs, bvals, voxel_offset: int = 0) -> Volume:
    v = Volume()
    v.nvox, v.ndir = int(data.shape[0]), int(data.shape[1])
    v.data, v.bvecs, v.bvals = _ptr(data), _ptr(bvecs), _ptr(bvals)
    v.grad = None
    v.voxel_offset = voxel_offset
    return v


def to_device(x, torch=None):
    torch = torch or _torch()
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x, np.float32))
    return x.to(device="cuda", dtype=torch.float32).contiguous()


def prepare_data(data) -> None:
    """remove_NonPositive_entries in place on a device tensor [nvox][ndir]."""
    torch = _torch()
    _check(load().bpx_prepare_data_dev(data.shape[0], data.shape[1], _ptr(data), _stream(torch)), "bpx_prepare_data_dev")


def fit(opts: Options, data, bvecs, bvals):
    """LM initial fits (+ tau under rician).  Returns (params, tau, status) device tensors."""
    torch = _torch()
    nvox = data.shape[0]
    params = torch.zeros((nvox, opts.nparams_fit), device="cuda", dtype=torch.float32)
    tau = torch.zeros(nvox, device="cuda", dtype=torch.float32)
    status = torch.zeros(nvox, device="cuda", dtype=torch.int32)
    vol = make_volume(data, bvecs, bvals)
    _check(load().bpx_fit_dev(C.byref(opts), C.byref(vol), _ptr(params), _ptr(tau), _ptr(status), _stream(torch)),
           "bpx_fit_dev")
    return params, tau, status


def mcmc_ex(opts: Options, data, bvecs, bvals, params, tau=None, props_in=None, freeze: int = 0,
            want_props: bool = False, voxel_offset: int = 0, status=None):
    """MCMC with per-voxel proposal widths (freeze: 0 adapt, 1 never, 2 burn-in only).
    Returns (records, props_out or None)."""
    torch = _torch()
    nvox = data.shape[0]
    rec = torch.zeros((nrec(opts.nfibres), opts.nsamples, nvox), device="cuda", dtype=torch.float32)
    pout = torch.zeros((6 + 3 * opts.nfibres, nvox), device="cuda", dtype=torch.float32) if want_props else None
    vol = make_volume(data, bvecs, bvals, voxel_offset)
    _check(load().bpx_mcmc_ex_dev(C.byref(opts), C.byref(vol), _ptr(params), _ptr(tau), _ptr(props_in), _ptr(pout),
                                  int(freeze), _ptr(rec), _ptr(status), _stream(torch)), "bpx_mcmc_ex_dev")
    return rec, pout


def mcmc_stretch(opts: Options, data, bvecs, bvals, it_begin: int, it_end: int, params=None, tau=None,
                 state=None, records=None, voxel_offset: int = 0, freeze: int = 0):
    """Iterations [it_begin, it_end) of the chain (bpx_mcmc_stretch_dev).  `state` is the previous
    stretch's return value (a dict of state/props/acc tensors) or None to start from params/tau.
    Returns (records, state at it_end); pass the same records tensor to every stretch of a chain."""
    torch = _torch()
    nvox = data.shape[0]
    rows = 6 + 3 * opts.nfibres
    if records is None:
        records = torch.zeros((nrec(opts.nfibres), opts.nsamples, nvox), device="cuda", dtype=torch.float32)
    out = {"state": torch.empty((rows, nvox), device="cuda", dtype=torch.float32),
           "props": torch.empty((rows, nvox), device="cuda", dtype=torch.float32),
           "acc": torch.empty((rows, nvox), device="cuda", dtype=torch.int32)}
    vol = make_volume(data, bvecs, bvals, voxel_offset)
    s_in = state or {}
    _check(load().bpx_mcmc_stretch_dev(C.byref(opts), C.byref(vol), _ptr(params), _ptr(tau), _ptr(s_in.get("state")),
                                       _ptr(s_in.get("props")), _ptr(s_in.get("acc")), int(it_begin), int(it_end),
                                       int(freeze), _ptr(records), _ptr(out["state"]), _ptr(out["props"]),
                                       _ptr(out["acc"]), None, _stream(torch)), "bpx_mcmc_stretch_dev")
    return records, out


def gemm_bf16(a, b, M: int, N: int, K: int, a_mn: bool = False, b_mn: bool = False):
    """C [M][N] fp32 = A B^T on the tcgen05 tensor cores; a, b are bf16 device tensors (see bpx_gemm_bf16_dev)."""
    torch = _torch()
    c = torch.zeros((M, N), device="cuda", dtype=torch.float32)
    _check(load().bpx_gemm_bf16_dev(M, N, K, _ptr(a), a.shape[1], 1 if a_mn else 0, _ptr(b), b.shape[1],
                                    1 if b_mn else 0, _ptr(c), N, _stream(torch)), "bpx_gemm_bf16_dev")
    return c


def synth(model: int, nfib: int, nvox: int, bvecs, bvals, seed: int, snr=(10.0, 40.0), voxel_offset: int = 0):
    """Forward-model voxels with Rician noise on the device: (data [nvox][ndir], truth [nvox][15])."""
    torch = _torch()
    ndir = bvals.shape[0]
    data = torch.empty((nvox, ndir), device="cuda", dtype=torch.float32)
    truth = torch.empty((nvox, BPX_NSTATE), device="cuda", dtype=torch.float32)
    _check(load().bpx_synth_dev(model, nfib, nvox, ndir, seed, voxel_offset, float(snr[0]), float(snr[1]),
                                _ptr(bvecs), _ptr(bvals), _ptr(data), _ptr(truth), _stream(torch)), "bpx_synth_dev")
    return data, truth


def poll_error() -> int:
    """Reads and clears the tensor-core kernels' device error word (synchronous)."""
    code = C.c_int32()
    _check(load().bpx_mlp_poll_error(C.byref(code)), "bpx_mlp_poll_error")
    return code.value


def mcmc(opts: Options, data, bvecs, bvals, params, tau=None, voxel_offset: int = 0, status=None):
    """Burn-in + recording.  Returns records [nrec][nsamples][nvox] (device)."""
    torch = _torch()
    nvox = data.shape[0]
    rec = torch.zeros((nrec(opts.nfibres), opts.nsamples, nvox), device="cuda", dtype=torch.float32)
    vol = make_volume(data, bvecs, bvals, voxel_offset)
    _check(load().bpx_mcmc_dev(C.byref(opts), C.byref(vol), _ptr(params), _ptr(tau), _ptr(rec), _ptr(status),
                               _stream(torch)), "bpx_mcmc_dev")
    return rec


OUT_KEYS = ["th", "ph", "f", "mean_d", "mean_dstd", "mean_R", "mean_f0", "mean_tau", "mean_S0", "mean_f", "dyads",
            "status"]


def alloc_outputs(opts: Options, nvox: int, device: str = "cuda", pin: bool = False):
    """Output arrays (torch tensors on `device`) and the Outputs struct pointing at them."""
    import torch

    K, ns = opts.nfibres, opts.nsamples
    shapes = dict(th=(K, ns, nvox), ph=(K, ns, nvox), f=(K, ns, nvox), mean_d=(nvox,), mean_dstd=(nvox,),
                  mean_R=(nvox,), mean_f0=(nvox,), mean_tau=(nvox,), mean_S0=(nvox,), mean_f=(K, nvox),
                  dyads=(K, 3, nvox), status=(nvox,))
    t = {}
    for k, s in shapes.items():
        dt = torch.int32 if k == "status" else torch.float32
        t[k] = torch.zeros(s, device=device, dtype=dt, pin_memory=(pin and device == "cpu"))
    o = Outputs()
    for k in OUT_KEYS:
        setattr(o, k, t[k].data_ptr())
    return t, o


def finish(opts: Options, records):
    torch = _torch()
    nvox = records.shape[2]
    t, o = alloc_outputs(opts, nvox)
    _check(load().bpx_finish_dev(C.byref(opts), nvox, _ptr(records), C.byref(o), _stream(torch)), "bpx_finish_dev")
    return t


def xfibres_dev(opts: Options, data, bvecs, bvals, voxel_offset: int = 0, out=None):
    """Whole pipeline on device tensors; returns the output dict (device tensors)."""
    torch = _torch()
    nvox = data.shape[0]
    if out is None:
        t, o = alloc_outputs(opts, nvox)
    else:
        t, o = out
    vol = make_volume(data, bvecs, bvals, voxel_offset)
    _check(load().bpx_xfibres_dev(C.byref(opts), C.byref(vol), C.byref(o), _stream(torch)), "bpx_xfibres_dev")
    return t


def xfibres_host(opts: Options, data: np.ndarray, bvecs: np.ndarray, bvals: np.ndarray, grad: np.ndarray | None = None,
                 voxel_offset: int = 0, out=None):
    """Drop-in for xfibres_gpu() with host arrays (synchronous).  Returns dict of host tensors."""
    data = np.ascontiguousarray(data, np.float32)
    bvecs = np.ascontiguousarray(bvecs, np.float32)
    bvals = np.ascontiguousarray(bvals, np.float32)
    nvox = data.shape[0]
    if out is None:
        t, o = alloc_outputs(opts, nvox, device="cpu")
    else:
        t, o = out
    vol = Volume()
    vol.nvox, vol.ndir = data.shape
    vol.data, vol.bvecs, vol.bvals = data.ctypes.data, bvecs.ctypes.data, bvals.ctypes.data
    g = None
    if grad is not None:
        g = np.ascontiguousarray(grad, np.float32)
        vol.grad = g.ctypes.data
    vol.voxel_offset = voxel_offset
    _check(load().bpx_xfibres_host(C.byref(opts), C.byref(vol), C.byref(o)), "bpx_xfibres_host")
    return t


def energy(opts: Options, data, bvecs, bvals, states):
    """FP32 likelihood and prior energies of states [nvox][15] (device)."""
    torch = _torch()
    nvox = data.shape[0]
    lik = torch.zeros(nvox, device="cuda", dtype=torch.float32)
    prior = torch.zeros(nvox, device="cuda", dtype=torch.float32)
    vol = make_volume(data, bvecs, bvals)
    _check(load().bpx_energy_dev(C.byref(opts), C.byref(vol), _ptr(states), _ptr(lik), _ptr(prior), _stream(torch)),
           "bpx_energy_dev")
    return lik, prior


def gradnonlin(grad, bvecs, bvals):
    """Per-voxel corrected b-matrix on the device: returns (bvecs [nvox][3][ndir], bvals [nvox][ndir])."""
    torch = _torch()
    nvox, ndir = grad.shape[0], bvals.shape[0]
    bv = torch.zeros((nvox, 3, ndir), device="cuda", dtype=torch.float32)
    bl = torch.zeros((nvox, ndir), device="cuda", dtype=torch.float32)
    _check(load().bpx_gradnonlin_dev(nvox, ndir, _ptr(grad), _ptr(bvecs), _ptr(bvals), _ptr(bv), _ptr(bl),
                                     _stream(torch)), "bpx_gradnonlin_dev")
    return bv, bl


def mcmc_layouts() -> list[tuple[int, int]]:
    L = load()
    n = L.bpx_mcmc_layouts(None, None, 0)
    tpv = (C.c_int32 * n)()
    mpl = (C.c_int32 * n)()
    L.bpx_mcmc_layouts(tpv, mpl, n)
    return list(zip(list(tpv), list(mpl)))


def measure_pipes() -> tuple[float, float]:
    """(MUFU ops/s, FP32 FMA ops/s) measured on the current device."""
    _torch()
    m, f = C.c_double(), C.c_double()
    _check(load().bpx_measure_pipes(C.byref(m), C.byref(f)), "bpx_measure_pipes")
    return m.value, f.value


def states_from_records(opts: Options, records, sample: int):
    """Chain states [nvox][15] (S0, d, d_std, R, tau, f0, (th, ph, f)*3) of one recorded sample."""
    torch = _torch()
    nvox = records.shape[2]
    st = torch.zeros((nvox, BPX_NSTATE), device=records.device, dtype=torch.float32)
    r = records[:, sample, :]
    st[:, 0] = r[5]
    st[:, 1] = r[0]
    st[:, 2] = r[3]
    st[:, 3] = r[4]
    st[:, 4] = r[2]
    st[:, 5] = r[1]
    for k in range(opts.nfibres):
        st[:, 6 + 3 * k] = r[6 + 3 * k]
        st[:, 7 + 3 * k] = r[7 + 3 * k]
        st[:, 8 + 3 * k] = r[8 + 3 * k]
    return st


def track_volume(th, ph, f, mask, voxel_size=(2.0, 2.0, 2.0), avoid=None, stop=None, waypoints=None,
                 nwaypoints: int = 0) -> TrackVolume:
    """TrackVolume over device tensors th/ph/f [nfib][nsamples][nz][ny][nx] and mask [nz][ny][nx];
    optional avoid and stop masks (float32 [nz][ny][nx]) and waypoint bits (int32 [nz][ny][nx], bit w
    for waypoint mask w < nwaypoints).  The tensors must outlive the call that uses the volume."""
    v = TrackVolume()
    v.nfib, v.nsamples, v.nz, v.ny, v.nx = (int(x) for x in th.shape)
    v.dx, v.dy, v.dz = (float(x) for x in voxel_size)
    v.th, v.ph, v.f, v.mask = th.data_ptr(), ph.data_ptr(), f.data_ptr(), mask.data_ptr()
    for name, t in (("avoid", avoid), ("stop", stop), ("waypoints", waypoints)):
        if t is not None:
            if tuple(t.shape) != tuple(mask.shape) or t.element_size() != 4 or not t.is_contiguous():
                raise ValueError(f"{name}: a contiguous 4-byte array of the mask's shape is needed")
            setattr(v, name, t.data_ptr())
    v.nwaypoints = int(nwaypoints) if waypoints is not None else 0
    return v


def waypoint_bits(masks) -> np.ndarray:
    """Waypoint masks ([nz][ny][nx] each, != 0 inside) packed as bpx_track_volume.waypoints:
    int32 [nz][ny][nx] with bit w set inside mask w."""
    masks = list(masks)
    if not 1 <= len(masks) <= 32:
        raise ValueError("1 to 32 waypoint masks")
    bits = np.zeros(np.shape(masks[0]), np.uint32)
    for w, m in enumerate(masks):
        bits |= (np.asarray(m) != 0).astype(np.uint32) << np.uint32(w)
    return bits.view(np.int32)


def matrix2_lookup(lrmask) -> np.ndarray:
    """bpx_track_volume.m2_lookup for a tract-space mask [lz][ly][lx]: int32 of the same shape, the
    column of every voxel inside the mask (0, 1, ... in z, y, x order, as Counter::initialise_matrix2
    numbers them, streamlines.cc:515-549) and -1 outside."""
    m = np.asarray(lrmask) != 0
    lut = np.full(m.shape, -1, np.int32)
    lut[m] = np.arange(int(m.sum()), dtype=np.int32)
    return lut


def probtrack(topts: TrackOptions, th, ph, f, mask, seeds, voxel_size=(2.0, 2.0, 2.0), avoid=None, stop=None,
              waypoints=None, targets=None, matrix2=None, matrix1=None, prefdir=None):
    """probtrackx on device tensors: (paths [nz][ny][nx] int32, or [nseeds][nz][ny][nx] with
    topts.per_seed; waytotal int) for
    seeds [nseeds][3] (voxel coordinates x, y, z).  `avoid` and `stop`: device masks of the mask's
    shape (--avoid, --stop); `waypoints`: a list of 1 to 32 masks (host or device) that a kept
    streamline must all pass (--waypoints); `targets`: a list of 1 to 32 target masks, for which
    seeds_to_targets [ntargets][nseeds] (int32, host) follows waytotal (--targetmasks --os2t);
    `matrix2`: (tract-space mask [lz][ly][lx], its voxel size in mm), for which fdt_matrix2
    [nseeds][columns] (int32, host) follows (--omatrix2 --lrmask); `matrix1`: the seed mask
    [nz][ny][nx], for which fdt_matrix1 [nseeds][seed-mask voxels] (int32, host) comes last
    (--omatrix1: each seed's path distribution at the seed-mask voxels, in z, y, x order); `prefdir`:
    a preferred direction per voxel, [3][nz][ny][nx] (--prefdir)."""
    torch = _torch()
    way_bits = None
    nway = 0
    if waypoints is not None:
        nway = len(waypoints)
        bits = waypoint_bits([w.cpu().numpy() if hasattr(w, "cpu") else w for w in waypoints])
        way_bits = torch.from_numpy(bits).to("cuda")
    v = track_volume(th, ph, f, mask, voxel_size, avoid=avoid, stop=stop, waypoints=way_bits, nwaypoints=nway)
    sd = to_device(np.asarray(seeds, np.float32).reshape(-1, 3))
    lead = (int(sd.shape[0]),) if topts.per_seed else ()
    paths = torch.zeros(lead + tuple(mask.shape), device="cuda", dtype=torch.int32)
    way = torch.zeros(1, device="cuda", dtype=torch.int64)
    s2t = None
    if targets is not None:
        tb = torch.from_numpy(waypoint_bits([t.cpu().numpy() if hasattr(t, "cpu") else t for t in targets])).to("cuda")
        s2t = torch.zeros((len(targets), int(sd.shape[0])), device="cuda", dtype=torch.int32)
        v.ntargets, v.targets, v.seeds_to_targets = len(targets), tb.data_ptr(), s2t.data_ptr()
    m2 = None
    if matrix2 is not None:
        lrmask, lr_size = matrix2
        lut = matrix2_lookup(lrmask.cpu().numpy() if hasattr(lrmask, "cpu") else lrmask)
        ncols = int((lut >= 0).sum())
        lut_d = torch.from_numpy(lut).to("cuda")
        m2 = torch.zeros((int(sd.shape[0]), ncols), device="cuda", dtype=torch.int32)
        v.m2_ncols = ncols
        v.lr_nz, v.lr_ny, v.lr_nx = (int(x) for x in lut.shape)
        v.lr_dx, v.lr_dy, v.lr_dz = (float(x) for x in lr_size)
        v.m2_lookup, v.matrix2 = lut_d.data_ptr(), m2.data_ptr()
    m1 = None
    if matrix1 is not None:
        lut1 = matrix2_lookup(matrix1.cpu().numpy() if hasattr(matrix1, "cpu") else matrix1)
        if lut1.shape != tuple(mask.shape):
            raise BpxError("matrix1: the seed mask must have the mask's shape")
        lut1_d = torch.from_numpy(lut1).to("cuda")
        m1 = torch.zeros((int(sd.shape[0]), int((lut1 >= 0).sum())), device="cuda", dtype=torch.int32)
        v.m1_ncols = int(m1.shape[1])
        v.m1_lookup, v.matrix1 = lut1_d.data_ptr(), m1.data_ptr()
    pd = None
    if prefdir is not None:
        pd = to_device(prefdir.cpu().numpy() if hasattr(prefdir, "cpu") else np.asarray(prefdir))
        if tuple(pd.shape) != (3,) + tuple(mask.shape):
            raise BpxError("prefdir: expected [3][nz][ny][nx] on the mask's grid")
        v.prefdir = pd.data_ptr()
    _check(load().bpx_probtrack_dev(C.byref(topts), C.byref(v), int(sd.shape[0]), _ptr(sd), _ptr(paths), _ptr(way),
                                    _stream(torch)), "bpx_probtrack_dev")
    out = (paths, int(way.item()))
    if targets is not None:
        out += (s2t.cpu().numpy(),)
    if matrix2 is not None:
        out += (m2.cpu().numpy(),)
    if matrix1 is not None:
        out += (m1.cpu().numpy(),)
    return out


class Handle:
    """Private workspaces for the workspace-using entries (bpx_handle_*).  ``with handle:`` binds it
    to the calling thread for the block, so that calls from different threads with different
    handles may run concurrently on different streams."""

    def __init__(self):
        h = C.c_void_p()
        _check(load().bpx_handle_create(C.byref(h)), "bpx_handle_create")
        self.h = h

    def __enter__(self):
        _check(load().bpx_handle_bind(self.h), "bpx_handle_bind")
        return self

    def __exit__(self, *exc):
        load().bpx_handle_bind(None)
        return False

    def close(self):
        if getattr(self, "h", None):
            _check(load().bpx_handle_destroy(self.h), "bpx_handle_destroy")
            self.h = None


class Batch:
    """A batch of items run as one CUDA-graph launch (bpx_batch_*).  `items` is a list of dicts
    with keys data, bvecs, bvals (device tensors), model, nfibres, and optionally voxel_offset,
    mlp (device FP32 initialiser parameters: learned start), nburn, freeze; the outputs are
    allocated here (device) and returned by run() as a list of output dicts."""

    def __init__(self, opts: Options, items: list, autotune: bool = True):
        torch = _torch()
        self.opts = opts
        self._keep = []
        arr = (Item * len(items))()
        self.outputs = []
        for i, it in enumerate(items):
            o = Options.make(**{f: getattr(opts, f) for f, _ in Options._fields_ if f != "reserved"})
            o.model, o.nfibres = it["model"], it["nfibres"]
            t, out = alloc_outputs(o, int(it["data"].shape[0]))
            self.outputs.append(t)
            arr[i].vol = make_volume(it["data"], it["bvecs"], it["bvals"], int(it.get("voxel_offset", 0)))
            arr[i].model, arr[i].nfibres = it["model"], it["nfibres"]
            arr[i].out = out
            arr[i].mlp_params = _ptr(it.get("mlp"))
            arr[i].nburn = int(it.get("nburn", -1))
            arr[i].freeze_props = int(it.get("freeze", 0))
            if it.get("mlp") is not None:
                self._keep.append(it["mlp"])
            self._keep.append((it["data"], it["bvecs"], it["bvals"]))
        h = C.c_void_p()
        _check(load().bpx_batch_create(C.byref(opts), arr, len(items), 1 if autotune else 0, C.byref(h)),
               "bpx_batch_create")
        self.handle = h
        del torch

    def buckets(self) -> list[dict]:
        L = load()
        n = L.bpx_batch_buckets(self.handle, None, 0)
        d = (C.c_int32 * (7 * max(n, 1)))()
        L.bpx_batch_buckets(self.handle, d, n)
        keys = ["model", "nfibres", "ndir", "tpv", "mpl", "voxels", "items"]
        return [dict(zip(keys, list(d[7 * i : 7 * i + 7]))) for i in range(n)]

    def run(self):
        torch = _torch()
        _check(load().bpx_batch_run(self.handle, _stream(torch)), "bpx_batch_run")
        return self.outputs

    def close(self):
        if getattr(self, "handle", None):
            load().bpx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_layout(opts: Options, bvecs, bvals, sample: int = 2048):
    """(tpv, mpl, {layout: seconds per voxel}) from bpx_autotune_layout."""
    _torch()
    L = load()
    lays = mcmc_layouts()
    t = (C.c_float * len(lays))()
    tpv, mpl = C.c_int32(), C.c_int32()
    _check(L.bpx_autotune_layout(C.byref(opts), int(bvals.shape[0]), _ptr(bvecs), _ptr(bvals), sample, C.byref(tpv),
                                 C.byref(mpl), t, None), "bpx_autotune_layout")
    return tpv.value, mpl.value, {lays[i]: t[i] for i in range(len(lays)) if t[i] >= 0}


def postproc(opts: Options, outputs: dict, thr: float = 0.05) -> dict:
    """bedpostx_postproc arithmetic on finished device outputs: mean_th, mean_ph, dispersion
    [K][n], dyads_thr, dyads_modf [K][3][n] (fibres 2..K), mean_fsum [n] (device tensors)."""
    torch = _torch()
    K, n = opts.nfibres, int(outputs["mean_d"].shape[0])
    r = dict(mean_th=torch.zeros((K, n), device="cuda"), mean_ph=torch.zeros((K, n), device="cuda"),
             dispersion=torch.zeros((K, n), device="cuda"), dyads_thr=torch.zeros((K, 3, n), device="cuda"),
             dyads_modf=torch.zeros((K, 3, n), device="cuda"), mean_fsum=torch.zeros(n, device="cuda"))
    o = Outputs()
    for k in OUT_KEYS:
        setattr(o, k, outputs[k].data_ptr())
    pp = PostProc()
    for k in r:
        setattr(pp, k, r[k].data_ptr())
    _check(load().bpx_postproc_dev(C.byref(opts), n, C.byref(o), thr, C.byref(pp), _stream(torch)),
           "bpx_postproc_dev")
    return r
