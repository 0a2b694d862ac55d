"""The allocation-free entry point (bpx_xfibres_noalloc_dev) against the allocating one.

Callers that cannot allocate device memory once running -- frameworks that reserve the GPU's memory
for their own pool, services that cannot afford cudaMalloc's implicit synchronisation -- use
bpx_xfibres_noalloc_dev, whose intermediates live in a fixed 40 MiB array inside the library.  It
runs the same kernels as bpx_xfibres_dev, so on the same inputs both must give the same outputs
(compared exactly, with the FP32 tolerance of the other parity tests as the bound), on two calls
in a row (the second call reuses the array the first one left behind).  The file name makes
pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from fdt_b200 import synth
from fdt_b200.abi import BPX_ERR_UNSUPPORTED, BPX_OK, Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(torch, lib, entry, opts, y, prot, with_status=True):
    d = lib.to_device(y)  # a fresh copy: the Rician clean-up works in place
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    t, o = lib.alloc_outputs(opts, y.shape[0])
    if not with_status:  # the entry then keeps the per-voxel status in its own array
        o.status = None
        del t["status"]
    vol = lib.make_volume(d, bv, bl)
    rc = entry(C.byref(opts), C.byref(vol), C.byref(o), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, {k: v.cpu().numpy() for k, v in t.items()}


@pytest.mark.parametrize("with_status", [True, False])
def test_noalloc_entry_matches_allocating_entry_twice(torch, with_status):
    from fdt_b200 import lib

    L = lib.load()
    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=60, njumps=100, sampleevery=10)
    prot = synth.three_shell(18, 90)
    y, _ = synth.make_volume(700, prot, 3, True, 25.0, seed=71)
    # the warm-up call a host makes at start-up: no voxels, only the array's address is resolved
    t0, o0 = lib.alloc_outputs(opts, 1)
    vol0 = lib.make_volume(lib.to_device(y[:1]), lib.to_device(prot.bvecs), lib.to_device(prot.bvals))
    vol0.nvox = 0
    assert L.bpx_xfibres_noalloc_dev(C.byref(opts), C.byref(vol0), C.byref(o0), None) == BPX_OK, L.bpx_last_error()
    rc, want = _run(torch, lib, L.bpx_xfibres_dev, opts, y, prot, with_status)
    assert rc == BPX_OK, L.bpx_last_error()
    for call in range(2):
        rc, got = _run(torch, lib, L.bpx_xfibres_noalloc_dev, opts, y, prot, with_status)
        assert rc == BPX_OK, L.bpx_last_error()
        for k in want:
            assert np.allclose(got[k], want[k], rtol=1e-6, atol=0), (call, k)


@pytest.mark.parametrize("bad", ["model", "njumps_below_sampleevery", "negative_njumps", "ndir"])
def test_noalloc_entry_rejects_bad_calls_before_touching_data(torch, bad):
    from fdt_b200 import lib

    L = lib.load()
    kw = dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=20, njumps=40, sampleevery=10)
    if bad == "model":
        kw["model"] = 4
    elif bad == "njumps_below_sampleevery":
        kw["njumps"] = 5
    elif bad == "negative_njumps":
        kw["njumps"] = -10
    opts = Options.make(**kw)
    prot = synth.three_shell(18, 90)
    y, _ = synth.make_volume(64, prot, 3, True, 25.0, seed=5)
    y[:, :4] = -1.0  # non-positive samples the Rician clean-up would replace in place
    d = lib.to_device(y)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    t, o = lib.alloc_outputs(opts if bad != "negative_njumps" else Options.make(model=2, nfibres=3), 64)
    vol = lib.make_volume(d, bv, bl)
    if bad == "ndir":
        vol.ndir = 5  # below the smallest protocol the fits accept
    rc = L.bpx_xfibres_noalloc_dev(C.byref(opts), C.byref(vol), C.byref(o), None)
    torch.cuda.synchronize()
    assert rc != BPX_OK
    assert np.array_equal(d.cpu().numpy(), y), "a rejected call modified the caller's data"


def test_noalloc_entry_rejects_volumes_beyond_its_array(torch):
    from fdt_b200 import lib

    L = lib.load()
    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1)  # 50 samples: ~3 KB per voxel
    prot = synth.three_shell(18, 90)
    n = 20000
    d = torch.zeros((n, prot.ndir), device="cuda")
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    t, o = lib.alloc_outputs(opts, 1)  # never written: the call is rejected before any launch
    vol = lib.make_volume(d, bv, bl)
    rc = L.bpx_xfibres_noalloc_dev(C.byref(opts), C.byref(vol), C.byref(o), None)
    assert rc == BPX_ERR_UNSUPPORTED
    msg = L.bpx_last_error().decode()
    assert "at most" in msg and str(n) in msg
