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


def _run(torch, lib, entry, opts, y, prot):
    d = lib.to_device(y)  # a fresh copy: the Rician clean-up works in place
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    t, o = lib.alloc_outputs(opts, y.shape[0])
    vol = lib.make_volume(d, bv, bl)
    rc = entry(C.byref(opts), C.byref(vol), C.byref(o), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, {k: v.cpu().numpy() for k, v in t.items()}


def test_noalloc_entry_matches_allocating_entry_twice(torch):
    from fdt_b200 import lib

    L = lib.load()
    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=60, njumps=100, sampleevery=10)
    prot = synth.three_shell(18, 90)
    y, _ = synth.make_volume(700, prot, 3, True, 25.0, seed=71)
    rc, want = _run(torch, lib, L.bpx_xfibres_dev, opts, y, prot)
    assert rc == BPX_OK, L.bpx_last_error()
    for call in range(2):
        rc, got = _run(torch, lib, L.bpx_xfibres_noalloc_dev, opts, y, prot)
        assert rc == BPX_OK, L.bpx_last_error()
        for k in want:
            assert np.allclose(got[k], want[k], rtol=1e-6, atol=0), (call, k)


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
