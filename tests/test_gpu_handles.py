"""Workspace handles: pipeline calls bound to different handles run concurrently from different host
threads on different streams and give the same outputs as the same calls run one after another.

Each thread's volume has its own size, so every thread grows its handle's workspace while the other
threads' kernels are running: with the shared per-device workspace that grow would free a buffer
another thread's later stages still use.
"""
import threading

import numpy as np
import pytest

from fdt_b200 import synth
from fdt_b200.abi import Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_handles_run_concurrently_with_sequential_results(torch):
    from fdt_b200 import lib

    lib.load()
    o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=40, njumps=80, sampleevery=8)
    prot = synth.three_shell(18, 90)
    sizes = [300, 700, 1100, 500]
    vols = [synth.make_volume(n, prot, 3, True, 25.0, seed=50 + i)[0] for i, n in enumerate(sizes)]
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)

    def run(i, out):
        d = lib.to_device(vols[i])
        return lib.xfibres_dev(o, d, bv, bl, voxel_offset=i * 10_000, out=out)

    want = []
    for i in range(len(sizes)):
        t = run(i, lib.alloc_outputs(o, sizes[i]))
        torch.cuda.synchronize()
        want.append({k: v.cpu().numpy() for k, v in t.items()})

    handles = [lib.Handle() for _ in sizes]
    outs = [lib.alloc_outputs(o, n) for n in sizes]
    errors = []
    barrier = threading.Barrier(len(sizes))

    def worker(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s), handles[i]:
                barrier.wait()
                for _ in range(2):  # the second call reuses the grown workspace
                    run(i, outs[i])
            s.synchronize()
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append((i, repr(e)))

    th = [threading.Thread(target=worker, args=(i,)) for i in range(len(sizes))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    for h in handles:
        h.close()
    assert not errors, errors
    for i in range(len(sizes)):
        got = {k: v.cpu().numpy() for k, v in outs[i][0].items()}
        for k in want[i]:
            assert np.array_equal(got[k], want[i][k]), (i, k)


def test_unbound_calls_use_the_shared_workspace_after_a_handle_is_unbound(torch):
    from fdt_b200 import lib

    L = lib.load()
    h = lib.Handle()
    with h:
        pass  # bind + unbind
    o = Options.make(model=1, nfibres=2, nburn=10, njumps=20, sampleevery=5)
    prot = synth.single_shell_64()
    y, _ = synth.make_volume(64, prot, 2, False, 20.0, seed=3)
    t = lib.xfibres_dev(o, lib.to_device(y), lib.to_device(prot.bvecs), lib.to_device(prot.bvals))
    torch.cuda.synchronize()
    assert np.all(np.isfinite(t["mean_f"].cpu().numpy()))
    h.close()
    assert L.bpx_handle_destroy(None) == 0


def test_released_shared_workspace_is_made_again_with_the_same_outputs(torch):
    """bpx_release_workspace frees the device's shared workspaces; the next call allocates them
    again and gives the same outputs bit for bit."""
    from fdt_b200 import lib

    L = lib.load()
    o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=20, njumps=40, sampleevery=8)
    prot = synth.three_shell(18, 90)
    y, _ = synth.make_volume(257, prot, 3, True, 25.0, seed=91)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    first = lib.xfibres_dev(o, lib.to_device(y), bv, bl)
    torch.cuda.synchronize()
    assert L.bpx_release_workspace() == 0, L.bpx_last_error()
    assert L.bpx_release_workspace() == 0  # nothing left to free: still fine
    again = lib.xfibres_dev(o, lib.to_device(y), bv, bl)
    torch.cuda.synchronize()
    for k in first:
        assert torch.equal(first[k], again[k]), k


def test_measure_pipes_reports_plausible_issue_rates(torch):
    """bpx_measure_pipes (the roofline denominators of the bench): MUFU ex2 and FP32 FMA rates are
    positive, the FMA rate well above the MUFU rate, and both below 2x the B200's nominal figures
    (148 SMs x 16 MUFU lanes and 128 FMA lanes per clock at up to 1.965 GHz)."""
    import ctypes as C

    from fdt_b200 import lib

    L = lib.load()
    m, f = C.c_double(), C.c_double()
    assert L.bpx_measure_pipes(C.byref(m), C.byref(f)) == 0, L.bpx_last_error()
    nominal_mufu, nominal_fma = 148 * 16 * 1.965e9, 148 * 128 * 1.965e9
    assert 0.2 * nominal_mufu < m.value < 2 * nominal_mufu, m.value
    assert 0.2 * nominal_fma < f.value < 2 * nominal_fma, f.value
    assert f.value > 4 * m.value
