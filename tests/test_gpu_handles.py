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
