"""Multi-GPU sharding host logic (fdt_b200/shard.py) on CPU with world-size-2 gloo ranks.

Each rank processes a contiguous voxel range with the RNG keyed by the global voxel index, so a
sharded run must reproduce the single-process run exactly.  Without a GPU the per-rank pipeline is
the CPU oracle's (clean-up, LM fits, chains keyed by voxel_offset, finishing), the same stages and
output layouts as bpx_xfibres_dev; a cheap deterministic stand-in checks the gather's padding over
uneven ranges.  tests/test_gpu_shard.py runs the library itself across ranks on a GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch

from fdt_b200.shard import partition, run_sharded

K, NS = 3, 5


def fake_pipeline(start, end):
    """Outputs of voxels [start, end) as the pipeline lays them out (voxel axis last)."""
    v = torch.arange(start, end, dtype=torch.float64)
    f = torch.stack([torch.stack([torch.sin(v * (k + 1) + s) for s in range(NS)]) for k in range(K)]).float()
    dy = torch.stack([torch.stack([torch.cos(v + 3 * k + c) for c in range(3)]) for k in range(K)]).float()
    return {"f": f, "dyads": dy, "mean_d": (v * 1e-6).float(), "status": (v.long() % 3).int()}


def test_partition_covers_and_balances():
    for n, w in [(10, 3), (1, 4), (0, 2), (131072, 8)]:
        r = partition(n, w)
        assert len(r) == w and r[0][0] == 0 and r[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [e - s for s, e in r]
        assert max(sizes) - min(sizes) <= 1
    rng = np.random.default_rng(0)
    cost = rng.choice([1.0, 2.5, 6.0], size=5000)  # e.g. models/fibre counts mixed
    r = partition(5000, 4, cost)
    loads = [cost[s:e].sum() for s, e in r]
    assert r[0][0] == 0 and r[-1][1] == 5000 and all(a[1] == b[0] for a, b in zip(r, r[1:]))
    assert max(loads) - min(loads) <= 2 * cost.max()
    with pytest.raises(ValueError):
        partition(3, 2, [1.0, -1.0, 2.0])


def oracle_pipeline(start, end):
    """The whole per-voxel path on the CPU oracle for voxels [start, end) of the shared test volume."""
    from oracle import oracle as O

    o, y, prot = _oracle_case()
    yy = O.prepare_data(y[start:end])
    p, tau, _ = O.fit(o, yy, prot.bvecs, prot.bvals, nthreads=1)
    rec = O.mcmc(o, yy, prot.bvecs, prot.bvals, p, tau, voxel_offset=start, nthreads=1)
    fin = O.finish(o, rec)
    return {k: torch.from_numpy(np.ascontiguousarray(fin[k])) for k in ("f", "th", "dyads", "mean_d", "mean_tau")}


def _oracle_case():
    from fdt_b200 import synth
    from fdt_b200.abi import Options

    o = Options.make(model=2, nfibres=2, rician=1, f0=1, nburn=20, njumps=40, sampleevery=10)
    prot = synth.three_shell(9, 90)
    y, _ = synth.make_volume(37, prot, 2, True, 25.0, seed=21)
    return o, y, prot


def _worker(rank, world, port, q, which):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        if which == "oracle":
            out = run_sharded(37, rank, world, oracle_pipeline, dist=dist)
        else:
            out = run_sharded(1001, rank, world, fake_pipeline, dist=dist)
        if rank == 0:
            q.put({k: v.numpy() for k, v in out.items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run_two_ranks(which):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, which)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return got


def test_two_rank_gloo_gather_over_uneven_ranges():
    got = _run_two_ranks("fake")
    want = fake_pipeline(0, 1001)
    for k, v in want.items():
        assert got[k].shape == tuple(v.shape), k
        assert np.array_equal(got[k], v.numpy()), k


def test_two_rank_gloo_oracle_pipeline_equals_single_run():
    got = _run_two_ranks("oracle")
    want = oracle_pipeline(0, 37)
    for k, v in want.items():
        assert got[k].shape == tuple(v.shape), k
        assert np.array_equal(got[k], v.numpy()), k
