"""Multi-GPU sharding host logic (fdt_b200/shard.py) on CPU with world-size-2 gloo ranks.

Each rank processes a contiguous voxel range with the RNG keyed by the global voxel index, so a
sharded run must reproduce the single-process run exactly; the stand-in for the GPU pipeline here
is a deterministic function of the global voxel index with the output layouts of bpx_outputs.
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


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
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


def test_two_rank_gloo_run_equals_single_run():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = fake_pipeline(0, 1001)
    for k, v in want.items():
        assert got[k].shape == tuple(v.shape), k
        assert np.array_equal(got[k], v.numpy()), k
