"""The sharded path with the library itself: two ranks (processes) each run bpx_xfibres_dev on their
voxel range, keyed by the range's first voxel, and rank 0 gathers the outputs (fdt_b200/shard.py);
the result equals one process running the whole volume, bit for bit.

Only one GPU is available here, so both ranks use it and gather over gloo; their kernels never wait
on each other (the path has no collective in any kernel), so sharing the device is safe.  With one
GPU per rank the same code gathers over NCCL (bench.py's weak-scaling runs).
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    from fdt_b200 import synth
    from fdt_b200.abi import Options

    o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=60, njumps=100, sampleevery=10)
    prot = synth.three_shell(18, 90)
    y, _ = synth.make_volume(1537, prot, 3, True, 25.0, seed=33)
    return o, y, prot


def library_range(start, end):
    import torch

    from fdt_b200 import lib

    o, y, prot = _case()
    t = lib.xfibres_dev(o, lib.to_device(y[start:end]), lib.to_device(prot.bvecs), lib.to_device(prot.bvals),
                        voxel_offset=start)
    torch.cuda.synchronize()
    return {k: t[k] for k in ("th", "ph", "f", "mean_d", "mean_S0", "mean_f", "dyads", "status")}


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from fdt_b200.shard import run_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = run_sharded(1537, rank, world, library_range, dist=dist)
        if rank == 0:
            q.put({k: v.numpy() for k, v in out.items()})
    finally:
        dist.destroy_process_group()


def test_two_ranks_of_the_library_equal_one_run():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = {k: v.cpu().numpy() for k, v in library_range(0, 1537).items()}
    for k, v in want.items():
        assert got[k].shape == v.shape, k
        assert np.array_equal(got[k], v), k
