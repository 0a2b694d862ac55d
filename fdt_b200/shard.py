"""Multi-GPU sharding of a volume: one process per GPU, each running its own voxel range.

Voxels are independent in the per-voxel path (no coupling between voxels in the GPU path of the
reference either), so a volume is split into contiguous voxel ranges, one per rank, with no
collective on the data path.  The Philox streams are keyed by the global voxel index
(`voxel_offset` + local index), so a sharded run reproduces the single-GPU run bit for bit.  The
outputs are gathered to rank 0 at the end (the reference's equivalent is the file-based
split_parts_gpu / merge_parts_gpu pair, CUDA/split_parts_gpu.cc:123-147, merge_parts_gpu.cc:17-82).

For mixed batches the ranges are cost-weighted: voxel v costs c_v (e.g. the MCMC work of its
model, fibre count and measurement count, J*(T*c_sig + L*M*c_lik)), and rank r gets the voxels
whose cumulative cost falls in [r/W, (r+1)/W) of the total.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def partition(nvox: int, world: int, cost: Sequence[float] | np.ndarray | None = None) -> list[tuple[int, int]]:
    """Contiguous [start, end) voxel ranges, one per rank, of about equal total cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if nvox <= 0:
        return [(0, 0)] * world
    if cost is None:
        bounds = [(r * nvox) // world for r in range(world + 1)]
    else:
        c = np.asarray(cost, np.float64)
        if c.shape != (nvox,) or not np.all(np.isfinite(c)) or np.any(c < 0):
            raise ValueError("cost must hold one finite non-negative value per voxel")
        cum = np.concatenate([[0.0], np.cumsum(c)])
        total = cum[-1]
        if total <= 0:
            return partition(nvox, world)
        # first voxel whose preceding cumulative cost reaches r/W of the total
        bounds = [0] + [int(np.searchsorted(cum, total * r / world, side="left")) for r in range(1, world)] + [nvox]
        bounds = [min(max(b, 0), nvox) for b in bounds]
        for r in range(1, world + 1):
            bounds[r] = max(bounds[r], bounds[r - 1])
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def run_sharded(nvox: int, rank: int, world: int, run_range: Callable[[int, int], dict], dist=None,
                cost=None) -> dict | None:
    """Runs `run_range(start, end)` for this rank's range and gathers the per-voxel outputs to
    rank 0.  `run_range` returns a dict of tensors (CPU or CUDA) whose LAST axis is the voxel axis
    (the layout of every bpx output array); the range's first voxel must key its chains
    (bpx_volume.voxel_offset).  The gather goes through the process group's backend: CUDA tensors
    for NCCL, CPU tensors for gloo.  Returns the assembled dict (CPU tensors) on rank 0, None
    elsewhere.  With world == 1 (or dist None) no collective is made."""
    import torch

    ranges = partition(nvox, world, cost)
    start, end = ranges[rank]
    mine = run_range(start, end)
    if world == 1 or dist is None:
        return {k: v.cpu() for k, v in mine.items()}
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    keys = sorted(mine)
    width = max(e - s for s, e in ranges)
    gathered = {}
    for k in keys:
        t = mine[k].contiguous().to(dev)
        # pad to the largest range so every rank sends the same shape
        pad = torch.zeros(t.shape[:-1] + (width,), dtype=t.dtype, device=dev)
        pad[..., : t.shape[-1]] = t
        parts = [torch.zeros_like(pad) for _ in range(world)] if rank == 0 else None
        dist.gather(pad, gather_list=parts, dst=0)
        if rank == 0:
            gathered[k] = torch.cat([parts[r][..., : ranges[r][1] - ranges[r][0]] for r in range(world)], dim=-1).cpu()
    return gathered if rank == 0 else None
