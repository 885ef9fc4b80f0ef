"""Multi-GPU host logic: one process per GPU, independent meshes sharded
across ranks with no data-path collective (weak scaling), device times
reduced as the maximum over ranks.

The reference distributes one octree over MPI ranks along the space-filling
curve (par::partitionW, include/par/parUtils.txx:1011); for independent
meshes the equivalent split is by contiguous ranges of meshes balanced by
element count.
"""
from __future__ import annotations

import numpy as np


def shard_meshes(weights, rank: int, world: int):
    """Contiguous range [lo, hi) of meshes for `rank`, balancing the summed
    weights (element counts) like a weighted SFC partition."""
    w = np.asarray(weights, np.float64)
    if world <= 1 or len(w) == 0:
        return 0, len(w)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")))
    cuts.append(len(w))
    cuts = np.maximum.accumulate(np.minimum(cuts, len(w)))
    return int(cuts[rank]), int(cuts[rank + 1])


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. a device time) over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
