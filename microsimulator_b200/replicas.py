"""One process per GPU: how work is split across ranks and how their timings
combine.  There is no data-path collective: a single colony does not shard
(each rank steps its own replica), and the colonies of a sweep are
independent (each rank steps its share).  The only collective is the
reduction of the timings, the maximum over ranks."""

from __future__ import annotations

import numpy as np


def shard(sizes, rank: int, world_size: int) -> np.ndarray:
    """The colonies (indices into `sizes`) rank `rank` of `world_size` steps:
    largest first, each to the rank with the fewest cells so far (ties to the
    lower rank), so that ranks carry near-equal cells.  Every colony goes to
    exactly one rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must lie in [0, world_size)")
    load = np.zeros(world_size, dtype=np.int64)
    owner = np.empty(len(sizes), dtype=np.int64)
    for i in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += sizes[i]
    return np.flatnonzero(owner == rank)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest of every rank's `value` (this rank's alone without a
    process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of every rank's `value` (a count of the units processed)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
