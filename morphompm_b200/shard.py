"""Sharding of independent growth scenes over ranks (one process per GPU).

Scenes are independent units: a rank advances its own subset and no data-path
collective is needed.  ``lpt_assign`` balances a fixed set of scenes by
longest-processing-time bin packing on particles x steps; ``max_over_ranks``
is the device-time reduction used for timing (the slowest rank sets the time).
"""
from __future__ import annotations

from typing import List, Sequence


def lpt_assign(costs: Sequence[float], world: int) -> List[List[int]]:
    """Scene indices per rank, largest cost first onto the least loaded rank
    (ties to the lowest rank), each rank's list sorted ascending."""
    loads = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += costs[i]
    return [sorted(x) for x in out]


def sum_over_ranks(value: float, device=None) -> float:
    """Sum of a per-rank float over the default process group (identity when
    torch.distributed is not initialised): e.g. the particles all ranks
    processed, when every rank runs a batch of its own."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over the default process group (identity when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
