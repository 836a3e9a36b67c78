"""Sharding of independent growth scenes over ranks (one process per GPU).

Scenes are independent units: a rank advances its own subset and no data-path
collective is needed.  ``lpt_assign`` balances a fixed set of scenes by
longest-processing-time bin packing on particles x steps; after the run,
``gather_scenes`` brings every scene's results (loss, d loss / d theta) to
every rank in scene order, and ``fixed_order_sum`` reduces a parameter shared
by all scenes in that order, so the result is bitwise that of one process
running the whole batch.  ``max_over_ranks`` is the device-time reduction used
for timing (the slowest rank sets the time).
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


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


def gather_scenes(local, mine: Sequence[int], n_scenes: int, device=None) -> np.ndarray:
    """Per-scene results of all ranks, in scene order, on every rank.

    ``local`` is this rank's (len(mine), m) array for its scenes ``mine``
    (global indices).  Every rank contributes a (n_scenes, m) float64 array
    holding its own rows and zeros elsewhere, summed over ranks: each entry has
    exactly one contribution, so the gathered values are the ranks' values
    unchanged, whatever the reduction order.  Identity without a process group.
    """
    import torch
    import torch.distributed as dist
    local = np.asarray(local, dtype=np.float64).reshape(len(mine), -1)
    full = np.zeros((n_scenes, local.shape[1]), dtype=np.float64)
    full[list(mine)] = local
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return full
    t = torch.from_numpy(full).to(device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def fixed_order_sum(values: Sequence[float]) -> float:
    """Sum in index order, left to right in float64: the reduction of a
    parameter shared by all scenes (e.g. one growth amplitude), independent
    of how the scenes were spread over ranks."""
    acc = 0.0
    for v in values:
        acc += float(v)
    return acc
