"""Particle layout in HBM: cell order.

Every per-particle kernel visits particles in the order of the step's cell
sort and reads their state through the sort permutation.  When the particles
of one warp (32 consecutive sorted slots) also sit next to each other in
memory, each of its loads touches about four 32-byte sectors; in a random
input order it touches 32.  So the batch engine stores particles in the cell
order of their initial positions: the stable order of the binning key
(stencil base + 2, flattened over the padded (N+2)^3 cell grid, z fastest),
the same key the device sort uses.  The order changes only the memory layout:
per-scene losses and gradients are sums over the same particles.

Measured on the 256-scene batch (4.49M particles, 200 steps fwd+adj, FP32):
a random order within each scene runs at 0.91e9 particle-steps/s, cell order
at 1.72e9.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch


def cell_keys_host(x: np.ndarray, dx: float, shape: Sequence[int]) -> np.ndarray:
    """Binning key of each particle (host).  Particles whose stencil misses
    the grid get the largest key and go last."""
    nx, ny, nz = (int(s) for s in shape)
    c = np.floor(np.asarray(x, dtype=np.float64) * (1.0 / dx) - 0.5).astype(np.int64) + 2
    dims = np.array([nx + 2, ny + 2, nz + 2])
    inside = np.all((c >= 0) & (c < dims), axis=1)
    key = (c[:, 0] * dims[1] + c[:, 1]) * dims[2] + c[:, 2]
    return np.where(inside, key, int(np.prod(dims)))


def cell_order_host(x: np.ndarray, dx: float, shape: Sequence[int]) -> np.ndarray:
    """Stable permutation that puts particles in cell order."""
    return np.argsort(cell_keys_host(x, dx, shape), kind="stable")


def cell_order_device(x: torch.Tensor, dx: float, shape: Sequence[int]) -> Optional[torch.Tensor]:
    """cell_order_host for an (n, 3) device tensor; None when the particles
    are already in cell order."""
    nx, ny, nz = (int(s) for s in shape)
    c = torch.floor(x.double() * (1.0 / dx) - 0.5).long() + 2
    dims = torch.tensor([nx + 2, ny + 2, nz + 2], device=x.device)
    inside = ((c >= 0) & (c < dims)).all(dim=1)
    key = (c[:, 0] * (ny + 2) + c[:, 1]) * (nz + 2) + c[:, 2]
    key = torch.where(inside, key, torch.full_like(key, (nx + 2) * (ny + 2) * (nz + 2)))
    if x.shape[0] < 2 or bool((key[1:] >= key[:-1]).all()):
        return None
    return torch.argsort(key, stable=True)


def batch_order(scenes, offsets: Sequence[int], scene_perm: Optional[Sequence[int]] = None,
                cell_order: bool = True) -> Optional[np.ndarray]:
    """Batch-wide permutation (slot -> input particle index).  The input holds
    the scenes in their given order, scene s at offsets[s]; the slots hold
    them in the order scene_perm (default: the given order), and each scene's
    particles in cell order within its range (cell_order).  None when that is
    the identity."""
    n = int(offsets[-1])
    perm = list(range(len(scenes))) if scene_perm is None else [int(i) for i in scene_perm]
    order = np.empty(n, dtype=np.int64)
    changed = perm != list(range(len(scenes)))
    q = 0
    for s in perm:
        sc, p0 = scenes[s], int(offsets[s])
        k = sc["x"].shape[0]
        o = np.arange(k)
        if cell_order and k >= 2:
            o = cell_order_host(sc["x"], float(sc["dx"]), sc["shape"])
            changed = changed or bool(np.any(o != np.arange(k)))
        order[q:q + k] = p0 + o
        q += k
    return order if changed else None
