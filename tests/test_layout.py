"""Cell-order particle layout (host side, no GPU): the binning key equals the
oracle's, the orders are stable permutations that sort the keys, and a batch
whose scenes are already in cell order keeps its layout."""
import numpy as np
import torch

from morphompm_b200 import layout
from oracle import mpm_oracle as O


def _scene_points(rng, n, N):
    x = rng.uniform(-0.05, 1.05, size=(n, 3))      # some stencils leave the grid
    x[: n // 4] = (rng.integers(0, N, size=(n // 4, 3)) + 0.5) / N     # exact binning ties
    return x


def test_keys_match_oracle_binning():
    rng = np.random.default_rng(0)
    for N in (8, 13, 32):
        x = _scene_points(rng, 4000, N)
        sc = O.Scene(shape=(N, N, N), dx=1.0 / N, dt=1e-3, damping=0.05, pmass=1.0, vol0=1.0)
        assert np.array_equal(layout.cell_keys_host(x, 1.0 / N, (N, N, N)), O.cell_keys(x, sc))


def test_orders_are_stable_sorting_permutations():
    rng = np.random.default_rng(1)
    x = _scene_points(rng, 5000, 16)
    k = layout.cell_keys_host(x, 1 / 16, (16, 16, 16))
    o = layout.cell_order_host(x, 1 / 16, (16, 16, 16))
    assert np.array_equal(np.sort(o), np.arange(len(x)))
    ks = k[o]
    assert np.all(np.diff(ks) >= 0)
    ties = np.diff(ks) == 0
    assert np.all(np.diff(o)[ties] > 0)           # stable: input order within a cell
    od = layout.cell_order_device(torch.as_tensor(x), 1 / 16, (16, 16, 16))
    assert np.array_equal(od.numpy(), o)
    assert layout.cell_order_device(torch.as_tensor(x[o]), 1 / 16, (16, 16, 16)) is None


def test_batch_order():
    from morphompm_b200 import scenes
    sc = scenes.config4(seed=5, n_scenes=4, n_lo=300, n_hi=2000)
    off = np.concatenate([[0], np.cumsum([s["x"].shape[0] for s in sc])])
    assert layout.batch_order(sc, off) is None      # the generator emits cell order
    rng = np.random.default_rng(2)
    sh = [dict(s, x=s["x"][rng.permutation(s["x"].shape[0])]) for s in sc]
    order = layout.batch_order(sh, off)
    assert np.array_equal(np.sort(order), np.arange(off[-1]))
    for s, p0, p1 in zip(sh, off[:-1], off[1:]):
        seg = order[p0:p1]
        assert seg.min() == p0 and seg.max() == p1 - 1          # stays inside its scene
        k = layout.cell_keys_host(s["x"], s["dx"], s["shape"])[seg - p0]
        assert np.all(np.diff(k) >= 0)
