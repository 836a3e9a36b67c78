"""The reference's C++ forward solver (growth_solver.h), built from the
reference tree by oracle/build_ref.py, pinned against the reference's own
recorded results: the numpy <-> C++ parity scene (test_growth.cpp:333-357,
recorded max|dF| 2.33e-5 through a 6-digit CSV) and the T2 free-swelling gate
(test_growth.cpp:95-115, mean det F within 8% of g^3)."""
import numpy as np
import pytest

from oracle import growth_ref as G

pytestmark = pytest.mark.skipif(not G.available(), reason="oracle/_ref not built (no reference tree)")

HERE = __import__("os").path.dirname(__import__("os").path.abspath(__file__))


def _pmass(density, sp):
    d, s = np.float32(density), np.float32(sp)
    return np.float32(np.float32(np.float32(d * s) * s) * s)


def test_cpp_parity_scene_against_numpy_fixture():
    g = np.load(f"{HERE}/golden/gates.npz")
    pts = G.parity_cube()
    assert np.abs(pts - g["parity27_pts"]).max() < 1e-7
    s = G.RefSolver(12, 0.05, 1e4, 0.3, 0.05)
    s.add(pts, _pmass(1000.0, 0.03), 1000.0)
    s.set_growth(1.05)
    s.step(1e-3, 30)
    x, _, F, _ = s.get()
    dF = np.abs(F - g["parity27_F"]).max()
    # the reference records 2.33e-5 for this comparison
    assert 1e-6 < dF < 3e-5, dF
    assert np.abs(x - g["parity27_x"]).max() < 2e-6


def test_cpp_free_swelling_gate():
    s = G.RefSolver(24, 0.05, 1e4, 0.3, 0.05)
    pts = G.parity_cube(sp=0.025, lo=0.5, hi=0.7)
    assert pts.shape == (729, 3)
    s.add(pts, _pmass(1000.0, 0.025), 1000.0)
    per = np.float32(1.5) ** np.float32(0.1)
    g = np.float32(1.0)
    for _ in range(10):
        g = np.float32(g * per)
        s.set_growth(g)
        s.step(1e-3, 250)
    _, _, F, _ = s.get()
    det = np.linalg.det(F.astype(np.float64)).mean()
    assert abs(det - 3.375) < 0.08 * 3.375, det
