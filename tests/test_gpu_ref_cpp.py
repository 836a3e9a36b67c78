"""The FP32 device path against the reference's own C++ FP32 forward solver
(growth_solver.h, built into oracle/_ref), run with the C++ solver's
semantics: Hencky, mass threshold 1e-9, per-step damping, no walls, advected
positions, explicit Fg = g I.  Scenes: the numpy <-> C++ parity cube
(test_growth.cpp:333-357) and the T2 free-swelling blob with stepwise growth
(test_growth.cpp:95-115)."""
import numpy as np
import pytest

from oracle import growth_ref as G

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not G.available(), reason="oracle/_ref not built (no reference tree)")]
torch = pytest.importorskip("torch")


def _pmass(density, sp):
    d, s = np.float32(density), np.float32(sp)
    return np.float32(np.float32(np.float32(d * s) * s) * s)


def _device_run(pts, N, dx, dt, damping, pm, vol0, E, nu, growth):
    """growth: list of (g, steps) blocks; returns x, F (float64 numpy)."""
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import Plan, SceneSpec, slab_particles, SLAB_ROWS, ROW_X, ROW_F
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    n = pts.shape[0]
    spec = SceneSpec(shape=(N, N, N), n=n, model=L.MODEL_HENCKY, dx=dx, dt=dt, damping=damping,
                     pmass=float(pm), vol0=float(vol0), mu=mu, lam=lam, mass_eps=1e-9, wall=0, growth_mode=0)
    plan = Plan([spec], dtype=torch.float32, device="cuda")
    a = torch.zeros(SLAB_ROWS, n, dtype=torch.float32, device="cuda")
    a[ROW_X:ROW_X + 3] = torch.as_tensor(pts.T.copy(), device="cuda")
    for i in range(3):
        a[ROW_F + 4 * i] = 1.0
    b = torch.empty_like(a)
    Fg = torch.zeros(9, n, dtype=torch.float32, device="cuda")
    t = 0
    for g, steps in growth:
        for i in range(3):
            Fg[4 * i] = float(g)
        for _ in range(steps):
            plan.step_fwd(slab_particles(a, Fg), slab_particles(b, Fg), True, t, None)
            a, b = b, a
            t += 1
    torch.cuda.synchronize()
    assert plan.status() == 0
    s = a.double().cpu().numpy()
    return s[ROW_X:ROW_X + 3].T, s[ROW_F:ROW_F + 9].T.reshape(n, 3, 3)


def test_parity_cube_fp32_against_cpp():
    pts = G.parity_cube()
    pm = _pmass(1000.0, 0.03)
    vol0 = np.float32(pm / np.float32(1000.0))
    ref = G.RefSolver(12, 0.05, 1e4, 0.3, 0.05)
    ref.add(pts, pm, 1000.0)
    ref.set_growth(1.05)
    ref.step(1e-3, 30)
    xr, _, Fr, _ = ref.get()
    x, F = _device_run(pts, 12, 0.05, 1e-3, 0.05, pm, vol0, 1e4, 0.3, [(1.05, 30)])
    # both FP32; the C++ Hencky stress goes through an SVD clamped at 1e-6
    assert np.abs(F - Fr).max() < 3e-5, np.abs(F - Fr).max()
    assert np.abs(x - xr).max() < 2e-6


def test_free_swelling_fp32_against_cpp():
    pts = G.parity_cube(sp=0.025, lo=0.5, hi=0.7)
    pm = _pmass(1000.0, 0.025)
    vol0 = np.float32(pm / np.float32(1000.0))
    per = np.float32(1.5) ** np.float32(0.1)
    blocks, g = [], np.float32(1.0)
    for _ in range(10):
        g = np.float32(g * per)
        blocks.append((float(g), 250))
    ref = G.RefSolver(24, 0.05, 1e4, 0.3, 0.05)
    ref.add(pts, pm, 1000.0)
    for gb, steps in blocks:
        ref.set_growth(gb)
        ref.step(1e-3, steps)
    _, _, Fr, _ = ref.get()
    _, F = _device_run(pts, 24, 0.05, 1e-3, 0.05, pm, vol0, 1e4, 0.3, blocks)
    det, det_r = np.linalg.det(F).mean(), np.linalg.det(Fr.astype(np.float64)).mean()
    # the reference's gate (test_growth.cpp:111), and agreement with its solver
    assert abs(det - 3.375) < 0.08 * 3.375, det
    assert abs(det - det_r) < 1e-4 * det_r, (det, det_r)
    assert np.abs(F - Fr).max() < 1e-3, np.abs(F - Fr).max()
