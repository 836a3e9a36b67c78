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


def _two_density_blob():
    pts = G.blob(0.6, 0.10, 0.025)
    density = np.where(pts[:, 0] < np.float32(0.6), np.float32(1000.0), np.float32(400.0)).astype(np.float32)
    sp = np.float32(0.025)
    mass = np.float32(density * sp * sp * sp)
    vol0 = np.float32(mass / density)
    return pts, mass, vol0, density


def _plan(n, dtype, pm, vol0, model=None):
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import Plan, SceneSpec
    spec = SceneSpec(shape=(24, 24, 24), n=n, model=L.MODEL_HENCKY if model is None else model, dx=0.05,
                     dt=1e-3, damping=0.05, pmass=float(pm), vol0=float(vol0), mu=1e4 / 2.6,
                     lam=1e4 * 0.3 / (1.3 * 0.4), mass_eps=1e-9, wall=0, growth_mode=0)
    return Plan([spec], dtype=dtype, device="cuda")


def _traj(plan, pts, g, steps, dtype):
    """loss (sum det F) and d loss/d g of a trajectory with Fg = g I (explicit)."""
    from morphompm_b200.runtime import SLAB_ROWS, ROW_X, ROW_F
    from morphompm_b200.trajectory import Rollout
    n = pts.shape[0]
    slab = torch.zeros(SLAB_ROWS, n, dtype=dtype, device="cuda")
    slab[ROW_X:ROW_X + 3] = torch.as_tensor(pts.T.astype(np.float64), dtype=dtype, device="cuda")
    for i in range(3):
        slab[ROW_F + 4 * i] = 1.0
    Fg = torch.zeros(9, n, dtype=dtype, device="cuda")
    for i in range(3):
        Fg[4 * i] = g
    ro = Rollout(plan, steps, advect=True, Fg=Fg)
    bar0 = ro.run(slab).clone()
    torch.cuda.synchronize()
    dg = float(ro.Fg_bar[0].sum() + ro.Fg_bar[4].sum() + ro.Fg_bar[8].sum())
    return float(ro.loss.sum()), dg, ro.final.clone(), bar0


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_particle_mass_arrays_with_scene_values_change_nothing(dtype):
    dt = getattr(torch, dtype)
    pts = G.blob(0.6, 0.10, 0.025)
    n = pts.shape[0]
    pm = _pmass(1000.0, 0.025)
    vol0 = np.float32(pm / np.float32(1000.0))
    a = _traj(_plan(n, dt, pm, vol0), pts, 1.2, 8, dt)
    p = _plan(n, dt, pm, vol0)
    p.set_particle_mass(torch.full((n,), float(pm), dtype=dt), torch.full((n,), float(vol0), dtype=dt))
    b = _traj(p, pts, 1.2, 8, dt)
    assert a[0] == b[0] and a[1] == b[1]
    assert torch.equal(a[2], b[2]) and torch.equal(a[3], b[3])


def test_particle_mass_fp32_against_cpp():
    pts, mass, vol0, density = _two_density_blob()
    ref = G.RefSolver(24, 0.05, 1e4, 0.3, 0.05)
    ref.add_each(pts, mass, density)
    ref.set_growth(1.2)
    ref.step(1e-3, 300)
    _, _, Fr, _ = ref.get()
    n = pts.shape[0]
    p = _plan(n, torch.float32, mass[0], vol0[0])
    p.set_particle_mass(torch.as_tensor(mass), torch.as_tensor(vol0))
    _, _, fin, _ = _traj(p, pts, 1.2, 300, torch.float32)
    F = fin[15:24].double().cpu().numpy().T.reshape(n, 3, 3)
    assert np.abs(F - Fr).max() < 5e-5, np.abs(F - Fr).max()


def test_particle_mass_gradient_vs_fd_fp64():
    pts, mass, vol0, _ = _two_density_blob()
    n = pts.shape[0]

    def run(g):
        p = _plan(n, torch.float64, mass[0], vol0[0])
        p.set_particle_mass(torch.as_tensor(mass.astype(np.float64)), torch.as_tensor(vol0.astype(np.float64)))
        return _traj(p, pts, g, 6, torch.float64)
    L, dg, _, _ = run(1.15)
    h = 1e-6
    fd = (run(1.15 + h)[0] - run(1.15 - h)[0]) / (2 * h)
    assert abs(dg - fd) < 1e-6 * abs(fd), (dg, fd)
