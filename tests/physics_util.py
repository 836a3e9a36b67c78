"""Helpers shared by the GPU tests that run the reference's C++ physics
scenes (tests/test_growth.cpp of the reference) on the device FP32 path with
the C++ solver's semantics: Hencky, gravity 0, per-step damping, mass
threshold 1e-9, no walls, advected positions, explicit per-particle Fg."""
import numpy as np


def pmass(density, sp):
    """density * sp * sp * sp evaluated left to right in single precision."""
    d, s = np.float32(density), np.float32(sp)
    return np.float32(np.float32(np.float32(d * s) * s) * s)


def device_run(pts, N, dx, dt, damping, density, sp, E, nu, blocks):
    """blocks: list of (Fg (n,3,3), steps); consecutive steps with the same Fg
    are chained.  Returns the final x (n,3) and F (n,3,3) in float64."""
    import torch
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import Plan, SceneSpec, slab_particles, SLAB_ROWS, ROW_X, ROW_F
    n = pts.shape[0]
    pm = pmass(density, sp)
    vol0 = np.float32(pm / np.float32(density))
    spec = SceneSpec(shape=(N, N, N), n=n, model=L.MODEL_HENCKY, dx=dx, dt=dt, damping=damping,
                     pmass=float(pm), vol0=float(vol0), mu=E / (2.0 * (1.0 + nu)),
                     lam=E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mass_eps=1e-9, wall=0, growth_mode=0)
    plan = Plan([spec], dtype=torch.float32, device="cuda")
    a = torch.zeros(SLAB_ROWS, n, dtype=torch.float32, device="cuda")
    a[ROW_X:ROW_X + 3] = torch.as_tensor(np.ascontiguousarray(pts.T), device="cuda")
    for i in range(3):
        a[ROW_F + 4 * i] = 1.0
    b = torch.empty_like(a)
    Fg = torch.empty(9, n, dtype=torch.float32, device="cuda")
    t = 0
    for G, steps in blocks:
        Fg.copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(G, np.float32).reshape(n, 9).T), device="cuda"))
        for k in range(steps):
            plan.step_fwd(slab_particles(a, Fg), slab_particles(b, Fg), True, t, None,
                          chained=k > 0, emit=k + 1 < steps)
            a, b = b, a
            t += 1
    torch.cuda.synchronize()
    assert plan.status() == 0
    s = a.double().cpu().numpy()
    return s[ROW_X:ROW_X + 3].T, s[ROW_F:ROW_F + 9].T.reshape(n, 3, 3)


def cpp_run(pts, N, dx, dt, damping, density, sp, E, nu, blocks):
    from oracle import growth_ref as G
    r = G.RefSolver(N, dx, E, nu, damping)
    r.add(pts, pmass(density, sp), density)
    for Fg, steps in blocks:
        r.set_growth_tensors(Fg)
        r.step(dt, steps)
    x, _, F, _ = r.get()
    return x.astype(np.float64), F.astype(np.float64)


def eps_norm(F, Fg):
    """||ln s|| of Fe = F Fg^-1 per particle, s clamped at 1e-6 (growth_solver.h:82-99)."""
    Fe = np.einsum("pij,pjk->pik", F, np.linalg.inv(Fg))
    s = np.linalg.svd(Fe, compute_uv=False)
    return np.linalg.norm(np.log(np.maximum(s, 1e-6)), axis=1)


def bend(x):
    """|mean y of the middle third - average of the outer thirds| (test_growth.cpp:140-145)."""
    xlo, xhi = x[:, 0].min(), x[:, 0].max()
    bw = (xhi - xlo) / 3.0 + 1e-9
    b = np.minimum(2, ((x[:, 0] - xlo) / bw).astype(int))
    m = [x[b == k, 1].mean() for k in range(3)]
    return abs(m[1] - 0.5 * (m[0] + m[2]))


def curvature(x, nb=9):
    """|2a| of the least-squares parabola through the per-bin mean centreline
    (test_growth.cpp:268-295)."""
    xlo, xhi = x[:, 0].min(), x[:, 0].max()
    bw = (xhi - xlo) / nb + 1e-9
    b = np.clip(((x[:, 0] - xlo) / bw).astype(int), 0, nb - 1)
    xs = np.array([x[b == k, 0].mean() for k in range(nb) if np.any(b == k)])
    ys = np.array([x[b == k, 1].mean() for k in range(nb) if np.any(b == k)])
    a = np.polyfit(xs - xs.mean(), ys, 2)[0]
    return abs(2.0 * a)


def iso(n, g):
    return np.tile(np.float32(g) * np.eye(3, dtype=np.float32), (n, 1, 1))


def layered(pts, cy, g_bot, g_top, axial=False):
    """Bilayer growth: g_top where y >= cy, else g_bot (diag(g,1,1) when axial)."""
    g = np.where(pts[:, 1] >= np.float32(cy), np.float32(g_top), np.float32(g_bot))
    Fg = np.zeros((pts.shape[0], 3, 3), np.float32)
    Fg[:, 0, 0] = g
    Fg[:, 1, 1] = 1.0 if axial else g
    Fg[:, 2, 2] = 1.0 if axial else g
    return Fg
