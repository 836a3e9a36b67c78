"""Seeded synthetic scenes for the five growth workloads (numpy only).

Every generator is deterministic in its seed (``numpy.random.default_rng``) and
returns plain numpy arrays plus the scene constants.  Particles are placed with
cell-stratified jitter: each grid cell holds 2x2x2 sub-cells with one uniformly
jittered particle in each (8 particles per cell, spacing sp = dx/2, so
pmass = rho*sp^3 and vol0 = sp^3 as in the reference ``SimConfig``).  Particles
are returned in the order of their stencil cell, the order the step kernels
sort into, so the device gathers through that order start out coalesced.

Workloads (sizes as named by the growth benchmarks):
  config1  32^3 grid, 8^3-cell cube, 4096 particles, neo-Hookean, ramp 1 -> 1.1 / 100 steps
  config2  96x32x32 grid, 64x8x8-cell strip, 32768 particles, Hencky bilayer
  config3  64^3 grid, 16^3-cell cube, 32768 particles, neo-Hookean, MSE position loss
  config4  256 uneven scenes, n log-uniform in [2048, 65536], grids 32^3..64^3
  config5  256^3 grid, 128x128x16-cell sheet, 2,097,152 particles, Herschel-Bulkley
"""
from __future__ import annotations

import math

import numpy as np


def stencil_order(x, dx):
    """Stable order of particles by the cell of their stencil base
    floor(x/dx - 0.5) (x-major, z fastest): the order the step kernels sort into."""
    b = np.floor(x / dx - 0.5).astype(np.int64)
    b -= b.min(axis=0)
    span = b.max(axis=0) + 1
    key = (b[:, 0] * span[1] + b[:, 1]) * span[2] + b[:, 2]
    return np.argsort(key, kind="stable")


def stratified_cells(rng, cell_lo, cell_hi, dx, limit=None):
    """8 particles per cell over the cell box [cell_lo, cell_hi), jittered in
    2x2x2 sub-cells, returned in stencil-cell order (see ``stencil_order``)."""
    lo = np.asarray(cell_lo, dtype=np.int64)
    hi = np.asarray(cell_hi, dtype=np.int64)
    ci = np.stack(np.meshgrid(*[np.arange(a, b) for a, b in zip(lo, hi)], indexing="ij"), -1).reshape(-1, 3)
    sub = np.stack(np.meshgrid([0, 1], [0, 1], [0, 1], indexing="ij"), -1).reshape(-1, 3)
    corner = (ci[:, None, :] * 2 + sub[None, :, :]).reshape(-1, 3).astype(np.float64)
    jit = rng.uniform(0.0, 1.0, size=corner.shape)
    x = (corner + jit) * (dx / 2.0)
    if limit is not None:
        x = x[:limit]
    return x[stencil_order(x, dx)]


def _elastic(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


def config1(seed=1):
    dx = 1.0 / 32
    rng = np.random.default_rng(seed)
    x = stratified_cells(rng, (12, 12, 12), (20, 20, 20), dx)
    mu, lam = _elastic(1e3, 0.3)
    return dict(name="free-swell cube 32^3, 4096 particles", x=x, shape=(32, 32, 32), dx=dx,
                dt=1e-4, damping=0.05, density=1.0, model="nh", E=1e3, nu=0.3, mu=mu, lam=lam,
                growth_A=0.1, ramp_steps=100, phi=None, wall=2, steps=100)


def config2(seed=2, length=64, steps=2000):
    """Bilayer strip of `length` x 8 x 8 cells from x-cell 16 (64 for the full
    workload), top half growing to g = 1.2 over `steps` steps, clamped end."""
    dx = 1.0 / 32
    rng = np.random.default_rng(seed)
    x = stratified_cells(rng, (16, 12, 12), (16 + length, 20, 20), dx)
    mu, lam = _elastic(1e3, 0.3)
    phi = (x[:, 1] >= 0.5).astype(np.float64)      # top layer grows
    return dict(name=f"bilayer strip 96x32x32, {x.shape[0]} particles", x=x, shape=(96, 32, 32), dx=dx,
                dt=5e-5, damping=0.05, density=1.0, model="hencky", E=1e3, nu=0.3, mu=mu, lam=lam,
                growth_A=0.2, ramp_steps=steps, phi=phi, wall=0,
                clamp_lo=(0, 0, 0), clamp_hi=(18, 32, 32), steps=steps)


def config3(seed=3):
    dx = 1.0 / 64
    rng = np.random.default_rng(seed)
    x = stratified_cells(rng, (24, 24, 24), (40, 40, 40), dx)
    mu, lam = _elastic(1e3, 0.3)
    return dict(name="inverse growth cube 64^3, 32768 particles", x=x, shape=(64, 64, 64), dx=dx,
                dt=1e-4, damping=0.05, density=1.0, model="nh", E=1e3, nu=0.3, mu=mu, lam=lam,
                g_true=1.15, g_eval=1.10, wall=2, steps=400, ckpt_every=20)


def config4(seed=4, n_scenes=256, n_lo=2048, n_hi=65536):
    """Uneven batch: per scene n ~ log-uniform, grid edge ~ U{32..64}, dx = 1/edge,
    a centred cube of ceil((n/8)^(1/3)) cells holding the first n particles,
    g ~ U(1.0, 1.3), E ~ U(5e2, 5e3), nu ~ U(0.2, 0.45), model 50/50 NH/Hencky."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_scenes):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        edge = int(rng.integers(32, 65))
        g = float(rng.uniform(1.0, 1.3))
        E = float(rng.uniform(5e2, 5e3))
        nu = float(rng.uniform(0.2, 0.45))
        model = "nh" if rng.uniform() < 0.5 else "hencky"
        c = int(math.ceil((n / 8.0) ** (1.0 / 3.0)))
        lo = (edge - c) // 2
        dx = 1.0 / edge
        x = stratified_cells(rng, (lo, lo, lo), (lo + c, lo + c, lo + c), dx, limit=n)
        mu, lam = _elastic(E, nu)
        out.append(dict(name=f"scene{s}", x=x, shape=(edge, edge, edge), dx=dx, dt=2e-5,
                        damping=0.05, density=1.0, model=model, E=E, nu=nu, mu=mu, lam=lam,
                        growth_A=g - 1.0, ramp_steps=0, phi=None, wall=2))
    return out


def config5(seed=5, cells=(128, 128, 16), edge=256, steps=1000):
    """Herschel-Bulkley sheet of `cells` cells centred in an edge^3 grid with
    the radial growth field g(r) = 1 + 0.2 exp(-r^2 / 0.05)."""
    dx = 1.0 / edge
    rng = np.random.default_rng(seed)
    lo = [(edge - c) // 2 for c in cells]
    hi = [a + c for a, c in zip(lo, cells)]
    x = stratified_cells(rng, lo, hi, dx)
    r2 = (x[:, 0] - 0.5) ** 2 + (x[:, 1] - 0.5) ** 2
    phi = np.exp(-r2 / 0.05)
    return dict(name=f"HB sheet {edge}^3, {x.shape[0]} particles", x=x, shape=(edge, edge, edge), dx=dx,
                dt=1e-5, damping=0.05, density=1.0, model="hb",
                hb=dict(kappa=1e4, K=1.0, n=0.5, tau_y=10.0, m=100.0, eps=1e-4),
                growth_A=0.2, ramp_steps=0, phi=phi, wall=2, steps=steps)
