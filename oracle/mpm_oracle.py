"""CPU oracle for the MLS-MPM growth step -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs
of ``bench.py`` may import it.  The product path (``morphompm_b200``) never calls
into it and has no CPU fallback.

It is a vectorised numpy FP64 restatement of the reference's per-particle Python
loops (2nugu/morphompm), organised so that every function cites the reference
lines it follows:

* quadratic B-spline weights ``wts``           -- python/morphompm/transfer.py:18-24
* weight gradient ``dwdx``                     -- python/morphompm/transfer.py:27-30
* ``step`` (P2G + grid update + G2P)            -- python/morphompm/transfer.py:33-79
* ``step_vjp`` (G2P / grid / P2G adjoints)      -- python/morphompm/transfer.py:82-158
* constitutive stress + VJP (NH, Hencky, HB)    -- python/morphompm/constitutive.py:25-147
* ``rollout`` / ``rollout_vjp`` / losses        -- python/morphompm/integrate.py:15-52

Parity is pinned: ``tests/golden/make_golden.py`` runs the unmodified reference
package on small scenes and the fixtures it wrote are checked against this oracle
by ``tests/test_oracle.py`` (max abs difference <= 1e-12 relative).

Extensions the reference does not have (each defaults to the reference
behaviour and is pinned only by finite-difference gates, "parity unpinned"):
non-cubic grids, sticky/clamped grid boundary conditions, gravity, a
configurable grid-mass threshold, a per-particle isotropic growth law
``g_p(t) = 1 + A * ramp(t) * phi_p`` and the mean-squared position loss.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

I3 = np.eye(3)
DEGEN = 1.0e-9  # Hencky divided-difference switch, constitutive.py:17,70

STEN = [(i, j, k) for i in range(3) for j in range(3) for k in range(3)]


# ----------------------------------------------------------------------------
# scene description (one grid + one material model)
# ----------------------------------------------------------------------------
@dataclass
class Model:
    """Constitutive model: kind in {"nh", "hencky", "hb"} plus its parameters.

    nh / hencky: mu, lam (Lame, config.py:12-18).
    hb: kappa, K, n, tau_y, m, eps (constitutive.py:115).
    """
    kind: str
    mu: float = 0.0
    lam: float = 0.0
    kappa: float = 1.0e4
    K: float = 1.0
    n: float = 0.5
    tau_y: float = 50.0
    m: float = 100.0
    eps: float = 1.0e-4

    @staticmethod
    def elastic(kind: str, E: float, nu: float) -> "Model":
        mu = E / (2.0 * (1.0 + nu))
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        return Model(kind=kind, mu=mu, lam=lam)


@dataclass
class Scene:
    """Grid + step constants.  Defaults reproduce the reference ``SimConfig``
    (config.py:21-40) on a cubic grid with no boundary conditions."""
    shape: Sequence[int] = (8, 8, 8)
    dx: float = 0.1
    dt: float = 1.0e-3
    damping: float = 0.05
    pmass: float = 1000.0 * 0.02 ** 3
    vol0: float = 0.02 ** 3
    mass_eps: float = 1.0e-12          # transfer.py:56 (gm > 1e-12)
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    wall: int = 0                      # sticky nodes: index < wall or >= N - wall
    clamp_lo: Sequence[int] = (0, 0, 0)  # sticky box [lo, hi) (empty if lo >= hi)
    clamp_hi: Sequence[int] = (0, 0, 0)

    @property
    def inv_dx(self) -> float:
        return 1.0 / self.dx

    def node_mask(self) -> np.ndarray:
        """1.0 for free nodes, 0.0 for sticky ones, flattened (x-major, z fastest)."""
        nx, ny, nz = self.shape
        ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        free = np.ones((nx, ny, nz), dtype=bool)
        if self.wall > 0:
            w = self.wall
            for a, n in ((ii, nx), (jj, ny), (kk, nz)):
                free &= (a >= w) & (a < n - w)
        lo, hi = self.clamp_lo, self.clamp_hi
        if all(h > l for l, h in zip(lo, hi)):
            inside = ((ii >= lo[0]) & (ii < hi[0]) & (jj >= lo[1]) & (jj < hi[1])
                      & (kk >= lo[2]) & (kk < hi[2]))
            free &= ~inside
        return free.reshape(-1).astype(np.float64)

    def plain(self) -> bool:
        return (self.wall == 0 and not all(h > l for l, h in zip(self.clamp_lo, self.clamp_hi))
                and not any(self.gravity))


# ----------------------------------------------------------------------------
# batched small linear algebra
# ----------------------------------------------------------------------------
def _inv(A):
    return np.linalg.inv(A)


def _det(A):
    return np.linalg.det(A)


def _T(A):
    return np.swapaxes(A, -1, -2)


def _sym(A):
    return 0.5 * (A + _T(A))


def _tr(A):
    return np.trace(A, axis1=-2, axis2=-1)


# ----------------------------------------------------------------------------
# constitutive models: stress + VJP  (constitutive.py:25-147)
# ----------------------------------------------------------------------------
def stress(model: Model, F, Fg, C=None):
    """Kirchhoff stress, batched over the leading axis."""
    k = model.kind
    if k == "nh":                                     # constitutive.py:25-28
        Fe = F @ _inv(Fg)
        J = _det(Fe)
        return model.mu * (Fe @ _T(Fe) - I3) + model.lam * np.log(J)[..., None, None] * I3
    if k == "hencky":                                 # constitutive.py:42-47
        Fe = F @ _inv(Fg)
        U, s, _ = np.linalg.svd(Fe)
        ls = np.log(s)
        h = 2.0 * model.mu * ls + model.lam * np.sum(ls, axis=-1, keepdims=True)
        return (U * h[..., None, :]) @ _T(U)
    if k == "hb":                                     # constitutive.py:118-132
        Je = _det(F) / _det(Fg)
        D, gdot = _hb_rate(model, C)
        eta = _hb_eta(model, gdot)
        return model.kappa * np.log(Je)[..., None, None] * I3 + 2.0 * eta[..., None, None] * D
    raise ValueError(k)


def _hb_rate(model, C):
    D = _sym(C)
    gdot = np.sqrt(2.0 * np.sum(D * D, axis=(-2, -1)) + model.eps ** 2)
    return D, gdot


def _hb_eta(model, gdot):
    return model.K * gdot ** (model.n - 1) + model.tau_y * (1 - np.exp(-model.m * gdot)) / gdot


def stress_vjp(model: Model, F, Fg, C, tau_bar):
    """(F_bar, Fg_bar, C_bar) for a cotangent tau_bar of the Kirchhoff stress."""
    k = model.kind
    tb = _sym(tau_bar)
    if k == "nh":                                     # constitutive.py:31-39
        Fg_inv = _inv(Fg)
        Fe = F @ Fg_inv
        Fe_invT = _T(_inv(Fe))
        Fe_bar = 2.0 * model.mu * (tb @ Fe) + model.lam * _tr(tb)[..., None, None] * Fe_invT
    elif k == "hencky":                               # constitutive.py:50-75
        Fg_inv = _inv(Fg)
        Fe = F @ Fg_inv
        U, s, _ = np.linalg.svd(Fe)
        beta = s * s
        lb = np.log(beta)
        M = model.mu * tb + 0.5 * model.lam * _tr(tb)[..., None, None] * I3
        UtMU = _T(U) @ M @ U
        d = beta[..., :, None] - beta[..., None, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            dd = (lb[..., :, None] - lb[..., None, :]) / d
        L = np.where(np.abs(d) > DEGEN, dd, 1.0 / beta[..., :, None] * np.ones_like(d))
        Bbar = U @ (UtMU * L) @ _T(U)
        Fe_bar = 2.0 * Bbar @ Fe
    elif k == "hb":                                   # constitutive.py:134-147
        trtb = _tr(tb)
        F_bar = model.kappa * trtb[..., None, None] * _T(_inv(F))
        Fg_bar = -model.kappa * trtb[..., None, None] * _T(_inv(Fg))
        D, gdot = _hb_rate(model, C)
        K, n, ty, m = model.K, model.n, model.tau_y, model.m
        deta = (K * (n - 1) * gdot ** (n - 2)
                + ty * ((m * np.exp(-m * gdot)) * gdot - (1 - np.exp(-m * gdot))) / gdot ** 2)
        tbD = np.sum(tb * D, axis=(-2, -1))
        eta = _hb_eta(model, gdot)
        C_bar = (2.0 * eta[..., None, None] * tb
                 + (4.0 * tbD * deta / gdot)[..., None, None] * D)
        return F_bar, Fg_bar, C_bar
    else:
        raise ValueError(k)
    F_bar = Fe_bar @ _T(Fg_inv)
    Fg_bar = -_T(Fg_inv) @ _T(F) @ Fe_bar @ _T(Fg_inv)
    return F_bar, Fg_bar, np.zeros_like(F_bar)


# ----------------------------------------------------------------------------
# weights and binning  (transfer.py:18-30)
# ----------------------------------------------------------------------------
def wts(x, inv_dx):
    """base (int64), fx, w[p, stencil, dim], dw[p, stencil, dim]."""
    X = x * inv_dx
    base = np.floor(X - 0.5).astype(np.int64)
    fx = X - base
    w = np.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2], axis=1)
    dw = np.stack([-(1.5 - fx), -2.0 * (fx - 1.0), (fx - 0.5)], axis=1)
    return base, fx, w, dw


def dwdx(i, j, k, w, dw, inv_dx):
    return np.stack([dw[:, i, 0] * w[:, j, 1] * w[:, k, 2],
                     w[:, i, 0] * dw[:, j, 1] * w[:, k, 2],
                     w[:, i, 0] * w[:, j, 1] * dw[:, k, 2]], axis=1) * inv_dx


def cell_keys(x, scene: Scene):
    """Sort key of each particle: its stencil base shifted by +2 on each axis and
    flattened over the padded (N+2)^3 cell grid (z fastest).  Particles whose
    stencil misses the grid entirely get the key (N+2)^3 (sorted last)."""
    nx, ny, nz = scene.shape
    base, _, _, _ = wts(x, scene.inv_dx)
    c = base + 2
    dims = np.array([nx + 2, ny + 2, nz + 2])
    inside = np.all((c >= 0) & (c < dims), axis=1)
    key = (c[:, 0] * dims[1] + c[:, 1]) * dims[2] + c[:, 2]
    return np.where(inside, key, int(np.prod(dims))).astype(np.int64)


# ----------------------------------------------------------------------------
# one MLS-MPM step and its VJP  (transfer.py:33-158)
# ----------------------------------------------------------------------------
@dataclass
class State:
    x: np.ndarray
    v: np.ndarray
    C: np.ndarray
    F: np.ndarray
    Fg: np.ndarray

    @staticmethod
    def rest(x0, g=1.0):
        n = x0.shape[0]
        I = np.tile(I3, (n, 1, 1))
        return State(x0.copy(), np.zeros((n, 3)), np.zeros((n, 3, 3)), I.copy(), g * I)

    def copy(self):
        return State(*(a.copy() for a in (self.x, self.v, self.C, self.F, self.Fg)))


def _stencil(base, fx, w, scene: Scene, o):
    nx, ny, nz = scene.shape
    i, j, k = o
    wt = w[:, i, 0] * w[:, j, 1] * w[:, k, 2]
    dpos = (np.array([i, j, k]) - fx) * scene.dx
    node = base + np.array([i, j, k])
    ok = ((node[:, 0] >= 0) & (node[:, 0] < nx) & (node[:, 1] >= 0) & (node[:, 1] < ny)
          & (node[:, 2] >= 0) & (node[:, 2] < nz))
    idx = (node[:, 0] * ny + node[:, 1]) * nz + node[:, 2]
    idx = np.where(ok, idx, 0)
    return wt, dpos, idx, ok


def p2g(st: State, model: Model, scene: Scene):
    """Particle-to-grid with stress, then the grid update (transfer.py:42-59).
    Returns (gm, gmom, gv, per-particle cache)."""
    x, v, C, F, Fg = st.x, st.v, st.C, st.F, st.Fg
    nx, ny, nz = scene.shape
    G = nx * ny * nz
    inv_dx, dt = scene.inv_dx, scene.dt
    k4 = 4.0 * inv_dx * inv_dx
    tau = stress(model, F, Fg, C)
    c = -k4 * scene.vol0 * _det(Fg)
    sk = c[:, None, None] * tau
    base, fx, w, dw = wts(x, inv_dx)
    gm = np.zeros(G)
    gmom = np.zeros((G, 3))
    for o in STEN:
        wt, dpos, idx, ok = _stencil(base, fx, w, scene, o)
        q = wt[:, None] * (scene.pmass * (v + np.einsum("nij,nj->ni", C, dpos))
                           + np.einsum("nij,nj->ni", sk, dpos) * dt)
        gm += np.bincount(idx[ok], weights=(wt * scene.pmass)[ok], minlength=G)
        for d in range(3):
            gmom[:, d] += np.bincount(idx[ok], weights=q[ok, d], minlength=G)
    act = gm > scene.mass_eps
    s = 1.0 - scene.damping
    gv = np.zeros((G, 3))
    gv[act] = s * (gmom[act] / gm[act, None] + dt * np.asarray(scene.gravity, dtype=np.float64))
    gv *= scene.node_mask()[:, None]
    pc = (base, fx, w, dw, tau, c, sk)
    return gm, gmom, gv, pc


def step(st: State, model: Model, scene: Scene, advect=True):
    """One MLS-MPM step (transfer.py:33-79).  Returns (new_state, cache)."""
    gm, gmom, gv, pc = p2g(st, model, scene)
    base, fx, w, dw, tau, c, sk = pc
    n = st.x.shape[0]
    k4 = 4.0 * scene.inv_dx ** 2
    nv = np.zeros((n, 3))
    nC = np.zeros((n, 3, 3))
    for o in STEN:
        wt, dpos, idx, ok = _stencil(base, fx, w, scene, o)
        vi = np.where(ok[:, None], gv[idx], 0.0)
        nv += wt[:, None] * vi
        nC += (k4 * wt)[:, None, None] * (vi[:, :, None] * dpos[:, None, :])
    xn = st.x + scene.dt * nv if advect else st.x.copy()
    Fn = (I3 + scene.dt * nC) @ st.F
    new = State(xn, nv, nC, Fn, st.Fg.copy())
    cache = (st, scene, model, gm, gv, pc, nC)
    return new, cache


def step_vjp(cache, xn_b, vn_b, Cn_b, Fn_b, Fgn_b, advect=True):
    """Reverse of ``step`` (transfer.py:82-158); same advect contract:
    with advect=False x is frozen and x_b is returned as 0."""
    st, scene, model, gm, gv, pc, Cn = cache
    x, v, C, F, Fg = st.x, st.v, st.C, st.F, st.Fg
    base, fx, w, dw, tau, c, sk = pc
    n = x.shape[0]
    nx, ny, nz = scene.shape
    G = nx * ny * nz
    inv_dx, dt = scene.inv_dx, scene.dt
    s, pmass, vol0 = 1.0 - scene.damping, scene.pmass, scene.vol0
    k4 = 4.0 * inv_dx * inv_dx

    F_b = np.zeros((n, 3, 3))
    v_b = np.zeros((n, 3))
    C_b = np.zeros((n, 3, 3))
    Fg_b = Fgn_b.copy()
    x_b = np.zeros((n, 3))
    gv_b = np.zeros((G, 3))

    # g2p adjoint (transfer.py:99-119)
    nv_b = vn_b + (dt * xn_b if advect else 0.0)
    if advect:
        x_b += xn_b
    Cnb = Cn_b + dt * (Fn_b @ _T(F))
    F_b += _T(I3 + dt * Cn) @ Fn_b
    for (i, j, k) in STEN:
        wt, dpos, idx, ok = _stencil(base, fx, w, scene, (i, j, k))
        vi = np.where(ok[:, None], gv[idx], 0.0)
        q = wt[:, None] * nv_b + (k4 * wt)[:, None] * np.einsum("nij,nj->ni", Cnb, dpos)
        for d in range(3):
            gv_b[:, d] += np.bincount(idx[ok], weights=q[ok, d], minlength=G)
        if advect:
            dW = dwdx(i, j, k, w, dw, inv_dx)
            t1 = np.sum(nv_b * vi, axis=1)
            t2 = k4 * np.einsum("ni,nij,nj->n", vi, Cnb, dpos)
            contrib = (t1 + t2)[:, None] * dW - (k4 * wt)[:, None] * np.einsum("nji,nj->ni", Cnb, vi)
            x_b += np.where(ok[:, None], contrib, 0.0)

    # grid adjoint (transfer.py:121-127), with the sticky mask and gravity
    act = gm > scene.mass_eps
    mask = scene.node_mask()
    gmom_b = np.zeros((G, 3))
    gm_b = np.zeros(G)
    gmom_b[act] = (s * mask[act])[:, None] * gv_b[act] / gm[act, None]
    if advect:
        grav_term = (s * mask[act])[:, None] * dt * np.asarray(scene.gravity, dtype=np.float64)
        gm_b[act] = -np.sum(gv_b[act] * (gv[act] - grav_term), axis=1) / gm[act]

    # p2g adjoint + constitutive VJP + volume path (transfer.py:129-156)
    sk_b = np.zeros((n, 3, 3))
    for (i, j, k) in STEN:
        wt, dpos, idx, ok = _stencil(base, fx, w, scene, (i, j, k))
        mb = np.where(ok[:, None], gmom_b[idx], 0.0)
        v_b += (wt * pmass)[:, None] * mb
        C_b += (wt * pmass)[:, None, None] * (mb[:, :, None] * dpos[:, None, :])
        sk_b += (wt * dt)[:, None, None] * (mb[:, :, None] * dpos[:, None, :])
        if advect:
            dW = dwdx(i, j, k, w, dw, inv_dx)
            Q2 = pmass * (v + np.einsum("nij,nj->ni", C, dpos)) + np.einsum("nij,nj->ni", sk, dpos) * dt
            gmb = np.where(ok, gm_b[idx], 0.0)
            contrib = ((np.sum(mb * Q2, axis=1) + gmb * pmass)[:, None] * dW
                       - (pmass * np.einsum("nji,nj->ni", C, mb) + dt * np.einsum("nji,nj->ni", sk, mb)) * wt[:, None])
            x_b += np.where(ok[:, None], contrib, 0.0)
    tau_b = c[:, None, None] * sk_b
    Fp_b, Fg_bar_stress, C_bar = stress_vjp(model, F, Fg, C, tau_b)
    F_b += Fp_b
    C_b += C_bar
    Fg_b += Fg_bar_stress
    Fg_b += (np.sum(sk_b * tau, axis=(1, 2)) * (-k4 * vol0) * _det(Fg))[:, None, None] * _T(_inv(Fg))
    return x_b, v_b, C_b, F_b, Fg_b


# ----------------------------------------------------------------------------
# trajectories, growth law, losses  (integrate.py:15-52)
# ----------------------------------------------------------------------------
@dataclass
class Growth:
    """Isotropic growth law Fg_p(t) = g_p(t) I, g_p(t) = 1 + A * ramp(t) * phi_p,
    ramp(t) = min(1, (t + 1) / ramp_steps) (1 when ramp_steps == 0)."""
    A: float
    ramp_steps: int = 0
    phi: Optional[np.ndarray] = None

    def ramp(self, t):
        return 1.0 if self.ramp_steps <= 0 else min(1.0, (t + 1) / self.ramp_steps)

    def g(self, t, n):
        phi = np.ones(n) if self.phi is None else self.phi
        return 1.0 + self.A * self.ramp(t) * phi


def rollout(st0: State, model, scene, n_steps, advect=False, growth: Optional[Growth] = None,
            keep_caches=True):
    st = st0
    caches = []
    for t in range(n_steps):
        if growth is not None:
            st = st.copy()
            st.Fg = growth.g(t, st.x.shape[0])[:, None, None] * I3
        st, cache = step(st, model, scene, advect=advect)
        if keep_caches:
            caches.append(cache)
    return st, caches


def rollout_vjp(caches, xf_b, vf_b, Cf_b, Ff_b, Fgf_b, advect=False, growth: Optional[Growth] = None):
    """Reverse sweep.  With a growth law, Fg is re-set before every step, so the
    Fg cotangent does not pass through; dL/dA is accumulated instead and
    returned as a sixth value."""
    xb, vb, Cb, Fb, Fgb = xf_b, vf_b, Cf_b, Ff_b, Fgf_b
    dA = 0.0
    T = len(caches)
    for t in range(T - 1, -1, -1):
        if growth is not None:
            Fgb = np.zeros_like(Fgb)
        xb, vb, Cb, Fb, Fgb = step_vjp(caches[t], xb, vb, Cb, Fb, Fgb, advect=advect)
        if growth is not None:
            n = xb.shape[0]
            phi = np.ones(n) if growth.phi is None else growth.phi
            dA += float(np.sum(_tr(Fgb) * growth.ramp(t) * phi))
    if growth is not None:
        return xb, vb, Cb, Fb, Fgb, dA
    return xb, vb, Cb, Fb, Fgb


def loss_detF(F):
    return float(np.sum(_det(F)))


def seed_detF(F):
    return _det(F)[:, None, None] * _T(_inv(F))


def loss_mse(x, x_obs):
    return float(np.mean(np.sum((x - x_obs) ** 2, axis=1)))


def seed_mse(x, x_obs):
    return 2.0 * (x - x_obs) / x.shape[0]


def dloss_dg(pts, model, scene, g, n_steps, advect):
    """d(sum det F_final)/dg (integrate.py:45-52)."""
    st, caches = rollout(State.rest(pts, g), model, scene, n_steps, advect=advect)
    n = st.x.shape[0]
    Ff_b = seed_detF(st.F)
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    _, _, _, _, Fg_b = rollout_vjp(caches, z3, z3, z33, Ff_b, z33, advect=advect)
    return loss_detF(st.F), float(np.sum(_tr(Fg_b)))


def scene_from_cfg(N, dx, dt, damping, sp, density):
    """Reference SimConfig (cubic) -> Scene (config.py:21-40)."""
    return Scene(shape=(N, N, N), dx=dx, dt=dt, damping=damping,
                 pmass=density * sp ** 3, vol0=sp ** 3)
