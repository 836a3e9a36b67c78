"""[4] Integrate -- trajectory rollout and adjoint with the reference's
signatures (python/morphompm/integrate.py:15-52):

    rollout(state0, model, cfg, n_steps, advect)          -> final state, caches
    rollout_vjp(caches, xf_b, vf_b, Cf_b, Ff_b, Fgf_b, advect) -> state cotangents
    iso_growth_state(pts, g), iso_growth_grad(Fg_b), loss_detF(F)
    dloss_dg(pts, model, cfg, g, n_steps, advect)         -> (loss, dloss/dg)

``rollout``/``rollout_vjp`` keep one cache per step like the reference (device
memory O(n_steps)).  ``dloss_dg`` runs the device trajectory engine
(trajectory.Rollout) instead, on the particles in cell order (layout.py), with optional checkpoint-every-k recomputation
(``ckpt_every``) and an optional mean-squared final-position loss
(``loss="mse"``, ``x_obs``); with the defaults it returns what the reference
returns.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .devarray import like_input, to_device
from .runtime import SLAB_ROWS, ROW_F, ROW_X
from .state import ParticleState
from .constitutive import is_external
from .config import compute_target
from .layout import cell_order_device
from .transfer import get_plan, scene_spec, step, step_vjp


def _dev_state(state0: ParticleState, cfg=None) -> ParticleState:
    x = to_device(state0.x, *compute_target(cfg)).contiguous()
    dt, dev = x.dtype, x.device
    return ParticleState(x, *(to_device(a, dt, dev).contiguous() for a in (state0.v, state0.C, state0.F, state0.Fg)))


def rollout(state0: ParticleState, model, cfg, n_steps, advect=False):
    ref = state0.x
    st = _dev_state(state0, cfg)
    caches = []
    for t in range(n_steps):
        st, cache = step(st, model, cfg, advect=advect)
        cache.ref = ref
        caches.append(cache)
    return ParticleState(*(like_input(a, ref) for a in (st.x, st.v, st.C, st.F, st.Fg))), caches


def rollout_vjp(caches, xf_b, vf_b, Cf_b, Ff_b, Fgf_b, advect=False):
    if not caches:
        return xf_b, vf_b, Cf_b, Ff_b, Fgf_b
    ref = caches[0].ref
    dt, dev = caches[0].x.dtype, caches[0].x.device
    bars = [to_device(a, dt, dev) for a in (xf_b, vf_b, Cf_b, Ff_b)] + [to_device(Fgf_b, torch.float64, dev)]
    for cache in reversed(caches):
        r = cache.ref
        cache.ref = bars[0]          # keep intermediate results on the device
        bars = list(step_vjp(cache, *bars, advect=advect))
        cache.ref = r
    out = [like_input(a, ref) for a in bars[:4]]
    out.append(like_input(bars[4], ref) if not isinstance(ref, torch.Tensor) else bars[4])
    return tuple(out)


def iso_growth_state(pts, g):
    st = ParticleState.rest(pts)
    if isinstance(st.Fg, torch.Tensor):
        st.Fg = g * torch.eye(3, dtype=st.Fg.dtype, device=st.Fg.device).expand_as(st.Fg).clone()
    else:
        st.Fg[:] = g * np.eye(3)
    return st


def iso_growth_grad(Fg_b):
    if isinstance(Fg_b, torch.Tensor):
        return float(torch.diagonal(Fg_b, dim1=-2, dim2=-1).sum().item())
    return float(sum(np.trace(Fg_b[p]) for p in range(len(Fg_b))))


def loss_detF(F):
    if isinstance(F, torch.Tensor):
        return float(torch.linalg.det(F.double()).sum().item())
    return float(sum(np.linalg.det(F[p]) for p in range(len(F))))


def _slab_from_points(pts_dev: torch.Tensor) -> torch.Tensor:
    n = pts_dev.shape[0]
    slab = torch.zeros(SLAB_ROWS, n, dtype=pts_dev.dtype, device=pts_dev.device)
    slab[ROW_X:ROW_X + 3] = pts_dev.t()
    for i in range(3):
        slab[ROW_F + 4 * i] = 1.0
    return slab


def check_loss(loss: str, x_obs) -> None:
    """The trajectory losses: "detF" (sum det F of the final state, the
    reference's, integrate.py:41-52) and "mse" (mean squared distance of the
    final positions to x_obs, which it needs)."""
    if loss not in ("detF", "mse"):
        raise ValueError(f"loss must be 'detF' or 'mse', not {loss!r}")
    if loss == "mse" and x_obs is None:
        raise ValueError("loss='mse' needs x_obs, the observed final positions (n, 3)")


def dloss_dg(pts, model, cfg, g, n_steps, advect, loss: str = "detF", x_obs=None,
             ckpt_every: Optional[int] = None):
    """d(loss of the final state)/dg for Fg = g I (integrate.py:45-52).
    loss="detF": sum det F_final (the reference's); loss="mse": mean
    |x_final - x_obs|^2."""
    from .trajectory import Rollout
    check_loss(loss, x_obs)
    if is_external(model):
        return _dloss_dg_steps(pts, model, cfg, g, n_steps, advect, loss, x_obs)
    if ckpt_every is None:
        ckpt_every = getattr(cfg, "checkpoint_every", None)
    p = to_device(pts, *compute_target(cfg)).contiguous()
    n = p.shape[0]
    if n == 0:
        return 0.0, 0.0     # no particles: sum det F over none
    order = cell_order_device(p, cfg.dx, cfg.grid_shape)     # memory layout only
    if order is not None:
        p = p[order].contiguous()
    plan = get_plan([scene_spec(cfg, model, n)], p.dtype, p.device)
    Fg = torch.zeros(9, n, dtype=p.dtype, device=p.device)
    for i in range(3):
        Fg[4 * i] = g
    xo = None
    if loss == "mse":
        xo_t = to_device(x_obs, p.dtype, p.device).reshape(n, 3)
        if order is not None:
            xo_t = xo_t[order]
        xo = xo_t.t().contiguous()
    ro = Rollout(plan, n_steps, advect=advect, ckpt_every=ckpt_every, Fg=Fg, loss=loss, x_obs=xo)
    ro.run(_slab_from_points(p))
    L = float(ro.loss.sum().item())
    dg = float(ro.Fg_bar[0].sum().item() + ro.Fg_bar[4].sum().item() + ro.Fg_bar[8].sum().item())
    return L, dg


def _dloss_dg_steps(pts, model, cfg, g, n_steps, advect, loss, x_obs):
    """dloss_dg through the single-step API (per-step caches, as the
    reference's rollout / rollout_vjp): the path of user-defined materials,
    whose stress is a callback evaluated every step."""
    p = to_device(pts, *compute_target(cfg)).contiguous()
    n = p.shape[0]
    if n == 0:
        return 0.0, 0.0
    st, caches = rollout(iso_growth_state(p, g), model, cfg, n_steps, advect)
    F = st.F.double()
    z3 = torch.zeros(n, 3, dtype=p.dtype, device=p.device)
    z33 = torch.zeros(n, 3, 3, dtype=p.dtype, device=p.device)
    if loss == "detF":
        L = float(torch.linalg.det(F).sum())
        Fb = (torch.linalg.det(F)[:, None, None] * torch.linalg.inv(F).transpose(1, 2)).to(p.dtype)
        xb = z3
    elif loss == "mse":
        xo = to_device(x_obs, torch.float64, p.device).reshape(n, 3)
        d = st.x.double() - xo
        L = float((d * d).sum() / n)
        xb, Fb = (2.0 * d / n).to(p.dtype), z33
    else:
        raise ValueError(loss)
    bars = rollout_vjp(caches, xb, z3, z33, Fb, torch.zeros(n, 3, 3, dtype=torch.float64, device=p.device),
                       advect)
    return L, float(torch.diagonal(bars[4], dim1=-2, dim2=-1).sum())


def lame_to_young(mu_bar: float, lam_bar: float, E: float, nu: float):
    """d/dE and d/dnu from d/dmu and d/dlambda: mu = E/(2(1+nu)),
    lambda = E nu/((1+nu)(1-2nu))."""
    dmu_dE = 1.0 / (2.0 * (1.0 + nu))
    dmu_dnu = -E / (2.0 * (1.0 + nu) ** 2)
    dlam_dE = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    dlam_dnu = E * (1.0 + 2.0 * nu * nu) / ((1.0 + nu) ** 2 * (1.0 - 2.0 * nu) ** 2)
    return mu_bar * dmu_dE + lam_bar * dlam_dE, mu_bar * dmu_dnu + lam_bar * dlam_dnu


def dloss_dparams(pts, model, cfg, g, n_steps, advect, loss: str = "detF", x_obs=None,
                  ckpt_every: Optional[int] = None):
    """Loss of the final state and its gradient with respect to the growth
    factor g (Fg = g I) and the material parameters: returns
    (L, {"g", "mu", "lam", "E", "nu"}).  The material-parameter gradients have
    no counterpart in the reference (its VJPs stop at F, Fg and C); they come
    from mpm_step_bwd_params.  Elastic models only (mu, lambda of the model)."""
    from .trajectory import Rollout
    check_loss(loss, x_obs)
    if is_external(model):
        raise TypeError("material-parameter gradients need a built-in elastic model (mu, lambda)")
    if ckpt_every is None:
        ckpt_every = getattr(cfg, "checkpoint_every", None)
    p = to_device(pts, *compute_target(cfg)).contiguous()
    n = p.shape[0]
    if n == 0:
        return 0.0, {"g": 0.0, "mu": 0.0, "lam": 0.0, "E": 0.0, "nu": 0.0}
    order = cell_order_device(p, cfg.dx, cfg.grid_shape)     # memory layout only
    if order is not None:
        p = p[order].contiguous()
    plan = get_plan([scene_spec(cfg, model, n)], p.dtype, p.device)
    Fg = torch.zeros(9, n, dtype=p.dtype, device=p.device)
    for i in range(3):
        Fg[4 * i] = g
    xo = None
    if loss == "mse":
        xo_t = to_device(x_obs, p.dtype, p.device).reshape(n, 3)
        if order is not None:
            xo_t = xo_t[order]
        xo = xo_t.t().contiguous()
    ro = Rollout(plan, n_steps, advect=advect, ckpt_every=ckpt_every, Fg=Fg, loss=loss, x_obs=xo,
                 material_grads=True)
    ro.run(_slab_from_points(p))
    L = float(ro.loss.sum().item())
    dg = float(ro.Fg_bar[0].sum().item() + ro.Fg_bar[4].sum().item() + ro.Fg_bar[8].sum().item())
    mu_b, lam_b = (float(v) for v in ro.material_grad[0].tolist())
    mu, lam = float(model.mu), float(model.lam)
    E, nu = mu * (3.0 * lam + 2.0 * mu) / (lam + mu), lam / (2.0 * (lam + mu))
    dE, dnu = lame_to_young(mu_b, lam_b, E, nu)
    return L, {"g": dg, "mu": mu_b, "lam": lam_b, "E": dE, "nu": dnu}
