"""[3] Transfer seam -- one MLS-MPM growth step and its hand-written VJP, with
the reference's signatures (python/morphompm/transfer.py:33,82):

    step(state, model, cfg, advect=True)                    -> (state', cache)
    step_vjp(cache, xn_b, vn_b, Cn_b, Fn_b, Fgn_b, advect)   -> (x_b, v_b, C_b, F_b, Fg_b)

Both run as sm_100a kernels behind the C ABI (``mpm_step_fwd`` /
``mpm_step_bwd``): cell binning and a deterministic radix sort, the stress
prepass, atomic-free P2G into node tiles with the grid update fused, G2P with
advection and the F update; and in reverse the G2P adjoint scatter, grid
adjoint, P2G adjoint with the constitutive VJP and the volume path.

Contract kept from the reference: inputs are never mutated, outputs are fresh
arrays, Fg is copied, the cache is opaque, and with advect=False x is frozen
and x_b is returned as 0 (transfer.py:83-86).  numpy inputs run in FP64 and
return numpy; torch CUDA tensors stay on the device in their own dtype.  Fg_b
is always float64 (it carries the growth-parameter gradient).
"""
from __future__ import annotations

import os
from collections import OrderedDict

import torch

from . import _lib as L
from .constitutive import is_external, model_fields
from .config import compute_target
from .devarray import like_input, to_device
from .runtime import Plan, SceneSpec, aos_cotangents, aos_particles
from .state import ParticleState

_PLAN_CACHE: "OrderedDict[tuple, Plan]" = OrderedDict()
_PLAN_CACHE_MAX = 16
STRICT = os.environ.get("MORPHOMPM_STRICT", "0") == "1"


def scene_spec(cfg, model, n: int, **extra) -> SceneSpec:
    f = model_fields(model)
    return SceneSpec(shape=cfg.grid_shape, n=n, dx=cfg.dx, dt=cfg.dt, damping=cfg.damping, pmass=cfg.pmass,
                     vol0=cfg.vol0, mass_eps=cfg.mass_eps, gravity=tuple(cfg.gravity), wall=cfg.wall,
                     clamp_lo=tuple(cfg.clamp_lo), clamp_hi=tuple(cfg.clamp_hi), **f, **extra)


def _key(spec: SceneSpec):
    d = dict(spec.__dict__)
    d["hb"] = tuple(sorted(d["hb"].items())) if d.get("hb") else None
    return tuple((k, tuple(v) if isinstance(v, (list, tuple)) else v) for k, v in sorted(d.items()))


def get_plan(specs, dtype, device, tuning=None) -> Plan:
    key = (tuple(_key(s) for s in specs), dtype, str(device), tuple(sorted((tuning or {}).items())))
    p = _PLAN_CACHE.get(key)
    if p is not None:
        _PLAN_CACHE.move_to_end(key)
        return p
    p = Plan(list(specs), dtype=dtype, tuning=tuning, device=device)
    _PLAN_CACHE[key] = p
    while len(_PLAN_CACHE) > _PLAN_CACHE_MAX:
        _PLAN_CACHE.popitem(last=False)
    return p


class StepCache:
    """Opaque record of one forward step (the reference's cache tuple)."""
    __slots__ = ("plan", "tape", "x", "v", "C", "F", "Fg", "Cn", "advect", "ref", "t", "model", "tau")

    def __init__(self, **kw):
        for k, v in kw.items():
            setattr(self, k, v)


def _check(plan: Plan):
    if STRICT:
        st = plan.status()
        if st & (L.MPM_ERR_NONFINITE | L.MPM_ERR_ARG):
            raise L.MpmError(st, "step")


def _check_shapes(state: ParticleState):
    """x, v: (n, 3); C, F, Fg: (n, 3, 3) -- the reference's layout (state.py:11-21)."""
    n = tuple(state.x.shape)[0] if len(tuple(state.x.shape)) == 2 else None
    want = {"x": (n, 3), "v": (n, 3), "C": (n, 3, 3), "F": (n, 3, 3), "Fg": (n, 3, 3)}
    for k, w in want.items():
        got = tuple(getattr(state, k).shape)
        if n is None or got != w:
            raise ValueError(f"ParticleState.{k} has shape {got}, expected {w if n is not None else '(n, 3)'}")


def step(state: ParticleState, model, cfg, advect=True, t: int = 0):
    _check_shapes(state)
    ref = state.x
    want_dt, want_dev = compute_target(cfg)
    x = to_device(state.x, want_dt, want_dev).contiguous()
    dev, dt = x.device, x.dtype
    v = to_device(state.v, dt, dev).contiguous()
    Cm = to_device(state.C, dt, dev).contiguous()
    F = to_device(state.F, dt, dev).contiguous()
    Fg = to_device(state.Fg, dt, dev).contiguous()
    n = x.shape[0]
    if n == 0:
        # no particles: an empty grid, nothing moves (transfer.py:33-79 loops over none)
        new = ParticleState(*(like_input(a.clone(), ref) for a in (x, v, Cm, F, Fg)))
        return new, StepCache(plan=None, tape=None, x=x, v=v, C=Cm, F=F, Fg=Fg, Cn=Cm, advect=bool(advect),
                              ref=ref, t=t, model=model, tau=None)
    plan = get_plan([scene_spec(cfg, model, n)], dt, dev)
    xn, vn = torch.empty_like(x), torch.empty_like(v)
    Cn, Fn, Fgn = torch.empty_like(Cm), torch.empty_like(F), torch.empty_like(Fg)
    tape = plan.new_tape()
    tau = None
    if is_external(model):
        # a user-defined material: its batched stress, consumed by the kernels
        tau = to_device(model.stress(F, Fg, Cm), dt, dev).reshape(n, 3, 3).contiguous()
        plan.set_external_stress(tau, None)
    plan.step_fwd(aos_particles(x, v, Cm, F, Fg), aos_particles(xn, vn, Cn, Fn, Fgn), advect, t, tape)
    if tau is not None:
        plan.set_external_stress(None, None)
    _check(plan)
    new = ParticleState(*(like_input(a, ref) for a in (xn, vn, Cn, Fn, Fgn)))
    cache = StepCache(plan=plan, tape=tape, x=x, v=v, C=Cm, F=F, Fg=Fg, Cn=Cn, advect=bool(advect), ref=ref, t=t,
                      model=model, tau=tau)
    return new, cache


def step_vjp(cache: StepCache, xn_b, vn_b, Cn_b, Fn_b, Fgn_b, advect=True):
    """Reverse of ``step``.  CONTRACT (transfer.py:83-86): with advect=False, x is
    a frozen input and x_b is returned as 0."""
    plan = cache.plan
    dt, dev = cache.x.dtype, cache.x.device
    if plan is None:
        # the step of an empty state: empty cotangents
        ref = cache.ref
        out = [like_input(torch.zeros_like(a), ref) for a in (cache.x, cache.v, cache.C, cache.F)]
        Fgb = torch.zeros(cache.Fg.shape, dtype=torch.float64, device=dev)
        out.append(like_input(Fgb, ref) if not isinstance(ref, torch.Tensor) else Fgb)
        return tuple(out)
    xb_in = to_device(xn_b, dt, dev).contiguous()
    vb_in = to_device(vn_b, dt, dev).contiguous()
    Cb_in = to_device(Cn_b, dt, dev).contiguous()
    Fb_in = to_device(Fn_b, dt, dev).contiguous()
    Fgb_in = to_device(Fgn_b, torch.float64, dev).contiguous()
    xb, vb = torch.empty_like(xb_in), torch.empty_like(vb_in)
    Cb, Fb = torch.empty_like(Cb_in), torch.empty_like(Fb_in)
    Fgb = torch.empty_like(Fgb_in)
    tau_bar = None
    if cache.tau is not None:
        tau_bar = torch.zeros_like(cache.tau)
        plan.set_external_stress(cache.tau, tau_bar)
    plan.step_bwd(aos_particles(cache.x, cache.v, cache.C, cache.F, cache.Fg), cache.Cn.data_ptr(),
                  aos_cotangents(xb_in, vb_in, Cb_in, Fb_in, Fgb_in), aos_cotangents(xb, vb, Cb, Fb, Fgb),
                  None, advect, cache.t, cache.tape)
    if tau_bar is not None:
        plan.set_external_stress(None, None)
        # the user material's own VJP of the stress it supplied
        F_s, Fg_s, C_s = cache.model.stress_vjp(cache.F, cache.Fg, cache.C, tau_bar)
        n = cache.F.shape[0]
        Fb += to_device(F_s, dt, dev).reshape(n, 3, 3)
        Fgb += to_device(Fg_s, torch.float64, dev).reshape(n, 3, 3)
        if C_s is not None:
            Cb += to_device(C_s, dt, dev).reshape(n, 3, 3)
    _check(plan)
    ref = cache.ref
    out = [like_input(a, ref) for a in (xb, vb, Cb, Fb)]
    out.append(like_input(Fgb, ref) if not isinstance(ref, torch.Tensor) else Fgb)
    return tuple(out)
