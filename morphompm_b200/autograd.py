"""torch.autograd entry points over the hand-written adjoints.

``step``          one MLS-MPM growth step as a differentiable function of the
                  particle state (x, v, C, F, Fg); its backward is
                  ``transfer.step_vjp`` (transfer.py:82-158 of the reference).
                  Chaining calls builds an ordinary autograd graph.
``rollout_loss``  a whole trajectory from the rest state at positions x0 with
                  growth Fg = g I (scalar g) or a per-particle Fg, reduced to
                  the loss of its final state (sum det F, as integrate.py:41-52,
                  or the mean squared position error); one autograd node whose
                  backward is the device adjoint of ``trajectory.Rollout``
                  (checkpoint-every-k recompute), giving d loss/d x0 and
                  d loss/d g (or d loss/d Fg).

Tensors are CUDA tensors, float64 (the plain path) or float32.
"""
from __future__ import annotations

from typing import Optional

import torch

from .layout import cell_order_device
from .runtime import ROW_X
from .state import ParticleState


class _Step(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, C, F, Fg, model, cfg, advect, t):
        from . import transfer
        st = ParticleState(x.detach(), v.detach(), C.detach(), F.detach(), Fg.detach())
        new, cache = transfer.step(st, model, cfg, advect=advect, t=t)
        ctx.cache = cache
        ctx.advect = advect
        ctx.fg_dtype = Fg.dtype
        return new.x, new.v, new.C, new.F

    @staticmethod
    def backward(ctx, xb, vb, Cb, Fb):
        from . import transfer
        c = ctx.cache
        z = lambda a, ref: a if a is not None else torch.zeros_like(ref)
        xb, vb, Cb, Fb = z(xb, c.x), z(vb, c.v), z(Cb, c.C), z(Fb, c.F)
        Fg_out_b = torch.zeros(c.Fg.shape, dtype=torch.float64, device=c.Fg.device)   # Fg is not an output
        gx, gv, gC, gF, gFg = transfer.step_vjp(c, xb, vb, Cb, Fb, Fg_out_b, advect=ctx.advect)
        return gx, gv, gC, gF, gFg.to(ctx.fg_dtype), None, None, None, None


def step(x, v, C, F, Fg, model, cfg, advect: bool = True, t: int = 0):
    """(x, v, C, F) of the next step; differentiable in all five inputs.
    With advect=False, x is a frozen input and its gradient is zero
    (transfer.py:83-86)."""
    return _Step.apply(x, v, C, F, Fg, model, cfg, bool(advect), int(t))


class _RolloutLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, growth, model, cfg, n_steps, advect, loss, x_obs, ckpt_every):
        from .integrate import _slab_from_points
        from .trajectory import Rollout
        from .transfer import get_plan, scene_spec
        p = x0.detach().contiguous()
        n = p.shape[0]
        order = cell_order_device(p, cfg.dx, cfg.grid_shape)     # memory layout only
        if order is not None:
            p = p[order].contiguous()
        plan = get_plan([scene_spec(cfg, model, n)], p.dtype, p.device)
        g = growth.detach()
        if g.dim() == 0:
            Fg = torch.zeros(9, n, dtype=p.dtype, device=p.device)
            for i in range(3):
                Fg[4 * i] = g.to(p.dtype)
        else:
            gp = g.to(p.dtype).reshape(n, 9)
            Fg = (gp if order is None else gp[order]).t().contiguous()
        xo = None
        if loss == "mse":
            xo = x_obs.detach().to(device=p.device, dtype=p.dtype).reshape(n, 3)
            xo = (xo if order is None else xo[order]).t().contiguous()
        ro = Rollout(plan, n_steps, advect=advect, ckpt_every=ckpt_every, Fg=Fg, loss=loss, x_obs=xo)
        ro.forward(_slab_from_points(p))
        ro.seed()
        ctx.ro = ro
        ctx.order = order
        ctx.scalar_g = g.dim() == 0
        ctx.g_dtype = growth.dtype
        return ro.loss.sum().to(p.dtype)

    @staticmethod
    def backward(ctx, gL):
        ro = ctx.ro
        bar0 = ro.backward()
        n = ro.plan.n
        gx = (bar0[ROW_X:ROW_X + 3].t() * gL).contiguous()
        Fg_b = ro.Fg_bar.t().reshape(n, 3, 3) * gL.double()
        if ctx.order is not None:
            # back to the caller's particle order
            gx = torch.empty_like(gx).index_copy_(0, ctx.order, gx)
            Fg_b = torch.empty_like(Fg_b).index_copy_(0, ctx.order, Fg_b)
        gg = (Fg_b[:, 0, 0] + Fg_b[:, 1, 1] + Fg_b[:, 2, 2]).sum() if ctx.scalar_g else Fg_b
        ctx.ro = None
        ctx.order = None
        return gx, gg.to(ctx.g_dtype), None, None, None, None, None, None, None


def rollout_loss(x0, growth, model, cfg, n_steps: int, advect: bool = True, loss: str = "detF",
                 x_obs: Optional[torch.Tensor] = None, ckpt_every: Optional[int] = None):
    """Loss of the final state of an n_steps trajectory from the rest state at
    x0 (n, 3) with Fg = growth I (0-d tensor) or growth (n, 3, 3); the same
    functional as ``integrate.dloss_dg``, differentiable in x0 and growth."""
    from .integrate import check_loss
    check_loss(loss, x_obs)
    if not isinstance(growth, torch.Tensor):
        growth = torch.tensor(float(growth), dtype=x0.dtype, device=x0.device)
    if ckpt_every is None:
        ckpt_every = getattr(cfg, "checkpoint_every", None)
    return _RolloutLoss.apply(x0, growth, model, cfg, int(n_steps), bool(advect), loss, x_obs, ckpt_every)
