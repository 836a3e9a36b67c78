"""Full-trajectory forward and adjoint on the device with checkpoint-every-k
recomputation (the reference keeps every step's cache in RAM,
python/morphompm/integrate.py:15-28; this engine keeps one state per segment
and recomputes a segment's k states and tapes just before reversing it).

States are (24, n) slabs (runtime.py); cotangent slabs have the same layout.
The Fg cotangent is a (9, n) float64 slab (explicit growth) or, for scenes in
growth-law mode, the per-scene d loss / d A accumulated in float64.

Everything a trajectory needs is allocated up front, so a whole
forward+adjoint can be captured once in a CUDA graph and replayed
(``Rollout.capture``).
"""
from __future__ import annotations

import math
from typing import List, Optional

import torch

from . import _lib as L
from .runtime import Plan, SLAB_ROWS, ROW_F, ROW_X, slab_cotangents, slab_particles, stream_ptr


def sqrt_schedule(n_steps: int) -> int:
    """Checkpoint interval of the sqrt(N) schedule."""
    return max(1, int(math.ceil(math.sqrt(n_steps))))


def budget_schedule(n_steps: int, state_bytes: int, tape_bytes: int, budget: int) -> int:
    """Largest checkpoint interval k whose storage fits the byte budget:
    ceil(N/k) checkpoints + (k+1) segment states + k tapes (k = N stores every
    step and needs no recompute)."""
    best = 1
    for k in range(1, n_steps + 1):
        need = ((n_steps + k - 1) // k + k + 1 + 5) * state_bytes + k * tape_bytes
        if need <= budget:
            best = k
    return best


class Rollout:
    """One batch (plan) rolled for n_steps with checkpoints every ``ckpt_every``.

    Fg: (9, n) slab for explicit growth (growth_mode 0 scenes), or None when
    every scene follows its growth law.
    """

    def __init__(self, plan: Plan, n_steps: int, advect: bool = True, ckpt_every: Optional[int] = None,
                 Fg: Optional[torch.Tensor] = None, loss: str = "detF", x_obs: Optional[torch.Tensor] = None,
                 material_grads: bool = False):
        if any(int(sc.model) == L.MODEL_EXTERNAL for sc in plan.scenes):
            raise TypeError("user-defined materials run through transfer.step / integrate.rollout "
                            "(their stress is a callback evaluated every step)")
        self.plan = plan
        self.n_steps = int(n_steps)
        self.advect = bool(advect)
        self.k = int(ckpt_every) if ckpt_every else self.n_steps
        self.k = max(1, min(self.k, self.n_steps))
        self.n_seg = (self.n_steps + self.k - 1) // self.k
        n, dt, dev = plan.n, plan.dtype, plan.device
        self.Fg = Fg
        self.loss_kind = loss
        self.x_obs = x_obs
        self.recompute = self.k < self.n_steps
        # checkpoints (state at the start of every segment) + final state
        self.ckpt = [torch.empty(SLAB_ROWS, n, dtype=dt, device=dev) for _ in range(self.n_seg)]
        # per-segment states t0..t0+k and tapes t0..t0+k-1
        self.seg_states = [torch.empty(SLAB_ROWS, n, dtype=dt, device=dev) for _ in range(self.k + 1)]
        self.tapes = [plan.new_tape() for _ in range(self.k)]
        self.final = torch.empty(SLAB_ROWS, n, dtype=dt, device=dev)
        self.scratch = [torch.empty(SLAB_ROWS, n, dtype=dt, device=dev) for _ in range(2)]
        self.bars = [torch.empty(SLAB_ROWS, n, dtype=dt, device=dev) for _ in range(2)]
        self.Fg_bar = torch.zeros(9, n, dtype=torch.float64, device=dev) if Fg is not None else None
        S = len(plan.scenes)
        self.loss = torch.zeros(S, dtype=torch.float64, device=dev)
        self.growth_grad = torch.zeros(S, dtype=torch.float64, device=dev)
        # d loss / d (mu, lambda) per scene, when asked for
        self.material_grad = torch.zeros(S, 2, dtype=torch.float64, device=dev) if material_grads else None
        self.bar0 = None
        self.graph = None

    def memory_bytes(self) -> int:
        es = self.plan.real_bytes
        n = self.plan.n
        slabs = len(self.ckpt) + len(self.seg_states) + 1 + 4
        return slabs * SLAB_ROWS * n * es + len(self.tapes) * self.plan.tape_bytes

    # -- forward --------------------------------------------------------------
    def _pp(self, slab):
        return slab_particles(slab, self.Fg)

    def forward(self, slab0: torch.Tensor, stream=None) -> torch.Tensor:
        """Run all steps from slab0; keeps the segment checkpoints.  When no
        recompute is needed (k == n_steps), the tapes of the single segment are
        recorded on the way."""
        p = self.plan
        self.ckpt[0].copy_(slab0)
        if not self.recompute:
            cur = self.seg_states[0]
            cur.copy_(slab0)
            for t in range(self.n_steps):
                nxt = self.seg_states[t + 1]
                p.step_fwd(self._pp(cur), self._pp(nxt), self.advect, t, self.tapes[t], stream,
                           chained=t > 0, emit=t + 1 < self.n_steps)
                cur = nxt
            self.final.copy_(cur)
            return self.final
        cur = self.ckpt[0]
        for t in range(self.n_steps):
            if t + 1 == self.n_steps:
                nxt = self.final
            elif (t + 1) % self.k == 0:
                nxt = self.ckpt[(t + 1) // self.k]
            else:
                nxt = self.scratch[t % 2] if cur is not self.scratch[t % 2] else self.scratch[(t + 1) % 2]
            p.step_fwd(self._pp(cur), self._pp(nxt), self.advect, t, None, stream,
                       chained=t > 0, emit=t + 1 < self.n_steps)
            cur = nxt
        return self.final

    # -- loss -----------------------------------------------------------------
    def seed(self, stream=None):
        """Loss of the final state and its cotangent slab (bars[0])."""
        p = self.plan
        n = p.n
        es = self.final.element_size()
        b = self.bars[0]
        b.zero_()
        if self.Fg_bar is not None:
            self.Fg_bar.zero_()
        if self.loss_kind == "detF":
            p.loss_detF(self.final.data_ptr() + ROW_F * n * es, 1, n, self.loss, b.data_ptr() + ROW_F * n * es,
                        stream)
        elif self.loss_kind == "mse":
            p.loss_mse(self.final.data_ptr() + ROW_X * n * es, 1, n, self.x_obs.data_ptr(), self.loss,
                       b.data_ptr() + ROW_X * n * es, stream)
        else:
            raise ValueError(self.loss_kind)
        return b

    # -- adjoint --------------------------------------------------------------
    def backward(self, bar_T: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """Reverse sweep from cotangent slab bar_T (defaults to the loss seed in
        bars[0]); returns the cotangent slab of the initial state."""
        p = self.plan
        if bar_T is not None and bar_T is not self.bars[0]:
            self.bars[0].copy_(bar_T)
        self.growth_grad.zero_()
        if self.material_grad is not None:
            self.material_grad.zero_()
        cur_bar, nxt_bar = self.bars[0], self.bars[1]
        for seg in range(self.n_seg - 1, -1, -1):
            t0 = seg * self.k
            t1 = min(self.n_steps, t0 + self.k)
            if self.recompute:
                st = self.seg_states
                st[0].copy_(self.ckpt[seg])
                for t in range(t0, t1):
                    j = t - t0
                    p.step_fwd(self._pp(st[j]), self._pp(st[j + 1]), self.advect, t, self.tapes[j], stream,
                               chained=t > t0, emit=t + 1 < t1)
            for t in range(t1 - 1, t0 - 1, -1):
                j = t - t0
                s_in = self.seg_states[j]
                s_out = self.seg_states[j + 1]
                n = p.n
                es = s_out.element_size()
                p.step_bwd(self._pp(s_in), s_out.data_ptr() + 6 * n * es,
                           slab_cotangents(cur_bar, self.Fg_bar), slab_cotangents(nxt_bar, self.Fg_bar),
                           self.growth_grad, self.advect, t, self.tapes[j], stream,
                           material_grad=self.material_grad)
                cur_bar, nxt_bar = nxt_bar, cur_bar
        self.bar0 = cur_bar
        return cur_bar

    # -- graph capture ----------------------------------------------------------
    def run(self, slab0: torch.Tensor, stream=None):
        self.forward(slab0, stream)
        self.seed(stream)
        return self.backward(None, stream)

    def capture(self, slab0: torch.Tensor, pre_capture=None):
        """Capture forward + loss + adjoint from the fixed input slab0 into one
        CUDA graph (replay with ``replay()``).  ``pre_capture`` runs after the
        eager warm-up, just before capture begins."""
        self._graph_in = slab0
        s = torch.cuda.Stream(device=self.plan.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run(slab0)          # warm-up outside the graph (loads, attributes)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        if pre_capture is not None:
            pre_capture()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(slab0)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()
        return self.bar0
