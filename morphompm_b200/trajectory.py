"""Full-trajectory forward and adjoint on the device with checkpoint-every-k
recomputation (the reference keeps every step's cache in RAM,
python/morphompm/integrate.py:15-28; this engine keeps one state per segment
and recomputes a segment's k states and tapes just before reversing it).  The
step loops run natively behind the C ABI (mpm_rollout_fwd / mpm_rollout_bwd);
this class owns their device buffers, the loss seed and graph capture.

States are (24, n) slabs (runtime.py); cotangent slabs have the same layout.
The Fg cotangent is a (9, n) float64 slab (explicit growth) or, for scenes in
growth-law mode, the per-scene d loss / d A accumulated in float64.

Everything a trajectory needs is allocated up front, so a whole
forward+adjoint can be captured once in a CUDA graph and replayed
(``Rollout.capture``).
"""
from __future__ import annotations

import math
from typing import Optional

import torch

from . import _lib as L
from .runtime import Plan, SLAB_ROWS, ROW_F, ROW_X


def sqrt_schedule(n_steps: int) -> int:
    """Checkpoint interval of the sqrt(N) schedule."""
    return max(1, int(math.ceil(math.sqrt(n_steps))))


def budget_schedule(n_steps: int, state_bytes: int, tape_bytes: int, budget: int) -> int:
    """Largest checkpoint interval k whose storage fits the byte budget:
    (k+1) segment states, 2 cotangent slabs, the final state, the loss seed
    and the initial-state cotangents, k tapes, and with recompute (k < N)
    ceil(N/k) checkpoints and 2 scratch states (k = N stores every step)."""
    best = 1
    for k in range(1, n_steps + 1):
        extra = (n_steps + k - 1) // k + 2 if k < n_steps else 0
        need = (extra + k + 1 + 5) * state_bytes + k * tape_bytes
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
        # the checkpoints, segment states, tapes and cotangent ping-pong of the
        # native trajectory engine (mpm_rollout_fwd / mpm_rollout_bwd)
        self.ws_bytes = plan.rollout_workspace_bytes(self.n_steps, self.k)
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=dev)
        self.ws_ptr = (self.ws.data_ptr() + 255) // 256 * 256
        self.final = torch.empty(SLAB_ROWS, n, dtype=dt, device=dev)
        self.seed_bar = torch.empty(SLAB_ROWS, n, dtype=dt, device=dev)     # loss seed: final-state cotangents
        self.bar0_buf = torch.empty(SLAB_ROWS, n, dtype=dt, device=dev)     # initial-state cotangents
        self.Fg_bar = torch.zeros(9, n, dtype=torch.float64, device=dev) if Fg is not None else None
        S = len(plan.scenes)
        self.loss = torch.zeros(S, dtype=torch.float64, device=dev)
        self.growth_grad = torch.zeros(S, dtype=torch.float64, device=dev)
        # d loss / d (mu, lambda) per scene, when asked for
        self.material_grad = torch.zeros(S, 2, dtype=torch.float64, device=dev) if material_grads else None
        self.bar0 = None
        self.graph = None

    def memory_bytes(self) -> int:
        return self.ws_bytes + 3 * SLAB_ROWS * self.plan.n * self.plan.real_bytes

    # -- forward --------------------------------------------------------------
    def forward(self, slab0: torch.Tensor, stream=None) -> torch.Tensor:
        """Run all steps from slab0 (mpm_rollout_fwd); keeps the segment
        checkpoints, or, when no recompute is needed (k == n_steps), every
        state and tape of the single segment."""
        self.plan.rollout_fwd(slab0, self.Fg, self.n_steps, self.k, self.advect, self.ws_ptr, self.final, stream)
        return self.final

    # -- loss -----------------------------------------------------------------
    def seed(self, stream=None):
        """Loss of the final state and its cotangent slab."""
        p = self.plan
        n = p.n
        es = self.final.element_size()
        b = self.seed_bar
        b.zero_()
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
        """Reverse sweep (mpm_rollout_bwd) from cotangent slab bar_T (defaults
        to the loss seed); returns the cotangent slab of the initial state.
        Fg_bar, growth_grad and material_grad receive this trajectory's sums."""
        self.plan.rollout_bwd(self.Fg, bar_T if bar_T is not None else self.seed_bar, self.n_steps, self.k,
                              self.advect, self.ws_ptr, self.bar0_buf, self.Fg_bar, self.growth_grad,
                              self.material_grad, stream)
        self.bar0 = self.bar0_buf
        return self.bar0

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
