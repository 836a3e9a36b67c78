"""Batched growth scenes: many instances with uneven particle counts, grids,
materials and growth parameters advanced together.

One plan holds every scene (scene table, per-scene cell/tile ranges); each
step is one launch sequence over all scenes, and the whole forward + loss +
adjoint trajectory is captured once in a CUDA graph and replayed.  Growth is
the per-scene isotropic law Fg = g_s I (growth_mode 1, g_s = 1 + A_s), so the
adjoint returns d loss / d g_s per scene, accumulated in float64.

The schedule (node-tile edge, P2G CTAs per SM, stencil offsets per pass,
particle block size) is chosen by ``autotune``, which times short forward
trajectories of the actual batch for each candidate on the current GPU.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib as L
from .runtime import Plan, SceneSpec, SLAB_ROWS, ROW_F, ROW_X
from .trajectory import Rollout, budget_schedule, sqrt_schedule
from .layout import batch_order

MODEL_KIND = {"nh": L.MODEL_NEOHOOKEAN, "hencky": L.MODEL_HENCKY, "hb": L.MODEL_HERSCHEL_BULKLEY}


def scene_spec_from_dict(s: dict, growth_mode: int = 1) -> SceneSpec:
    dx = float(s["dx"])
    sp = dx / 2.0
    return SceneSpec(shape=tuple(s["shape"]), n=int(s["x"].shape[0]), model=MODEL_KIND[s["model"]], dx=dx,
                     dt=float(s["dt"]), damping=float(s.get("damping", 0.05)),
                     pmass=float(s.get("density", 1.0)) * sp ** 3, vol0=sp ** 3, mu=float(s.get("mu", 0.0)),
                     lam=float(s.get("lam", 0.0)), hb=s.get("hb"), wall=int(s.get("wall", 0)),
                     clamp_lo=tuple(s.get("clamp_lo", (0, 0, 0))), clamp_hi=tuple(s.get("clamp_hi", (0, 0, 0))),
                     growth_mode=growth_mode, growth_A=float(s.get("growth_A", 0.0)),
                     ramp_steps=float(s.get("ramp_steps", 0)))


def host_slab(scenes: List[dict], dtype=np.float32) -> np.ndarray:
    """(24, n_total) rest-state slab of all scenes (x from the scenes, F = I)."""
    n = sum(int(s["x"].shape[0]) for s in scenes)
    slab = np.zeros((SLAB_ROWS, n), dtype=dtype)
    p = 0
    for s in scenes:
        k = s["x"].shape[0]
        slab[ROW_X:ROW_X + 3, p:p + k] = s["x"].T
        p += k
    for i in range(3):
        slab[ROW_F + 4 * i] = 1.0
    return slab


def host_phi(scenes: List[dict], dtype=np.float32) -> Optional[np.ndarray]:
    if all(s.get("phi") is None for s in scenes):
        return None
    return np.concatenate([s["phi"] if s.get("phi") is not None else np.ones(s["x"].shape[0])
                           for s in scenes]).astype(dtype)


class Batch:
    """A batch of scenes with a graph-captured forward+adjoint trajectory."""

    def __init__(self, scenes: List[dict], n_steps: int, dtype=torch.float32, advect: bool = True,
                 ckpt_every=None, tuning: Optional[dict] = None, loss: str = "detF",
                 x_obs: Optional[np.ndarray] = None, device=None, active_cap="auto",
                 memory_fraction: float = 0.75, slab_host: Optional[np.ndarray] = None,
                 material_grads: bool = False, reorder: bool = True):
        """ckpt_every: int, None (store every step), "sqrt", or "auto" (largest
        interval that fits memory_fraction of the free device memory).
        active_cap: "auto" sizes the tapes' active-tile lists from a probe
        forward run of slab_host (1.25x its maximum), None keeps every tile.
        material_grads: also accumulate d loss / d (mu, lambda) per scene
        (dloss_dmaterial, dloss_dE, dloss_dnu).
        reorder: store each scene's particles in the cell order of their
        initial positions (layout.py); inputs and the state accessors keep the
        caller's particle order."""
        from .integrate import check_loss
        check_loss(loss, x_obs)
        self.scenes = [dict(s) for s in scenes]   # set_params edits these copies
        self.n_steps = n_steps
        self.dtype = dtype
        # The plan holds the scenes grouped by material model (stable), so that
        # each model's particles are one run of slots and get the kernels
        # specialised for that model; per-scene results come back in the
        # caller's scene order.
        self.scene_perm = np.array(sorted(range(len(scenes)), key=lambda i: (MODEL_KIND[scenes[i]["model"]], i)),
                                   dtype=np.int64)
        self.specs = [scene_spec_from_dict(scenes[i]) for i in self.scene_perm]
        self.n = sum(sp.n for sp in self.specs)
        npd = np.float32 if dtype == torch.float32 else np.float64
        tuning = dict(tuning or {})
        offsets = np.concatenate([[0], np.cumsum([s["x"].shape[0] for s in scenes])]).astype(np.int64)
        # slot -> input particle
        self.order = batch_order(scenes, offsets, self.scene_perm, cell_order=reorder)
        self._scene_inv = None
        if np.any(self.scene_perm != np.arange(len(scenes))):
            self._scene_inv = torch.as_tensor(np.argsort(self.scene_perm))
        phi = host_phi(scenes, npd)
        if phi is not None and self.order is not None:
            phi = np.ascontiguousarray(phi[self.order])
        if active_cap == "auto":
            probe = Plan(self.specs, dtype=dtype, tuning=tuning, device=device)
            self._set_phi(probe, phi)
            sh = slab_host if slab_host is not None else host_slab(scenes, npd)
            if self.order is not None:
                sh = np.ascontiguousarray(np.asarray(sh)[:, self.order])
            tuning["active_tile_cap"] = self._probe_active(probe, sh, advect)
            del probe
        elif active_cap:
            tuning["active_tile_cap"] = int(active_cap)
        self.plan = Plan(self.specs, dtype=dtype, tuning=tuning, device=device)
        self.phi = self._set_phi(self.plan, phi)
        state_bytes = SLAB_ROWS * self.n * self.plan.real_bytes
        if ckpt_every == "sqrt":
            ckpt_every = sqrt_schedule(n_steps)
        elif ckpt_every == "auto":
            free, _ = torch.cuda.mem_get_info(self.plan.device)
            ckpt_every = budget_schedule(n_steps, state_bytes, self.plan.tape_bytes, int(memory_fraction * free))
        self.ckpt_every = ckpt_every or n_steps
        xo = None
        if loss == "mse":
            xob = x_obs if self.order is None else x_obs[self.order]
            xo = torch.as_tensor(np.ascontiguousarray(xob.T.astype(npd))).to(self.plan.device)
        self.rollout = Rollout(self.plan, n_steps, advect=advect, ckpt_every=self.ckpt_every, Fg=None, loss=loss,
                               x_obs=xo, material_grads=material_grads)
        self.slab0 = torch.empty(SLAB_ROWS, self.n, dtype=dtype, device=self.plan.device)
        if self._scene_inv is not None:
            self._scene_inv = self._scene_inv.to(self.plan.device)
        self.order_dev = self.inverse_dev = self._stage = None
        if self.order is not None:
            dev = self.plan.device
            self.order_dev = torch.as_tensor(self.order).to(dev)
            self.inverse_dev = torch.as_tensor(np.argsort(self.order)).to(dev)
            self._stage = torch.empty(SLAB_ROWS, self.n, dtype=dtype, device=dev)
        self._copy_stream = None      # prefetch(): side-stream input copies
        self._pending = False
        self.graph = None

    @staticmethod
    def _set_phi(plan, phi):
        if phi is None:
            return None
        t = torch.as_tensor(phi).to(plan.device)
        plan.set_growth_field(t)
        return t

    def _probe_active(self, plan, slab_host, advect) -> int:
        """Run the forward trajectory once without tapes and return a tape
        capacity of 1.25x the largest active-tile count seen (+16)."""
        from .runtime import slab_particles
        dev = plan.device
        a = torch.as_tensor(slab_host).to(dev)
        b = torch.empty_like(a)
        mx = 0
        for t in range(self.n_steps):
            plan.step_fwd(slab_particles(a), slab_particles(b), advect, t, None, chained=t > 0,
                          emit=t + 1 < self.n_steps)
            mx = max(mx, plan.active_tiles(None))
            a, b = b, a
        return int(1.25 * mx) + 16

    def particle_steps(self) -> int:
        return self.n * self.n_steps

    def load(self, slab_host: np.ndarray, non_blocking=True):
        """Copy a (24, n) host slab (pinned for async) into the device input;
        it replaces a prefetched input that no run has taken yet."""
        src = torch.from_numpy(slab_host) if isinstance(slab_host, np.ndarray) else slab_host
        self._pending = False
        if self.order is None:
            self.slab0.copy_(src, non_blocking=non_blocking)
        else:
            # the caller's particle order -> the batch's cell order, on the device
            self._stage.copy_(src, non_blocking=non_blocking)
            torch.index_select(self._stage, 1, self.order_dev, out=self.slab0)

    def prefetch(self, slab_host):
        """Start the host -> device copy of the next trajectory's (24, n) host
        slab (pinned) on a side stream, so that it overlaps the trajectory that
        is running; the next run() / replay() waits for it and moves it into
        the input, in the batch's cell order.  The host slab must stay
        unchanged until that run starts."""
        src = torch.from_numpy(slab_host) if isinstance(slab_host, np.ndarray) else slab_host
        dev = self.plan.device
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(device=dev)
            self._inbox = torch.empty(SLAB_ROWS, self.n, dtype=self.dtype, device=dev)
            self._inbox_ready = torch.cuda.Event()
            self._inbox_free = torch.cuda.Event()
            self._inbox_free.record(torch.cuda.current_stream(dev))
        cs = self._copy_stream
        cs.wait_event(self._inbox_free)          # the previous prefetch has been taken
        with torch.cuda.stream(cs):
            self._inbox.copy_(src, non_blocking=True)
            self._inbox_ready.record(cs)
        self._pending = True

    def _take_prefetched(self):
        if not self._pending:
            return
        cur = torch.cuda.current_stream(self.plan.device)
        cur.wait_event(self._inbox_ready)
        if self.order is None:
            self.slab0.copy_(self._inbox)
        else:
            torch.index_select(self._inbox, 1, self.order_dev, out=self.slab0)
        self._inbox_free.record(cur)
        self._pending = False

    def _to_input_order(self, slab: torch.Tensor) -> torch.Tensor:
        if self.order is None:
            return slab
        return torch.index_select(slab, 1, self.inverse_dev)

    def final_state(self) -> torch.Tensor:
        """(24, n) final state of the last trajectory, in the caller's particle order."""
        return self._to_input_order(self.rollout.final)

    def initial_cotangents(self) -> torch.Tensor:
        """(24, n) d loss / d (initial state) of the last trajectory, in the
        caller's particle order."""
        return self._to_input_order(self.rollout.bar0)

    def run(self):
        self._take_prefetched()
        return self.rollout.run(self.slab0)

    def capture(self, pre_capture=None):
        self.graph = self.rollout.capture(self.slab0, pre_capture)
        return self.graph

    def replay(self):
        self._take_prefetched()
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def _scene_order(self, t: torch.Tensor) -> torch.Tensor:
        """Per-scene values of the plan (grouped by model) in the caller's scene order."""
        return t if self._scene_inv is None else torch.index_select(t, 0, self._scene_inv)

    @property
    def loss(self) -> torch.Tensor:
        return self._scene_order(self.rollout.loss)

    @property
    def dloss_dg(self) -> torch.Tensor:
        """d loss_s / d g_s (growth law g_s = 1 + A_s, so d/dA = d/dg)."""
        return self._scene_order(self.rollout.growth_grad)

    @property
    def dloss_dmaterial(self) -> torch.Tensor:
        """(S, 2): d loss_s / d mu_s, d loss_s / d lambda_s (material_grads=True)."""
        return self._scene_order(self.rollout.material_grad)

    def dloss_dE_nu(self) -> np.ndarray:
        """(S, 2) on the host: d loss_s / d E_s, d loss_s / d nu_s."""
        from .integrate import lame_to_young
        mg = self.dloss_dmaterial.cpu().numpy()
        out = np.zeros_like(mg)
        for s, sc in enumerate(self.scenes):
            out[s] = lame_to_young(mg[s, 0], mg[s, 1], float(sc["E"]), float(sc["nu"]))
        return out

    def set_params(self, growth_A=None, E=None, nu=None):
        """New per-scene growth amplitudes and/or Young's moduli and Poisson
        ratios (arrays of length S) for the same batch; the captured graph
        replays with them (mpm_plan_update_scenes)."""
        for s, sc in enumerate(self.scenes):
            if growth_A is not None:
                sc["growth_A"] = float(growth_A[s])
            if E is not None:
                sc["E"] = float(E[s])
            if nu is not None:
                sc["nu"] = float(nu[s])
            if E is not None or nu is not None:
                sc["mu"] = sc["E"] / (2.0 * (1.0 + sc["nu"]))
                sc["lam"] = sc["E"] * sc["nu"] / ((1.0 + sc["nu"]) * (1.0 - 2.0 * sc["nu"]))
        self.specs = [scene_spec_from_dict(self.scenes[i]) for i in self.scene_perm]
        self.plan.update_scenes(self.specs)


# ---------------------------------------------------------------------------
# autotuner
# ---------------------------------------------------------------------------
CANDIDATES = {
    "tile_xy": [4, 8],
    "tile_z": [4, 8, 16],
    "scatter_ctas_per_sm": [1, 2],
    "scatter_oxb": [1, 3],
    "particle_block": [128, 256],
}
TUNE_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")


def _signature(scenes: List[dict], dtype) -> str:
    n = sum(int(s["x"].shape[0]) for s in scenes)
    g = sum(int(np.prod(s["shape"])) for s in scenes)
    return f"{len(scenes)}s-{n}p-{g}g-{str(dtype).split('.')[-1]}"


def _gpu_name() -> str:
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "none"


def load_tuned(scenes: List[dict], dtype) -> Optional[dict]:
    try:
        table = json.load(open(TUNE_CACHE))
    except Exception:
        return None
    return table.get(_gpu_name(), {}).get(_signature(scenes, dtype))


def autotune(scenes: List[dict], dtype=torch.float32, steps: int = 4, budget_s: float = 90.0,
             save: bool = False, verbose: bool = False) -> Dict:
    """Time a `steps`-step forward + adjoint trajectory of the batch for every
    candidate schedule (coordinate search: one knob at a time, starting from
    the defaults) and return the fastest.  Results are deterministic whatever
    the schedule (the summation order per node does not depend on it)."""
    t_start = time.time()
    best = {"tile_xy": 4, "tile_z": 4, "scatter_ctas_per_sm": 1, "scatter_oxb": 3 if dtype == torch.float32 else 1,
            "particle_block": 256}
    slab = torch.as_tensor(host_slab(scenes, np.float32 if dtype == torch.float32 else np.float64))

    def measure(cfg):
        b = Batch(scenes, steps, dtype=dtype, tuning=cfg, ckpt_every=steps, active_cap=None)
        b.load(slab.to(b.plan.device), non_blocking=False)
        ro = b.rollout
        ro.run(b.slab0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ro.run(b.slab0)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    results = {}
    t_best = measure(best)
    results[json.dumps(best, sort_keys=True)] = t_best
    for knob, vals in CANDIDATES.items():
        for v in vals:
            if time.time() - t_start > budget_s:
                break
            if dtype == torch.float64 and knob == "scatter_oxb" and v == 3:
                continue
            cfg = dict(best, **{knob: v})
            key = json.dumps(cfg, sort_keys=True)
            if key in results:
                continue
            t = measure(cfg)
            results[key] = t
            if verbose:
                print(f"autotune {cfg} {t:.3f} ms", flush=True)
            if t < t_best:
                best, t_best = cfg, t
    if save:
        try:
            table = json.load(open(TUNE_CACHE))
        except Exception:
            table = {}
        table.setdefault(_gpu_name(), {})[_signature(scenes, dtype)] = best
        json.dump(table, open(TUNE_CACHE, "w"), indent=1, sort_keys=True)
    return dict(best, _ms=t_best)


def main():
    """python -m morphompm_b200.batch --autotune [--scenes 256] [--budget 120]:
    tune the config-4 batch on this GPU and store the schedule in tuned.json."""
    import argparse
    from . import scenes as S
    ap = argparse.ArgumentParser()
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--budget", type=float, default=120.0)
    ap.add_argument("--dtype", default="float32", choices=["float32", "float64"])
    a = ap.parse_args()
    if a.autotune:
        dt = torch.float32 if a.dtype == "float32" else torch.float64
        best = autotune(S.config4(n_scenes=a.scenes), dt, budget_s=a.budget, save=True, verbose=True)
        print(json.dumps(best))


if __name__ == "__main__":
    main()
