"""Device runtime around the C ABI: batch plans, workspaces, tapes and the
device particle layout.  torch provides device memory and streams only; all
arithmetic runs in the library's sm_100a kernels.

Device state layout ("slab"): one (24, n) tensor per state, rows
x(3) v(3) C(9) F(9), component-major so every kernel access is coalesced
(element (p, c) of a 3x3 field at row 6+c / 15+c, column p).  Fg (explicit
growth) lives in its own (9, n) slab since it does not change along a
trajectory.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import torch

from . import _lib as L

ROW_X, ROW_V, ROW_C, ROW_F = 0, 3, 6, 15
SLAB_ROWS = 24


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("morphompm_b200 needs a CUDA device (sm_100a); there is no CPU fallback")


def dtype_bytes(dtype) -> int:
    if dtype == torch.float32:
        return 4
    if dtype == torch.float64:
        return 8
    raise TypeError(f"unsupported dtype {dtype} (float32 or float64)")


def _ptr(t: Optional[torch.Tensor]) -> int:
    return t.data_ptr() if t is not None else 0


def stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


@dataclass
class SceneSpec:
    """One scene of a batch (fields of the C struct MpmScene)."""
    shape: Sequence[int]
    n: int
    model: int
    dx: float
    dt: float
    damping: float
    pmass: float
    vol0: float
    mu: float = 0.0
    lam: float = 0.0
    hb: Optional[dict] = None
    mass_eps: float = 1e-12
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    wall: int = 0
    clamp_lo: Sequence[int] = (0, 0, 0)
    clamp_hi: Sequence[int] = (0, 0, 0)
    growth_mode: int = 0
    growth_A: float = 0.0
    ramp_steps: float = 0.0

    def to_c(self, p_begin: int) -> L.MpmScene:
        s = L.MpmScene()
        for d in range(3):
            s.shape[d] = int(self.shape[d])
            s.clamp_lo[d] = int(self.clamp_lo[d])
            s.clamp_hi[d] = int(self.clamp_hi[d])
            s.gravity[d] = float(self.gravity[d])
        s.model = int(self.model)
        s.p_begin = int(p_begin)
        s.p_end = int(p_begin + self.n)
        s.wall = int(self.wall)
        s.growth_mode = int(self.growth_mode)
        s.dx, s.dt, s.damping = float(self.dx), float(self.dt), float(self.damping)
        s.pmass, s.vol0, s.mass_eps = float(self.pmass), float(self.vol0), float(self.mass_eps)
        s.mu, s.lam = float(self.mu), float(self.lam)
        hb = dict(kappa=1.0e4, K=1.0, n=0.5, tau_y=50.0, m=100.0, eps=1e-4)
        if self.hb:
            hb.update(self.hb)
        s.kappa, s.K, s.n_exp = hb["kappa"], hb["K"], hb["n"]
        s.tau_y, s.m_pap, s.eps = hb["tau_y"], hb["m"], hb["eps"]
        s.growth_A, s.ramp_steps = float(self.growth_A), float(self.ramp_steps)
        return s


def tuning_struct(t: Optional[dict]) -> L.MpmTuning:
    c = L.MpmTuning()
    t = t or {}
    c.tile_xy = int(t.get("tile_xy", 0))
    c.scatter_ctas_per_sm = int(t.get("scatter_ctas_per_sm", 0))
    c.scatter_oxb = int(t.get("scatter_oxb", 0))
    c.particle_block = int(t.get("particle_block", 0))
    c.active_tile_cap = int(t.get("active_tile_cap", 0))
    c.fp64_gap_thresh = float(t.get("fp64_gap_thresh", 0.0))
    c.tile_z = int(t.get("tile_z", 0))
    return c


class Plan:
    """A bound batch plan: scene table + workspace on one CUDA device
    (``device``, default the current one).  The library launches on the
    current device, so every later call on the plan must run with that device
    current (one process per GPU, as torchrun launches them, satisfies this);
    ``stream=None`` means the current stream of the current device."""

    def __init__(self, scenes: List[SceneSpec], dtype=torch.float64, tuning: Optional[dict] = None,
                 device=None, stream=None):
        require_cuda()
        self.lib = L.load()
        self.dtype = dtype
        self.real_bytes = dtype_bytes(dtype)
        self.scenes = list(scenes)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        arr = (L.MpmScene * len(self.scenes))()
        p = 0
        self.offsets = []
        for i, sc in enumerate(self.scenes):
            arr[i] = sc.to_c(p)
            self.offsets.append(p)
            p += int(sc.n)
        self.offsets.append(p)
        self.n = p
        self._c_scenes = arr
        self.tuning = dict(tuning or {})
        handle = C.c_void_p()
        L.check(self.lib.mpm_plan_create(arr, len(self.scenes), self.real_bytes, C.byref(tuning_struct(tuning)),
                                         C.byref(handle)), "mpm_plan_create")
        self.handle = handle
        nb = C.c_size_t()
        L.check(self.lib.mpm_plan_workspace_bytes(handle, C.byref(nb)), "workspace_bytes")
        self.ws_bytes = nb.value
        L.check(self.lib.mpm_plan_tape_bytes(handle, C.byref(nb)), "tape_bytes")
        self.tape_bytes = nb.value
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=self.device)
            base = self.workspace.data_ptr()
            self.ws_ptr = (base + 255) // 256 * 256
            L.check(self.lib.mpm_plan_bind(handle, C.c_void_p(self.ws_ptr), C.c_void_p(stream_ptr(stream))),
                    "mpm_plan_bind")
        self._phi = None

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                self.lib.mpm_plan_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:
            pass

    # -- tapes -------------------------------------------------------------
    def new_tape(self) -> "TapeBuf":
        return TapeBuf(self)

    def update_scenes(self, scenes: List[SceneSpec], stream=None):
        """New physical parameters for the same scene structure
        (mpm_plan_update_scenes); captured graphs replay with them."""
        scenes = list(scenes)
        arr = (L.MpmScene * len(scenes))()
        for i, sc in enumerate(scenes):
            arr[i] = sc.to_c(self.offsets[i])
        L.check(self.lib.mpm_plan_update_scenes(self.handle, arr, len(scenes), C.c_void_p(stream_ptr(stream))),
                "mpm_plan_update_scenes")
        self.scenes = scenes
        self._c_scenes = arr

    def set_external_stress(self, tau: Optional[torch.Tensor], tau_bar: Optional[torch.Tensor] = None):
        """Caller-supplied Kirchhoff stress (n, 3, 3) for MPM_MODEL_EXTERNAL
        scenes, and the buffer the reverse step writes its cotangent to."""
        for a in (tau, tau_bar):
            assert a is None or (a.is_contiguous() and a.dtype == self.dtype and a.numel() == 9 * self.n)
        self._ext = (tau, tau_bar)
        L.check(self.lib.mpm_plan_set_external_stress(
            self.handle, C.c_void_p(tau.data_ptr() if tau is not None else 0),
            C.c_void_p(tau_bar.data_ptr() if tau_bar is not None else 0)), "set_external_stress")

    def set_particle_mass(self, mass: Optional[torch.Tensor], vol0: Optional[torch.Tensor] = None):
        """Per-particle masses and reference volumes (None: the scenes' pmass / vol0)."""
        prep = lambda a: (a.to(device=self.device, dtype=self.dtype).contiguous() if a is not None else None)
        mass, vol0 = prep(mass), prep(vol0)
        for a in (mass, vol0):
            assert a is None or a.numel() == self.n
        self._mass = (mass, vol0)     # kept alive while the plan uses them
        L.check(self.lib.mpm_plan_set_particle_mass(
            self.handle, C.c_void_p(mass.data_ptr() if mass is not None else 0),
            C.c_void_p(vol0.data_ptr() if vol0 is not None else 0)), "set_particle_mass")

    def set_growth_field(self, phi: Optional[torch.Tensor]):
        if phi is not None:
            phi = phi.to(device=self.device, dtype=self.dtype).contiguous()
            assert phi.numel() == self.n
        self._phi = phi
        L.check(self.lib.mpm_plan_set_growth_field(self.handle, C.c_void_p(phi.data_ptr() if phi is not None else 0)),
                "set_growth_field")

    # -- status --------------------------------------------------------------
    def status(self, stream=None) -> int:
        v = C.c_int32()
        L.check(self.lib.mpm_plan_read_status(self.handle, C.byref(v), C.c_void_p(stream_ptr(stream))), "status")
        return v.value

    def fp64_fallbacks(self, stream=None) -> int:
        v = C.c_int64()
        L.check(self.lib.mpm_plan_read_fp64_fallbacks(self.handle, C.byref(v), C.c_void_p(stream_ptr(stream))),
                "fallbacks")
        return v.value

    # -- profiling ---------------------------------------------------------------
    def profile_begin(self, kinds, max_launches: int = 1 << 16):
        """Bracket the launches of the named kernel kinds with CUDA events."""
        mask = 0
        for k in kinds:
            mask |= 1 << L.KERNELS.index(k)
        L.check(self.lib.mpm_plan_profile_begin(self.handle, mask, int(max_launches)), "profile_begin")

    def profile_end(self) -> dict:
        """{kind: (total_ms, launches)} of the bracketed launches."""
        ms = (C.c_double * len(L.KERNELS))()
        cnt = (C.c_int32 * len(L.KERNELS))()
        L.check(self.lib.mpm_plan_profile_end(self.handle, ms, cnt), "profile_end")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(L.KERNELS) if cnt[i] > 0}

    def active_tiles(self, tape: Optional["TapeBuf"] = None, stream=None) -> int:
        v = C.c_int32()
        L.check(self.lib.mpm_plan_active_tiles(self.handle, C.c_void_p(tape.ptr if tape is not None else 0),
                                               C.byref(v), C.c_void_p(stream_ptr(stream))), "active_tiles")
        return v.value

    def launch_count(self) -> int:
        return int(self.lib.mpm_plan_launch_count(self.handle))

    # -- steps ---------------------------------------------------------------
    def step_fwd(self, pin: L.MpmParticles, pout: L.MpmParticles, advect: bool, t: int,
                 tape: Optional["TapeBuf"] = None, stream=None, chained: bool = False, emit: bool = False):
        """One forward step.  chained/emit: consecutive steps of a trajectory
        (mpm_step_fwd_chain): emit forms the next step's cell keys and P2G
        records in this step's G2P, chained uses them."""
        flags = (L.MPM_FWD_CHAINED if chained else 0) | (L.MPM_FWD_EMIT if emit else 0)
        L.check(self.lib.mpm_step_fwd_chain(self.handle, C.byref(pin), C.byref(pout), int(bool(advect)), int(t),
                                            C.c_void_p(tape.ptr if tape is not None else 0), flags,
                                            C.c_void_p(stream_ptr(stream))), "mpm_step_fwd")

    def step_bwd(self, pin: L.MpmParticles, out_C_ptr: int, ob: L.MpmCotangents, ib: L.MpmCotangents,
                 growth_grad: Optional[torch.Tensor], advect: bool, t: int, tape: "TapeBuf", stream=None,
                 material_grad: Optional[torch.Tensor] = None):
        """Reverse of one step.  growth_grad (S,) and material_grad (S, 2:
        d/dmu, d/dlambda) are float64 accumulators, or None."""
        gg = growth_grad.data_ptr() if growth_grad is not None else 0
        if material_grad is None:
            L.check(self.lib.mpm_step_bwd(self.handle, C.byref(pin), C.c_void_p(out_C_ptr), C.byref(ob),
                                          C.byref(ib), C.c_void_p(gg), int(bool(advect)), int(t),
                                          C.c_void_p(tape.ptr), C.c_void_p(stream_ptr(stream))), "mpm_step_bwd")
            return
        assert material_grad.dtype == torch.float64 and material_grad.is_contiguous()
        assert material_grad.numel() == 2 * len(self.scenes)
        L.check(self.lib.mpm_step_bwd_params(self.handle, C.byref(pin), C.c_void_p(out_C_ptr), C.byref(ob),
                                             C.byref(ib), C.c_void_p(gg), C.c_void_p(material_grad.data_ptr()),
                                             int(bool(advect)), int(t), C.c_void_p(tape.ptr),
                                             C.c_void_p(stream_ptr(stream))), "mpm_step_bwd_params")

    def rollout_workspace_bytes(self, n_steps: int, ckpt_every: int) -> int:
        nb = C.c_size_t(0)
        L.check(self.lib.mpm_rollout_workspace_bytes(self.handle, int(n_steps), int(ckpt_every), C.byref(nb)),
                "mpm_rollout_workspace_bytes")
        return nb.value

    def rollout_fwd(self, state0: torch.Tensor, Fg: Optional[torch.Tensor], n_steps: int, ckpt_every: int,
                    advect: bool, ws_ptr: int, final: torch.Tensor, stream=None):
        """n_steps forward steps of (24, n) slab state0 into final, keeping the
        checkpoints (or every step's state and tape) in the rollout workspace
        (mpm_rollout_fwd)."""
        for t in (state0, final):
            assert t.dtype == self.dtype and t.shape == (SLAB_ROWS, self.n) and t.is_contiguous()
        L.check(self.lib.mpm_rollout_fwd(self.handle, C.c_void_p(state0.data_ptr()), C.c_void_p(_ptr(Fg)),
                                         int(n_steps), int(ckpt_every), int(bool(advect)), C.c_void_p(ws_ptr),
                                         C.c_void_p(final.data_ptr()), C.c_void_p(stream_ptr(stream))),
                "mpm_rollout_fwd")

    def rollout_bwd(self, Fg: Optional[torch.Tensor], final_bar: torch.Tensor, n_steps: int, ckpt_every: int,
                    advect: bool, ws_ptr: int, state0_bar: torch.Tensor, Fg_bar: Optional[torch.Tensor] = None,
                    growth_grad: Optional[torch.Tensor] = None, material_grad: Optional[torch.Tensor] = None,
                    stream=None):
        """Reverse sweep of the last rollout_fwd on the workspace
        (mpm_rollout_bwd); Fg_bar, growth_grad and material_grad are
        overwritten float64 outputs."""
        for t in (final_bar, state0_bar):
            assert t.dtype == self.dtype and t.shape == (SLAB_ROWS, self.n) and t.is_contiguous()
        for t in (Fg_bar, growth_grad, material_grad):
            assert t is None or (t.dtype == torch.float64 and t.is_contiguous())
        L.check(self.lib.mpm_rollout_bwd(self.handle, C.c_void_p(_ptr(Fg)), C.c_void_p(final_bar.data_ptr()),
                                         int(n_steps), int(ckpt_every), int(bool(advect)), C.c_void_p(ws_ptr),
                                         C.c_void_p(state0_bar.data_ptr()), C.c_void_p(_ptr(Fg_bar)),
                                         C.c_void_p(_ptr(growth_grad)), C.c_void_p(_ptr(material_grad)),
                                         C.c_void_p(stream_ptr(stream))), "mpm_rollout_bwd")

    def loss_detF(self, F_ptr: int, sp9: int, sc9: int, loss: torch.Tensor, F_bar_ptr: int = 0, stream=None):
        L.check(self.lib.mpm_loss_detF(self.handle, C.c_void_p(F_ptr), sp9, sc9, C.c_void_p(loss.data_ptr()),
                                       C.c_void_p(F_bar_ptr), C.c_void_p(stream_ptr(stream))), "mpm_loss_detF")

    def loss_mse(self, x_ptr: int, sp3: int, sc3: int, xo_ptr: int, loss: torch.Tensor, x_bar_ptr: int = 0,
                 stream=None):
        L.check(self.lib.mpm_loss_mse(self.handle, C.c_void_p(x_ptr), sp3, sc3, C.c_void_p(xo_ptr),
                                      C.c_void_p(loss.data_ptr()), C.c_void_p(x_bar_ptr),
                                      C.c_void_p(stream_ptr(stream))), "mpm_loss_mse")


class TapeBuf:
    """Device buffer recording one forward step for its reverse."""

    def __init__(self, plan: Plan):
        self.plan = plan
        self.buf = torch.empty(plan.tape_bytes + 256, dtype=torch.uint8, device=plan.device)
        self.ptr = (self.buf.data_ptr() + 255) // 256 * 256


# ---------------------------------------------------------------------------
# particle views
# ---------------------------------------------------------------------------
def slab_particles(slab: torch.Tensor, Fg: Optional[torch.Tensor] = None) -> L.MpmParticles:
    """MpmParticles over a (24, n) slab (and an optional (9, n) Fg slab)."""
    assert slab.dim() == 2 and slab.shape[0] == SLAB_ROWS and slab.is_contiguous()
    n = slab.shape[1]
    es = slab.element_size()
    b = slab.data_ptr()
    p = L.MpmParticles()
    p.x, p.v, p.C, p.F = b + ROW_X * n * es, b + ROW_V * n * es, b + ROW_C * n * es, b + ROW_F * n * es
    p.Fg = Fg.data_ptr() if Fg is not None else 0
    if Fg is not None:
        assert Fg.shape == (9, n) and Fg.is_contiguous() and Fg.dtype == slab.dtype
    p.sp3, p.sc3, p.sp9, p.sc9 = 1, n, 1, n
    return p


def slab_cotangents(slab: torch.Tensor, Fg_bar: Optional[torch.Tensor] = None) -> L.MpmCotangents:
    n = slab.shape[1]
    es = slab.element_size()
    b = slab.data_ptr()
    c = L.MpmCotangents()
    c.x, c.v, c.C, c.F = b + ROW_X * n * es, b + ROW_V * n * es, b + ROW_C * n * es, b + ROW_F * n * es
    c.Fg = Fg_bar.data_ptr() if Fg_bar is not None else 0
    if Fg_bar is not None:
        assert Fg_bar.shape == (9, n) and Fg_bar.dtype == torch.float64 and Fg_bar.is_contiguous()
    c.sp3, c.sc3, c.sp9, c.sc9 = 1, n, 1, n
    return c


def aos_particles(x, v, Cm, F, Fg) -> L.MpmParticles:
    """MpmParticles over (n,3)/(n,3,3) C-contiguous tensors."""
    p = L.MpmParticles()
    p.x, p.v, p.C, p.F = x.data_ptr(), v.data_ptr(), Cm.data_ptr(), F.data_ptr()
    p.Fg = Fg.data_ptr() if Fg is not None else 0
    p.sp3, p.sc3, p.sp9, p.sc9 = 3, 1, 9, 1
    return p


def aos_cotangents(x, v, Cm, F, Fg) -> L.MpmCotangents:
    c = L.MpmCotangents()
    c.x, c.v, c.C, c.F = x.data_ptr(), v.data_ptr(), Cm.data_ptr(), F.data_ptr()
    c.Fg = Fg.data_ptr() if Fg is not None else 0
    c.sp3, c.sc3, c.sp9, c.sc9 = 3, 1, 9, 1
    return c


def slab_from_aos(x, v, Cm, F) -> torch.Tensor:
    n = x.shape[0]
    return torch.cat([x.reshape(n, 3).t(), v.reshape(n, 3).t(), Cm.reshape(n, 9).t(), F.reshape(n, 9).t()],
                     0).contiguous()


def aos_from_slab(slab: torch.Tensor):
    n = slab.shape[1]
    t = slab.t()
    return (t[:, 0:3].contiguous(), t[:, 3:6].contiguous(), t[:, 6:15].reshape(n, 3, 3).contiguous(),
            t[:, 15:24].reshape(n, 3, 3).contiguous())
