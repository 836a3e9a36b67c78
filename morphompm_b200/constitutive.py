"""[2] Constitutive seam -- the reference's pluggable models
(python/morphompm/constitutive.py:1-147) with the same interface:

    model.stress(F, Fg, C=None)           -> tau   (Kirchhoff, 3x3 sym)
    model.stress_vjp(F, Fg, C, tau_bar)   -> (F_bar, Fg_bar, C_bar)

Both run on the GPU (``mpm_stress`` / ``mpm_stress_vjp``) for a single 3x3
matrix or a batch (n,3,3).  numpy inputs come back as numpy, torch CUDA inputs
stay on the device.  Inside ``transfer.step`` the same device code is fused into
the P2G prepass and the reverse particle kernel; these objects carry the model
kind and parameters that the step kernels read.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L
from .config import Material
from .devarray import to_device, like_input


class _Model:
    kind = None

    def scene_fields(self) -> dict:
        raise NotImplementedError

    def _scene(self):
        from .runtime import SceneSpec
        f = self.scene_fields()
        return SceneSpec(shape=(1, 1, 1), n=0, dx=1.0, dt=0.0, damping=0.0, pmass=0.0, vol0=0.0, **f).to_c(0)

    def stress(self, F, Fg, C=None):
        lib = L.load()
        (Fd, Fgd, Cd), ref, single = _prep([F, Fg, C])
        import torch
        tau = torch.empty_like(Fd)
        from .runtime import dtype_bytes, stream_ptr
        L.check(lib.mpm_stress(ct.byref(self._scene()), dtype_bytes(Fd.dtype), Fd.shape[0], Fd.data_ptr(),
                               Fgd.data_ptr(), Cd.data_ptr() if Cd is not None else None, tau.data_ptr(),
                               ct.c_void_p(stream_ptr())), "mpm_stress")
        return like_input(tau[0] if single else tau, ref)

    def stress_vjp(self, F, Fg, C, tau_bar):
        lib = L.load()
        (Fd, Fgd, Cd, tb), ref, single = _prep([F, Fg, C, tau_bar])
        import torch
        Fb, Fgb, Cb = torch.empty_like(Fd), torch.empty_like(Fd), torch.empty_like(Fd)
        from .runtime import dtype_bytes, stream_ptr
        L.check(lib.mpm_stress_vjp(ct.byref(self._scene()), dtype_bytes(Fd.dtype), Fd.shape[0], Fd.data_ptr(),
                                   Fgd.data_ptr(), Cd.data_ptr() if Cd is not None else None, tb.data_ptr(),
                                   Fb.data_ptr(), Fgb.data_ptr(), Cb.data_ptr(), ct.c_void_p(stream_ptr())),
                "mpm_stress_vjp")
        out = (Fb, Fgb, Cb)
        if single:
            out = tuple(o[0] for o in out)
        return tuple(like_input(o, ref) for o in out)


def _prep(arrs):
    """Move a list of (3,3)/(n,3,3) arrays (None allowed) to contiguous device tensors."""
    ref = next(a for a in arrs if a is not None)
    single = (ref.ndim == 2)
    dev = to_device(ref)
    out = []
    for a in arrs:
        if a is None:
            out.append(None)
            continue
        t = to_device(a, dtype=dev.dtype, device=dev.device)
        if single:
            t = t.reshape(1, 3, 3)
        out.append(t.contiguous())
    return out, ref, single


class _ElasticModel(_Model):
    """Rate-independent: C ignored, C_bar = 0 (constitutive.py:79-93)."""

    def __init__(self, material: Material):
        self.mu = material.mu
        self.lam = material.lam

    def scene_fields(self):
        return dict(model=self.kind, mu=self.mu, lam=self.lam)


class NeoHookean(_ElasticModel):
    """tau = mu (Fe Fe^T - I) + lam ln J I   (constitutive.py:25-39)."""
    kind = L.MODEL_NEOHOOKEAN


class Hencky(_ElasticModel):
    """tau = U diag(2 mu ln s + lam sum ln s) U^T  (constitutive.py:42-75)."""
    kind = L.MODEL_HENCKY


class HerschelBulkley(_Model):
    """Rate-dependent bioink, Papanastasiou-regularised (constitutive.py:106-147)."""
    kind = L.MODEL_HERSCHEL_BULKLEY

    def __init__(self, kappa=1.0e4, K=1.0, n=0.5, tau_y=50.0, m=100.0, eps=1e-4):
        self.kappa, self.K, self.n, self.tau_y, self.m, self.eps = kappa, K, n, tau_y, m, eps

    def scene_fields(self):
        return dict(model=self.kind, hb=dict(kappa=self.kappa, K=self.K, n=self.n, tau_y=self.tau_y,
                                             m=self.m, eps=self.eps))


def is_external(model) -> bool:
    """A user-defined material: not built in, but with batched
    ``stress(F, Fg, C) -> tau`` and ``stress_vjp(F, Fg, C, tau_bar) ->
    (F_bar, Fg_bar, C_bar)`` on (n, 3, 3) device tensors."""
    return (not isinstance(model, _Model) and callable(getattr(model, "stress", None))
            and callable(getattr(model, "stress_vjp", None)))


def model_fields(model) -> dict:
    """Scene fields of a model.  A built-in model runs inside the kernels; a
    user-defined one (``is_external``) runs as a batched callback whose stress
    the kernels consume (``transfer.step`` / ``step_vjp`` only).  Anything
    else is rejected: the GPU path has no CPU fallback."""
    if isinstance(model, _Model):
        return model.scene_fields()
    if is_external(model):
        return dict(model=L.MODEL_EXTERNAL)
    raise TypeError(f"{type(model).__name__} is not a morphompm_b200 model: use NeoHookean, Hencky, "
                    "HerschelBulkley, or an object with batched stress(F, Fg, C) and stress_vjp(F, Fg, C, tau_bar)")


class PerParticle:
    """Batched adapter for a material written like the reference's models
    (constitutive.py:3-5: ``stress`` and ``stress_vjp`` on one particle's
    3x3 numpy arrays).  It loops over the particles on the host, so it is
    slow; it lets such a material run unchanged through ``transfer.step``."""

    def __init__(self, model):
        self.model = model

    @staticmethod
    def _np(a):
        return a.detach().double().cpu().numpy() if hasattr(a, "detach") else np.asarray(a, dtype=np.float64)

    def stress(self, F, Fg, C=None):
        import torch
        Fh, Fgh = self._np(F), self._np(Fg)
        Ch = self._np(C) if C is not None else np.zeros_like(Fh)
        tau = np.stack([np.asarray(self.model.stress(Fh[p], Fgh[p], Ch[p])) for p in range(Fh.shape[0])])
        return torch.as_tensor(tau, dtype=F.dtype, device=F.device)

    def stress_vjp(self, F, Fg, C, tau_bar):
        import torch
        Fh, Fgh, tb = self._np(F), self._np(Fg), self._np(tau_bar)
        Ch = self._np(C) if C is not None else np.zeros_like(Fh)
        outs = [self.model.stress_vjp(Fh[p], Fgh[p], Ch[p], tb[p]) for p in range(Fh.shape[0])]
        return tuple(torch.as_tensor(np.stack([o[k] for o in outs]), dtype=F.dtype, device=F.device)
                     for k in range(3))


def confined_swell_neohookean(mat, g: float = 1.5):
    """Closed-form check of the neo-Hookean model (constitutive.py:150-170):
    a block growing by Fg = g I, confined laterally (F = diag(1, 1, s)) and
    free along z, settles where tau_zz = 0, i.e. where
        r(s) = mu (s^2/g^2 - 1) + lambda ln(s / g^3) = 0,
    and then carries tau_xx = mu (1 - s^2) / g^2.  Returns (s, tau_xx).
    r is strictly increasing (r' = 2 mu s/g^2 + lambda/s > 0) with r(g) < 0
    for g > 1, so Newton's method from the upper side converges monotonically;
    a bracket keeps every iterate inside [lo, hi]."""
    mu, lam = float(mat.mu), float(mat.lam)
    g = float(g)
    r = lambda s: mu * (s * s / (g * g) - 1.0) + lam * np.log(s / g ** 3)
    dr = lambda s: 2.0 * mu * s / (g * g) + lam / s
    lo, hi = 1e-6, max(g, 1.0)
    while r(hi) < 0.0:
        lo, hi = hi, 2.0 * hi
    s = hi
    for _ in range(100):
        v = r(s)
        if v > 0.0:
            hi = s
        else:
            lo = s
        step = s - v / dr(s)
        s_new = step if lo < step < hi else 0.5 * (lo + hi)
        if abs(s_new - s) <= 1e-15 * s:
            s = s_new
            break
        s = s_new
    return float(s), float(mu * (1.0 - s * s) / (g * g))
