"""The allocation-free forward step (mpm_step_fwd_noalloc), for callers that
cannot call cudaMalloc: a host application that owns every device allocation,
or a run that must not fail on an allocation part-way through.  It must give
the same particles as the planned entry point mpm_step_fwd, on two calls in a
row (the fixed scratch array keeps the previous call's contents), and refuse a
scene that does not fit the fixed scratch with MPM_ERR_TOO_LARGE.

This file is collected last so that a failure here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _scene(kind, n, shape, dx, E=1e3, nu=0.3):
    from morphompm_b200.runtime import SceneSpec
    from morphompm_b200 import _lib as L
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    sp = dx / 2
    model = {"nh": L.MODEL_NEOHOOKEAN, "hencky": L.MODEL_HENCKY}[kind]
    return SceneSpec(shape=shape, n=n, model=model, dx=dx, dt=1e-4, damping=0.05, pmass=sp ** 3, vol0=sp ** 3,
                     mu=mu, lam=lam, wall=2)


def _state(x, dtype, rng):
    n = x.shape[0]
    t = lambda a: torch.tensor(a, dtype=dtype, device="cuda").contiguous()
    v = 0.05 * rng.standard_normal((n, 3))
    Cm = 0.1 * rng.standard_normal((n, 3, 3))
    F = np.eye(3) + 0.02 * rng.standard_normal((n, 3, 3))
    Fg = 1.05 * np.eye(3) + 0.01 * rng.standard_normal((n, 3, 3))
    return [t(x), t(v), t(Cm), t(F), t(Fg)]


def _planned(spec, st, dtype):
    from morphompm_b200.runtime import Plan, aos_particles
    plan = Plan([spec], dtype=dtype)
    out = [torch.empty_like(a) for a in st]
    plan.step_fwd(aos_particles(*st), aos_particles(*out), True, 0, plan.new_tape())
    torch.cuda.synchronize()
    return out


def _noalloc(spec, st, dtype):
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import aos_particles, dtype_bytes
    out = [torch.empty_like(a) for a in st]
    status = C.c_int32(-1)
    rc = L.load().mpm_step_fwd_noalloc(C.byref(spec.to_c(0)), dtype_bytes(dtype), C.byref(aos_particles(*st)),
                                      C.byref(aos_particles(*out)), 1, 0, C.byref(status),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.MPM_OK, rc
    assert status.value == 0, status.value
    return out


@pytest.mark.parametrize("kind,dtype,tol", [("nh", torch.float64, 1e-12), ("hencky", torch.float32, 1e-6)])
def test_noalloc_matches_planned_step_twice(kind, dtype, tol):
    from morphompm_b200 import scenes
    rng = np.random.default_rng(21)
    c = scenes.config1()
    spec = _scene(kind, c["x"].shape[0], c["shape"], c["dx"])
    # two different inputs, one call each, then the first input again: the
    # shared scratch must not carry anything from one call into the next
    st_a = _state(c["x"], dtype, rng)
    st_b = _state(c["x"] + 0.003 * rng.standard_normal(c["x"].shape), dtype, rng)
    for st in (st_a, st_b, st_a):
        ref = _planned(spec, st, dtype)
        got = _noalloc(spec, st, dtype)
        for r, g in zip(ref, got):
            err = (r - g).abs().max().item() / max(r.abs().max().item(), 1e-300)
            assert err <= tol, err


def test_noalloc_rejects_scene_beyond_scratch():
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import aos_particles
    n = 400_000
    spec = _scene("nh", n, (64, 64, 64), 1 / 64)
    st = [torch.zeros(n, 3, device="cuda", dtype=torch.float64), torch.zeros(n, 3, device="cuda", dtype=torch.float64)]
    st += [torch.zeros(n, 3, 3, device="cuda", dtype=torch.float64) for _ in range(3)]
    out = [torch.empty_like(a) for a in st]
    rc = L.load().mpm_step_fwd_noalloc(C.byref(spec.to_c(0)), 8, C.byref(aos_particles(*st)),
                                      C.byref(aos_particles(*out)), 1, 0, None,
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.MPM_ERR_TOO_LARGE
