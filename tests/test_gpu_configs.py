"""Growth workloads 1, 2 and 5 on the device, against the reference and the oracle.

- Config 1 at full length: the 100-step free-swell cube (ramp 1 -> 1.1) and
  its trajectory adjoint, against the fixture that the unmodified reference
  produced (tests/golden/make_golden.py ``make_c1_full``): device FP64
  max|dF| <= 1e-10, d loss / d A and the initial-state cotangents.
- Config 2, reduced: a 16 x 8 x 8-cell Hencky bilayer strip in the 96x32x32
  grid with the clamp box and a layered growth ramp (top half to g = 1.2) over
  20 steps.
- Config 5, reduced: a 32 x 32 x 2-cell Herschel-Bulkley sheet (tau_y = 10) in
  a 64^3 grid with the radial growth field g(r) = 1 + A exp(-r^2 / 0.05),
  30 steps with sqrt(N) checkpoints; the gradient is d loss / d A.

For 2 and 5: device FP64 against the oracle (state 1e-12, gradient 1e-9
relative), against central differences of the device loss (h = 1e-6), and the
FP32 error in F, x and d loss / d A against device FP64, stated and bounded.
The loss is sum det F of the final state (integrate.py:41-52).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from oracle import mpm_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _oracle_run(c, steps):
    """Oracle forward + adjoint of a scene dict: final state, loss, d loss / d A."""
    sp = c["dx"] / 2
    sc = O.Scene(shape=c["shape"], dx=c["dx"], dt=c["dt"], damping=c["damping"], pmass=c["density"] * sp ** 3,
                 vol0=sp ** 3, wall=c["wall"], clamp_lo=c.get("clamp_lo", (0, 0, 0)),
                 clamp_hi=c.get("clamp_hi", (0, 0, 0)))
    if c["model"] == "hb":
        h = c["hb"]
        m = O.Model(kind="hb", kappa=h["kappa"], K=h["K"], n=h["n"], tau_y=h["tau_y"], m=h["m"], eps=h["eps"])
    else:
        m = O.Model.elastic(c["model"], c["E"], c["nu"])
    gr = O.Growth(A=c["growth_A"], ramp_steps=c["ramp_steps"], phi=c["phi"])
    st, caches = O.rollout(O.State.rest(c["x"]), m, sc, steps, advect=True, growth=gr)
    n = c["x"].shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    out = O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True, growth=gr)
    return st, O.loss_detF(st.F), out[5]


def _device_run(c, steps, dtype, ckpt):
    """Device trajectory of one scene: (final (24, n) slab as float64 numpy,
    loss, d loss / d A, the batch)."""
    from morphompm_b200.batch import Batch, host_slab
    b = Batch([c], steps, dtype=dtype, ckpt_every=ckpt)
    b.load(host_slab([c], np.float64 if dtype == torch.float64 else np.float32), non_blocking=False)
    b.run()
    torch.cuda.synchronize()
    fin = b.final_state().double().cpu().numpy()
    assert b.plan.status() & (1 | 4) == 0, b.plan.status()     # no bad argument, nothing non-finite
    return fin, float(b.loss[0]), float(b.dloss_dg[0]), b


def _fd(b, A, h=1e-6):
    """Central difference of the device loss in the growth amplitude."""
    out = []
    for a in (A + h, A - h):
        b.set_params(growth_A=[a])
        b.run()
        out.append(float(b.loss[0]))
    b.set_params(growth_A=[A])
    return (out[0] - out[1]) / (2 * h)


def _F(slab):
    return slab[15:24].T.reshape(-1, 3, 3)


def _x(slab):
    return slab[0:3].T


def _check_scene(c, steps, ckpt, tol_state=1e-12):
    st, L_o, dA_o = _oracle_run(c, steps)
    f64, L64, dA64, b64 = _device_run(c, steps, torch.float64, ckpt)
    errF = np.max(np.abs(_F(f64) - st.F))
    errx = np.max(np.abs(_x(f64) - st.x))
    assert errF <= tol_state and errx <= tol_state, (errF, errx)
    assert abs(L64 - L_o) <= 1e-12 * abs(L_o), (L64, L_o)
    assert abs(dA64 - dA_o) <= 1e-9 * abs(dA_o), (dA64, dA_o)
    fd = _fd(b64, c["growth_A"])
    assert abs(dA64 - fd) <= 1e-6 * abs(fd), (dA64, fd)
    del b64
    f32, L32, dA32, _ = _device_run(c, steps, torch.float32, ckpt)
    err32 = {"F": float(np.max(np.abs(_F(f32) - _F(f64)))), "x": float(np.max(np.abs(_x(f32) - _x(f64)))),
             "dLdA_rel": abs(dA32 - dA64) / abs(dA64)}
    print(f"{c['name']}: FP64 vs oracle |dF| {errF:.2e} |dx| {errx:.2e}; dL/dA {dA64:.10e} "
          f"(oracle {dA_o:.10e}, FD {fd:.10e}); FP32 error {err32}")
    return err32


def test_config1_full_length_matches_reference():
    """The whole 100-step config-1 trajectory and its adjoint against the
    reference's own run: FP64 max|dF| <= 1e-10 (the plain drop-in's bar)."""
    from morphompm_b200 import scenes
    g = np.load(os.path.join(GOLDEN, "c1_full.npz"))
    c = scenes.config1()
    steps = int(g["steps"])
    assert steps == c["steps"]
    f64, L64, dA64, b = _device_run(c, steps, torch.float64, 10)
    errF = np.max(np.abs(_F(f64) - g["F"]))
    errx = np.max(np.abs(_x(f64) - g["x"]))
    assert errF <= 1e-10 and errx <= 1e-10, (errF, errx)
    assert abs(L64 - float(g["loss"])) <= 1e-12 * abs(float(g["loss"]))
    assert abs(dA64 - float(g["dloss_dA"])) <= 1e-9 * abs(float(g["dloss_dA"])), (dA64, float(g["dloss_dA"]))
    bar0 = b.initial_cotangents().cpu().numpy()
    xb, Fb = bar0[0:3].T, bar0[15:24].T.reshape(-1, 3, 3)
    assert np.max(np.abs(xb - g["x0_bar"])) <= 1e-9 * np.max(np.abs(g["x0_bar"]))
    assert np.max(np.abs(Fb - g["F0_bar"])) <= 1e-9 * np.max(np.abs(g["F0_bar"]))
    f32, _, dA32, _ = _device_run(c, steps, torch.float32, 10)
    assert np.max(np.abs(_F(f32) - g["F"])) <= 1e-4
    assert abs(dA32 - dA64) <= 1e-4 * abs(dA64)


def test_config2_bilayer_strip_reduced():
    """Hencky bilayer with the clamped end and the layered ramp."""
    from morphompm_b200 import scenes
    c = scenes.config2(length=16, steps=20)
    err = _check_scene(c, 20, 5)
    assert err["F"] <= 1e-4 and err["x"] <= 1e-5 and err["dLdA_rel"] <= 1e-4, err


def test_config5_hb_sheet_reduced():
    """Herschel-Bulkley sheet with the radial growth field, sqrt(N) checkpoints."""
    from morphompm_b200 import scenes
    from morphompm_b200.trajectory import sqrt_schedule
    c = scenes.config5(cells=(32, 32, 2), edge=64, steps=30)
    err = _check_scene(c, 30, sqrt_schedule(30))
    assert err["F"] <= 1e-4 and err["x"] <= 1e-5 and err["dLdA_rel"] <= 1e-4, err
