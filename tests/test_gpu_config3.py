"""Inverse-growth workload (config 3): 32768 particles in a 64^3 grid, 400
steps, checkpoint every 20 with recomputation, mean squared position loss
against the final positions from g* = 1.15.  dL/dg on the device in FP64
against central differences (h = 1e-6), against the oracle on a 10-step
trajectory, and the FP32 error against FP64 (rel. <= 1e-4)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from oracle import mpm_oracle as O


def _cfg(c):
    from morphompm_b200.config import SimConfig, Material
    return SimConfig(N=64, dx=c["dx"], dt=c["dt"], damping=c["damping"], sp=c["dx"] / 2,
                     material=Material(E=c["E"], nu=c["nu"], density=c["density"]), wall=c["wall"])


def test_config3_gradient_fd_and_fp32():
    from morphompm_b200 import scenes, integrate
    from morphompm_b200.constitutive import NeoHookean
    c = scenes.config3()
    cfg = _cfg(c)
    m = NeoHookean(cfg.material)
    x0 = torch.tensor(c["x"], dtype=torch.float64, device="cuda")
    # observation: final positions from g*
    xT = _final_x(c, cfg, m, c["g_true"], torch.float64)
    g = c["g_eval"]
    L64, d64 = integrate.dloss_dg(x0, m, cfg, g, c["steps"], True, loss="mse", x_obs=xT, ckpt_every=c["ckpt_every"])
    h = 1e-6
    Lp, _ = integrate.dloss_dg(x0, m, cfg, g + h, c["steps"], True, loss="mse", x_obs=xT, ckpt_every=c["ckpt_every"])
    Lm, _ = integrate.dloss_dg(x0, m, cfg, g - h, c["steps"], True, loss="mse", x_obs=xT, ckpt_every=c["ckpt_every"])
    fd = (Lp - Lm) / (2 * h)
    assert abs(d64 - fd) <= 1e-5 * abs(fd), (d64, fd)
    x32 = x0.float()
    L32, d32 = integrate.dloss_dg(x32, m, cfg, g, c["steps"], True, loss="mse", x_obs=xT.float(),
                                  ckpt_every=c["ckpt_every"])
    assert abs(d32 - d64) <= 1e-4 * abs(d64), (d32, d64)


def _final_x(c, cfg, m, g, dtype):
    from morphompm_b200 import integrate
    from morphompm_b200.transfer import get_plan, scene_spec
    from morphompm_b200.trajectory import Rollout
    p = torch.tensor(c["x"], dtype=dtype, device="cuda")
    n = p.shape[0]
    plan = get_plan([scene_spec(cfg, m, n)], dtype, p.device)
    Fg = torch.zeros(9, n, dtype=dtype, device="cuda")
    for i in range(3):
        Fg[4 * i] = g
    ro = Rollout(plan, c["steps"], advect=True, ckpt_every=c["ckpt_every"], Fg=Fg)
    ro.forward(integrate._slab_from_points(p))
    return ro.final[0:3].t().contiguous()


def test_config3_short_trajectory_matches_oracle():
    from morphompm_b200 import scenes, integrate
    from morphompm_b200.constitutive import NeoHookean
    c = scenes.config3()
    cfg = _cfg(c)
    m = NeoHookean(cfg.material)
    steps = 10
    rng = np.random.default_rng(3)
    x_obs = c["x"] + 1e-3 * rng.standard_normal(c["x"].shape)
    L, dg = integrate.dloss_dg(c["x"], m, cfg, c["g_eval"], steps, True, loss="mse", x_obs=x_obs, ckpt_every=4)
    sp = c["dx"] / 2
    sc = O.Scene(shape=(64, 64, 64), dx=c["dx"], dt=c["dt"], damping=c["damping"], pmass=c["density"] * sp ** 3,
                 vol0=sp ** 3, wall=c["wall"])
    st, caches = O.rollout(O.State.rest(c["x"], c["g_eval"]), O.Model.elastic("nh", c["E"], c["nu"]), sc, steps,
                           advect=True)
    n = c["x"].shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    Fgb = O.rollout_vjp(caches, O.seed_mse(st.x, x_obs), z3, z33, z33, z33, advect=True)[4]
    ref = float(np.trace(Fgb, axis1=1, axis2=2).sum())
    assert abs(L - O.loss_mse(st.x, x_obs)) <= 1e-11 * abs(L)
    assert abs(dg - ref) <= 1e-9 * abs(ref), (dg, ref)
