"""The CPU oracle (oracle/mpm_oracle.py) against the golden fixtures written by
the unmodified reference (tests/golden/make_golden.py), and finite-difference
gates for the oracle's extensions (boundary conditions, gravity, growth law,
position loss) that the reference does not have."""
import os

import numpy as np
import pytest

from oracle import mpm_oracle as O
from oracle.build_ref import ref_root

REF = ref_root()


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def _models(d):
    return {"nh": O.Model.elastic("nh", float(d["E"]), float(d["nu"])),
            "hencky": O.Model.elastic("hencky", float(d["E"]), float(d["nu"])),
            "hb": O.Model("hb")}


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
@pytest.mark.parametrize("adv", [False, True])
def test_step_matches_reference(golden, name, adv):
    d = golden("step.npz")
    n = d["x"].shape[0]
    sc = O.scene_from_cfg(int(d["N"]), float(d["dx"]), float(d["dt"]), float(d["damping"]),
                          float(d["sp"]), float(d["density"]))
    m = _models(d)[name]
    st = O.State(d["x"].copy(), d["v"].copy(), d["C"].copy(), d["F"].copy(), d["Fg"].copy())
    ns, cache = O.step(st, m, sc, advect=adv)
    tag = f"{name}_{'adv' if adv else 'fix'}"
    new = np.concatenate([ns.x, ns.v, ns.C.reshape(n, 9), ns.F.reshape(n, 9)], 1)
    assert rel(new, d[tag + "_new"]) < 1e-13
    assert rel(cache[3], d[tag + "_gm"].reshape(-1)) < 1e-13
    g = O.step_vjp(cache, d["xn_b"], d["vn_b"], d["Cn_b"], d["Fn_b"], d["Fgn_b"], advect=adv)
    grads = np.concatenate([g[0], g[1], g[2].reshape(n, 9), g[3].reshape(n, 9), g[4].reshape(n, 9)], 1)
    assert rel(grads, d[tag + "_grads"]) < 1e-13


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
def test_constitutive_matches_reference(golden, name):
    d = golden("constitutive.npz")
    m = O.Model.elastic(name, 1e4, 0.3) if name != "hb" else O.Model("hb")
    tau = O.stress(m, d["F"], d["Fg"], d["C"])
    assert rel(tau, d[f"{name}_tau"]) < 1e-13
    Fb, Fgb, Cb = O.stress_vjp(m, d["F"], d["Fg"], d["C"], d["tau_bar"])
    assert rel(Fb, d[f"{name}_F_bar"]) < 1e-11
    assert rel(Fgb, d[f"{name}_Fg_bar"]) < 1e-11
    if name == "hb":
        assert rel(Cb, d[f"{name}_C_bar"]) < 1e-12


def test_reference_gates(golden):
    d = golden("gates.npz")
    pts = np.array([[0.40, 0.40, 0.40], [0.42, 0.40, 0.41], [0.40, 0.43, 0.40],
                    [0.41, 0.40, 0.44], [0.44, 0.44, 0.43]])
    sc = O.scene_from_cfg(8, 0.1, 1e-3, 0.05, 0.02, 1000.0)
    nh = O.Model.elastic("nh", 1e4, 0.3)
    assert abs(float(d["single_step_dg"]) - 3.548014e-01) < 5e-7        # transfer.py gate value
    st, cache = O.step(O.State.rest(pts, 1.3), nh, sc, advect=False)
    z3, z33 = np.zeros((5, 3)), np.zeros((5, 3, 3))
    Fgb = O.step_vjp(cache, z3, z3, z33, O.seed_detF(st.F), z33, advect=False)[4]
    assert abs(np.trace(Fgb, axis1=1, axis2=2).sum() - float(d["single_step_dg"])) < 1e-13
    for tag, model, adv, val in (("nh_fix", nh, False, 2.142598), ("nh_adv", nh, True, 2.138035),
                                 ("hb_fix", O.Model("hb"), False, 2.885411)):
        L, dg = O.dloss_dg(pts, model, sc, 1.30, 3, adv)
        assert abs(dg - float(d[f"traj_{tag}_dg"])) < 1e-12 * abs(dg)
        assert abs(dg - val) < 1e-6
        assert abs(L - float(d[f"traj_{tag}_loss"])) < 1e-12


def test_free_swell_and_parity_scene(golden):
    d = golden("gates.npz")
    sc = O.scene_from_cfg(12, 0.05, 1e-3, 0.05, 0.03, 1000.0)
    for name in ("nh", "hencky", "hb"):
        m = O.Model.elastic(name, 1e4, 0.3) if name != "hb" else O.Model("hb")
        st, _ = O.rollout(O.State.rest(d["swell_pts"], 1.5), m, sc, 150, advect=True, keep_caches=False)
        assert rel(st.F, d[f"swell_{name}_F"]) < 1e-11
        assert abs(np.mean(np.linalg.det(st.F)) - float(d[f"swell_{name}_detF"])) < 1e-11
    st, _ = O.rollout(O.State.rest(d["parity27_pts"], 1.05), O.Model.elastic("hencky", 1e4, 0.3), sc, 30,
                      advect=True, keep_caches=False)
    assert rel(st.F, d["parity27_F"]) < 1e-12


def test_c1_head(golden):
    from morphompm_b200 import scenes
    d = golden("c1_head.npz")
    c = scenes.config1()
    assert np.array_equal(c["x"], d["x0"])
    sc = O.Scene(shape=(32, 32, 32), dx=c["dx"], dt=c["dt"], damping=c["damping"],
                 pmass=c["density"] * (c["dx"] / 2) ** 3, vol0=(c["dx"] / 2) ** 3)
    m = O.Model.elastic("nh", c["E"], c["nu"])
    gr = O.Growth(A=c["growth_A"], ramp_steps=c["ramp_steps"])
    st, _ = O.rollout(O.State.rest(c["x"]), m, sc, int(d["steps"]), advect=True, growth=gr, keep_caches=False)
    assert rel(st.F, d["F"]) < 1e-12
    assert rel(st.x, d["x"]) < 1e-14


def test_c1_full_length_and_adjoint(golden):
    """The whole 100-step config-1 trajectory and its adjoint (sum det F, d/dA
    of the growth ramp) against the reference's own run of them."""
    from morphompm_b200 import scenes
    d = golden("c1_full.npz")
    c = scenes.config1()
    sc = O.Scene(shape=(32, 32, 32), dx=c["dx"], dt=c["dt"], damping=c["damping"],
                 pmass=c["density"] * (c["dx"] / 2) ** 3, vol0=(c["dx"] / 2) ** 3)
    gr = O.Growth(A=c["growth_A"], ramp_steps=c["ramp_steps"])
    st, caches = O.rollout(O.State.rest(c["x"]), O.Model.elastic("nh", c["E"], c["nu"]), sc, int(d["steps"]),
                           advect=True, growth=gr)
    assert np.max(np.abs(st.F - d["F"])) < 1e-12
    assert np.max(np.abs(st.x - d["x"])) < 1e-13
    assert abs(O.loss_detF(st.F) - float(d["loss"])) < 1e-12 * float(d["loss"])
    n = c["x"].shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    xb, _, _, Fb, _, dA = O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True, growth=gr)
    assert abs(dA - float(d["dloss_dA"])) < 1e-11 * abs(float(d["dloss_dA"]))
    assert rel(xb, d["x0_bar"]) < 1e-11
    assert rel(Fb, d["F0_bar"]) < 1e-11


def _ext_scene():
    return O.Scene(shape=(10, 9, 11), dx=0.1, dt=1e-3, damping=0.05, pmass=1000 * 0.05 ** 3, vol0=0.05 ** 3,
                   gravity=(0.0, -9.8, 0.5), wall=2, clamp_lo=(0, 0, 0), clamp_hi=(4, 9, 11))


def test_extension_fd_growth_law_mse():
    """Extensions (non-cubic grid, walls, clamp box, gravity, growth ramp with a
    per-particle field, MSE loss): adjoint d loss/dA vs central FD."""
    rng = np.random.default_rng(5)
    sc = _ext_scene()
    pts = rng.uniform(0.3, 0.7, size=(30, 3))
    phi = rng.uniform(0.2, 1.0, size=30)
    m = O.Model.elastic("hencky", 1e4, 0.3)
    x_obs = pts + 0.01 * rng.standard_normal(pts.shape)

    def run(A):
        gr = O.Growth(A=A, ramp_steps=3, phi=phi)
        st, caches = O.rollout(O.State.rest(pts), m, sc, 4, advect=True, growth=gr)
        return st, caches, gr

    A0 = 0.2
    st, caches, gr = run(A0)
    n = pts.shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    out = O.rollout_vjp(caches, O.seed_mse(st.x, x_obs), z3, z33, z33, z33, advect=True, growth=gr)
    h = 1e-6
    fd = (O.loss_mse(run(A0 + h)[0].x, x_obs) - O.loss_mse(run(A0 - h)[0].x, x_obs)) / (2 * h)
    assert abs(out[5] - fd) < 1e-6 * abs(fd)


def test_extension_fd_explicit_fg_detF():
    rng = np.random.default_rng(6)
    sc = _ext_scene()
    pts = rng.uniform(0.3, 0.7, size=(24, 3))
    m = O.Model.elastic("nh", 1e4, 0.3)

    def L(g):
        st, _ = O.rollout(O.State.rest(pts, g), m, sc, 3, advect=True, keep_caches=False)
        return O.loss_detF(st.F)
    st, caches = O.rollout(O.State.rest(pts, 1.2), m, sc, 3, advect=True)
    n = pts.shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    Fgb = O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True)[4]
    dg = np.trace(Fgb, axis1=1, axis2=2).sum()
    fd = (L(1.2 + 1e-6) - L(1.2 - 1e-6)) / 2e-6
    assert abs(dg - fd) < 1e-6 * abs(fd)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "python", "morphompm")), reason="reference not mounted")
def test_oracle_vs_live_reference():
    """Fresh random scene through the reference package itself (read-only)."""
    import sys
    sys.path.insert(0, os.path.join(REF, "python"))
    from morphompm import config, constitutive, transfer, state
    rng = np.random.default_rng(99)
    cfg = config.SimConfig(N=9, dx=0.11, dt=7e-4, damping=0.1, sp=0.04)
    n = 20
    x = rng.uniform(0.1, 0.9, size=(n, 3))
    v = rng.standard_normal((n, 3)) * 0.3
    Cm = rng.standard_normal((n, 3, 3)) * 0.3
    F = np.eye(3) + 0.05 * rng.standard_normal((n, 3, 3))
    Fg = 1.2 * np.eye(3) + 0.03 * rng.standard_normal((n, 3, 3))
    bars = [rng.standard_normal(s) for s in ((n, 3), (n, 3), (n, 3, 3), (n, 3, 3), (n, 3, 3))]
    sc = O.scene_from_cfg(9, 0.11, 7e-4, 0.1, 0.04, 1000.0)
    for rm, om in ((constitutive.Hencky(cfg.material), O.Model.elastic("hencky", 1e4, 0.3)),
                   (constitutive.HerschelBulkley(), O.Model("hb"))):
        ns_r, c_r = transfer.step(state.ParticleState(x, v, Cm, F, Fg), rm, cfg, advect=True)
        g_r = transfer.step_vjp(c_r, *bars, advect=True)
        ns_o, c_o = O.step(O.State(x, v, Cm, F, Fg), om, sc, advect=True)
        g_o = O.step_vjp(c_o, *bars, advect=True)
        assert rel(ns_o.F, ns_r.F) < 1e-13 and rel(ns_o.x, ns_r.x) < 1e-15
        for a, b in zip(g_o, g_r):
            assert rel(a, b) < 1e-12


def _confined_root(tau_zz, lo=1.0, hi=4.0, it=200):
    """Bisection for tau_zz(lam) = 0 (tau_zz increasing in lam)."""
    for _ in range(it):
        mid = 0.5 * (lo + hi)
        if tau_zz(mid) > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def test_confined_swell_gate():
    """The reference's confined-swell check (constitutive.py:155-179): neo-Hookean,
    E = 1e4, nu = 0.3, Fg = 1.5 I, laterally confined F = diag(1, 1, lam);
    tau_zz(lam*) = 0 at lam* = 2.0028 with tau_xx = -5147.403."""
    m = O.Model.elastic("nh", 1e4, 0.3)
    Fg = 1.5 * np.eye(3)[None]
    tau = lambda lam: O.stress(m, np.diag([1.0, 1.0, lam])[None], Fg)[0]
    lam = _confined_root(lambda l: tau(l)[2, 2])
    assert abs(lam - 2.0028) < 5e-5
    assert abs(tau(lam)[0, 0] - (-5147.403)) < 1e-3
    assert abs(tau(lam)[2, 2]) < 1e-9


def test_confined_swell_helper_matches_the_model():
    """constitutive.confined_swell_neohookean (the reference's closed-form
    helper, constitutive.py:150-170): the reference's numbers at g = 1.5, and
    at other materials and growths the oracle's neo-Hookean stress at the
    returned stretch has tau_zz = 0 and the returned tau_xx."""
    from morphompm_b200.config import Material
    from morphompm_b200.constitutive import confined_swell_neohookean
    s, txx = confined_swell_neohookean(Material(E=1e4, nu=0.3))
    assert abs(s - 2.0028) < 5e-5 and abs(txx + 5147.403) < 1e-3
    for E, nu, g in ((1e4, 0.3, 1.5), (2e3, 0.45, 1.2), (5e2, 0.2, 1.05), (1e4, 0.3, 1.0)):
        mat = Material(E=E, nu=nu)
        s, txx = confined_swell_neohookean(mat, g)
        tau = O.stress(O.Model.elastic("nh", E, nu), np.diag([1.0, 1.0, s])[None], g * np.eye(3)[None])[0]
        assert abs(tau[2, 2]) < 1e-9 * mat.mu
        assert abs(tau[0, 0] - txx) < 1e-9 * mat.mu
