"""Generate the golden fixtures in this folder by running the UNMODIFIED reference
package (2nugu/morphompm, ``python/morphompm``) read-only.

    python tests/golden/make_golden.py --ref /path/to/reference [--only io|c1full]

The reference cannot travel to the GPU machine, so its outputs are committed as
small ``.npz`` fixtures.  Every fixture records the exact inputs it was made from.
Known-answer values quoted by the reference's own gates (transfer.py:162-193,
integrate.py:55-128, diff.py:27-45, constitutive.py:155-179) are recomputed here
and stored next to the arrays.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_ref(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "python"))
    import morphompm  # noqa: F401  (the reference package)
    from morphompm import config, constitutive, transfer, integrate, diff, state
    return config, constitutive, transfer, integrate, diff, state


PTS5 = np.array([[0.40, 0.40, 0.40], [0.42, 0.40, 0.41], [0.40, 0.43, 0.40],
                 [0.41, 0.40, 0.44], [0.44, 0.44, 0.43]])   # transfer.py:167-168


def make_constitutive(ref):
    config, constitutive, *_ = ref
    mat = config.Material()
    rng = np.random.default_rng(11)
    out = {}
    models = {"nh": constitutive.NeoHookean(mat), "hencky": constitutive.Hencky(mat),
              "hb": constitutive.HerschelBulkley()}
    n = 24
    F = np.eye(3) + 0.08 * rng.standard_normal((n, 3, 3))
    Fg = np.diag([1.3, 1.1, 0.9]) + 0.05 * rng.standard_normal((n, 3, 3))
    C = 0.5 * rng.standard_normal((n, 3, 3))
    # degenerate / isotropic rows (the Hencky rest regime, constitutive.py:220-230)
    F[0] = 1.3 * np.eye(3)
    Fg[0] = np.eye(3)
    F[1] = np.diag([1.5, 1.5, 1.2]) + 1e-4 * rng.standard_normal((3, 3))
    Fg[1] = np.eye(3)
    F[2] = 1.2 * np.eye(3)
    Fg[2] = 1.2 * np.eye(3)
    C[2] = 0.0
    tb = rng.standard_normal((n, 3, 3))
    tb = 0.5 * (tb + np.swapaxes(tb, 1, 2))
    out.update(F=F, Fg=Fg, C=C, tau_bar=tb)
    for name, m in models.items():
        taus, Fbs, Fgbs, Cbs = [], [], [], []
        for p in range(n):
            taus.append(m.stress(F[p], Fg[p], C[p]))
            a, b, c = m.stress_vjp(F[p], Fg[p], C[p], tb[p])
            Fbs.append(a); Fgbs.append(b); Cbs.append(c)
        out[f"{name}_tau"] = np.array(taus)
        out[f"{name}_F_bar"] = np.array(Fbs)
        out[f"{name}_Fg_bar"] = np.array(Fgbs)
        out[f"{name}_C_bar"] = np.array(Cbs)
    lz, txx = constitutive.confined_swell_neohookean(config.Material(E=1e4, nu=0.3), g=1.5)
    out["confined_lz"] = lz
    out["confined_txx"] = txx
    np.savez_compressed(os.path.join(HERE, "constitutive.npz"), **out)


def _rand_scene_state(rng, n, lo, hi, g):
    x = rng.uniform(lo, hi, size=(n, 3))
    v = 0.2 * rng.standard_normal((n, 3))
    C = 0.5 * rng.standard_normal((n, 3, 3))
    F = np.eye(3) + 0.05 * rng.standard_normal((n, 3, 3))
    Fg = g * np.eye(3) + 0.02 * rng.standard_normal((n, 3, 3))
    return x, v, C, F, Fg


def make_step(ref):
    """One step + step_vjp on a random 48-particle scene, every model, both
    advect modes, including particles whose stencil leaves the grid."""
    config, constitutive, transfer, integrate, diff, state = ref
    rng = np.random.default_rng(12)
    cfg = config.SimConfig(N=10, dx=0.1, dt=1.0e-3, damping=0.05, sp=0.05)
    n = 48
    x, v, C, F, Fg = _rand_scene_state(rng, n, 0.2, 0.8, 1.1)
    x[0] = [0.04, 0.5, 0.5]       # stencil clipped at the low wall
    x[1] = [0.5, 0.97, 0.5]       # clipped at the high wall
    x[2] = [0.5, 0.5, 1.12]       # entirely outside the grid
    bars = [rng.standard_normal((n, 3)), rng.standard_normal((n, 3)),
            rng.standard_normal((n, 3, 3)), rng.standard_normal((n, 3, 3)),
            rng.standard_normal((n, 3, 3))]
    out = dict(x=x, v=v, C=C, F=F, Fg=Fg, xn_b=bars[0], vn_b=bars[1], Cn_b=bars[2],
               Fn_b=bars[3], Fgn_b=bars[4], N=cfg.N, dx=cfg.dx, dt=cfg.dt,
               damping=cfg.damping, sp=cfg.sp, density=cfg.material.density,
               E=cfg.material.E, nu=cfg.material.nu)
    models = {"nh": constitutive.NeoHookean(cfg.material), "hencky": constitutive.Hencky(cfg.material),
              "hb": constitutive.HerschelBulkley()}
    for name, m in models.items():
        for adv in (False, True):
            st = state.ParticleState(x.copy(), v.copy(), C.copy(), F.copy(), Fg.copy())
            ns, cache = transfer.step(st, m, cfg, advect=adv)
            grads = transfer.step_vjp(cache, *[b.copy() for b in bars], advect=adv)
            tag = f"{name}_{'adv' if adv else 'fix'}"
            out[f"{tag}_new"] = np.concatenate([ns.x, ns.v, ns.C.reshape(n, 9), ns.F.reshape(n, 9)], axis=1)
            out[f"{tag}_gm"] = cache[3]
            out[f"{tag}_gv"] = cache[4]
            out[f"{tag}_grads"] = np.concatenate([grads[0], grads[1], grads[2].reshape(n, 9),
                                                   grads[3].reshape(n, 9), grads[4].reshape(n, 9)], axis=1)
    np.savez_compressed(os.path.join(HERE, "step.npz"), **out)


def make_gates(ref):
    """Known answers of the reference's own gates."""
    config, constitutive, transfer, integrate, diff, state = ref
    out = {}
    cfg = config.SimConfig()
    nh = constitutive.NeoHookean(cfg.material)
    hb = constitutive.HerschelBulkley()
    # single-step assembly (transfer.py:162-193)
    st = integrate.iso_growth_state(PTS5, 1.30)
    ns, cache = transfer.step(st, nh, cfg, advect=False)
    n = 5
    Fn_b = np.stack([np.linalg.det(ns.F[p]) * np.linalg.inv(ns.F[p]).T for p in range(n)])
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    Fg_b = transfer.step_vjp(cache, z3, z3, z33, Fn_b, z33, advect=False)[4]
    out["single_step_dg"] = float(sum(np.trace(Fg_b[p]) for p in range(n)))
    out["single_step_F"] = ns.F
    # 3-step trajectories (integrate.py:113-128)
    for tag, model, adv in (("nh_fix", nh, False), ("nh_adv", nh, True), ("hb_fix", hb, False)):
        L, dg = integrate.dloss_dg(PTS5, model, cfg, 1.30, 3, adv)
        out[f"traj_{tag}_loss"] = L
        out[f"traj_{tag}_dg"] = dg
    # inverse (diff.py:27-45)
    st, _ = integrate.rollout(integrate.iso_growth_state(PTS5, 1.40), nh, cfg, 3)
    target = integrate.loss_detF(st.F)
    g_rec, iters = diff.infer_growth(PTS5, nh, cfg, target, 3, g_init=1.15)
    out["inverse_target"] = target
    out["inverse_g"] = g_rec
    out["inverse_iters"] = iters
    # forward physics free swell (integrate.py:67-89)
    fcfg = config.SimConfig(N=12, dx=0.05, dt=1.0e-3, damping=0.05, sp=0.03)
    c = np.arange(0.30 - 0.015, 0.30 + 0.015 + 1e-9, 0.03)
    pts8 = np.array([(a, b, d) for a in c for b in c for d in c])
    out["swell_pts"] = pts8
    for name, model in (("nh", constitutive.NeoHookean(fcfg.material)),
                        ("hencky", constitutive.Hencky(fcfg.material)),
                        ("hb", constitutive.HerschelBulkley())):
        st, _ = integrate.rollout(integrate.iso_growth_state(pts8, 1.5), model, fcfg, 150, advect=True)
        out[f"swell_{name}_detF"] = float(np.mean([np.linalg.det(st.F[p]) for p in range(st.n)]))
        out[f"swell_{name}_F"] = st.F
        out[f"swell_{name}_x"] = st.x
    # numpy <-> C++ parity scene (test_growth.cpp:337-357, parity.py:34-38)
    coords = np.arange(0.27, 0.33 + 1e-9, 0.03)
    pts27 = np.array([(a, b, d) for a in coords for b in coords for d in coords])
    st, _ = integrate.rollout(integrate.iso_growth_state(pts27, 1.05), constitutive.Hencky(fcfg.material),
                              fcfg, 30, advect=True)
    out["parity27_pts"] = pts27
    out["parity27_F"] = st.F
    out["parity27_x"] = st.x
    np.savez_compressed(os.path.join(HERE, "gates.npz"), **out)


def make_c1_head(ref):
    """First 3 steps of the 4096-particle free-swell cube (32^3 grid, dx=1/32,
    dt=1e-4, neo-Hookean E=1e3 nu=0.3 rho=1, growth ramp 1 -> 1.1 over 100
    steps) run through the reference step; Fg is re-set between steps, the same
    way a caller drives the reference's growth-agnostic step."""
    config, constitutive, transfer, integrate, diff, state = ref
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from morphompm_b200 import scenes
    sc = scenes.config1()
    cfg = config.SimConfig(N=32, dx=sc["dx"], dt=sc["dt"], damping=sc["damping"], sp=sc["dx"] / 2,
                           material=config.Material(E=1e3, nu=0.3, density=1.0))
    model = constitutive.NeoHookean(cfg.material)
    st = state.ParticleState.rest(sc["x"])
    steps = 3
    for t in range(steps):
        g = 1.0 + sc["growth_A"] * min(1.0, (t + 1) / sc["ramp_steps"])
        st.Fg[:] = g * np.eye(3)
        st, _ = transfer.step(st, model, cfg, advect=True)
    np.savez_compressed(os.path.join(HERE, "c1_head.npz"), x0=sc["x"], steps=steps,
                        x=st.x, F=st.F, v=st.v)


def make_c1_full(ref):
    """The whole 100-step free-swell cube of ``make_c1_head`` through the
    reference step, then its trajectory adjoint through the reference
    ``step_vjp`` for the loss sum det F (integrate.py:45-52).  The caller
    re-sets Fg = g(t) I before every step, so each step's Fg is an input of
    its own: its cotangent does not flow back into the previous step, and
    d loss / d A = sum_t ramp(t) sum_p tr(Fg_bar_t).  Takes about 15 minutes
    on one core."""
    config, constitutive, transfer, integrate, diff, state = ref
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from morphompm_b200 import scenes
    sc = scenes.config1()
    cfg = config.SimConfig(N=32, dx=sc["dx"], dt=sc["dt"], damping=sc["damping"], sp=sc["dx"] / 2,
                           material=config.Material(E=1e3, nu=0.3, density=1.0))
    model = constitutive.NeoHookean(cfg.material)
    st = state.ParticleState.rest(sc["x"])
    steps = sc["steps"]
    caches, ramps = [], []
    for t in range(steps):
        r = min(1.0, (t + 1) / sc["ramp_steps"])
        st.Fg[:] = (1.0 + sc["growth_A"] * r) * np.eye(3)
        st, cache = transfer.step(st, model, cfg, advect=True)
        caches.append(cache)
        ramps.append(r)
    n = st.n
    loss = integrate.loss_detF(st.F)
    xb, vb = np.zeros((n, 3)), np.zeros((n, 3))
    Cb = np.zeros((n, 3, 3))
    Fb = np.stack([np.linalg.det(st.F[p]) * np.linalg.inv(st.F[p]).T for p in range(n)])
    dA = 0.0
    for t in reversed(range(steps)):
        xb, vb, Cb, Fb, Fgb = transfer.step_vjp(caches[t], xb, vb, Cb, Fb, np.zeros((n, 3, 3)), advect=True)
        dA += ramps[t] * integrate.iso_growth_grad(Fgb)
        caches[t] = None
    np.savez_compressed(os.path.join(HERE, "c1_full.npz"), steps=steps, x=st.x, F=st.F, loss=loss,
                        dloss_dA=dA, x0_bar=xb, F0_bar=Fb)


def make_io(ref_root):
    """Files written by the reference's own I/O adapters (io.py:29-111) for a
    small state and config, so that the device-side writers are checked byte
    for byte."""
    sys.path.insert(0, os.path.join(ref_root, "python"))
    from morphompm import io as rio
    from morphompm.state import ParticleState
    from morphompm.config import SimConfig, Material
    rng = np.random.default_rng(13)
    n = 7
    st = ParticleState(rng.standard_normal((n, 3)), rng.standard_normal((n, 3)), rng.standard_normal((n, 3, 3)),
                       np.tile(np.eye(3), (n, 1, 1)) + 0.05 * rng.standard_normal((n, 3, 3)),
                       np.tile(1.2 * np.eye(3), (n, 1, 1)))
    st.x[0, 1] = -0.0          # formatting of signed zero
    st.v[1, 2] = 1.0e-5        # and of an exponent
    np.savez_compressed(os.path.join(HERE, "io_state.npz"), x=st.x, v=st.v, C=st.C, F=st.F, Fg=st.Fg)
    rio.save_state(st, os.path.join(HERE, "io_state.csv"))
    rio.save_state(st, os.path.join(HERE, "io_state.vtk"))
    rio.save_config(SimConfig(N=12, dx=0.05, dt=2e-4, damping=0.07, sp=0.025,
                              material=Material(E=3.0e3, nu=0.35, density=900.0)),
                    os.path.join(HERE, "io_config.json"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MORPHOMPM_REF"),
                    help="root of the reference project (or set MORPHOMPM_REF)")
    ap.add_argument("--skip-c1", action="store_true")
    ap.add_argument("--only", choices=["io", "c1full"], default=None, help="write one group of fixtures")
    a = ap.parse_args()
    if not a.ref:
        ap.error("the reference root is required: --ref PATH or MORPHOMPM_REF")
    if a.only == "io":
        make_io(a.ref)
        print("golden I/O fixtures written to", HERE)
        return
    ref = _import_ref(a.ref)
    if a.only == "c1full":
        make_c1_full(ref)
        print("golden c1_full fixture written to", HERE)
        return
    make_constitutive(ref)
    make_step(ref)
    make_gates(ref)
    if not a.skip_c1:
        make_c1_head(ref)
        make_c1_full(ref)
    make_io(a.ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
