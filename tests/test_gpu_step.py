"""GPU parity of the sm_100a kernels against the reference's golden outputs and
the oracle: constitutive seam, binning, one step + VJP, the reference's gates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import mpm_oracle as O


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


PTS5 = np.array([[0.40, 0.40, 0.40], [0.42, 0.40, 0.41], [0.40, 0.43, 0.40],
                 [0.41, 0.40, 0.44], [0.44, 0.44, 0.43]])


def _models(E=1e4, nu=0.3):
    from morphompm_b200 import constitutive as K
    from morphompm_b200.config import Material
    mat = Material(E=E, nu=nu)
    return {"nh": K.NeoHookean(mat), "hencky": K.Hencky(mat), "hb": K.HerschelBulkley()}


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
def test_constitutive_fp64(golden, name):
    d = golden("constitutive.npz")
    m = _models()[name]
    tau = m.stress(d["F"], d["Fg"], d["C"])
    assert rel(tau, d[f"{name}_tau"]) < 1e-12
    Fb, Fgb, Cb = m.stress_vjp(d["F"], d["Fg"], d["C"], d["tau_bar"])
    tol = 1e-10 if name != "hencky" else 1e-8    # Hencky: reference's 1e-9 divided-difference switch
    assert rel(Fb, d[f"{name}_F_bar"]) < tol
    assert rel(Fgb, d[f"{name}_Fg_bar"]) < tol
    if name == "hb":
        assert rel(Cb, d["hb_C_bar"]) < 1e-11
    # single-matrix call returns a 3x3
    assert m.stress(d["F"][3], d["Fg"][3], d["C"][3]).shape == (3, 3)


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
def test_constitutive_fp32(golden, name):
    d = golden("constitutive.npz")
    m = _models()[name]
    f32 = lambda a: torch.tensor(a, dtype=torch.float32, device="cuda")
    tau = m.stress(f32(d["F"]), f32(d["Fg"]), f32(d["C"]))
    assert tau.dtype == torch.float32
    assert rel(tau, d[f"{name}_tau"]) < 2e-5
    Fb, Fgb, Cb = m.stress_vjp(f32(d["F"]), f32(d["Fg"]), f32(d["C"]), f32(d["tau_bar"]))
    assert rel(Fb, d[f"{name}_F_bar"]) < 5e-5
    assert rel(Fgb, d[f"{name}_Fg_bar"]) < 5e-5


def _spectra_cases(rng):
    """Deformations F = Q diag(s) R^T with chosen singular values s (random
    rotations Q, R) and growth Fg = g I: the FP32 Hencky eigensolve's hard cases."""
    def rot():
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        q = q * np.sign(np.diag(r))
        return q if np.linalg.det(q) > 0 else -q
    s_sets = {
        "pair_gap_1e-5": [1.2, 1.2 * (1 + 1e-5), 0.9],       # just above the 1e-6 FP64-fallback gap
        "pair_gap_1e-3": [1.1, 1.1 * (1 + 1e-3), 1.1 * (1 - 1e-3)],
        "near_iso_1e-4": [1.05, 1.05 * (1 + 1e-4), 1.05 * (1 - 2e-4)],
        "exact_pair": [1.2, 1.2, 0.9],                         # below the gap: FP64 recompute
        "isotropic": [1.07, 1.07, 1.07],
        "rotation": [1.0, 1.0, 1.0],
        "large_stretch": [2.0, 0.5, 1.0],
        "compressed": [0.6, 0.7, 0.8],
    }
    out = {}
    for k, s in s_sets.items():
        F = np.stack([rot() @ np.diag(s) @ rot().T for _ in range(64)])
        Fg = np.broadcast_to(np.eye(3) * rng.uniform(0.9, 1.1), F.shape).copy()
        out[k] = (F, Fg)
    F = np.eye(3) + 0.2 * rng.standard_normal((64, 3, 3))
    F[np.linalg.det(F) < 0.3] = np.eye(3)
    out["random"] = (F, np.broadcast_to(np.eye(3), F.shape).copy())
    return out


@pytest.mark.parametrize("case", ["pair_gap_1e-5", "pair_gap_1e-3", "near_iso_1e-4", "exact_pair", "isotropic",
                                  "rotation", "large_stretch", "compressed", "random"])
def test_hencky_fp32_spectra_vs_fp64(case):
    """FP32 Hencky stress and VJP (closed-form eigensolve, FP64 recompute below
    the singular-value gap threshold) against the FP64 path (Jacobi sweeps),
    for spectra with close, equal and far-apart singular values."""
    rng = np.random.default_rng(11)
    F, Fg = _spectra_cases(rng)[case]
    C = np.zeros_like(F)
    tb = rng.standard_normal(F.shape)
    m = _models()["hencky"]
    dev = lambda a, dt: torch.tensor(a, dtype=dt, device="cuda")
    t64 = m.stress(dev(F, torch.float64), dev(Fg, torch.float64), dev(C, torch.float64))
    b64 = m.stress_vjp(dev(F, torch.float64), dev(Fg, torch.float64), dev(C, torch.float64), dev(tb, torch.float64))
    # the FP32 path sees the FP32-rounded inputs; compare against FP64 on the same values
    F32, Fg32, tb32 = (a.astype(np.float32) for a in (F, Fg, tb))
    t64r = m.stress(dev(F32, torch.float64), dev(Fg32, torch.float64), dev(C, torch.float64))
    b64r = m.stress_vjp(dev(F32, torch.float64), dev(Fg32, torch.float64), dev(C, torch.float64),
                        dev(tb32, torch.float64))
    t32 = m.stress(dev(F32, torch.float32), dev(Fg32, torch.float32), dev(C, torch.float32))
    b32 = m.stress_vjp(dev(F32, torch.float32), dev(Fg32, torch.float32), dev(C, torch.float32),
                       dev(tb32, torch.float32))
    assert torch.isfinite(t32).all() and torch.isfinite(b32[0]).all() and torch.isfinite(b32[1]).all()
    # error relative to the largest entry of the batch (tau vanishes for a pure rotation)
    scale = lambda a: max(float(a.abs().max()), 1.0)
    e_tau = float((t32.double() - t64r).abs().max()) / scale(t64r)
    e_fb = float((b32[0].double() - b64r[0]).abs().max()) / scale(b64r[0])
    e_fgb = float((b32[1].double() - b64r[1]).abs().max()) / scale(b64r[1])
    assert e_tau < 2e-5 and e_fb < 5e-5 and e_fgb < 5e-5, (case, e_tau, e_fb, e_fgb)
    assert float((t64r - t64).abs().max()) / scale(t64) < 1e-5          # input rounding only
    assert b64[0].shape == b32[0].shape


def test_bin_keys_bit_exact():
    """Cell keys of the device binning equal the oracle's (transfer.py:19-21),
    including particles exactly on half-cell boundaries and outside the grid."""
    import ctypes as C
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import SceneSpec
    rng = np.random.default_rng(3)
    for shape, dx in (((32, 32, 32), 1 / 32), ((10, 9, 11), 0.1), ((96, 32, 32), 1 / 32)):
        sc = O.Scene(shape=shape, dx=dx)
        n = 20000
        x = rng.uniform(-0.1, 1.1, size=(n, 3)) * np.array(shape) * dx
        x[:2000] = (rng.integers(-3, max(shape) + 3, size=(2000, 3)) + 0.5) * dx   # exact half-cells
        x[2000:3000] = rng.integers(0, max(shape), size=(1000, 3)) * dx           # exact nodes
        ref = O.cell_keys(x, sc)
        spec = SceneSpec(shape=shape, n=n, model=0, dx=dx, dt=0, damping=0, pmass=0, vol0=0).to_c(0)
        for dt in (torch.float64, torch.float32):
            xd = torch.tensor(x, dtype=dt, device="cuda").contiguous()
            keys = torch.empty(n, dtype=torch.int32, device="cuda")
            L.check(L.load().mpm_bin_keys(C.byref(spec), xd.element_size(), n, xd.data_ptr(), keys.data_ptr(),
                                          C.c_void_p(torch.cuda.current_stream().cuda_stream)))
            got = keys.cpu().numpy()
            if dt == torch.float64:
                assert np.array_equal(got, ref)
            else:
                ref32 = O.cell_keys(x.astype(np.float32).astype(np.float64), sc)
                if dx in (1 / 32,):        # power-of-two inv_dx: FP32 binning is exact
                    assert np.array_equal(got, ref32)
                else:
                    # non-power-of-two inv_dx: only points planted on cell
                    # boundaries may bin differently in FP32
                    assert np.array_equal(got[3000:], ref32[3000:]) or np.mean(got[3000:] == ref32[3000:]) > 0.9995


def _step_inputs(d):
    return [d[k].copy() for k in ("x", "v", "C", "F", "Fg")]


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
@pytest.mark.parametrize("adv", [False, True])
def test_step_and_vjp_fp64_vs_reference(golden, name, adv):
    from morphompm_b200 import transfer
    from morphompm_b200.config import SimConfig
    from morphompm_b200.state import ParticleState
    d = golden("step.npz")
    n = d["x"].shape[0]
    cfg = SimConfig(N=int(d["N"]), dx=float(d["dx"]), dt=float(d["dt"]), damping=float(d["damping"]),
                    sp=float(d["sp"]))
    m = _models()[name]
    ns, cache = transfer.step(ParticleState(*_step_inputs(d)), m, cfg, advect=adv)
    tag = f"{name}_{'adv' if adv else 'fix'}"
    new = np.concatenate([ns.x, ns.v, ns.C.reshape(n, 9), ns.F.reshape(n, 9)], 1)
    assert isinstance(ns.x, np.ndarray)
    assert rel(new, d[tag + "_new"]) < 1e-12
    assert np.array_equal(ns.Fg, d["Fg"])
    g = transfer.step_vjp(cache, d["xn_b"], d["vn_b"], d["Cn_b"], d["Fn_b"], d["Fgn_b"], advect=adv)
    grads = np.concatenate([g[0], g[1], g[2].reshape(n, 9), g[3].reshape(n, 9), g[4].reshape(n, 9)], 1)
    tol = 1e-10 if name != "hencky" else 1e-8
    assert rel(grads, d[tag + "_grads"]) < tol
    if not adv:
        assert np.all(g[0] == 0)


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
def test_step_fp32_close(golden, name):
    from morphompm_b200 import transfer
    from morphompm_b200.config import SimConfig
    from morphompm_b200.state import ParticleState
    d = golden("step.npz")
    cfg = SimConfig(N=int(d["N"]), dx=float(d["dx"]), dt=float(d["dt"]), damping=float(d["damping"]),
                    sp=float(d["sp"]))
    t32 = [torch.tensor(a, dtype=torch.float32, device="cuda") for a in _step_inputs(d)]
    ns, cache = transfer.step(ParticleState(*t32), _models()[name], cfg, advect=True)
    assert ns.F.dtype == torch.float32 and ns.F.is_cuda
    ref = d[f"{name}_adv_new"][:, 15:24].reshape(-1, 3, 3)
    assert rel(ns.F, ref) < 1e-5


def test_reference_gate_values(golden):
    """Known answers of the reference's own gates, through the GPU FP64 path."""
    from morphompm_b200 import transfer, integrate, diff
    from morphompm_b200.config import SimConfig
    g = golden("gates.npz")
    cfg = SimConfig()
    nh = _models()["nh"]
    st = integrate.iso_growth_state(PTS5, 1.30)
    ns, cache = transfer.step(st, nh, cfg, advect=False)
    Fn_b = np.stack([np.linalg.det(ns.F[p]) * np.linalg.inv(ns.F[p]).T for p in range(5)])
    z3, z33 = np.zeros((5, 3)), np.zeros((5, 3, 3))
    Fg_b = transfer.step_vjp(cache, z3, z3, z33, Fn_b, z33, advect=False)[4]
    dg = integrate.iso_growth_grad(Fg_b)
    assert abs(dg - float(g["single_step_dg"])) < 1e-12 * abs(dg)
    for tag, model, adv in (("nh_fix", nh, False), ("nh_adv", nh, True), ("hb_fix", _models()["hb"], False)):
        L, dg = integrate.dloss_dg(PTS5, model, cfg, 1.30, 3, adv)
        assert abs(dg - float(g[f"traj_{tag}_dg"])) < 1e-11 * abs(dg), tag
        assert abs(L - float(g[f"traj_{tag}_loss"])) < 1e-12 * abs(L), tag
    # reference-style rollout / rollout_vjp with per-step caches
    st, caches = integrate.rollout(integrate.iso_growth_state(PTS5, 1.3), nh, cfg, 3, advect=True)
    Ff_b = np.stack([np.linalg.det(st.F[p]) * np.linalg.inv(st.F[p]).T for p in range(5)])
    Fg_b = integrate.rollout_vjp(caches, z3, z3, z33, Ff_b, z33, advect=True)[4]
    assert abs(integrate.iso_growth_grad(Fg_b) - float(g["traj_nh_adv_dg"])) < 1e-11
    # inverse (diff.py:27-45), unchanged driver
    g_rec, iters = diff.infer_growth(PTS5, nh, cfg, float(g["inverse_target"]), 3, g_init=1.15)
    assert abs(g_rec - 1.40) < 1e-4 and iters == int(g["inverse_iters"])


def test_free_swell_and_cpp_parity_scene(golden):
    from morphompm_b200 import integrate
    from morphompm_b200.config import SimConfig
    g = golden("gates.npz")
    cfg = SimConfig(N=12, dx=0.05, dt=1.0e-3, damping=0.05, sp=0.03)
    for name, m in _models().items():
        st, _ = integrate.rollout(integrate.iso_growth_state(g["swell_pts"], 1.5), m, cfg, 150, advect=True)
        assert rel(st.F, g[f"swell_{name}_F"]) < 1e-10, name
    st, _ = integrate.rollout(integrate.iso_growth_state(g["parity27_pts"], 1.05), _models()["hencky"], cfg, 30,
                              advect=True)
    assert rel(st.F, g["parity27_F"]) < 1e-11


def test_confined_swell_gate_on_device():
    """constitutive.py:155-179 through the device stress (FP64): the root of
    tau_zz for a laterally confined swelling block, and tau_xx there, equal the
    oracle's and the reference's 2.0028 / -5147.403."""
    from oracle import mpm_oracle as O
    m = _models()["nh"]
    om = O.Model.elastic("nh", 1e4, 0.3)
    Fg = 1.5 * np.eye(3)
    lo, hi = 1.0, 4.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if m.stress(np.diag([1.0, 1.0, mid]), Fg)[2, 2] > 0:
            hi = mid
        else:
            lo = mid
    lam = 0.5 * (lo + hi)
    tau = m.stress(np.diag([1.0, 1.0, lam]), Fg)
    assert abs(lam - 2.0028) < 5e-5
    assert abs(tau[0, 0] - (-5147.403)) < 1e-3
    otau = O.stress(om, np.diag([1.0, 1.0, lam])[None], Fg[None])[0]
    assert np.max(np.abs(tau - otau)) < 1e-12 * 5147.403
