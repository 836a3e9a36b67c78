"""GPU trajectories: checkpoint recompute, finite-difference gates on the
device FP64 path, the growth-law batch against the oracle, batching and
determinism, and the 4096-particle free-swell scene against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from oracle import mpm_oracle as O


def _cfg(**kw):
    from morphompm_b200.config import SimConfig
    return SimConfig(**kw)


def _mat(E=1e4, nu=0.3):
    from morphompm_b200.config import Material
    return Material(E=E, nu=nu)


def test_checkpoint_recompute_is_bitwise_identical():
    from morphompm_b200 import integrate
    from morphompm_b200.constitutive import Hencky
    rng = np.random.default_rng(0)
    pts = rng.uniform(0.35, 0.65, size=(200, 3))
    cfg = _cfg(N=16, dx=1 / 16, dt=5e-4, sp=1 / 32, wall=2)
    m = Hencky(_mat())
    a = integrate.dloss_dg(pts, m, cfg, 1.2, 12, True)
    b = integrate.dloss_dg(pts, m, cfg, 1.2, 12, True, ckpt_every=5)
    c = integrate.dloss_dg(pts, m, cfg, 1.2, 12, True, ckpt_every=1)
    assert a == b == c


@pytest.mark.parametrize("kind", ["nh", "hencky", "hb"])
def test_trajectory_gradient_vs_fd_fp64(kind):
    from morphompm_b200 import integrate
    from morphompm_b200.constitutive import NeoHookean, Hencky, HerschelBulkley
    rng = np.random.default_rng(1)
    pts = rng.uniform(0.3, 0.6, size=(60, 3))
    cfg = _cfg(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2, gravity=(0.0, -1.0, 0.0))
    m = {"nh": NeoHookean(_mat()), "hencky": Hencky(_mat()), "hb": HerschelBulkley()}[kind]
    for adv in (False, True):
        _, dg = integrate.dloss_dg(pts, m, cfg, 1.15, 5, adv)
        h = 1e-6
        fp, _ = integrate.dloss_dg(pts, m, cfg, 1.15 + h, 5, adv)
        fm, _ = integrate.dloss_dg(pts, m, cfg, 1.15 - h, 5, adv)
        fd = (fp - fm) / (2 * h)
        assert abs(dg - fd) < 1e-6 * abs(fd), (kind, adv, dg, fd)


def test_mse_loss_gradient_vs_oracle_and_fd():
    from morphompm_b200 import integrate
    from morphompm_b200.constitutive import NeoHookean
    rng = np.random.default_rng(2)
    pts = rng.uniform(0.35, 0.6, size=(80, 3))
    x_obs = pts + 0.01 * rng.standard_normal(pts.shape)
    cfg = _cfg(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2)
    m = NeoHookean(_mat())
    L, dg = integrate.dloss_dg(pts, m, cfg, 1.1, 6, True, loss="mse", x_obs=x_obs, ckpt_every=4)
    sc = O.Scene(shape=(12, 12, 12), dx=1 / 12, dt=4e-4, damping=0.05, pmass=1000 / 24 ** 3, vol0=1 / 24 ** 3,
                 wall=2)
    om = O.Model.elastic("nh", 1e4, 0.3)
    st, caches = O.rollout(O.State.rest(pts, 1.1), om, sc, 6, advect=True)
    z3, z33 = np.zeros((80, 3)), np.zeros((80, 3, 3))
    Fgb = O.rollout_vjp(caches, O.seed_mse(st.x, x_obs), z3, z33, z33, z33, advect=True)[4]
    assert abs(L - O.loss_mse(st.x, x_obs)) < 1e-12 * abs(L)
    assert abs(dg - np.trace(Fgb, axis1=1, axis2=2).sum()) < 1e-9 * abs(dg)


def _small_batch_scenes():
    from morphompm_b200 import scenes
    sc = scenes.config4(seed=7, n_scenes=3, n_lo=300, n_hi=3000)
    sc[0]["model"] = "nh"
    sc[1]["model"] = "hencky"
    sc[2]["model"] = "hencky"
    return sc


def _oracle_scene(s):
    sp = s["dx"] / 2
    return O.Scene(shape=s["shape"], dx=s["dx"], dt=s["dt"], damping=s["damping"], pmass=s["density"] * sp ** 3,
                   vol0=sp ** 3, wall=s["wall"])


def test_growth_law_batch_vs_oracle_fp64():
    from morphompm_b200.batch import Batch, host_slab
    scn = _small_batch_scenes()
    steps = 8
    b = Batch(scn, steps, dtype=torch.float64, ckpt_every=3)
    b.load(host_slab(scn, np.float64), non_blocking=False)
    b.run()
    torch.cuda.synchronize()
    loss = b.loss.cpu().numpy()
    dA = b.dloss_dg.cpu().numpy()
    for i, s in enumerate(scn):
        m = O.Model.elastic(s["model"], s["E"], s["nu"])
        gr = O.Growth(A=s["growth_A"])
        st, caches = O.rollout(O.State.rest(s["x"]), m, _oracle_scene(s), steps, advect=True, growth=gr)
        n = s["x"].shape[0]
        z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
        out = O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True, growth=gr)
        assert abs(loss[i] - O.loss_detF(st.F)) < 1e-12 * abs(loss[i])
        assert abs(dA[i] - out[5]) < 1e-9 * abs(out[5]), (i, dA[i], out[5])


def test_batch_equals_single_scene_runs_and_is_deterministic():
    from morphompm_b200.batch import Batch, host_slab
    scn = _small_batch_scenes()
    b = Batch(scn, 5, dtype=torch.float32)
    b.load(host_slab(scn), non_blocking=False)
    b.run()
    l1, g1 = b.loss.clone(), b.dloss_dg.clone()
    b.run()
    assert torch.equal(l1, b.loss) and torch.equal(g1, b.dloss_dg)
    b.capture()
    b.replay()
    torch.cuda.synchronize()
    assert torch.equal(l1, b.loss) and torch.equal(g1, b.dloss_dg)
    for i, s in enumerate(scn):
        one = Batch([s], 5, dtype=torch.float32)
        one.load(host_slab([s]), non_blocking=False)
        one.run()
        assert torch.equal(one.loss[0], l1[i]) and torch.equal(one.dloss_dg[0], g1[i])


def test_config1_free_swell_fp64_matches_oracle_1e10():
    """4096-particle cube, 32^3 grid, growth ramp 1 -> 1.1 over 100 steps:
    device FP64 vs the oracle, max|dF| <= 1e-10; FP32 error stated."""
    from morphompm_b200 import scenes
    from morphompm_b200.batch import Batch, host_slab
    c = scenes.config1()
    sp = c["dx"] / 2
    sc = O.Scene(shape=c["shape"], dx=c["dx"], dt=c["dt"], damping=c["damping"], pmass=c["density"] * sp ** 3,
                 vol0=sp ** 3, wall=c["wall"])
    st, _ = O.rollout(O.State.rest(c["x"]), O.Model.elastic("nh", c["E"], c["nu"]), sc, c["steps"], advect=True,
                      growth=O.Growth(A=c["growth_A"], ramp_steps=c["ramp_steps"]), keep_caches=False)
    res = {}
    for dt in (torch.float64, torch.float32):
        b = Batch([c], c["steps"], dtype=dt, ckpt_every=10)
        b.load(host_slab([c], np.float64 if dt == torch.float64 else np.float32), non_blocking=False)
        b.rollout.forward(b.slab0)
        fin = b.final_state().double().cpu().numpy()
        F = fin[15:24].T.reshape(-1, 3, 3)
        x = fin[0:3].T
        res[dt] = (np.max(np.abs(F - st.F)), np.max(np.abs(x - st.x)))
    assert res[torch.float64][0] <= 1e-10, res
    assert res[torch.float32][0] <= 1e-4, res
    assert abs(np.mean(np.linalg.det(st.F)) - 1.1 ** 3) < 0.1


@pytest.mark.parametrize("kind", ["nh", "hencky"])
def test_material_gradients_vs_fd_fp64(kind):
    """d loss / d (E, nu) of a device FP64 trajectory (mpm_step_bwd_params)
    against central differences of the loss in E and nu."""
    from morphompm_b200 import integrate
    from morphompm_b200.config import Material
    from morphompm_b200.constitutive import NeoHookean, Hencky
    rng = np.random.default_rng(5)
    pts = rng.uniform(0.3, 0.6, size=(60, 3))
    cfg = _cfg(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2)
    x_obs = pts + 0.02 * rng.standard_normal(pts.shape)
    cls = {"nh": NeoHookean, "hencky": Hencky}[kind]
    E, nu = 2.0e4, 0.28
    for loss in ("detF", "mse"):
        L, grads = integrate.dloss_dparams(pts, cls(Material(E=E, nu=nu)), cfg, 1.2, 5, True, loss=loss,
                                           x_obs=x_obs)
        L0, dg = integrate.dloss_dg(pts, cls(Material(E=E, nu=nu)), cfg, 1.2, 5, True, loss=loss, x_obs=x_obs)
        assert L == L0 and grads["g"] == dg
        for name, h in (("E", 1e-4 * E), ("nu", 1e-5)):
            kp = dict(E=E, nu=nu)
            km = dict(E=E, nu=nu)
            kp[name] += h
            km[name] -= h
            fp, _ = integrate.dloss_dg(pts, cls(Material(**kp)), cfg, 1.2, 5, True, loss=loss, x_obs=x_obs)
            fm, _ = integrate.dloss_dg(pts, cls(Material(**km)), cfg, 1.2, 5, True, loss=loss, x_obs=x_obs)
            fd = (fp - fm) / (2 * h)
            assert abs(grads[name] - fd) < 1e-6 * max(abs(fd), 1e-12) + 1e-14, (kind, loss, name, grads[name], fd)


def test_save_batch_writes_each_scene(tmp_path):
    from morphompm_b200 import io as mio, scenes
    from morphompm_b200.batch import Batch, host_slab
    sc = scenes.config4(seed=3, n_scenes=2, n_lo=300, n_hi=600)
    b = Batch(sc, 3, dtype=torch.float32, active_cap=None)
    b.load(host_slab(sc, np.float32), non_blocking=False)
    b.rollout.forward(b.slab0)
    paths = mio.save_batch(b, str(tmp_path / "scene{s}.npz"))
    fin = b.final_state().double().cpu().numpy()
    p0 = 0
    for s, path in enumerate(paths):
        st = mio.load_state(path)
        k = st.n
        assert k == sc[s]["x"].shape[0]
        np.testing.assert_array_equal(st.x, fin[0:3, p0:p0 + k].T)
        np.testing.assert_array_equal(st.F.reshape(k, 9), fin[15:24, p0:p0 + k].T)
        assert np.allclose(st.Fg, (1.0 + sc[s]["growth_A"]) * np.eye(3))
        p0 += k


def test_prefetch_matches_load():
    """Batch.prefetch (side-stream input copy overlapping the running
    trajectory) feeds each replay exactly the slab a blocking load would."""
    from morphompm_b200.batch import Batch, host_slab
    scn = _small_batch_scenes()
    b = Batch(scn, 5, dtype=torch.float32)
    s1 = host_slab(scn)
    s2 = s1.copy()
    s2[0:3] += 0.002
    pins = [torch.from_numpy(s).pin_memory() for s in (s1, s2)]
    ref = []
    for p in pins:
        b.load(p, non_blocking=False)
        b.replay()
        ref.append(b.loss.clone())
    got = []
    for i in (0, 1, 0, 1):
        b.prefetch(pins[i])
        b.replay()
        got.append(b.loss.clone())
    torch.cuda.synchronize()
    assert not torch.equal(ref[0], ref[1])
    for i, g in zip((0, 1, 0, 1), got):
        assert torch.equal(g, ref[i])


def test_config_dtype_and_checkpoint_fields():
    """SimConfig(dtype="float32") runs numpy inputs on the FP32 path (the
    result of passing FP32 tensors, returned as the input's numpy type);
    SimConfig(checkpoint_every=k) is the default ckpt_every of dloss_dg."""
    from morphompm_b200 import integrate, transfer
    from morphompm_b200.config import Material, SimConfig
    from morphompm_b200.constitutive import Hencky
    from morphompm_b200.state import ParticleState
    rng = np.random.default_rng(6)
    n = 40
    x = rng.uniform(0.3, 0.6, size=(n, 3))
    F = np.eye(3) + 0.02 * rng.standard_normal((n, 3, 3))
    st = ParticleState(x, 0.05 * rng.standard_normal((n, 3)), 0.1 * rng.standard_normal((n, 3, 3)), F,
                       1.1 * np.tile(np.eye(3), (n, 1, 1)))
    base = dict(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, material=Material(E=1e4, nu=0.3))
    m = Hencky(Material(E=1e4, nu=0.3))
    ns, _ = transfer.step(st, m, SimConfig(dtype="float32", **base))
    f32 = lambda a: torch.as_tensor(a, dtype=torch.float32, device="cuda")
    ref, _ = transfer.step(ParticleState(*(f32(a) for a in (st.x, st.v, st.C, st.F, st.Fg))), m, SimConfig(**base))
    assert isinstance(ns.F, np.ndarray) and ns.F.dtype == np.float64
    assert np.array_equal(ns.F, ref.F.double().cpu().numpy())
    a = integrate.dloss_dg(x, m, SimConfig(checkpoint_every=2, **base), 1.1, 5, True)
    b = integrate.dloss_dg(x, m, SimConfig(**base), 1.1, 5, True, ckpt_every=2)
    assert a == b
