"""Batched inverse problems on the device: new scene parameters replayed
through the captured trajectory graph (mpm_plan_update_scenes), the
reference's growth Gauss-Newton run for every scene of a batch at once, and a
multi-parameter fit with the material gradients."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _scenes(k=3, seed=21):
    from morphompm_b200 import scenes
    sc = scenes.config4(seed=seed, n_scenes=k, n_lo=600, n_hi=1500)
    for s in sc:
        s["dt"] = 1e-4           # long enough for the growth to move the particles
    return sc


def _batch(sc, steps, dtype=torch.float64, **kw):
    from morphompm_b200.batch import Batch, host_slab
    npd = np.float64 if dtype == torch.float64 else np.float32
    b = Batch(sc, steps, dtype=dtype, active_cap=None, **kw)
    b.load(host_slab(sc, npd), non_blocking=False)
    return b


def test_update_scenes_matches_a_fresh_batch():
    from morphompm_b200 import _lib as L
    sc = _scenes()
    b = _batch(sc, 6)
    b.replay()
    A = np.array([0.05, 0.25, 0.12])
    E = np.array([800.0, 3000.0, 1500.0])
    b.set_params(growth_A=A, E=E)
    b.replay()
    got = (b.loss.clone(), b.dloss_dg.clone(), b.rollout.bar0.clone())
    sc2 = [dict(s, growth_A=float(a), E=float(e)) for s, a, e in zip(sc, A, E)]
    for s in sc2:
        s["mu"] = s["E"] / (2 * (1 + s["nu"]))
        s["lam"] = s["E"] * s["nu"] / ((1 + s["nu"]) * (1 - 2 * s["nu"]))
    f = _batch(sc2, 6)
    f.replay()
    assert torch.equal(got[0], f.loss) and torch.equal(got[1], f.dloss_dg)
    assert torch.equal(got[2], f.rollout.bar0)
    # the structure cannot change
    from morphompm_b200.batch import scene_spec_from_dict
    specs = [scene_spec_from_dict(s) for s in b.scenes]
    specs[0].shape = (specs[0].shape[0] + 1,) * 3
    with pytest.raises(L.MpmError):
        b.plan.update_scenes(specs)


def test_infer_growth_batched_recovers_each_scene():
    from morphompm_b200 import diff
    sc = _scenes()
    b = _batch(sc, 8)
    g_true = np.array([1.10, 1.22, 1.15])
    b.set_params(growth_A=g_true - 1.0)
    b.replay()
    targets = b.loss.cpu().numpy().copy()
    g, its = diff.infer_growth_batched(b, targets, 1.0, iters=20, tol=1e-10)
    assert np.abs(g - g_true).max() < 1e-6, (g, g_true, its)
    assert its.max() <= 10


def test_fit_batched_recovers_modulus():
    from morphompm_b200 import diff
    sc = _scenes(k=2, seed=22)
    E_true = np.array([1200.0, 2500.0])
    truth = _batch(sc, 30)
    truth.set_params(E=E_true)
    truth.rollout.forward(truth.slab0)
    x_obs = truth.final_state()[0:3].t().cpu().numpy().copy()
    fit = _batch(sc, 30, loss="mse", x_obs=x_obs, material_grads=True)
    res = diff.fit_batched(fit, params=("E",), iters=60, lr=0.05, E0=E_true * np.array([1.5, 0.7]))
    assert (res["loss"][-1] < 1e-3 * res["loss"][0]).all(), res["loss"][[0, -1]]
    assert np.abs(res["E"] / E_true - 1).max() < 0.02, res["E"]
