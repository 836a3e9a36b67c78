"""Scenes grouped by material model.  A batch keeps its scenes in the plan
grouped by model (stable), so each model's particles form one run of slots
launched with the kernels specialised for that model; the caller's scene and
particle order is kept at the API.  With the models interleaved:

- every scene's loss, growth gradient, final state and initial-state
  cotangents are bitwise those of the scene run alone (also after
  set_params, which addresses scenes in the caller's order);
- a plan built in the interleaved order runs the kernels with the run-time
  model switch; its results agree with the grouped batch's to rounding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STEPS = 6


def _scenes():
    from morphompm_b200 import scenes
    sc = scenes.config4(seed=9, n_scenes=5, n_lo=300, n_hi=2500)
    for s, m in zip(sc, ("hencky", "nh", "hencky", "nh", "hencky")):
        s["model"] = m
    hb = dict(kappa=1e4, K=1.0, n=0.5, tau_y=10.0, m=100.0, eps=1e-4)
    sc[2] = dict(sc[2], model="hb", hb=hb)
    return sc


def _run(sc, dtype):
    from morphompm_b200.batch import Batch, host_slab
    b = Batch(sc, STEPS, dtype=dtype, ckpt_every=3)
    b.load(host_slab(sc, np.float64 if dtype == torch.float64 else np.float32), non_blocking=False)
    b.run()
    torch.cuda.synchronize()
    return b


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_grouped_batch_equals_scenes_alone(dtype):
    sc = _scenes()
    b = _run(sc, dtype)
    assert list(b.scene_perm) == [1, 3, 0, 4, 2]          # nh, nh, hencky, hencky, hb
    fin, bar0 = b.final_state(), b.initial_cotangents()
    off = np.concatenate([[0], np.cumsum([s["x"].shape[0] for s in sc])])
    for i, s in enumerate(sc):
        one = _run([s], dtype)
        assert torch.equal(b.loss[i], one.loss[0]) and torch.equal(b.dloss_dg[i], one.dloss_dg[0]), i
        assert torch.equal(fin[:, off[i]:off[i + 1]], one.final_state()), i
        assert torch.equal(bar0[:, off[i]:off[i + 1]], one.initial_cotangents()), i
    # new parameters land on the caller's scenes
    A = np.array([0.05, 0.2, 0.1, 0.15, 0.25])
    b.set_params(growth_A=A)
    b.run()
    torch.cuda.synchronize()
    for i, s in enumerate(sc):
        one = _run([dict(s, growth_A=float(A[i]))], dtype)
        assert torch.equal(b.dloss_dg[i], one.dloss_dg[0]), i


def test_runtime_model_switch_matches_specialised_kernels():
    from morphompm_b200.batch import host_slab, scene_spec_from_dict
    from morphompm_b200.runtime import Plan
    from morphompm_b200.trajectory import Rollout
    sc = _scenes()
    b = _run(sc, torch.float64)
    plan = Plan([scene_spec_from_dict(s) for s in sc], dtype=torch.float64, device="cuda")   # interleaved
    ro = Rollout(plan, STEPS, advect=True, ckpt_every=3, Fg=None)
    ro.run(torch.as_tensor(host_slab(sc, np.float64)).cuda())
    torch.cuda.synchronize()
    loss, grad = ro.loss.cpu().numpy(), ro.growth_grad.cpu().numpy()
    assert np.allclose(loss, b.loss.cpu().numpy(), rtol=1e-12, atol=0)
    assert np.allclose(grad, b.dloss_dg.cpu().numpy(), rtol=1e-10, atol=0)
