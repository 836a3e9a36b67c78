"""The native trajectory engine (mpm_rollout_fwd / mpm_rollout_bwd, driven by
trajectory.Rollout) against the same trajectory stepped one call at a time
through mpm_step_fwd_chain / mpm_step_bwd_params from Python: bitwise equal
final states, initial-state cotangents, Fg, growth and material gradients,
with and without checkpoint recompute, FP32 and FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch(dtype, explicit_fg):
    from morphompm_b200 import scenes
    from morphompm_b200.batch import host_slab, host_phi, scene_spec_from_dict
    from morphompm_b200.runtime import Plan
    sc = scenes.config4(seed=21, n_scenes=5, n_lo=500, n_hi=3000)
    sc[0]["model"], sc[1]["model"] = "nh", "hencky"
    sc[2] = dict(sc[2], model="hb", hb=dict(kappa=1e4, K=1.0, n=0.5, tau_y=10.0, m=100.0, eps=1e-4))
    npd = np.float32 if dtype == torch.float32 else np.float64
    specs = [scene_spec_from_dict(s, growth_mode=0 if explicit_fg else 1) for s in sc]
    plan = Plan(specs, dtype=dtype, device="cuda")
    n = plan.n
    Fg = None
    if explicit_fg:
        rng = np.random.default_rng(2)
        g = 1.0 + 0.2 * rng.random(n)
        Fg = torch.zeros(9, n, dtype=dtype, device="cuda")
        for i in range(3):
            Fg[4 * i] = torch.as_tensor(g, dtype=dtype)
    else:
        phi = host_phi(sc, npd)
        if phi is None:
            phi = np.linspace(0.0, 1.0, n).astype(npd)
        plan.set_growth_field(torch.as_tensor(phi).cuda())
    slab0 = torch.as_tensor(host_slab(sc, npd)).cuda()
    return plan, slab0, Fg


def _stepwise(plan, slab0, Fg, n_steps, k, advect, seed_bar):
    """Store-every-state trajectory through the single-step entry points."""
    from morphompm_b200.runtime import slab_cotangents, slab_particles, SLAB_ROWS, ROW_C
    n, S = plan.n, len(plan.scenes)
    states = [slab0.clone()] + [torch.empty_like(slab0) for _ in range(n_steps)]
    tapes = [plan.new_tape() for _ in range(n_steps)]
    for t in range(n_steps):
        # chained within each k-step segment, as the recomputed segments are
        plan.step_fwd(slab_particles(states[t], Fg), slab_particles(states[t + 1], Fg), advect, t, tapes[t],
                      chained=t % k != 0, emit=(t + 1) % k != 0 and t + 1 < n_steps)
    Fg_bar = torch.zeros(9, n, dtype=torch.float64, device="cuda") if Fg is not None else None
    gg = torch.zeros(S, dtype=torch.float64, device="cuda")
    mg = torch.zeros(S, 2, dtype=torch.float64, device="cuda")
    cur = seed_bar.clone()
    es = slab0.element_size()
    for t in range(n_steps - 1, -1, -1):
        nxt = torch.empty_like(cur)
        plan.step_bwd(slab_particles(states[t], Fg), states[t + 1].data_ptr() + ROW_C * n * es,
                      slab_cotangents(cur, Fg_bar), slab_cotangents(nxt, Fg_bar), gg, advect, t, tapes[t],
                      material_grad=mg)
        cur = nxt
    return states[-1], cur, Fg_bar, gg, mg


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("explicit_fg", [False, True])
@pytest.mark.parametrize("k", [None, 3])
def test_native_rollout_matches_stepwise(dtype, explicit_fg, k):
    from morphompm_b200.trajectory import Rollout
    dt = getattr(torch, dtype)
    plan, slab0, Fg = _batch(dt, explicit_fg)
    T = 7
    ro = Rollout(plan, T, advect=True, ckpt_every=k, Fg=Fg, material_grads=True)
    bar0 = ro.run(slab0)
    final, bar0_ref, Fg_bar, gg, mg = _stepwise(plan, slab0, Fg, T, k or T, True, ro.seed_bar)
    torch.cuda.synchronize()
    assert torch.equal(ro.final, final)
    assert torch.equal(bar0, bar0_ref)
    assert torch.equal(ro.material_grad, mg)
    if explicit_fg:
        assert torch.equal(ro.Fg_bar, Fg_bar)
    else:
        assert torch.equal(ro.growth_grad, gg)
        assert float(gg.abs().max()) > 0
    assert plan.status() == 0
    # a second run overwrites (does not accumulate) the gradient outputs
    ro.run(slab0)
    assert torch.equal(ro.material_grad, mg) and torch.equal(ro.bar0, bar0_ref)


def test_native_rollout_graph_and_edges():
    from morphompm_b200 import _lib as L
    from morphompm_b200.trajectory import Rollout
    plan, slab0, Fg = _batch(torch.float32, False)
    ro = Rollout(plan, 6, advect=True, ckpt_every=2)
    eager = ro.run(slab0).clone()
    ro.capture(slab0)
    for _ in range(2):
        assert torch.equal(ro.replay(), eager)
    # zero steps: the final state is the initial one, the cotangents pass through
    r0 = Rollout(plan, 0)
    r0.forward(slab0)
    assert torch.equal(r0.final, slab0)
    bar = torch.randn_like(slab0)
    assert torch.equal(r0.backward(bar), bar)
    # the input and output slabs must differ
    ws = ro.ws_ptr
    with pytest.raises(L.MpmError) as e:
        plan.rollout_fwd(slab0, None, 6, 2, True, ws, slab0)
    assert e.value.code == L.MPM_ERR_ARG
