"""Chained forward steps (mpm_step_fwd_chain): the G2P pass that forms the next
step's cell keys and P2G records must give exactly the states of independent
mpm_step_fwd calls, and a chained call that does not continue the last
emitting call must be refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch(dtype):
    from morphompm_b200 import scenes
    from morphompm_b200.batch import host_slab, host_phi, scene_spec_from_dict
    from morphompm_b200.runtime import Plan
    sc = scenes.config4(seed=11, n_scenes=6, n_lo=600, n_hi=4000)
    # one scene of each model, plus a Herschel-Bulkley scene with a growth field
    sc[0]["model"], sc[1]["model"] = "nh", "hencky"
    sc[2] = dict(sc[2], model="hb", hb=dict(kappa=1e4, K=1.0, n=0.5, tau_y=10.0, m=100.0, eps=1e-4),
                 phi=np.linspace(0.0, 1.0, sc[2]["x"].shape[0]))
    specs = [scene_spec_from_dict(s) for s in sc]
    npd = np.float32 if dtype == torch.float32 else np.float64
    plan = Plan(specs, dtype=dtype, device="cuda")
    phi = host_phi(sc, npd)
    if phi is not None:
        plan.set_growth_field(torch.as_tensor(phi).cuda())
    slab0 = torch.as_tensor(host_slab(sc, npd)).cuda()
    return plan, slab0


def _run(plan, slab0, n, chain):
    from morphompm_b200.runtime import slab_particles
    a, b = slab0.clone(), torch.empty_like(slab0)
    for t in range(n):
        plan.step_fwd(slab_particles(a), slab_particles(b), True, t, None,
                      chained=chain and t > 0, emit=chain and t + 1 < n)
        a, b = b, a
    torch.cuda.synchronize()
    return a


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_chained_steps_match_independent_steps(dtype):
    dt = getattr(torch, dtype)
    plan, slab0 = _batch(dt)
    ref = _run(plan, slab0, 8, chain=False)
    got = _run(plan, slab0, 8, chain=True)
    assert torch.equal(ref, got)
    assert plan.status() == 0


def test_chained_step_must_continue_the_emitting_call():
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import slab_particles
    plan, slab0 = _batch(torch.float32)
    a, b, c = slab0.clone(), torch.empty_like(slab0), torch.empty_like(slab0)
    # nothing emitted yet
    with pytest.raises(L.MpmError) as e:
        plan.step_fwd(slab_particles(a), slab_particles(b), True, 0, None, chained=True)
    assert e.value.code == L.MPM_ERR_ARG
    plan.step_fwd(slab_particles(a), slab_particles(b), True, 0, None, emit=True)
    # wrong step index, then wrong input state
    for t, src in ((2, b), (1, a)):
        with pytest.raises(L.MpmError) as e:
            plan.step_fwd(slab_particles(src), slab_particles(c), True, t, None, chained=True)
        assert e.value.code == L.MPM_ERR_ARG
    # a refused call leaves the chain in place; an unchained call ends it
    plan.step_fwd(slab_particles(b), slab_particles(c), True, 1, None, chained=True, emit=True)
    plan.step_fwd(slab_particles(c), slab_particles(a), True, 2, None)
    with pytest.raises(L.MpmError):
        plan.step_fwd(slab_particles(a), slab_particles(b), True, 3, None, chained=True)


@pytest.mark.parametrize("speed", [0.05, 0.6])
def test_incremental_resort_matches_full_sort(speed):
    """Chained steps re-sort incrementally from the previous step's order and
    the emitted cell changes; independent steps run the full radix sort.  With
    initial velocities that move `speed` cells per step, a few percent of the
    particles change cell each step (0.05, the incremental path) or more than
    the re-sort's 16384-particle capacity does (0.6, the device falls back to
    the full sort).  States must agree bitwise: the P2G sums run in the
    sorted order, so any difference in the permutation would show."""
    from morphompm_b200 import scenes
    from morphompm_b200.batch import host_slab, scene_spec_from_dict
    from morphompm_b200.runtime import Plan, ROW_V
    sc = scenes.config4(seed=12, n_scenes=5, n_lo=20000, n_hi=40000)
    plan = Plan([scene_spec_from_dict(s) for s in sc], dtype=torch.float32, device="cuda")
    slab = host_slab(sc, np.float32)
    rng = np.random.default_rng(3)
    off = 0
    for s in sc:
        k = s["x"].shape[0]
        slab[ROW_V:ROW_V + 3, off:off + k] = rng.standard_normal((3, k)) * (speed * s["dx"] / s["dt"])
        off += k
    slab0 = torch.as_tensor(slab).cuda()
    ref = _run(plan, slab0, 6, chain=False)
    got = _run(plan, slab0, 6, chain=True)
    assert torch.equal(ref, got)
    assert plan.status() & ~8 == 0      # particles leaving the grid only warn
