"""Failure detection without any GPU fault: conditions are created on the host
(non-finite input, particles off the grid) and the kernels report them in the
device status word; the step keeps the reference's semantics meanwhile."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _plan_and_state(n=64, dtype=torch.float64):
    from morphompm_b200.runtime import Plan, SceneSpec
    from morphompm_b200 import _lib as L
    rng = np.random.default_rng(4)
    spec = SceneSpec(shape=(10, 10, 10), n=n, model=L.MODEL_NEOHOOKEAN, dx=0.1, dt=1e-3, damping=0.05,
                     pmass=1e-3, vol0=1e-6, mu=3846.0, lam=5769.0)
    t = lambda a: torch.tensor(a, dtype=dtype, device="cuda").contiguous()
    x = rng.uniform(0.3, 0.7, size=(n, 3))
    st = [t(x), t(np.zeros((n, 3))), t(np.zeros((n, 3, 3))), t(np.tile(np.eye(3), (n, 1, 1))),
          t(np.tile(1.1 * np.eye(3), (n, 1, 1)))]
    return Plan([spec], dtype=dtype), st


def test_nonfinite_input_sets_status():
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import aos_particles
    plan, st = _plan_and_state()
    assert plan.status() == 0
    st[3][5, 0, 0] = float("nan")
    out = [torch.empty_like(a) for a in st]
    plan.step_fwd(aos_particles(*st), aos_particles(*out), True, 0, plan.new_tape())
    assert plan.status() & L.MPM_ERR_NONFINITE
    assert torch.isnan(out[3][5]).any()


def test_particle_outside_grid_keeps_reference_semantics():
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import aos_particles
    plan, st = _plan_and_state()
    st[0][7] = torch.tensor([1.5, 0.5, 0.5], dtype=st[0].dtype, device="cuda")     # stencil fully off the grid
    st[1][7] = torch.tensor([0.3, 0.0, 0.0], dtype=st[0].dtype, device="cuda")
    st[3][7] = torch.tensor([[1.1, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], dtype=st[0].dtype, device="cuda")
    out = [torch.empty_like(a) for a in st]
    plan.step_fwd(aos_particles(*st), aos_particles(*out), True, 0, plan.new_tape())
    assert plan.status() & L.MPM_WARN_OUTSIDE
    assert not plan.status() & L.MPM_ERR_NONFINITE
    # transfer.py:61-79 with every node out of range: v = C = 0, x and F unchanged
    assert torch.equal(out[0][7], st[0][7])
    assert torch.count_nonzero(out[1][7]) == 0 and torch.count_nonzero(out[2][7]) == 0
    assert torch.equal(out[3][7], st[3][7])


def test_bad_arguments_are_rejected_before_launch():
    from morphompm_b200 import _lib as L
    from morphompm_b200.runtime import aos_particles
    plan, st = _plan_and_state()
    p = aos_particles(*st)
    with pytest.raises(L.MpmError):
        plan.step_fwd(p, p, True, 0, plan.new_tape())          # in and out alias
    assert plan.status() == 0
