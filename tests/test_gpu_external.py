"""User-defined materials on the device: a batched torch stress callback whose
stress the kernels consume (MPM_MODEL_EXTERNAL), with the caller's VJP applied
to the tau_bar the reverse step returns.  A torch neo-Hookean written as a
user material must reproduce the built-in one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from morphompm_b200 import constitutive as K
from morphompm_b200.config import Material, SimConfig


class TorchNeoHookean:
    """tau = mu (Fe Fe^T - I) + lam ln J I, batched torch on the device."""

    def __init__(self, mat):
        self.mu, self.lam = mat.mu, mat.lam

    def stress(self, F, Fg, C):
        Fe = F @ torch.linalg.inv(Fg)
        I = torch.eye(3, dtype=F.dtype, device=F.device)
        lnJ = torch.log(torch.linalg.det(Fe))
        return self.mu * (Fe @ Fe.transpose(1, 2) - I) + self.lam * lnJ[:, None, None] * I

    def stress_vjp(self, F, Fg, C, tb):
        tb = 0.5 * (tb + tb.transpose(1, 2))
        tr = torch.diagonal(tb, dim1=1, dim2=2).sum(-1)
        Fgi = torch.linalg.inv(Fg)
        Fe = F @ Fgi
        Feb = 2.0 * self.mu * tb @ Fe + self.lam * tr[:, None, None] * torch.linalg.inv(Fe).transpose(1, 2)
        Fb = Feb @ Fgi.transpose(1, 2)
        Fgb = -Fgi.transpose(1, 2) @ F.transpose(1, 2) @ Feb @ Fgi.transpose(1, 2)
        return Fb, Fgb, torch.zeros_like(F)


class RefStyleNeoHookean:
    """The same material per particle on 3x3 numpy arrays (the reference's style)."""

    def __init__(self, mat):
        self.t = TorchNeoHookean(mat)

    def stress(self, F, Fg, C):
        return self.t.stress(torch.as_tensor(F)[None], torch.as_tensor(Fg)[None], None)[0].numpy()

    def stress_vjp(self, F, Fg, C, tb):
        out = self.t.stress_vjp(torch.as_tensor(F)[None], torch.as_tensor(Fg)[None], None, torch.as_tensor(tb)[None])
        return tuple(o[0].numpy() for o in out)


def _state(n=60, seed=3):
    from morphompm_b200.state import ParticleState
    rng = np.random.default_rng(seed)
    d = lambda a: torch.as_tensor(a, device="cuda")
    return ParticleState(d(rng.uniform(0.3, 0.7, (n, 3))), d(0.1 * rng.standard_normal((n, 3))),
                         d(0.3 * rng.standard_normal((n, 3, 3))), d(np.eye(3) + 0.03 * rng.standard_normal((n, 3, 3))),
                         d(1.1 * np.eye(3) + 0.01 * rng.standard_normal((n, 3, 3))))


@pytest.mark.parametrize("advect", [False, True])
def test_user_material_matches_builtin_step_and_vjp(advect):
    from morphompm_b200 import transfer
    cfg = SimConfig(N=10, dx=0.1, dt=1e-3, sp=0.05)
    mat = Material(E=2e4, nu=0.3)
    st = _state()
    a, ca = transfer.step(st, K.NeoHookean(mat), cfg, advect=advect)
    b, cb = transfer.step(st, TorchNeoHookean(mat), cfg, advect=advect)
    for k in ("x", "v", "C", "F"):
        assert torch.allclose(getattr(a, k), getattr(b, k), rtol=0, atol=1e-12), k
    rng = np.random.default_rng(4)
    bars = [torch.as_tensor(rng.standard_normal(s), device="cuda") for s in ((60, 3), (60, 3), (60, 3, 3), (60, 3, 3))]
    bars.append(torch.as_tensor(rng.standard_normal((60, 3, 3)), device="cuda"))
    ga = transfer.step_vjp(ca, *bars, advect=advect)
    gb = transfer.step_vjp(cb, *bars, advect=advect)
    for u, w in zip(ga, gb):
        assert torch.allclose(u, w, rtol=1e-10, atol=1e-10 * float(w.abs().max()))


def test_user_material_trajectory_gradient():
    from morphompm_b200 import integrate
    rng = np.random.default_rng(5)
    pts = rng.uniform(0.35, 0.6, size=(40, 3))
    cfg = SimConfig(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2)
    mat = Material(E=1e4, nu=0.3)
    L0, g0 = integrate.dloss_dg(pts, K.NeoHookean(mat), cfg, 1.15, 4, True)
    L1, g1 = integrate.dloss_dg(pts, TorchNeoHookean(mat), cfg, 1.15, 4, True)
    L2, g2 = integrate.dloss_dg(pts, K.PerParticle(RefStyleNeoHookean(mat)), cfg, 1.15, 4, True)
    assert abs(L1 - L0) < 1e-12 * abs(L0) and abs(L2 - L0) < 1e-12 * abs(L0)
    assert abs(g1 - g0) < 1e-10 * abs(g0) and abs(g2 - g0) < 1e-10 * abs(g0), (g0, g1, g2)


def test_user_material_refusals():
    from morphompm_b200 import _lib as L, integrate
    from morphompm_b200.runtime import Plan, SLAB_ROWS, slab_particles
    from morphompm_b200.transfer import scene_spec
    from morphompm_b200.trajectory import Rollout
    cfg = SimConfig(N=8, dx=0.125, dt=1e-3, sp=0.0625)
    model = TorchNeoHookean(Material())
    with pytest.raises(TypeError):
        integrate.dloss_dparams(np.full((4, 3), 0.5), model, cfg, 1.1, 2, True)
    plan = Plan([scene_spec(cfg, model, 8)], dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError):
        Rollout(plan, 2)
    a = torch.zeros(SLAB_ROWS, 8, dtype=torch.float64, device="cuda")
    a[0:3] = 0.5
    for i in range(3):
        a[15 + 4 * i] = 1.0
    b = torch.empty_like(a)
    Fg = torch.zeros(9, 8, dtype=torch.float64, device="cuda")
    Fg[0] = Fg[4] = Fg[8] = 1.0
    with pytest.raises(L.MpmError):          # no stress supplied
        plan.step_fwd(slab_particles(a, Fg), slab_particles(b, Fg), True, 0, None)
    plan.set_external_stress(torch.zeros(8, 3, 3, dtype=torch.float64, device="cuda"))
    with pytest.raises(L.MpmError):          # chaining would evaluate the stress inside G2P
        plan.step_fwd(slab_particles(a, Fg), slab_particles(b, Fg), True, 0, None, emit=True)
    plan.step_fwd(slab_particles(a, Fg), slab_particles(b, Fg), True, 0, None)
