"""torch.autograd over the device adjoints: differentiable single steps and a
differentiable checkpointed trajectory loss, against dloss_dg, against each
other, and against central differences (FP64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from morphompm_b200.config import Material, SimConfig
from morphompm_b200.constitutive import Hencky, NeoHookean

DEV = dict(dtype=torch.float64, device="cuda")


def _setup(seed=7, n=50):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(0.35, 0.6, size=(n, 3))
    cfg = SimConfig(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2)
    return pts, cfg


@pytest.mark.parametrize("cls", [NeoHookean, Hencky])
def test_chained_autograd_steps_match_trajectory_adjoint(cls):
    from morphompm_b200 import autograd, integrate
    pts, cfg = _setup()
    model = cls(Material(E=1e4, nu=0.3))
    n, T = pts.shape[0], 4
    x0 = torch.as_tensor(pts, **DEV).requires_grad_(True)
    x = x0
    v = torch.zeros(n, 3, **DEV)
    C = torch.zeros(n, 3, 3, **DEV)
    F = torch.eye(3, **DEV).repeat(n, 1, 1)
    g = torch.tensor(1.2, **DEV, requires_grad=True)
    Fg = g * torch.eye(3, **DEV).repeat(n, 1, 1)
    for t in range(T):
        x, v, C, F = autograd.step(x, v, C, F, Fg, model, cfg, advect=True, t=t)
    L = torch.linalg.det(F).sum()
    dx0, dg = torch.autograd.grad(L, (x0, g))
    L0, dg0 = integrate.dloss_dg(pts, model, cfg, 1.2, T, True)
    assert abs(L.item() - L0) < 1e-12 * abs(L0)
    assert abs(float(dg) - dg0) < 1e-10 * abs(dg0), (float(dg), dg0)
    # the same gradients from the one-node trajectory loss
    x1 = torch.as_tensor(pts, **DEV).requires_grad_(True)
    g1 = torch.tensor(1.2, **DEV, requires_grad=True)
    L1 = autograd.rollout_loss(x1, g1, model, cfg, T, True)
    L1.backward()
    assert abs(L1.item() - L0) < 1e-12 * abs(L0)
    assert abs(float(g1.grad) - float(dg)) < 1e-10 * abs(float(dg))
    scale = float(dx0.abs().max())
    assert scale > 0
    assert float((x1.grad - dx0).abs().max()) < 1e-10 * scale


def test_single_step_matches_step_vjp():
    from morphompm_b200 import autograd, transfer
    from morphompm_b200.state import ParticleState
    pts, cfg = _setup(seed=9)
    model = Hencky(Material(E=1e4, nu=0.3))
    n = pts.shape[0]
    rng = np.random.default_rng(3)
    x = torch.as_tensor(pts, **DEV).requires_grad_(True)
    v = torch.as_tensor(rng.normal(0, 0.05, (n, 3)), **DEV).requires_grad_(True)
    C = torch.as_tensor(rng.normal(0, 0.1, (n, 3, 3)), **DEV).requires_grad_(True)
    F = torch.as_tensor(np.eye(3) + rng.normal(0, 0.02, (n, 3, 3)), **DEV).requires_grad_(True)
    Fg = torch.as_tensor(1.1 * np.eye(3) + rng.normal(0, 0.01, (n, 3, 3)), **DEV).requires_grad_(True)
    outs = autograd.step(x, v, C, F, Fg, model, cfg, advect=True)
    cots = [torch.as_tensor(rng.normal(size=o.shape), **DEV) for o in outs]
    got = torch.autograd.grad(outs, (x, v, C, F, Fg), cots)
    st = ParticleState(*(a.detach() for a in (x, v, C, F, Fg)))
    _, cache = transfer.step(st, model, cfg, advect=True)
    want = transfer.step_vjp(cache, *cots, torch.zeros(n, 3, 3, **DEV), advect=True)
    for a, b in zip(got, want):
        assert torch.equal(a, b)


def test_rollout_loss_gradients():
    from morphompm_b200 import autograd, integrate
    pts, cfg = _setup(seed=8)
    model = NeoHookean(Material(E=1e4, nu=0.3))
    x_obs = pts + 0.01
    u = np.random.default_rng(5).normal(size=pts.shape)
    for loss in ("detF", "mse"):
        x0 = torch.as_tensor(pts, **DEV).requires_grad_(True)
        g = torch.tensor(1.15, **DEV, requires_grad=True)
        L = autograd.rollout_loss(x0, g, model, cfg, 5, True, loss=loss,
                                  x_obs=torch.as_tensor(x_obs, **DEV), ckpt_every=2)
        L.backward()
        L0, dg0 = integrate.dloss_dg(pts, model, cfg, 1.15, 5, True, loss=loss, x_obs=x_obs)
        assert abs(L.item() - L0) < 1e-12 * abs(L0)
        assert abs(float(g.grad) - dg0) < 1e-10 * abs(dg0)
        # d loss / d x0 along a random direction against central differences
        h = 1e-6
        f = lambda y: integrate.dloss_dg(y, model, cfg, 1.15, 5, True, loss=loss, x_obs=x_obs)[0]
        fd = (f(pts + h * u) - f(pts - h * u)) / (2 * h)
        got = float((x0.grad.cpu().numpy() * u).sum())
        assert abs(got - fd) < 1e-5 * abs(fd) + 1e-8, (loss, got, fd)


def test_rollout_loss_per_particle_growth():
    from morphompm_b200 import autograd
    pts, cfg = _setup(seed=10)
    model = NeoHookean(Material(E=1e4, nu=0.3))
    n = pts.shape[0]
    rng = np.random.default_rng(4)
    Fg0 = 1.1 * np.eye(3) + rng.normal(0, 0.02, (n, 3, 3))
    Fg = torch.as_tensor(Fg0, **DEV).requires_grad_(True)
    x0 = torch.as_tensor(pts, **DEV)
    L = autograd.rollout_loss(x0, Fg, model, cfg, 4, True)
    L.backward()
    W = rng.normal(size=(n, 3, 3))
    h = 1e-6
    f = lambda A: autograd.rollout_loss(x0, torch.as_tensor(A, **DEV), model, cfg, 4, True).item()
    fd = (f(Fg0 + h * W) - f(Fg0 - h * W)) / (2 * h)
    got = float((Fg.grad.cpu().numpy() * W).sum())
    assert abs(got - fd) < 1e-6 * abs(fd), (got, fd)
