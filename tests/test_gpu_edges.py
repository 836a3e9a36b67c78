"""Edge cases of the growth step: an empty state, empty and one-particle
scenes inside a batch, and particles exactly on cell boundaries and at the
grid's faces, against the oracle (FP64) and against single-scene runs."""
import numpy as np
import pytest

from oracle import mpm_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


def test_empty_state():
    """No particles: nothing to transfer; the step returns empty arrays of the
    input's shapes and type, its VJP empty cotangents, dloss_dg (0, 0)."""
    from morphompm_b200 import integrate, transfer
    from morphompm_b200.config import Material, SimConfig
    from morphompm_b200.constitutive import Hencky
    from morphompm_b200.state import ParticleState
    cfg = SimConfig()
    model = Hencky(Material())
    z3, z33 = np.zeros((0, 3)), np.zeros((0, 3, 3))
    ns, cache = transfer.step(ParticleState(z3, z3, z33, z33, z33), model, cfg, advect=True)
    assert all(isinstance(a, np.ndarray) for a in (ns.x, ns.v, ns.C, ns.F, ns.Fg))
    assert ns.x.shape == (0, 3) and ns.F.shape == (0, 3, 3)
    g = transfer.step_vjp(cache, z3, z3, z33, z33, z33, advect=True)
    assert [a.shape for a in g] == [(0, 3), (0, 3), (0, 3, 3), (0, 3, 3), (0, 3, 3)]
    assert integrate.dloss_dg(z3, model, cfg, 1.2, 3, True) == (0.0, 0.0)
    d = torch.zeros(0, 3, dtype=torch.float32, device="cuda")
    st = ParticleState.rest(d)
    ns, _ = transfer.step(st, model, cfg)
    assert ns.x.is_cuda and ns.x.dtype == torch.float32 and ns.x.shape == (0, 3)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_batch_with_empty_and_single_particle_scenes(dtype):
    from morphompm_b200 import scenes
    from morphompm_b200.batch import Batch, host_slab
    dt = getattr(torch, dtype)
    npd = np.float32 if dtype == "float32" else np.float64
    sc = scenes.config4(seed=3, n_scenes=3, n_lo=400, n_hi=1500)
    empty = dict(sc[1], x=sc[1]["x"][:0])
    single = dict(sc[2], x=sc[2]["x"][:1])
    batch = [sc[0], empty, single, sc[1]]
    b = Batch(batch, 5, dtype=dt)
    b.load(host_slab(batch, npd), non_blocking=False)
    b.run()
    torch.cuda.synchronize()
    assert float(b.loss[1]) == 0.0 and float(b.dloss_dg[1]) == 0.0
    assert b.plan.status() == 0
    for i in (0, 2, 3):
        one = Batch([batch[i]], 5, dtype=dt)
        one.load(host_slab([batch[i]], npd), non_blocking=False)
        one.run()
        assert torch.equal(one.loss[0], b.loss[i]) and torch.equal(one.dloss_dg[0], b.dloss_dg[i]), i
    # the lone particle of scene 2 swells freely: its det F stays that of one free step
    assert 0.0 < float(b.loss[2])


@pytest.mark.parametrize("name", ["nh", "hencky", "hb"])
def test_cell_boundaries_and_faces_fp64_vs_oracle(name):
    """Particles with x/dx - 1/2 an exact integer (the floor of the binning
    ties), and particles whose stencil crosses the lower and upper faces of
    the grid (their outside nodes are skipped, transfer.py:19-21, 48-50)."""
    from morphompm_b200 import constitutive as K, transfer
    from morphompm_b200.config import Material, SimConfig
    from morphompm_b200.state import ParticleState
    N, dx = 16, 1.0 / 16
    rng = np.random.default_rng(11)
    ties = (rng.integers(3, 12, size=(20, 3)) + 0.5) * dx            # X - 1/2 integral
    faces = np.array([[0.01, 0.5, 0.5], [0.99, 0.5, 0.5], [0.5, 0.002, 0.5], [0.5, 0.5, 0.998],
                      [0.02, 0.98, 0.03], [0.5 * dx, 0.5, 0.5], [1 - 0.5 * dx, 0.5, 0.5]])
    x = np.concatenate([ties, faces, rng.uniform(0.3, 0.7, size=(20, 3))])
    n = x.shape[0]
    v = 0.1 * rng.standard_normal((n, 3))
    C = 0.3 * rng.standard_normal((n, 3, 3))
    F = np.eye(3) + 0.02 * rng.standard_normal((n, 3, 3))
    Fg = 1.15 * np.eye(3) + 0.01 * rng.standard_normal((n, 3, 3))
    cfg = SimConfig(N=N, dx=dx, dt=5e-4, sp=dx / 2, material=Material(E=1e4, nu=0.3))
    models = {"nh": (K.NeoHookean(cfg.material), O.Model.elastic("nh", 1e4, 0.3)),
              "hencky": (K.Hencky(cfg.material), O.Model.elastic("hencky", 1e4, 0.3)),
              "hb": (K.HerschelBulkley(), O.Model(kind="hb"))}
    m, om = models[name]
    scene = O.scene_from_cfg(N, dx, 5e-4, cfg.damping, dx / 2, cfg.material.density)
    bars = [rng.standard_normal(s) for s in ((n, 3), (n, 3), (n, 3, 3), (n, 3, 3), (n, 3, 3))]
    for adv in (False, True):
        ns, cache = transfer.step(ParticleState(x, v, C, F, Fg), m, cfg, advect=adv)
        ons, oc = O.step(O.State(x, v, C, F, Fg), om, scene, advect=adv)
        for a, b in ((ns.x, ons.x), (ns.v, ons.v), (ns.C, ons.C), (ns.F, ons.F)):
            assert _rel(a, b) < 1e-12
        g = transfer.step_vjp(cache, *bars, advect=adv)
        og = O.step_vjp(oc, *bars, advect=adv)
        tol = 1e-10 if name != "hencky" else 1e-8
        for a, b in zip(g, og):
            assert _rel(a, b) < tol
