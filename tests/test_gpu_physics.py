"""The reference's C++ physics suite (tests/test_growth.cpp, T1-T8) run on the
device FP32 path with the C++ solver's semantics.  Every test applies the
reference's own gate; the simulated scenes are also compared with the
reference's C++ solver itself (oracle/_ref) run on the same inputs."""
import math

import numpy as np
import pytest

import physics_util as U
from oracle import growth_ref as G

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
needs_cpp = pytest.mark.skipif(not G.available(), reason="oracle/_ref not built (no reference tree)")

E, NU = 1.0e4, 0.3
MU, LAM = E / (2 * (1 + NU)), E * NU / ((1 + NU) * (1 - 2 * NU))


def _stress(F, Fg):
    from morphompm_b200.config import Material
    from morphompm_b200.constitutive import Hencky
    t = lambda a: torch.as_tensor(np.asarray(a, np.float32).reshape(-1, 3, 3), device="cuda")
    return Hencky(Material(E=E, nu=NU)).stress(t(F), t(Fg)).double().cpu().numpy()


def test_T1_isotropic_constitutive():
    g = 1.5
    tau = _stress(g * np.eye(3), g * np.eye(3))[0]
    assert np.abs(tau).max() < 1e-2                                  # F = Fg: Fe = I
    tau = _stress(np.eye(3), g * np.eye(3))[0]
    expected = -(2 * MU + 3 * LAM) * math.log(g)
    assert abs(tau[0, 0] - expected) < abs(expected) * 1e-3 + 1e-2
    assert abs(tau[1, 2]) < 1e-2


def test_T1b_anisotropic_constitutive():
    gs = (1.2, 1.0, 0.8)
    tau = _stress(np.eye(3), np.diag(gs))[0]
    e = [-math.log(v) for v in gs]
    for i in range(3):
        assert abs(tau[i, i] - (2 * MU * e[i] + LAM * sum(e))) < 1.0
    assert abs(tau[0, 1]) < 1.0


def test_T4_objectivity():
    F0 = np.array([[1.2, 0.10, 0.0], [0.0, 0.9, 0.05], [0.03, 0.0, 1.1]]).T    # from_columns
    Fg = np.diag([1.3, 1.0, 0.8])
    ax = np.array([0.3, 0.7, 0.6]) / np.linalg.norm([0.3, 0.7, 0.6])
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = np.eye(3) + math.sin(0.9) * K + (1 - math.cos(0.9)) * K @ K
    tau0 = _stress(F0, Fg)[0]
    tau1 = _stress(R @ F0, Fg)[0]
    d = np.abs(tau1 - R @ tau0 @ R.T).max()
    assert d < np.abs(tau0).max() * 1e-3 + 1e-2, d


SWELL = dict(N=24, dx=0.05, dt=1e-3, damping=0.05, density=1000.0, sp=0.025, E=E, nu=NU)


def _aniso_blocks(n, fac, K=10, M=250):
    per = [np.float32(f) ** np.float32(1.0 / K) for f in fac]
    g = [np.float32(1.0)] * 3
    blocks = []
    for _ in range(K):
        g = [np.float32(pi * gi) for pi, gi in zip(per, g)]
        blocks.append((np.tile(np.diag(g).astype(np.float32), (n, 1, 1)), M))
    return blocks


@needs_cpp
def test_T5_anisotropic_free_growth():
    pts = G.blob(0.6, 0.10, 0.025)
    fac = (1.3, 0.8, 1.1)
    blocks = _aniso_blocks(pts.shape[0], fac)
    x, F = U.device_run(pts, blocks=blocks, **SWELL)
    det = np.linalg.det(F).mean()
    expected = fac[0] * fac[1] * fac[2]
    Fg = blocks[-1][0].astype(np.float64)
    print(f"T5 device: mean det F {det:.5f} (det Fg {expected:.4f}), max eps {U.eps_norm(F, Fg).max():.4f}")
    assert abs(det - expected) < 0.08 * expected
    assert U.eps_norm(F, Fg).max() < 0.06
    xr, Fr = U.cpp_run(pts, blocks=blocks, **SWELL)
    det_r = np.linalg.det(Fr).mean()
    print(f"T5 C++:    mean det F {det_r:.5f}; max|dF| {np.abs(F - Fr).max():.2e}")
    assert abs(det - det_r) < 1e-4 * det_r


def test_T6_determinism():
    pts = G.blob(0.6, 0.10, 0.025)
    blocks = [(U.iso(pts.shape[0], 1.2), 300)]
    a = U.device_run(pts, blocks=blocks, **SWELL)
    b = U.device_run(pts, blocks=blocks, **SWELL)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


BILAYER = dict(N=28, dx=0.05, dt=1e-3, damping=0.05, density=1000.0, sp=0.025, E=E, nu=NU)


def _bilayer(g_b, g_t, cpp=False):
    pts = G.blob((0.7, 0.7, 0.7), (0.20, 0.05, 0.05), 0.025)
    Fg = U.layered(pts, 0.7, g_b, g_t)
    run = U.cpp_run if cpp else U.device_run
    x, F = run(pts, blocks=[(Fg, 4000)], **BILAYER)
    return U.eps_norm(F, Fg.astype(np.float64)).mean(), U.bend(x)


@pytest.fixture(scope="module")
def bilayers():
    return {"large": _bilayer(1.10, 1.50), "small": _bilayer(1.10, 1.20)}


def test_T3_differential_growth(bilayers):
    eps, bend = bilayers["large"]
    print(f"T3 device: mean eps {eps:.5f}, bend {bend:.5f}")
    assert eps > 0.02 and bend > 0.010


def test_T7_bend_monotonic(bilayers):
    assert bilayers["large"][1] > bilayers["small"][1] > 0.0


@needs_cpp
def test_T3_T7_against_cpp(bilayers):
    for key, (gb, gt) in (("large", (1.10, 1.50)), ("small", (1.10, 1.20))):
        eps_r, bend_r = _bilayer(gb, gt, cpp=True)
        eps, bend = bilayers[key]
        print(f"bilayer {key}: device eps {eps:.5f} bend {bend:.5f}; C++ eps {eps_r:.5f} bend {bend_r:.5f}")
        # measured: eps to 3e-4, bend to 1e-5 relative
        assert abs(eps - eps_r) < 2e-3 * eps_r
        assert abs(bend - bend_r) < 2e-3 * bend_r


BEAM = dict(N=48, dx=0.025, dt=1e-3, damping=0.05, density=1000.0, sp=0.0125, E=E, nu=NU)


def _beam(eps_m, cpp=False):
    pts = G.blob((0.6, 0.6, 0.6), (0.25, 0.025, 0.0125), 0.0125)
    Fg = U.layered(pts, 0.6, 1.0, 1.0 + eps_m)
    run = U.cpp_run if cpp else U.device_run
    x, _ = run(pts, blocks=[(Fg, 4000)], **BEAM)
    return U.curvature(x)


def test_T8_bilayer_timoshenko():
    h = 0.05
    k1, k2 = _beam(0.02), _beam(0.04)
    kT1 = 1.5 * 0.02 / h
    print(f"T8 device: kappa(0.02) {k1:.4f} kappa(0.04) {k2:.4f}; ratio to Timoshenko {k1 / kT1:.3f}; "
          f"scaling {k2 / k1:.3f}")
    assert 0.4 < k1 / kT1 < 1.7
    assert 1.6 < k2 / k1 < 2.4
    if G.available():
        k1r = _beam(0.02, cpp=True)
        print(f"T8 C++:    kappa(0.02) {k1r:.4f}")
        assert abs(k1 - k1r) < 2e-3 * k1r          # measured: 3e-4
