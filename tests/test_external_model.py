"""User-defined materials (no GPU needed here): classification and the
per-particle adapter for materials written like the reference's models."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from morphompm_b200 import constitutive as K
from morphompm_b200.config import Material


class NotAModel:
    pass


class RefStyleLinear:
    """Per-particle 3x3 numpy material, as the reference's models are written."""

    def stress(self, F, Fg, C):
        return 2.0 * (F - Fg) + 0.1 * C

    def stress_vjp(self, F, Fg, C, tb):
        return 2.0 * tb, -2.0 * tb, 0.1 * tb


def test_classification():
    assert not K.is_external(K.NeoHookean(Material()))
    assert K.is_external(K.PerParticle(RefStyleLinear()))
    assert K.model_fields(K.PerParticle(RefStyleLinear()))["model"] == 3
    with pytest.raises(TypeError):
        K.model_fields(NotAModel())


def test_per_particle_adapter_batches():
    rng = np.random.default_rng(0)
    F, Fg, C, tb = (torch.as_tensor(rng.standard_normal((5, 3, 3))) for _ in range(4))
    m = K.PerParticle(RefStyleLinear())
    np.testing.assert_allclose(m.stress(F, Fg, C).numpy(), (2.0 * (F - Fg) + 0.1 * C).numpy())
    a, b, c = m.stress_vjp(F, Fg, C, tb)
    np.testing.assert_allclose(a.numpy(), 2.0 * tb.numpy())
    np.testing.assert_allclose(b.numpy(), -2.0 * tb.numpy())
    np.testing.assert_allclose(c.numpy(), 0.1 * tb.numpy())
