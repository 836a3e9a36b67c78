"""transfer.step refuses a mis-shaped particle state before any device work
(no GPU needed for the refusal)."""
import numpy as np
import pytest

from morphompm_b200 import transfer
from morphompm_b200.config import Material, SimConfig
from morphompm_b200.constitutive import NeoHookean
from morphompm_b200.state import ParticleState


@pytest.mark.parametrize("field,shape", [("x", (5, 2)), ("v", (4, 3)), ("C", (5, 9)), ("F", (5, 3, 2)),
                                         ("Fg", (6, 3, 3))])
def test_misshaped_state_is_refused(field, shape):
    n = 5
    st = dict(x=np.zeros((n, 3)), v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)), F=np.tile(np.eye(3), (n, 1, 1)),
              Fg=np.tile(np.eye(3), (n, 1, 1)))
    st[field] = np.zeros(shape)
    with pytest.raises(ValueError, match=field):
        transfer.step(ParticleState(**st), NeoHookean(Material()), SimConfig())


@pytest.mark.parametrize("loss,x_obs", [("l2", None), ("mse", None)])
def test_trajectory_losses_are_checked_before_device_work(loss, x_obs):
    from morphompm_b200 import integrate
    from morphompm_b200.batch import Batch
    from morphompm_b200 import scenes
    pts = np.random.default_rng(0).uniform(0.3, 0.6, size=(10, 3))
    with pytest.raises(ValueError, match="loss"):
        integrate.dloss_dg(pts, NeoHookean(Material()), SimConfig(), 1.1, 2, True, loss=loss, x_obs=x_obs)
    with pytest.raises(ValueError, match="loss"):
        integrate.dloss_dparams(pts, NeoHookean(Material()), SimConfig(), 1.1, 2, True, loss=loss, x_obs=x_obs)
    with pytest.raises(ValueError, match="loss"):
        Batch(scenes.config4(n_scenes=2, n_lo=100, n_hi=200), 2, loss=loss, x_obs=x_obs)
