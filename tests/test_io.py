"""Device-boundary I/O against files written by the reference's own adapters
(io.py:29-111): byte-identical .csv/.vtk/.json, lossless .npz, round trips."""
import os

import numpy as np
import pytest

from morphompm_b200 import io as mio
from morphompm_b200.config import Material, SimConfig
from morphompm_b200.state import ParticleState

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _state():
    d = np.load(os.path.join(GOLD, "io_state.npz"))
    return ParticleState(d["x"], d["v"], d["C"], d["F"], d["Fg"])


@pytest.mark.parametrize("ext", [".csv", ".vtk"])
def test_files_match_the_reference_writer(tmp_path, ext):
    p = tmp_path / ("s" + ext)
    mio.save_state(_state(), str(p))
    assert p.read_bytes() == open(os.path.join(GOLD, "io_state" + ext), "rb").read()


def test_config_matches_and_round_trips(tmp_path):
    cfg = SimConfig(N=12, dx=0.05, dt=2e-4, damping=0.07, sp=0.025,
                    material=Material(E=3.0e3, nu=0.35, density=900.0))
    p = tmp_path / "c.json"
    mio.save_config(cfg, str(p))
    assert p.read_bytes() == open(os.path.join(GOLD, "io_config.json"), "rb").read()
    c2 = mio.load_config(str(p))
    assert (c2.N, c2.dx, c2.dt, c2.damping, c2.sp) == (cfg.N, cfg.dx, cfg.dt, cfg.damping, cfg.sp)
    assert c2.material.mu == cfg.material.mu and c2.material.lam == cfg.material.lam


def test_round_trips(tmp_path):
    st = _state()
    for ext, atol in ((".npz", 0.0), (".csv", 1e-6)):
        p = str(tmp_path / ("s" + ext))
        mio.save_state(st, p)
        back = mio.load_state(p)
        for k in ("x", "v", "C", "F", "Fg"):
            np.testing.assert_allclose(getattr(back, k), getattr(st, k), rtol=0, atol=atol)
    # the reference's reader accepts ours (same header, same dialect)
    with open(os.path.join(GOLD, "io_state.csv")) as f:
        assert f.readline().strip().split(",")[:3] == ["x", "y", "z"]
    with pytest.raises(ValueError):
        mio.save_state(st, str(tmp_path / "s.txt"))


def test_torch_tensors_and_empty_state(tmp_path):
    torch = pytest.importorskip("torch")
    st = _state()
    tst = ParticleState(*(torch.as_tensor(getattr(st, k)) for k in ("x", "v", "C", "F", "Fg")))
    for ext in (".csv", ".vtk"):
        p = tmp_path / ("t" + ext)
        mio.save_state(tst, str(p))
        assert p.read_bytes() == open(os.path.join(GOLD, "io_state" + ext), "rb").read()
    empty = ParticleState(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3, 3)), np.zeros((0, 3, 3)),
                          np.zeros((0, 3, 3)))
    mio.save_state(empty, str(tmp_path / "e.vtk"))
    mio.save_state(empty, str(tmp_path / "e.csv"))


def test_load_curve(tmp_path):
    p = tmp_path / "curve.csv"
    p.write_text("shear_rate,stress\n0.1,12.5\nbad,row\n1.0,20.0\n")
    x, y = mio.load_curve(str(p))
    assert list(x) == [0.1, 1.0] and list(y) == [12.5, 20.0]
