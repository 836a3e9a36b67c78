"""SimConfig's B200 extension fields default to the reference's behaviour,
validate their values, and stay out of the reference's JSON format."""
import json

import pytest

from morphompm_b200 import io
from morphompm_b200.config import SimConfig, compute_target


def test_defaults_ask_for_nothing():
    c = SimConfig()
    assert (c.dtype, c.device, c.checkpoint_every) == (None, None, None)
    assert compute_target(c) == (None, None)

    class RefLike:          # a config without the extension fields
        N, dx, dt, damping, sp = 8, 0.1, 1e-3, 0.05, 0.02
    assert compute_target(RefLike()) == (None, None)


def test_dtype_is_validated():
    import torch
    assert compute_target(SimConfig(dtype="float32", device="cuda:1")) == (torch.float32, "cuda:1")
    with pytest.raises(ValueError):
        compute_target(SimConfig(dtype="bfloat16"))


def test_json_keeps_reference_fields(tmp_path):
    p = str(tmp_path / "c.json")
    io.save_config(SimConfig(N=12, dtype="float32", checkpoint_every=5), p)
    d = json.load(open(p))
    assert set(d) == {"N", "dx", "dt", "damping", "sp", "material"}
    c = io.load_config(p)
    assert c.N == 12 and c.dtype is None and c.checkpoint_every is None
