"""Schedules do not change results: every schedule knob of the autotuner (node
tile shape, particle block size, P2G node-gather CTAs per SM, stencil
x-offsets per pass of the P2G phase-1 kernels) gives bitwise the default
schedule's losses, growth gradients, final state and initial-state
cotangents on a small uneven batch.  The per-node sum order (source cells
o = 0..26) and the per-cell order (sorted particles) are fixed whatever the
schedule, and so is the number of FP32 Hencky evaluations recomputed in FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SCHEDULES = [
    {"tile_xy": 8, "tile_z": 16, "particle_block": 128},
    {"tile_xy": 4, "tile_z": 8, "scatter_ctas_per_sm": 2},
    {"scatter_oxb": 1},
]


def _run(scn, dtype, tuning):
    from morphompm_b200.batch import Batch, host_slab
    b = Batch(scn, 12, dtype=dtype, tuning=tuning, ckpt_every=4)
    b.load(host_slab(scn, np.float64 if dtype == torch.float64 else np.float32), non_blocking=False)
    b.run()
    torch.cuda.synchronize()
    return (b.loss.cpu().numpy(), b.dloss_dg.cpu().numpy(), b.final_state().cpu().numpy(),
            b.initial_cotangents().cpu().numpy(), b.plan.fp64_fallbacks())


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_schedules_are_bitwise_equal(dtype):
    from morphompm_b200 import scenes
    scn = scenes.config4(n_scenes=10, n_lo=512, n_hi=8192)
    ref = _run(scn, dtype, None)
    for tun in SCHEDULES:
        if dtype == torch.float64 and tun.get("scatter_oxb") == 3:
            continue
        got = _run(scn, dtype, tun)
        for name, a, b in zip(("loss", "dloss_dg", "state", "cotangents"), ref[:4], got[:4]):
            assert np.array_equal(a, b), (dtype, tun, name, float(np.max(np.abs(a - b))))
        assert got[4] == ref[4], (dtype, tun, "fp64 fallbacks")
    if dtype == torch.float32:
        assert ref[4] > 0          # the batch exercises the FP64 recomputes
