"""The bounds-checked build (MPM_CHECK_BOUNDS: every index the kernels compute
into node, cell-sum, segment, tile and sort arrays is checked, counted and
skipped when out of range) runs the batched trajectories, FP32 and FP64, and a
single step with its VJP, without one violation, and gives bitwise the
results of the release build.  It stands in for a memory checker."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))


def test_checked_build_has_no_violations_and_matches_release(tmp_path):
    import checked_workload as W
    from morphompm_b200 import build as B
    B.build(checked=True)
    out = tmp_path / "checked.npz"
    env = dict(os.environ, MORPHOMPM_CHECKED="1")
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_workload.py"), str(out)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    got = dict(np.load(out))
    rc, cnt, site, idx = (int(v) for v in got.pop("violations"))
    assert rc == 0, "the child did not load the checked library"
    assert cnt == 0, f"{cnt} out-of-range indices, first at site {site} index {idx}"
    ref = W.run()
    assert W.violations()[0] != 0        # the release library has no checks
    assert set(ref) == set(got)
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
