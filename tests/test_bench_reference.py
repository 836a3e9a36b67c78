"""The reference arm of bench.py (the oracle port of the reference's
fwd+adj on the host cores) prints the contract's JSON line with the same
metric, unit and workload as the GPU arm; a rank other than 0 prints nothing."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--scenes", "3"]


def test_reference_arm_json_line():
    r = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert (d["metric"], d["unit"], d["config"]["workload"]) == (bench.METRIC, bench.UNIT, bench.WORKLOAD)
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]


def test_reference_arm_other_ranks_print_nothing():
    r = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, RANK="1", WORLD_SIZE="2"))
    assert r.returncode == 0 and r.stdout.strip() == ""
