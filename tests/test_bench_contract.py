"""bench.py's output contract on CPU: the reference arm's JSON line carries
every key of the contract with consistent values, and the ncu summaries the
bench's roofline reads its per-launch DRAM traffic from exist and parse."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


@pytest.mark.parametrize("tag", ["faces_tma_kernel_box128_mixed", "faces_kernel_box128_mixed",
                                 "stage_kernel_box128_mixed"])
def test_profile_traffic_parses(tag):
    import bench

    traffic = bench.ncu_traffic(tag)
    # a 128^3 face launch moves at least its 312 B per point of algorithmic bytes
    assert traffic is not None and traffic >= 312 * 128 ** 3, (tag, traffic)


@pytest.mark.timeout(300)
def test_reference_arm_line_has_every_key():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    missing = [k for k in KEYS if k not in line]
    assert not missing, missing
    assert line["impl"] == "reference" and line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["config"]["workload"] == "box128_9sp_viscous_rk3"
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
