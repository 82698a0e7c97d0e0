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


def test_clock_sampler_counts_only_the_timed_region(tmp_path, monkeypatch):
    """The sampler waits for nvidia-smi's first sample before the timed
    region starts and summarises only the samples taken after that; a region
    shorter than the sampling interval still gets the next sample.  A fake
    nvidia-smi on PATH prints one line per interval: 1200 MHz before the
    region (its first line), 1965 MHz after, sw_power_cap active."""
    import time

    import bench

    fake = tmp_path / "nvidia-smi"
    fake.write_text(
        "#!" + sys.executable + "\n"
        "import sys, time\n"
        "print('0, 1200, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active', flush=True)\n"
        "while True:\n"
        "    time.sleep(0.05)\n"
        "    print('0, 1965, 1965, 900.0, 0x4, Not Active, Not Active, Not Active, Active', flush=True)\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))
    with bench.ClockSampler(0) as clk:
        time.sleep(0.01)  # shorter than the 50 ms interval
    s = clk.summary()
    assert s["samples"] >= 1 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0, s
    assert s["reasons"] == ["sw_power_cap"], s
