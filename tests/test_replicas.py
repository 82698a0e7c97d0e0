"""The N>1 path of bench.py on CPU ranks (gloo, world size 2): the timed
region is the slowest rank's (max over ranks), the value is the whole job's,
and under torchrun the reference arm runs on rank 0 alone while every rank
exits cleanly.  The path does not shard across GPUs (replicas only), so
there is no data-path collective to test."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 * (rank + 1), dist)
    value = bench.whole_job_rate(world, 1000, 5, ms)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out, "rank%d.json" % rank), "w") as f:
        json.dump({"ms": ms, "value": value}, f)


def test_max_over_ranks_and_whole_job_rate(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        got = json.load(open(tmp_path / ("rank%d.json" % r)))
        assert got["ms"] == 20.0  # the slower rank's time on every rank
        assert abs(got["value"] - world * 1000 * 3 * 5 / 0.020 / 1e6) < 1e-12


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
