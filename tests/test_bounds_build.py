"""The bounds-checked build (libcc_b200_bounds.so, nvcc -DCC_BOUNDS_CHECK),
which stands in for compute-sanitizer's memory check: its kernels check the
arena, scratch and plane indices they compute (face and update kernels, the
halo program's nodes and copies, the TMA plane coordinates) and report an
index out of range as status bit 64 instead of accessing it.  On every parity
case, kernel variant and scheme it must report nothing and give the normal
build's states bit for bit.  Each build runs in a process of its own
(tests/bounds_runner.py, library chosen by CC_LIBRARY)."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "tests", "bounds_runner.py")
LIBS = {"normal": os.path.join(ROOT, "combustioncodegpu_b200", "libcc_b200.so"),
        "bounds": os.path.join(ROOT, "combustioncodegpu_b200", "libcc_b200_bounds.so")}
STATUS_BOUNDS = 64


def test_bounds_build_exists_and_exports_the_abi():
    import ctypes
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import build

    build.build(bounds=True)  # in-tree, only what is stale
    lib = ctypes.CDLL(LIBS["bounds"])
    for name in cc.EXPORTS:
        assert hasattr(lib, name), name


def _run(which, args, out):
    env = dict(os.environ, CC_LIBRARY=LIBS[which])
    r = subprocess.run([sys.executable, RUNNER, *args, str(out)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


@pytest.mark.gpu
@pytest.mark.parametrize("name,variant,precision,scheme", [
    ("box", "split-tma", "mixed", "rk3"), ("box", "split-tma-p", "fp64", "rk3"), ("box", "l1", "fp64", "steady"),
    ("channel", "split-tma", "mixed", "rk3"), ("channel", "split", "fp64", "lusgs"),
    ("multiblock", "split-tma", "mixed", "rk3"), ("multiblock", "tma", "mixed", "steady"),
    ("multiblock", "dq-tma", "mixed", "rk3"), ("sod", "split-tma", "fp64", "rk3"),
    ("mixing", "split-tma", "mixed", "rk3")])
def test_bounds_build_reports_nothing_and_matches(tmp_path, name, variant, precision, scheme):
    args = [name, variant, precision, scheme]
    got = _run("bounds", args, tmp_path / "bounds.npz")
    want = _run("normal", args, tmp_path / "normal.npz")
    assert str(got["lib"]) == "libcc_b200_bounds.so" and str(want["lib"]) == "libcc_b200.so"
    assert int(got["status"]) & STATUS_BOUNDS == 0, "an index outside its array was caught"
    assert int(got["status"]) == int(want["status"]) == 0
    for k in want.files:
        if k.startswith("b"):
            np.testing.assert_array_equal(got[k], want[k])
    np.testing.assert_array_equal(got["res"], want["res"])
