"""C++ code written against the reference's classes (include/cfd_b200.hpp:
cfd::Parameter, Mesh, ChemData, Driver, Field over the C ABI) runs a case
through the library and gets, bit for bit, the state the Python mirror of
the same calls gets.  The program is tests/cpp/driver_drop_in.cpp; it reads a
case dump written here."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "driver_drop_in.cpp")
SPECIES_TABLES = ("mw", "t_low", "t_mid", "t_high", "low_temp_coeff", "high_temp_coeff", "LJ_potent_inv",
                  "vis_coeff", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8")


def compile_driver(out_dir):
    """g++ -std=c++17 against include/ and the in-tree libcc_b200.so."""
    exe = os.path.join(str(out_dir), "driver_drop_in")
    lib_dir = os.path.dirname(cc.LIB_PATH)
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", exe, "-L", lib_dir, "-lcc_b200", "-Wl,-rpath," + lib_dir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def dump_case(case, d):
    os.makedirs(d, exist_ok=True)
    p = case["params"]
    sp = p.get("species")
    ns = 0 if sp is None else int(sp["n_spec"])
    with open(os.path.join(d, "params.txt"), "w") as f:
        for k in ("inviscid_scheme", "reconstruction", "limiter", "viscous_order", "ngg"):
            f.write("int %s %d\n" % (k, int(p[k])))
        for k in ("prandtl_number", "cfl", "schmidt_number"):
            f.write("double %s %.17g\n" % (k, float(p[k])))
        f.write("int n_spec %d\nint n_block %d\n" % (ns, len(case["blocks"])))
    if ns:
        with open(os.path.join(d, "species.bin"), "wb") as f:
            for k in SPECIES_TABLES:
                np.ascontiguousarray(sp[k], dtype=np.float64).tofile(f)
    for b, blk in enumerate(case["blocks"]):
        with open(os.path.join(d, "block_%d.txt" % b), "w") as f:
            f.write("%d %d %d %d %d\n" % (*blk["dims"], len(blk["boundaries"]), len(blk["inner_faces"])))
            for r in list(blk["boundaries"]) + list(blk["inner_faces"]):
                f.write(" ".join(str(int(x)) for x in r) + "\n")
        with open(os.path.join(d, "block_%d.bin" % b), "wb") as f:
            for a in (blk["jac"], blk["metric"], blk["bv"]) + ((blk["yk"],) if ns else ()):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
    with open(os.path.join(d, "bcs.bin"), "wb") as f:
        for bc in case["bcs"]:
            f.write(bytes(cc.make_bc(bc, ns)))


def test_cfd_header_compiles_against_the_library(tmp_path, cclib):
    assert ctypes.sizeof(cc.CCBc) == 4 * 4 + 7 * 8 + 16 * 8  # the cc_bc record the program reads raw
    compile_driver(tmp_path)


CASES = {
    "box": lambda: cases.case_box(10, species=cases.synthetic_species(), seed=3),
    "channel": lambda: cases.case_channel((11, 8, 6), species=cases.synthetic_species()),
    "multiblock": lambda: cases.case_multiblock(([6, 7], [6, 5], [5]), species=cases.synthetic_species()),
    "sod": lambda: cases.case_sod(40, 6, 6),
}


@pytest.mark.gpu
@pytest.mark.parametrize("precision,scheme", [("fp64", "rk3"), ("mixed", "lusgs"), ("fp64", "steady")])
@pytest.mark.parametrize("name", sorted(CASES))
def test_cpp_driver_equals_python_driver(name, precision, scheme, tmp_path):
    case = CASES[name]()
    exe = compile_driver(tmp_path)
    dump_case(case, str(tmp_path / "case"))
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, str(tmp_path / "case"), out, str(cc.PRECISIONS[precision]), str(cc.SCHEMES[scheme]), "3"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64)
    d = cc.Driver.from_case(case, precision)
    d.initialize_computation()
    d.simulate(3, scheme, residual=True)
    want = [np.concatenate([a.ravel() for a in d.field[b].get_state()]) for b in range(len(case["blocks"]))]
    want = np.concatenate(want + [d.residual()])
    d.close()
    assert got.size == want.size
    np.testing.assert_array_equal(got, want)
