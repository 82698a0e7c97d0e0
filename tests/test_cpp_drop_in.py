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
@pytest.mark.parametrize("precision,scheme,layout",
                         [("fp64", "rk3", 0), ("mixed", "lusgs", 0), ("fp64", "steady", 0), ("mixed", "rk3", 1)])
@pytest.mark.parametrize("name", sorted(CASES))
def test_cpp_driver_equals_python_driver(name, precision, scheme, layout, tmp_path):
    """layout 1: the C++ program sets and reads the state in the reference's
    VectorField3D order (CC_LAYOUT_POINT_MAJOR) and must still get the Python
    driver's field-major state bit for bit."""
    case = CASES[name]()
    exe = compile_driver(tmp_path)
    dump_case(case, str(tmp_path / "case"))
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, str(tmp_path / "case"), out, str(cc.PRECISIONS[precision]), str(cc.SCHEMES[scheme]), "3",
                        str(layout)], capture_output=True, text=True, timeout=600)
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


# ------------------------------------------------ C++ readers of the input files

READ_SRC = os.path.join(ROOT, "tests", "cpp", "read_case.cpp")


def compile_reader(out_dir):
    exe = os.path.join(str(out_dir), "read_case")
    lib_dir = os.path.dirname(cc.LIB_PATH)
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           READ_SRC, "-o", exe, "-L", lib_dir, "-lcc_b200", "-Wl,-rpath," + lib_dir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _parse_dump(path):
    v = np.fromfile(path, dtype=np.float64)
    o = [0]

    def take(n):
        a = v[o[0]:o[0] + n]
        o[0] += n
        return a

    nb, ngg, ns = (int(x) for x in take(3))
    out = {"ngg": ngg, "n_spec": ns, "params": take(7), "blocks": [], "bcs": []}
    sizes = (ns, ns, ns, ns, 7 * ns, 7 * ns, ns, ns, ns * ns, ns * ns)
    out["species"] = [take(n) for n in sizes]
    for _ in range(nb):
        mx, my, mz, n_b, n_i = (int(x) for x in take(5))
        b = {"dims": (mx, my, mz), "boundaries": take(7 * n_b).reshape(-1, 7).astype(int).tolist(),
             "inner_faces": take(13 * n_i).reshape(-1, 13).astype(int).tolist()}
        ng = (mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg)
        b["jac"], b["metric"], b["bv"], b["yk"] = take(ng), take(9 * ng), take(6 * ng), take(ns * ng)
        out["blocks"].append(b)
    for _ in range(int(take(1)[0])):
        c = take(10 + ns)
        out["bcs"].append({"label": int(c[0]), "kind": int(c[1]), "thermal_type": int(c[2]), "t_wall": c[3],
                           "state": c[4:10], "yk": c[10:]})
    assert o[0] == v.size
    return out


def _write(case, coords, d, init):
    from combustioncodegpu_b200 import io

    io.write_case(case, d, coords, init)
    return io.load_case(d)


def _coords(dims, lengths, offset=(0, 0, 0)):
    x, y, z = cases.block_coordinates(dims, lengths)
    sl = (slice(3, -3),) * 3
    h = [L / (n - 1) for L, n in zip(lengths, dims)]
    return [x[sl] + offset[0] * h[0], y[sl] + offset[1] * h[1], z[sl] + offset[2] * h[2]]


def _reader_cases():
    sp = cases.synthetic_species()
    init_sp = {"density": 1.0, "u": 1.0, "v": 0.0, "w": 0.0, "pressure": 101325.0, "temperature": 400.0,
               "yk": list(np.full(sp["n_spec"], 1.0 / sp["n_spec"]))}
    init_air = {"density": 1.2, "u": 1.0, "v": 0.0, "w": 0.0, "pressure": 101325.0, "temperature": 300.0, "yk": []}
    sizes = ([6, 7], [6, 5], [5])
    mb = cases.case_multiblock(sizes, species=sp)
    h = 2e-3 / 127
    starts = [np.concatenate([[0], np.cumsum([n - 1 for n in s])[:-1]]) for s in sizes]
    mb_coords = []
    for c in range(len(sizes[2])):
        for b in range(len(sizes[1])):
            for a in range(len(sizes[0])):
                dims = (sizes[0][a], sizes[1][b], sizes[2][c])
                mb_coords.append(_coords(dims, tuple(h * (d - 1) for d in dims), (starts[0][a], starts[1][b],
                                                                                   starts[2][c])))
    return {
        "multiblock": (mb, mb_coords, init_sp),
        "box": (cases.case_box(10, species=sp, seed=2), [_coords((10, 10, 10), (2e-3,) * 3)], init_sp),
        "channel": (cases.case_channel(species=sp), [_coords((12, 9, 6), (2e-3, 1.5e-3, 1e-3))], init_sp),
        "sod": (cases.case_sod(40, 6, 6), [_coords((40, 6, 6), (1.0, 0.03125, 0.03125))], init_air),
    }


@pytest.mark.parametrize("name", ["box", "channel", "multiblock", "sod"])
def test_cpp_readers_equal_python_readers(name, tmp_path, cclib):
    """The C++ readers (include/cfd_b200_io.hpp) and the Python readers give
    the same parameters, species tables, ghost-grid geometry, face records,
    initial state and conditions for a case written in the reference's
    formats."""
    case, coords, init = _reader_cases()[name]
    d = str(tmp_path / "input_files")
    want = _write(case, coords, d, init)
    exe = compile_reader(tmp_path)
    r = subprocess.run([exe, d, str(tmp_path / "dump.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = _parse_dump(str(tmp_path / "dump.bin"))
    p = want["params"]
    assert got["ngg"] == p["ngg"]
    np.testing.assert_array_equal(got["params"], [p["inviscid_scheme"], p["reconstruction"], p["limiter"],
                                                  p["viscous_order"], p["cfl"], p["prandtl_number"],
                                                  p["schmidt_number"]])
    sp = p.get("species")
    assert got["n_spec"] == (0 if sp is None else sp["n_spec"])
    if sp is not None:
        for k, a in zip(SPECIES_TABLES, got["species"]):
            np.testing.assert_array_equal(a, np.asarray(sp[k], dtype=np.float64).ravel(), err_msg=k)
    for gb, wb in zip(got["blocks"], want["blocks"]):
        assert tuple(gb["dims"]) == tuple(wb["dims"])
        assert gb["boundaries"] == [list(x) for x in wb["boundaries"]]
        assert gb["inner_faces"] == [list(x)[:13] for x in wb["inner_faces"]]
        np.testing.assert_array_equal(gb["jac"], np.ravel(wb["jac"]))
        np.testing.assert_array_equal(gb["metric"], np.ravel(wb["metric"]))
        np.testing.assert_allclose(gb["bv"], np.ravel(wb["bv"]), rtol=1e-14)
        np.testing.assert_allclose(gb["yk"], np.ravel(wb["yk"]), rtol=1e-14)
    assert [b["label"] for b in got["bcs"]] == [b["label"] for b in want["bcs"]]
    for gb, wb in zip(got["bcs"], want["bcs"]):
        assert gb["kind"] == wb["kind"]
        if wb["kind"] == 2:
            assert gb["thermal_type"] == wb.get("thermal_type", 0) and gb["t_wall"] == wb["t_wall"]
        if wb["kind"] == 5:
            np.testing.assert_allclose(gb["state"], [wb[k] for k in ("density", "u", "v", "w", "pressure",
                                                                     "temperature")], rtol=1e-14)
            np.testing.assert_allclose(gb["yk"], np.asarray(wb["yk"])[:got["n_spec"]], rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["channel", "multiblock", "sod"])
def test_cpp_main_runs_reference_case_files(name, tmp_path):
    """main.cu-style C++ (read the input files, Driver, initialize, steady
    loop) gives bit for bit the state of the Python readers and driver."""
    from combustioncodegpu_b200 import io

    case, coords, init = _reader_cases()[name]
    d = str(tmp_path / "input_files")
    io.write_case(case, d, coords, init)
    lib_dir = os.path.dirname(cc.LIB_PATH)
    exe = os.path.join(str(tmp_path), "run_case")
    r = subprocess.run([shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                        os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "run_case.cpp"), "-o", exe,
                        "-L", lib_dir, "-lcc_b200", "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, d, out, "3"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64)
    loaded = io.load_case(d)
    drv = cc.Driver.from_case(loaded, "fp64")
    drv.initialize_computation()
    drv.simulate(3, "steady", residual=True)
    want = [np.concatenate([a.ravel() for a in drv.field[b].get_state()]) for b in range(len(loaded["blocks"]))]
    want = np.concatenate(want + [drv.residual()])
    drv.close()
    assert got.size == want.size
    np.testing.assert_array_equal(got, want)
