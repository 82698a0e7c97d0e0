"""Readers of the reference's input files (combustioncodegpu_b200.io): the
synthetic workloads written in the reference's formats and read back give
the same geometry (ghost grid and metrics), faces, conditions, parameters and
species tables, so the reference's own case directories drive the library."""
import numpy as np
import pytest

from combustioncodegpu_b200 import cases, io


def _coords(dims, lengths, offset=(0, 0, 0)):
    x, y, z = cases.block_coordinates(dims, lengths)
    g = 3
    sl = (slice(g, -g),) * 3
    h = [L / (n - 1) for L, n in zip(lengths, dims)]
    return [x[sl] + offset[0] * h[0], y[sl] + offset[1] * h[1], z[sl] + offset[2] * h[2]]


def _roundtrip(case, coords, tmp_path, init=None):
    init = init or {"density": 1.0, "u": 1.0, "v": 0.0, "w": 0.0, "pressure": 101325.0, "temperature": 400.0,
                    "yk": [] if case["params"].get("species") is None else
                    list(np.full(case["params"]["species"]["n_spec"], 1.0 / case["params"]["species"]["n_spec"]))}
    io.write_case(case, str(tmp_path), coords, init)
    return io.load_case(str(tmp_path))


def _same_geometry(a, b):
    for ba, bb in zip(a["blocks"], b["blocks"]):
        assert tuple(ba["dims"]) == tuple(bb["dims"])
        np.testing.assert_allclose(bb["jac"], ba["jac"], rtol=1e-12)
        np.testing.assert_allclose(bb["metric"], ba["metric"], rtol=1e-9, atol=1e-9 * np.abs(ba["metric"]).max())
        assert [list(r) for r in bb["boundaries"]] == [list(r) for r in ba["boundaries"]]
        assert [list(r)[:13] for r in bb["inner_faces"]] == [list(r)[:13] for r in ba["inner_faces"]]


def test_box_roundtrip(tmp_path):
    sp = cases.synthetic_species()
    case = cases.case_box(10, species=sp, seed=2)
    got = _roundtrip(case, [_coords((10, 10, 10), (2e-3,) * 3)], tmp_path)
    _same_geometry(case, got)
    for k in ("inviscid_scheme", "reconstruction", "limiter", "viscous_order", "cfl", "prandtl_number",
              "schmidt_number"):
        assert got["params"][k] == case["params"][k]
    gs = got["params"]["species"]
    for k in ("mw", "low_temp_coeff", "high_temp_coeff", "t_low", "t_mid", "LJ_potent_inv", "vis_coeff"):
        np.testing.assert_array_equal(np.asarray(gs[k]), np.asarray(sp[k]))
    assert np.allclose(got["blocks"][0]["bv"][5], 400.0) and np.allclose(got["blocks"][0]["yk"].sum(0), 1.0)


def test_channel_conditions_roundtrip(tmp_path):
    sp = cases.synthetic_species()
    case = cases.case_channel(species=sp)
    dims, L = (12, 9, 6), (2e-3, 1.5e-3, 1e-3)
    got = _roundtrip(case, [_coords(dims, L)], tmp_path)
    _same_geometry(case, got)
    want = {bc["label"]: bc for bc in case["bcs"]}
    for bc in got["bcs"]:
        w = want[bc["label"]]
        assert bc["kind"] == w["kind"]
        if bc["kind"] == 2:
            assert bc["thermal_type"] == w["thermal_type"]
            if w["thermal_type"] == 0:
                assert bc["t_wall"] == w["t_wall"]
        if bc["kind"] == 5:
            for k in ("density", "u", "v", "w", "pressure", "temperature"):
                assert bc[k] == pytest.approx(w[k], rel=1e-14)
            np.testing.assert_allclose(bc["yk"], np.asarray(w["yk"])[:sp["n_spec"]], rtol=1e-14)


def test_multiblock_ghost_grid_from_neighbours(tmp_path):
    """Interface ghosts come from the neighbour block (Mesh.cpp:874-923): the
    metrics of every block equal those of the global uniform lattice."""
    sp = cases.synthetic_species()
    sizes = ([6, 7], [6, 5], [5])
    case = cases.case_multiblock(sizes, species=sp)
    h = 2e-3 / 127
    starts = [np.concatenate([[0], np.cumsum([n - 1 for n in s])[:-1]]) for s in sizes]
    coords = []
    for c in range(len(sizes[2])):
        for b in range(len(sizes[1])):
            for a in range(len(sizes[0])):
                dims = (sizes[0][a], sizes[1][b], sizes[2][c])
                coords.append(_coords(dims, tuple(h * (d - 1) for d in dims),
                                      (starts[0][a], starts[1][b], starts[2][c])))
    got = _roundtrip(case, coords, tmp_path)
    _same_geometry(case, got)


def test_parameter_files(tmp_path):
    (tmp_path / "2_scheme.txt").write_text("// comment\nint inviscid_scheme = 3\nint inviscid_scheme = 9\n"
                                           "double cfl = 0.25\nbool gradPInDiffusionFlux = 1\n"
                                           "string mechanism_file = chem/mech.inp\n")
    par = io.read_parameters(str(tmp_path))
    assert par == {"inviscid_scheme": 3, "cfl": 0.25, "gradPInDiffusionFlux": True,
                   "mechanism_file": "chem/mech.inp", "ngg": 2}
