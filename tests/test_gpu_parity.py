"""CUDA path (through the C ABI) against the CPU oracle and against the
reference's own kernels (golden fixtures).

Tolerances: FP64 plain path vs the FP64 oracle 1e-10 relative per field
group after a few steps (rounding only: FMA contraction and evaluation order
differ); mixed path (FP32 fluxes/transport, FP64 conserved variables and
Newton) vs the FP64 oracle 1e-4 after two steps (the long-run L2 bound of
1e-5 after 1000 steps is measured by bench.py)."""
import os
import sys

import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases
from oracle.oracle_py import Oracle

sys.path.insert(0, os.path.dirname(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from gpu_compare import bv_groups, cv_groups, group_errors, interior  # noqa: E402
import make_golden as mg  # noqa: E402

pytestmark = pytest.mark.gpu


def _cases():
    sp = cases.synthetic_species()
    return {
        "sod": cases.case_sod(40, 6, 6),
        "box": cases.case_box(12, species=sp, seed=3),
        "channel": cases.case_channel((11, 8, 6), species=sp),
        "multiblock": cases.case_multiblock(([6, 7], [6, 5], [5]), species=sp),
        "air_visc": mg.load("air_visc_o1")[0],
        "mixing": cases.case_mixing_layer(40, 24, 4, h=4e-3 / 39, delta=4e-4, species=sp),
        # curvilinear periodic grid: non-zero geometric term of the gauge-pressure momentum fluxes
        "box_distorted": cases.case_box_distorted(12, amp=0.3, species=sp),
    }


CASES = _cases()


def compare(case, scheme, n, precision, variant="auto", kz=0, tile_j=0):
    renorm = precision in ("mixed", "fp32") and case["params"].get("species") is not None
    o = Oracle(case)
    o.init()
    d = cc.Driver.from_case(case, precision)
    d.set_tuning(variant, kz, tile_j)
    d.initialize_computation()
    if variant != "auto":
        assert d.tuning()["variant"] == variant
    if scheme == "rk3":
        o.rk3_step(n, renorm_y=renorm)
    elif scheme == "lusgs":
        o.lusgs_step(n, renorm_y=renorm)
    else:
        o.steady_step(n, renorm_y=renorm)
    d.simulate(n, scheme, residual=True)
    errs = {}
    ns = o.ns
    for b, blk in enumerate(case["blocks"]):
        bv, yk, cv = d.field[b].get_state()
        obv, oyk, ocv = o.state(b)
        for k, v in group_errors(bv, obv, bv_groups()).items():
            errs["bv." + k] = max(errs.get("bv." + k, 0.0), v)
        for k, v in group_errors(cv, ocv, cv_groups(ns)).items():
            errs["cv." + k] = max(errs.get("cv." + k, 0.0), v)
        if ns:
            errs["yk"] = max(errs.get("yk", 0.0), float(np.abs(yk - oyk).max()))
        mul, cond, rd = d.field[b].get_props()
        omul, ocond, ord_ = o.props(b)
        errs["mul"] = max(errs.get("mul", 0.0), float(np.abs(mul - omul).max() / np.abs(omul).max()))
        errs["cond"] = max(errs.get("cond", 0.0), float(np.abs(cond - ocond).max() / np.abs(ocond).max()))
    res, ores = d.residual(), o.residual()
    errs["res"] = float(np.max(np.abs(res - ores) / np.maximum(np.abs(ores), 1e-300)))
    if scheme == "rk3":
        errs["dt"] = abs(d.last_dt() - o.last_dt()) / o.last_dt()
    status = d.status()
    d.close()
    return errs, status


@pytest.mark.parametrize("scheme", ["steady", "rk3"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_oracle(name, scheme):
    errs, status = compare(CASES[name], scheme, 2, "fp64")
    assert status == 0
    bad = {k: v for k, v in errs.items() if not v < 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("scheme", ["steady", "rk3"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_close_to_oracle(name, scheme):
    errs, status = compare(CASES[name], scheme, 2, "mixed")
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
    assert not bad, errs


# Every stage-kernel variant on every case, with k-chunks that split the
# sweep (kz=3) and that do not (kz=64).  The TMA variants exist for 0 or 9
# species; the fused one and the dq one for the FP32 bulk precision only.
@pytest.mark.parametrize("variant", ["tma", "split-tma", "split-tma-p", "dq-tma"])
@pytest.mark.parametrize("kz", [3, 64])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_variant_close_to_oracle(name, kz, variant):
    errs, status = compare(CASES[name], "rk3", 2, "mixed", variant, kz)
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
    assert not bad, errs


@pytest.mark.parametrize("variant", ["split", "split-tma", "split-tma-p"])
@pytest.mark.parametrize("scheme", ["steady", "rk3"])
@pytest.mark.parametrize("kz", [3, 64])
@pytest.mark.parametrize("name", sorted(CASES))
def test_split_variant_fp64_matches_oracle(name, kz, scheme, variant):
    errs, status = compare(CASES[name], scheme, 2, "fp64", variant, kz)
    assert status == 0
    bad = {k: v for k, v in errs.items() if not v < 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("name", sorted(CASES))
def test_split_variant_mixed_close_to_oracle(name):
    errs, status = compare(CASES[name], "rk3", 2, "mixed", "split", 3)
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
    assert not bad, errs


@pytest.mark.parametrize("tile_j", [4, 8, 16])
@pytest.mark.parametrize("name", sorted(CASES))
def test_dq_variant_tile_shapes_close_to_oracle(name, tile_j):
    """The face kernel that differences the faces inside its tile, at every
    tile height (32 x 4, 32 x 8, 32 x 16 points, k-chunks of 3), steady and
    RK3 steps against the oracle."""
    for scheme in ("steady", "rk3"):
        errs, status = compare(CASES[name], scheme, 2, "mixed", "dq-tma", 3, tile_j)
        assert status == 0
        tol = {"res": 5e-3, "dt": 1e-5}
        bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
        assert not bad, (scheme, errs)


def test_dq_variant_tile_shape_and_chunking_are_bit_identical():
    """Every face the dq kernel computes goes through one call site and every
    point's residual is summed in one order, whichever tile or k-chunk the
    point and its faces fall in: the state after two steps is the same for
    every tile height and k-chunk, bit for bit."""
    case = CASES["multiblock"]
    out = []
    for tile_j, kz in ((8, 1), (4, 2), (16, 64), (8, 3)):
        d = cc.Driver.from_case(case, "mixed")
        d.set_tuning("dq-tma", kz, tile_j)
        d.initialize_computation()
        assert d.tuning()["tile"] == (32, tile_j, kz)
        d.simulate(2, "rk3")
        out.append([d.field[b].get_state()[2] for b in range(len(case["blocks"]))])
        d.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("variant", ["split-tma", "split-tma-p"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["multiblock", "channel", "box_distorted"])
def test_face_tile_heights_are_bit_identical(name, precision, variant):
    """The TMA face kernel computes every face of a point once, whichever
    tile (32 x 4, 32 x 8, 32 x 16, 16 x 8, 16 x 16 points; 32 x 16 in FP32
    only) and k-chunk it falls in: the state after two RK3 steps does not
    depend on the tile shape, bit for bit."""
    case = CASES[name]
    shapes = [(32, 8, 4), (32, 4, 2), (32, 4, 64), (16, 8, 3), (16, 16, 2)]
    shapes += [(32, 16, 3), (32, 16, 64)] if precision == "mixed" else []
    out = []
    for tile_i, tile_j, kz in shapes:
        d = cc.Driver.from_case(case, precision)
        d.set_tuning(variant, kz, tile_j, tile_i)
        d.initialize_computation()
        assert d.tuning()["tile"] == (tile_i, tile_j, kz)
        d.simulate(2, "rk3")
        assert d.status() == 0
        out.append([d.field[b].get_state()[2] for b in range(len(case["blocks"]))])
        d.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("tile_j", [4, 16])
def test_face_tile_heights_close_to_oracle(tile_j):
    errs, status = compare(CASES["box"], "rk3", 2, "mixed", "split-tma", 3, tile_j)
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
    assert not bad, errs


def test_face_tile_height_16_refused_in_fp64():
    """The 32 x 16 tile's FP64 plane ring does not fit in shared memory (the
    16 x 16 one does)."""
    d = cc.Driver.from_case(CASES["box"], "fp64")
    d.set_tuning("split-tma", 4, 16, 32)
    with pytest.raises(RuntimeError, match="does not fit"):
        d.initialize_computation()
    d.close()


@pytest.mark.parametrize("variant", ["l1", "split", "split-tma", "split-tma-p"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_k_chunking_is_bit_identical(precision, variant):
    """A face at a k-chunk boundary is computed by both chunks through the
    same call site: the state after two steps must not depend on kz."""
    case = CASES["multiblock"]
    out = []
    for kz in (1, 2, 64):
        d = cc.Driver.from_case(case, precision)
        d.set_tuning(variant, kz)
        d.initialize_computation()
        assert d.tuning()["kz"] == kz
        d.simulate(2, "rk3")
        out.append([d.field[b].get_state()[2] for b in range(len(case["blocks"]))])
        d.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_variants_agree_at_64(precision):
    """All stage-kernel variants give the same state at 64^3 (a size whose
    split-variant edge tiles span several CTAs per face layer) after two
    RK3 steps: FP64 to 1e-13, mixed to 1e-6 relative per field."""
    case = cases.case_box(64, species=cases.synthetic_species(), seed=5)
    variants = ["l1", "split", "split-tma", "split-tma-p"] + (["tma", "dq-tma"] if precision == "mixed" else [])
    out = {}
    for v in variants:
        d = cc.Driver.from_case(case, precision)
        d.set_tuning(v, 4)
        d.initialize_computation()
        d.simulate(2, "rk3")
        assert d.status() == 0
        out[v] = d.field[0].get_state()[2].reshape(14, -1)
        d.close()
    tol = 1e-13 if precision == "fp64" else 1e-6
    ref = out["l1"]
    scale = np.abs(ref).max(axis=1)
    for v in variants[1:]:
        rel = np.abs(out[v] - ref).max(axis=1) / scale
        assert rel.max() < tol, (v, rel)


# Full-FP32 precision (conserved state rounded to FP32, FP32 Newton): close
# to the FP64 oracle after two steps, at the FP32 level.
@pytest.mark.parametrize("name", ["box", "channel", "mixing", "sod"])
def test_fp32_close_to_oracle(name):
    errs, status = compare(CASES[name], "rk3", 2, "fp32")
    assert status == 0
    tol = {"res": 5e-2, "dt": 1e-4}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-3)}
    assert not bad, errs


# The uneven 64-block periodic layout at small sizes (5..9 points per side).
MB64_SMALL = cases.case_multiblock(cases.multiblock_sizes(seed=3, lo=5, hi=9), species=cases.synthetic_species(),
                                   seed=3)


@pytest.mark.parametrize("variant", ["l1", "split"])
def test_multiblock64_small_fp64_matches_oracle(variant):
    errs, status = compare(MB64_SMALL, "rk3", 2, "fp64", variant, 4)
    assert status == 0
    bad = {k: v for k, v in errs.items() if not v < 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("variant,precision", [("l1", "fp64"), ("l1", "mixed"), ("split", "fp64"),
                                               ("split", "mixed"), ("dq-tma", "mixed")])
def test_per_block_launches_equal_batched(precision, variant):
    """One launch per block per kernel (the reference's granularity) gives
    bit-identical states to the batched launch over all blocks."""
    out = []
    for mode in ("batched", "per_block"):
        d = cc.Driver.from_case(MB64_SMALL, precision)
        d.set_tuning(variant, 4)
        d.set_launch_mode(mode)
        d.initialize_computation()
        d.simulate(2, "rk3", residual=True)
        out.append(([d.field[b].get_state()[2] for b in range(len(MB64_SMALL["blocks"]))], d.residual()))
        d.close()
    for a, b in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name", mg.NAMES)
def test_fp64_matches_reference_kernels(name):
    """Steady explicit-Euler loop on the golden inputs vs the reference's own
    kernels' outputs (state, transport properties, residual)."""
    case, ref = mg.load(name)
    d = cc.Driver.from_case(case, "fp64")
    d.initialize_computation()
    d.simulate(case["n_steps"], "steady", residual=True)
    ns = 0 if case["params"]["species"] is None else case["params"]["species"]["n_spec"]
    for b in range(len(case["blocks"])):
        bv, yk, cv = d.field[b].get_state()
        for k, v in group_errors(bv, ref["b%d_bv" % b], bv_groups()).items():
            assert v < 1e-10, (k, v)
        for k, v in group_errors(cv, ref["b%d_cv" % b], cv_groups(ns)).items():
            assert v < 1e-10, (k, v)
        mul, cond, rd = d.field[b].get_props()
        assert np.abs(mul - ref["b%d_mul" % b]).max() < 1e-10 * np.abs(ref["b%d_mul" % b]).max()
        if ns:
            assert np.abs(yk - ref["b%d_yk" % b]).max() < 1e-10
    np.testing.assert_allclose(d.residual(), ref["residual"], rtol=1e-8)
    d.close()


def test_graph_replay_equals_launches():
    case = CASES["box"]
    out = []
    for graph in (True, False):
        d = cc.Driver.from_case(case, "mixed")
        d.use_graph(graph)
        d.initialize_computation()
        d.simulate(3)
        out.append(d.field[0].get_state()[2])
        d.close()
    assert np.array_equal(out[0], out[1])


def test_status_flags_nonfinite_state():
    """A NaN seeded into the host state (one interior temperature) is reported
    through the status word; the context stays usable."""
    case = cases.case_box(10, species=cases.synthetic_species(), seed=4)
    bv = case["blocks"][0]["bv"].copy()
    n = 10 + 4
    bv[5, 5 + n * (5 + n * 5)] = np.nan  # interior point (3, 3, 3)
    case["blocks"][0]["bv"] = bv
    d = cc.Driver.from_case(case, "fp64")
    d.initialize_computation()
    d.simulate(1)
    assert d.status() & 2
    assert d.status() == 0  # cleared by the read
    d.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_conservation_and_mass_fractions(precision):
    """128^3 periodic box: conserved totals over the unique points are kept
    (flux form) and the mass fractions stay normalised."""
    n = 128
    case = cases.case_box(n, species=cases.synthetic_species(), seed=1234)
    d = cc.Driver.from_case(case, precision)
    d.set_renormalize(True)
    d.initialize_computation()
    sl = (slice(None), slice(2, -3), slice(2, -3), slice(2, -3))
    cv0 = d.field[0].get_state()[2].reshape(14, n + 4, n + 4, n + 4)[sl].sum(axis=(1, 2, 3))
    d.simulate(5)
    bv, yk, cv = d.field[0].get_state()
    cv1 = cv.reshape(14, n + 4, n + 4, n + 4)[sl].sum(axis=(1, 2, 3))
    scale = np.abs(cv0).max()
    assert np.abs(cv1 - cv0).max() < 1e-12 * scale
    ysum = interior(yk, (n, n, n)).sum(axis=0)
    assert np.abs(ysum - 1).max() < (1e-12 if precision == "fp64" else 5e-6)
    assert np.isfinite(bv).all()
    assert d.status() == 0
    d.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restart_is_bit_identical(precision, tmp_path):
    case = CASES["channel"]
    d = cc.Driver.from_case(case, precision)
    d.initialize_computation()
    d.simulate(3, "rk3")
    path = tmp_path / "state.ckpt"
    d.save_checkpoint(path)
    d.simulate(3, "rk3", residual=True)
    want, want_res = d.field[0].get_state(), d.residual()
    d.close()
    e = cc.Driver.from_case(case, precision)
    e.initialize_computation()
    e.load_checkpoint(path)
    e.simulate(3, "rk3", residual=True)
    got, got_res = e.field[0].get_state(), e.residual()
    assert e.status() == 0
    e.close()
    for a, b in zip(want, got):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(want_res, got_res)
    # a context of another precision refuses the file
    f = cc.Driver.from_case(case, "fp64" if precision == "mixed" else "mixed")
    f.initialize_computation()
    with pytest.raises(RuntimeError, match="another layout or precision"):
        f.load_checkpoint(path)
    f.close()


# LU-SGS steady steps (the implicit scheme of temporal_scheme 1) against the
# oracle's lexicographic sweeps: at the cases' CFL 0.5 and at CFL 5.
def _with_cfl(case, cfl):
    c = dict(case)
    c["params"] = dict(case["params"], cfl=cfl)
    return c


@pytest.mark.parametrize("cfl", [0.5, 5.0])
@pytest.mark.parametrize("name", sorted(CASES))
def test_lusgs_fp64_matches_oracle(name, cfl):
    errs, status = compare(_with_cfl(CASES[name], cfl), "lusgs", 3, "fp64")
    assert status == 0
    bad = {k: v for k, v in errs.items() if not v < 1e-10}
    assert not bad, errs


@pytest.mark.parametrize("name", sorted(CASES))
def test_lusgs_mixed_close_to_oracle(name):
    errs, status = compare(_with_cfl(CASES[name], 5.0), "lusgs", 3, "mixed")
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4)}
    assert not bad, errs


def test_lusgs_multiblock64_small_matches_oracle():
    errs, status = compare(_with_cfl(MB64_SMALL, 5.0), "lusgs", 3, "fp64")
    assert status == 0
    bad = {k: v for k, v in errs.items() if not v < 1e-10}
    assert not bad, errs


def test_lusgs_graph_replay_equals_launches():
    case = _with_cfl(CASES["multiblock"], 5.0)
    out = []
    for graph in (True, False):
        d = cc.Driver.from_case(case, "mixed")
        d.use_graph(graph)
        d.initialize_computation()
        d.simulate(3, "lusgs")
        out.append([d.field[b].get_state()[2] for b in range(len(case["blocks"]))])
        d.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ["box", "channel", "sod"])
def test_lusgs_fp32_close_to_oracle(name):
    """LU-SGS in the full-FP32 precision (conserved state rounded to FP32):
    at the FP32 level of the RK3 test."""
    errs, status = compare(_with_cfl(CASES[name], 5.0), "lusgs", 3, "fp32")
    assert status == 0
    tol = {"res": 5e-2, "dt": 1e-4}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-3)}
    assert not bad, errs


def test_lusgs_with_learned_closure():
    """LU-SGS steps with the transport of each new state from the learned
    closure: after five CFL-5 steps (ten times the time an RK3 step at CFL
    0.5 advances) the state stays within a few times the closure's ~1e-3
    transport error of the steps with the exact transport."""
    from combustioncodegpu_b200 import closure

    w, _ = closure.load()
    case = _with_cfl(cases.case_box(16, species=cases.synthetic_species(), seed=4), 5.0)
    out = {}
    for mode in ("exact", "closure"):
        d = cc.Driver.from_case(case, "mixed")
        if mode == "closure":
            d.set_closure(w)
            d.use_closure(True)
        d.initialize_computation()
        d.simulate(5, "lusgs")
        assert d.status() == 0
        out[mode] = d.field[0].get_state()[0]
        d.close()
    for f in (0, 4, 5):  # rho, p, T
        rel = np.abs(out["closure"][f] - out["exact"][f]).max() / np.abs(out["exact"][f]).max()
        assert rel < 5e-3, (f, rel)


# A species count without a compiled specialisation (4: H2, O2, H2O, N2) runs
# the kernels' runtime-count path.
SP4 = cases.synthetic_species([cases.H2O2_N2_SPECIES[i] for i in (0, 1, 2, 8)])


@pytest.mark.parametrize("variant", ["l1", "split"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_runtime_species_count_matches_oracle(precision, variant):
    case = cases.case_box_distorted(10, amp=0.3, species=SP4, seed=4)
    errs, status = compare(case, "rk3", 2, precision, variant, 3)
    assert status == 0
    tol = {"res": 5e-3, "dt": 1e-5} if precision == "mixed" else {}
    bad = {k: v for k, v in errs.items() if not v < tol.get(k, 1e-4 if precision == "mixed" else 1e-10)}
    assert not bad, errs


def test_fused_tma_variant_refused_in_fp64():
    """The fused TMA variant exists in the FP32 bulk precision only (its FP64
    planes do not fit in shared memory): pinning it on an FP64 context fails
    at cc_init, before any kernel runs."""
    for variant in ("tma", "dq-tma"):
        d = cc.Driver.from_case(CASES["box"], "fp64")
        d.set_tuning(variant, 4)
        with pytest.raises(RuntimeError, match="TMA variants"):
            d.initialize_computation()
        d.close()


def test_tma_variants_refused_without_tensor_maps():
    """Tensor maps exist for 0 or 9 species only: pinning a TMA variant on a
    context with another species count fails at cc_init."""
    case = cases.case_box(8, species=SP4, seed=2)
    for variant in ("tma", "split-tma", "split-tma-p", "dq-tma"):
        d = cc.Driver.from_case(case, "mixed")
        d.set_tuning(variant, 4)
        with pytest.raises(RuntimeError, match="TMA variants"):
            d.initialize_computation()
        d.close()


@pytest.mark.parametrize("name", ["channel", "multiblock", "mixing", "box"])
@pytest.mark.parametrize("precision,scheme", [("fp64", "rk3"), ("mixed", "rk3"), ("fp64", "steady")])
def test_ghost_conserved_state_written_before_read_out(name, precision, scheme):
    """Steps leave the conserved state of ghost points that nothing reads
    (the stage kernels read Q at interior points only) and cc_get_state
    writes it first.  A no-op exchange hook makes every step run every halo
    copy; both runs must give the same states at every point, ghost points
    included, bit for bit."""
    import ctypes

    case = CASES[name]
    out = []
    for hooked in (False, True):
        d = cc.Driver.from_case(case, precision)
        if hooked:
            def noop(user, event, stage, value):
                return 0  # the local time step is the global one on one process

            fn = cc.EXCHANGE_FN(noop)
            assert d.lib.cc_set_exchange(d.ctx, ctypes.cast(fn, ctypes.c_void_p), None) == 0
        d.initialize_computation()
        d.simulate(3, scheme)
        out.append([d.field[b].get_state()[2] for b in range(len(case["blocks"]))])
        if hooked:
            d.lib.cc_set_exchange(d.ctx, None, None)
        d.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
