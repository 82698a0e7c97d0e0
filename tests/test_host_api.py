"""Host-side checks of the C ABI (no device needed): the library loads and
exports every entry point include/cc_b200.h declares, face registration
matches the oracle's restatement of Mesh.cpp, and argument errors are
reported."""
import ctypes
import os
import re

import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases
from oracle.oracle_py import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cc_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cc_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(cclib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(cclib, n), n
    assert set(names) <= set(cc.EXPORTS), set(names) - set(cc.EXPORTS)


def test_version_and_no_device_error(cclib):
    assert cclib.cc_version() >= 10000
    if cc.device_count() == 0:
        d = cc.Driver.from_case(cases.case_sod(32, 5, 5))
        with pytest.raises(cc.CCError, match="no CUDA device"):
            d.initialize_computation()


@pytest.mark.parametrize("make", [lambda: cases.case_channel((9, 6, 5)),
                                  lambda: cases.case_multiblock(([6, 7], [6, 5], [5])),
                                  lambda: cases.case_sod(20, 5, 5)])
def test_face_registration_matches_oracle(cclib, make):
    case = make()
    o = Oracle(case)
    walls = {bc["label"] for bc in case["bcs"] if bc["kind"] == 2}
    for b, blk in enumerate(case["blocks"]):
        ob = o.boundaries(b)
        for raw, x in zip(blk["boundaries"], ob):
            y = cc.register_boundary(raw)
            if y.type_label in walls:  # BoundCond.cu:218-230, applied when the condition is registered
                for q in range(3):
                    if q != y.face:
                        y.range_start[q] += 2
                        y.range_end[q] -= 2
            assert cc.boundary_tuple(y) == (tuple(x.range_start), tuple(x.range_end), x.type_label, x.face,
                                            x.direction)
        for raw, x in zip(blk["inner_faces"], o.inner_faces(b)):
            assert cc.inner_face_tuple(cc.register_inner_face(raw)) == cc.inner_face_tuple(x)


def test_invalid_parameters_are_rejected(cclib):
    p, keep = cc.make_params(cc.Parameter(cases.default_params(None)), None)
    p.ngg = 3
    ctx = ctypes.c_void_p()
    assert cclib.cc_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    assert b"ngg" in cclib.cc_last_error()
    p.ngg = 2
    p.inviscid_scheme = 2
    assert cclib.cc_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    p.inviscid_scheme = 3
    assert cclib.cc_create(ctypes.byref(p), ctypes.byref(ctx)) == 0
    jac = np.ones(8 * 8 * 8)
    met = np.ones(9 * 8 * 8 * 8)
    bid = ctypes.c_int()
    assert cclib.cc_add_block(ctx, 0, 4, 4, cc._ptr(jac), cc._ptr(met), ctypes.byref(bid)) == -1
    assert cclib.cc_step(ctx, 1, 0, 0) == -2  # before cc_init
    # a state layout that is neither field- nor point-major
    assert cclib.cc_add_block(ctx, 4, 4, 4, cc._ptr(jac), cc._ptr(met), ctypes.byref(bid)) == 0
    bv = np.ones(6 * 8 * 8 * 8)
    assert cclib.cc_set_state(ctx, bid.value, cc._ptr(bv), None, 2) == -1
    assert b"layout" in cclib.cc_last_error()
    assert cclib.cc_set_state(ctx, bid.value, cc._ptr(bv), None, 1) == 0
    assert cclib.cc_destroy(ctx) == 0


def test_state_layout_names(cclib):
    """The Python mirror takes the layout by name: "field" ([n_field][Ng]) or
    "point" ([Ng][n_field], the reference's VectorField3D order); the
    point-major arrays reach the library before cc_init without a device."""
    case = cases.case_sod(8, 5, 5)
    blk = case["blocks"][0]
    d = cc.Driver.from_case(case)
    d.field[0].set_state(np.ascontiguousarray(blk["bv"].T), None, layout="point")
    with pytest.raises(ValueError):
        d.field[0].set_state(blk["bv"], None, layout="aos")
    d.close()


def test_struct_layouts_match_reference_pods():
    # cfd::Boundary is 9 ints, cfd::InnerFace 26 ints (Mesh.h:9-60)
    assert ctypes.sizeof(cc.CCBoundary) == 9 * 4
    assert ctypes.sizeof(cc.CCInnerFace) == 26 * 4


def test_multi_process_entry_points_validate_arguments(cclib):
    """cc_set_owned_blocks refuses blocks that do not exist, and the
    exchange's pack / unpack refuse to run outside cc_init and an exchange
    hook call (no device needed for either check)."""
    case = cases.case_multiblock(([6, 7], [6, 5], [5]), species=cases.synthetic_species())
    d = cc.Driver.from_case(case)
    bad = (ctypes.c_int * 1)(7)
    assert cclib.cc_set_owned_blocks(d.ctx, bad, 1) == -1
    assert b"no block 7" in cclib.cc_last_error()
    good = (ctypes.c_int * 2)(0, 3)
    assert cclib.cc_set_owned_blocks(d.ctx, good, 2) == 0
    assert cclib.cc_set_owned_blocks(d.ctx, None, 0) == 0  # every block again
    nf = ctypes.c_int()
    assert cclib.cc_exchange_fields(d.ctx, ctypes.byref(nf)) == 0
    assert nf.value == (6 + 9) + (2 + 9) + (5 + 9)
    idx = np.zeros(1, dtype=np.int64)
    out = np.zeros(nf.value)
    assert cclib.cc_pack_points(d.ctx, 0, idx.ctypes.data_as(ctypes.c_void_p), 1,
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == -2  # before cc_init
    d.close()


def test_tile_width_argument_checks(cclib):
    """cc_set_tile_width takes 0 (autotune), 16 or 32 points along i and
    refuses anything else (no device needed)."""
    d = cc.Driver.from_case(cases.case_sod(20, 5, 5))
    for ok in (0, 16, 32):
        assert cclib.cc_set_tile_width(d.ctx, ok) == 0
    assert cclib.cc_set_tile_width(d.ctx, 8) == -1
    assert b"tile_i" in cclib.cc_last_error()
    d.close()
