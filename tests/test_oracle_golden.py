"""Pins the CPU oracle to the reference's own kernels.

tests/golden/*.npz hold small seeded cases and the outputs of the
reference's CUDA kernels (built from the reference sources by
oracle/ref_harness/build_ref.sh and run on a B200 by
tests/golden/make_golden.py): processed face descriptors, the first step's
dq and local dt, and the state, transport properties and residual after n
steps of the reference's steady explicit-Euler loop."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as mg  # noqa: E402
from oracle.oracle_py import Oracle  # noqa: E402

# FP64 on both sides; the reference runs on the GPU (FMA contraction), the
# oracle on the host without contraction: agreement to rounding.
RTOL = 1e-12


def relmax(a, r):
    s = np.maximum(np.abs(r).max(axis=-1, keepdims=True), 1e-300)
    return float((np.abs(a - r) / s).max())


@pytest.mark.parametrize("name", mg.NAMES)
def test_oracle_matches_reference_kernels(name):
    case, ref = mg.load(name)
    o = Oracle(case)
    o.init()
    for b in range(len(case["blocks"])):
        got_b = [[*x.range_start, *x.range_end, x.type_label, x.face, x.direction] for x in o.boundaries(b)]
        assert np.array_equal(np.array(got_b, dtype=np.int64).reshape(-1, 9), ref["b%d_boundaries" % b])
        got_f = [[*x.range_start, *x.range_end, x.face, x.direction, *x.target_start, *x.target_end, x.target_block,
                  x.target_face, x.target_direction, *x.src_tar, *x.loop_dir, *x.target_loop_dir]
                 for x in o.inner_faces(b)]
        assert np.array_equal(np.array(got_f, dtype=np.int64).reshape(-1, 26), ref["b%d_inner_faces" % b])
    dq = [o.dq(b) for b in range(len(case["blocks"]))]
    o.steady_step(1)
    for b in range(len(case["blocks"])):
        assert relmax(dq[b], ref["b%d_dq1" % b]) < RTOL
        assert relmax(o.dt_local(b)[None], ref["b%d_dt1" % b][None]) < RTOL
    o.steady_step(case["n_steps"] - 1)
    for b in range(len(case["blocks"])):
        bv, yk, cv = o.state(b)
        assert relmax(bv, ref["b%d_bv" % b]) < 1e-12
        assert relmax(cv, ref["b%d_cv" % b]) < 1e-12
        mul, cond, rd = o.props(b)
        assert relmax(mul[None], ref["b%d_mul" % b][None]) < RTOL
        assert relmax(cond[None], ref["b%d_cond" % b][None]) < RTOL
        if o.ns:
            assert relmax(yk, ref["b%d_yk" % b]) < RTOL
            assert relmax(rd, ref["b%d_rho_d" % b]) < RTOL
    np.testing.assert_allclose(o.residual(), ref["residual"], rtol=1e-12)
