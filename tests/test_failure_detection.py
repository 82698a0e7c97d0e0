"""Failure detection on the GPU without a GPU fault.

* A device-side wait that gives up: the TMA plane waits of the face kernel
  check once without blocking, then poll at most cc_set_wait_limit times.
  With a limit of 0 the first plane of every tile, requested from memory a
  few instructions earlier, is not there yet: the kernel sets status bit 3,
  waits (with its own fixed bound) for the copies it has in flight and
  returns.  The context stays usable: after the limit is restored and the
  state set again, a step gives the same state as a fresh context.  The
  learned closure's tensor-core completion wait gives up the same way
  (status bit 4, reported as an error by cc_eval_transport).
* The temperature Newton's iteration cap (Thermo.cu:103-121 stops silently
  after 1000 iterations; here the cap is settable and reported): with a cap of
  one iteration, a state whose temperature changes by far more than the 1e-3
  tolerance in one stage (a 400 K / 1400 K jump at uniform pressure) sets
  status bit 0; with the default cap the same step converges everywhere.
"""
import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases

pytestmark = pytest.mark.gpu

STATUS_NEWTON_CAP, STATUS_TMA_TIMEOUT = 1, 8


def test_tma_wait_limit_gives_up_and_context_recovers():
    case = cases.case_box(128, species=cases.synthetic_species(), seed=1234)
    blk = case["blocks"][0]
    d = cc.Driver.from_case(case, "mixed")
    d.set_tuning("split-tma", 4)
    d.initialize_computation()
    d.set_wait_limit(0)
    d.simulate(1)
    assert d.status() & STATUS_TMA_TIMEOUT
    d.set_wait_limit(None)
    d.field[0].set_state(blk["bv"], blk["yk"])
    d.simulate(1)
    assert d.status() == 0
    got = d.field[0].get_state()[2]
    d.close()
    e = cc.Driver.from_case(case, "mixed")
    e.set_tuning("split-tma", 4)
    e.initialize_computation()
    e.simulate(1)
    want = e.field[0].get_state()[2]
    assert e.status() == 0
    e.close()
    np.testing.assert_array_equal(got, want)


def test_closure_wait_limit_gives_up_and_recovers():
    from combustioncodegpu_b200 import closure

    w, _ = closure.load()
    case = cases.case_box(8, species=cases.synthetic_species(), seed=2)
    d = cc.Driver.from_case(case, "mixed")
    d.initialize_computation()
    d.set_closure(w)
    T, Y, _ = closure.sample_states(4096, cases.synthetic_species(), seed=5)
    want = d.eval_transport(T, Y, "closure")
    d.set_wait_limit(0)
    with pytest.raises(RuntimeError, match="status 16"):
        d.eval_transport(T, Y, "closure")
    d.set_wait_limit(None)
    np.testing.assert_array_equal(d.eval_transport(T, Y, "closure"), want)
    d.close()


def _temperature_jump_case():
    sp = cases.synthetic_species()
    case = cases.case_box(12, species=sp, seed=6)
    blk = case["blocks"][0]
    bv, yk = blk["bv"].copy(), blk["yk"]
    n = 12 + 4
    i = np.arange(bv.shape[1]) % n
    T = np.where(i < n // 2, 400.0, 1400.0)
    mw = np.asarray(sp["mw"])[:, None]
    bv[5] = T
    bv[0] = bv[4] / (cases.R_U * T * (yk / mw).sum(axis=0))
    blk["bv"] = bv
    return case


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_newton_iteration_cap_is_reported(precision):
    case = _temperature_jump_case()
    d = cc.Driver.from_case(case, precision)
    d.initialize_computation()
    d.set_newton_max_iter(1)
    d.simulate(1)
    assert d.status() & STATUS_NEWTON_CAP
    d.close()
    d = cc.Driver.from_case(case, precision)
    d.initialize_computation()
    d.simulate(1)
    assert d.status() == 0
    d.close()
