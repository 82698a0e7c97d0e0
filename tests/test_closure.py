"""Learned transport closure (the tcgen05 MLP kernel) and the exact
pointwise transport it replaces.

* the exact FP64 transport kernel behind cc_eval_transport against the
  oracle's transport (Transport.cu:43-96 restated), 1e-12 relative;
* the tensor-core MLP kernel against a plain PyTorch FP32 reference of the
  same network with the kernel's rounding points (BF16 inputs as hi/lo pairs,
  BF16 weights and hidden activations, FP32 accumulation), on seeded random
  weights: differences come only from FP32 summation order flipping a BF16
  rounding, so log-space errors stay below 5e-3 (max) and 1e-4 (median);
* the trained closure inside the stages, and its exact fallback outside the
  training hull.
"""
import os

import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases, closure

pytestmark = pytest.mark.gpu

SP = cases.synthetic_species()


def _driver(case=None, precision="mixed"):
    return cc.Driver.from_case(case or cases.case_box(4, species=SP), precision)


def test_exact_transport_matches_oracle():
    from oracle.oracle_py import kat_transport

    T, Y, _ = closure.sample_states(64, SP, seed=1)
    d = _driver()
    got = d.eval_transport(T, Y, "exact")
    d.close()
    for i in range(T.size):
        mu, lam, rd = kat_transport(SP, T[i], Y[:, i])
        np.testing.assert_allclose(got[0, i], mu, rtol=1e-12)
        np.testing.assert_allclose(got[1, i], lam, rtol=1e-12)
        np.testing.assert_allclose(got[2:, i], rd, rtol=1e-12)


def test_closure_kernel_matches_torch_reference():
    import torch

    ns = SP["n_spec"]
    net = closure.ClosureNet(2 + 2 * ns, 2 + ns, "cuda", seed=3)
    w = net.export(np.zeros(2 + ns), np.ones(2 + ns))  # kernel output = exp(o)
    T, Y, _ = closure.sample_states(4096 + 77, SP, seed=2)  # not a multiple of the 128-point tile
    inv_mw = (1.0 / np.asarray(SP["mw"])).astype(np.float32)
    X32 = Y.astype(np.float32) * inv_mw[:, None]
    X32 = X32 / X32.sum(axis=0, keepdims=True)
    with torch.no_grad():
        ref = net.forward(closure.features(T.astype(np.float32), X32, "cuda")).cpu().numpy().T
    d = _driver()
    d.set_closure(w)
    got = np.log(d.eval_transport(T, Y, "closure"))
    d.close()
    err = np.abs(got - ref)
    assert np.median(err) < 1e-4, np.median(err)
    assert err.max() < 5e-3, err.max()


def _trained():
    if not os.path.exists(closure.DEFAULT_WEIGHTS):
        pytest.fail("trained closure weights missing: python -m combustioncodegpu_b200.closure")
    return closure.load()[0]


def test_trained_closure_accuracy():
    w = _trained()
    d = _driver()
    d.set_closure(w)
    rep = closure.validate(d, SP, n=50_000, seed=5)
    d.close()
    assert rep["median"] < 2e-3 and rep["p99"] < 2e-2, rep


def test_closure_in_stages_and_fallback():
    w = dict(_trained())
    case = cases.case_box(24, species=SP, seed=4)
    out = {}
    for mode in ("exact", "closure"):
        d = _driver(case)
        if mode == "closure":
            d.set_closure(w)
            d.use_closure(True)
        d.initialize_computation()
        d.simulate(5, "rk3")
        assert d.status() == 0
        out[mode] = d.field[0].get_state()[0]
        if mode == "closure":
            n_eval, n_fb = d.closure_stats()
            assert n_eval >= 24 ** 3 * 15 and n_fb == 0
        d.close()
    for f in (0, 4, 5):  # rho, p, T
        rel = np.abs(out["closure"][f] - out["exact"][f]).max() / np.abs(out["exact"][f]).max()
        assert rel < 1e-3, (f, rel)
    # outside the hull (here: T above 900 K) the exact transport is used
    w["t_max"] = 900.0
    T, Y, _ = closure.sample_states(2000, SP, seed=6, t_range=(300.0, 1500.0))
    d = _driver()
    d.set_closure(w)
    exact = d.eval_transport(T, Y, "exact")
    got = d.eval_transport(T, Y, "closure")
    n_eval, n_fb = d.closure_stats()
    d.close()
    hot = T > 900.0
    X = closure.mole_fractions(Y, SP["mw"])
    pure = X.max(axis=0) >= 0.9985  # clearly inside the near-pure-species fallback
    assert n_eval == T.size and int(hot.sum()) <= n_fb <= int((hot | (X.max(axis=0) >= 0.9975)).sum())
    np.testing.assert_allclose(got[:, hot | pure], exact[:, hot | pure], rtol=2e-5)
