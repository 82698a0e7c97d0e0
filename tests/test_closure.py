"""Learned transport closure (the tcgen05 MLP kernel) and the exact
pointwise transport it replaces.

* the exact FP64 transport kernel behind cc_eval_transport against the
  oracle's transport (Transport.cu:43-96 restated), 1e-12 relative;
* the tensor-core MLP kernel against a plain PyTorch FP32 reference of the
  same network with the kernel's rounding points (BF16 inputs as hi/lo pairs,
  BF16 weights, FP32 hidden activations, which the kernel carries as BF16
  hi/lo pairs, FP32 accumulation), on seeded random weights: differences
  come from the ~2^-17 relative residue of the hi/lo pairs and the FP32
  summation order, so log-space errors stay below 1e-3 (max) and 1e-5
  (median);
* the trained closure's accuracy against the exact transport (the measure
  of its error) with the run-time check off: median relative error at most
  1e-3; and the run-time check itself (4 samples per 128-point tile: a tile
  goes back to the exact transport when its sampled relative error exceeds
  1e-3 in root mean square, or 1e-2 in one output): with the trained weights
  it sends a minority of tiles back, with a deliberately perturbed network
  every tile, and the output is then the exact transport;
* the trained closure inside the stages, and its exact fallback outside the
  training hull;
* the training kernels (cc_mlp_grad, cc_mlp_adam) against the CPU
  restatement of the same quantisation-aware math (oracle/closure_mlp.py),
  and a short training run through them.
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
    d.set_closure_bound(0.0)  # the network itself, not the exact transport of failing tiles
    got = np.log(d.eval_transport(T, Y, "closure"))
    d.close()
    err = np.abs(got - ref)
    assert np.median(err) < 1e-5, np.median(err)
    assert err.max() < 1e-3, err.max()


def _trained():
    if not os.path.exists(closure.DEFAULT_WEIGHTS):
        pytest.fail("trained closure weights missing: python -m combustioncodegpu_b200.closure")
    return closure.load()[0]


@pytest.mark.parametrize("states", ["train", "edge", "box"])
def test_trained_closure_accuracy(states):
    """The network alone (run-time check off) on fresh states inside the
    hull, from the training distribution, from its Dirichlet(0.5) half, and
    from the synthetic box generator: median relative error over the 11
    outputs at most 1e-3."""
    w = _trained()
    d = _driver()
    d.set_closure(w)
    d.set_closure_bound(0.0)
    rep = closure.validate(d, SP, n=50_000, seed=5, states=states)
    d.close()
    assert rep["median"] <= 1e-3 and rep["p99"] < 1e-2, rep


def test_run_time_check_sends_bad_tiles_to_the_exact_transport():
    w = dict(_trained())
    T, Y, _ = closure.sample_states(128 * 400, SP, seed=21)
    d = _driver()
    exact = d.eval_transport(T, Y, "exact")
    d.set_closure(w)  # the trained network, check at the default 1e-3
    got = d.eval_transport(T, Y, "closure")
    n_eval, n_hull, n_chk = d.closure_stats()
    assert n_eval == T.size and n_chk < 0.5 * n_eval, (n_eval, n_hull, n_chk)
    rel = np.abs(got / exact - 1.0)
    assert np.median(rel) <= 1e-3
    # a network whose every output is off by 1 % (output bias shifted): every
    # tile fails its samples and takes the exact transport
    bad = dict(w)
    bad["out_mean"] = np.asarray(w["out_mean"], np.float32) + np.float32(0.01)
    d.set_closure(bad)
    got = d.eval_transport(T, Y, "closure")
    n_eval, n_hull, n_chk = d.closure_stats()
    d.close()
    assert n_eval == T.size and n_hull + n_chk == n_eval, (n_eval, n_hull, n_chk)
    np.testing.assert_allclose(got, exact, rtol=2e-5)


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
            # the box's compositions (every species present, none dominant) lie
            # where the Dirichlet(0.5) training set is thin: the network's
            # error there is near the bound, and the run-time check sends
            # many tiles to the exact transport
            n_eval, n_fb, n_chk = d.closure_stats()
            assert n_eval >= 24 ** 3 * 15 and n_fb == 0 and n_chk <= n_eval
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
    n_eval, n_fb, _ = d.closure_stats()
    d.close()
    hot = T > 900.0
    X = closure.mole_fractions(Y, SP["mw"])
    pure = X.max(axis=0) >= 0.9985  # clearly inside the near-pure-species fallback
    assert n_eval == T.size and int(hot.sum()) <= n_fb <= int((hot | (X.max(axis=0) >= 0.9975)).sum())
    np.testing.assert_allclose(got[:, hot | pure], exact[:, hot | pure], rtol=2e-5)


# ---------------------------------------------------------------- training kernels

H = closure.HIDDEN


def _mlp_batch(n, seed):
    """Features of sampled states (BF16 values), random targets and scales."""
    import torch

    ns = SP["n_spec"]
    T, Y, X = closure.sample_states(n, SP, seed=seed)
    x = closure.features(T, X, "cuda").contiguous()
    rng = np.random.default_rng(seed)
    y = torch.as_tensor(rng.standard_normal((n, 2 + ns)), dtype=torch.float32, device="cuda")
    scale = torch.as_tensor(rng.uniform(0.5, 2.0, 2 + ns), dtype=torch.float32, device="cuda")
    net = closure.ClosureNet(2 + 2 * ns, 2 + ns, "cuda", seed=seed)
    params = torch.cat([p.detach().reshape(-1) for p in net.params]).contiguous()
    params += 0.05 * torch.randn(params.numel(), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    return x, y, scale, params


def _grad(lib, x, y, scale, params):
    import ctypes
    import torch

    n_in, n_out, n = x.shape[1], y.shape[1], x.shape[0]
    grad = torch.zeros_like(params)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    work = torch.empty(lib.cc_mlp_workspace_bytes(n_in, H, n_out, n), dtype=torch.uint8, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.cc_mlp_grad(n_in, H, n_out, n, vp(params), vp(x), vp(y), vp(scale), vp(grad), vp(loss), vp(work),
                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.cc_last_error()
    torch.cuda.synchronize()
    return float(loss), grad.cpu().numpy()


def test_mlp_gradient_matches_oracle():
    """Loss and gradient of the quantisation-aware MLP: the kernels (FP32
    sums in a fixed order) against the FP64 restatement on the same rounded
    operands, on a batch that is not a multiple of the 32-row CTA tile."""
    from oracle import closure_mlp as om

    lib = cc.load_library()
    x, y, scale, params = _mlp_batch(300, seed=11)
    loss, grad = _grad(lib, x, y, scale, params)
    ns = SP["n_spec"]
    ref_loss, ref_grad = om.loss_and_grad(params.cpu().numpy(), x.cpu().numpy(), y.cpu().numpy(),
                                          scale.cpu().numpy(), 2 + 2 * ns, H, 2 + ns)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-5)
    lay, n = om.layout(2 + 2 * ns, H, 2 + ns)
    assert grad.size == n
    for ow, shp, ob, nb in lay:  # per weight matrix and bias: max error against that tensor's scale
        for a, b in ((ow, ow + shp[0] * shp[1]), (ob, ob + nb)):
            g, r = grad[a:b], ref_grad[a:b]
            tol = 1e-3 * np.abs(r).max()
            assert np.abs(g - r).max() <= tol, (a, np.abs(g - r).max(), tol)
            assert np.median(np.abs(g - r)) <= 1e-5 * np.abs(r).max()


def test_mlp_gradient_is_reproducible():
    lib = cc.load_library()
    x, y, scale, params = _mlp_batch(4096, seed=12)
    a = _grad(lib, x, y, scale, params)
    b = _grad(lib, x, y, scale, params)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])


def test_mlp_adam_matches_oracle():
    import ctypes
    import torch
    from oracle import closure_mlp as om

    lib = cc.load_library()
    rng = np.random.default_rng(3)
    n = 10379
    p0, g = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m0, v0 = (0.1 * rng.standard_normal(n)).astype(np.float32), rng.uniform(0, 0.1, n).astype(np.float32)
    t = [torch.as_tensor(a, device="cuda") for a in (p0, g, m0, v0)]
    vp = lambda a: ctypes.c_void_p(a.data_ptr())
    rc = lib.cc_mlp_adam(n, vp(t[0]), vp(t[1]), vp(t[2]), vp(t[3]), 1e-3, 0.9, 0.999, 1e-8, 7,
                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.cc_last_error()
    torch.cuda.synchronize()
    f32 = lambda v: float(np.float32(v))  # the kernel receives FP32 hyperparameters
    p1, m1, v1 = om.adam(p0.astype(np.float64), g.astype(np.float64), m0.astype(np.float64), v0.astype(np.float64),
                         f32(1e-3), f32(0.9), f32(0.999), f32(1e-8), 7)
    np.testing.assert_allclose(t[2].cpu().numpy(), m1, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(t[3].cpu().numpy(), v1, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(t[0].cpu().numpy(), p1, rtol=1e-6, atol=1e-6)


def test_short_training_run_learns_the_transport():
    """Ten epochs on 100k states through the training kernels: on held-out
    states the trained network's median relative error is a few per cent,
    a tenth or less of the same network's before training."""
    ns = SP["n_spec"]
    d = _driver()
    w, rep = closure.train(d, SP, n_samples=100_000, n_val=20_000, epochs=10, batch=4096, lr=5e-3,
                           log=lambda *a: None)
    d.set_closure_bound(0.0)  # the networks themselves
    d.set_closure(w)
    trained = closure.validate(d, SP, n=20_000, seed=8)
    d.set_closure(closure.ClosureNet(2 + 2 * ns, 2 + ns, "cuda", seed=7).export(w["out_mean"], w["out_scale"]))
    untrained = closure.validate(d, SP, n=20_000, seed=8)
    d.close()
    assert trained["median"] < 0.05, (trained, rep)
    assert trained["median"] < 0.1 * untrained["median"], (trained, untrained)
