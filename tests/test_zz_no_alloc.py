"""cc_residual_rms_noalloc: the residual norms without any device allocation.

This entry point is for callers that cannot call cudaMalloc where they need
the norms (an allocation-free time loop, or a host application whose own
allocator owns the device memory).  It reduces caller-provided device arrays
with a fixed scratch array compiled into the library, so it must give the
same answer as the context's own residual (cc_step with a residual request,
then cc_residual), including on a second call that finds the previous call's
partial sums still in the shared scratch.  This file is collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import combustioncodegpu_b200 as cc
from combustioncodegpu_b200 import cases

pytestmark = pytest.mark.gpu

RTOL = 1e-10  # the FP64 tolerance of the other GPU parity tests


def _rho_vel_p_t(bv, dims):
    """(rho, |V|, p, T) of the interior points as a [4][n] FP64 array."""
    mx, my, mz = dims
    b = bv.reshape(6, mz + 4, my + 4, mx + 4)[:, 2:-2, 2:-2, 2:-2].reshape(6, -1)
    vel = np.sqrt(b[1] * b[1] + b[2] * b[2] + b[3] * b[3])
    return np.ascontiguousarray(np.stack([b[0], vel, b[4], b[5]]))


def test_noalloc_residual_matches_context_residual_twice():
    import torch

    lib = cc.load_library()
    n_side = 16
    case = cases.case_box(n_side, species=cases.synthetic_species(), seed=8)
    dims = (n_side,) * 3
    d = cc.Driver.from_case(case, "fp64")
    d.initialize_computation()
    last = _rho_vel_p_t(d.field[0].get_state()[0], dims)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row share the library's scratch array
        d.simulate(1, residual=True)
        expected = d.residual()
        cur = _rho_vel_p_t(d.field[0].get_state()[0], dims)
        cur_d = torch.from_numpy(cur).cuda()
        last_d = torch.from_numpy(last).cuda()
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream().cuda_stream
        rc = lib.cc_residual_rms_noalloc(ctypes.c_void_p(cur_d.data_ptr()), ctypes.c_void_p(last_d.data_ptr()),
                                         cur.shape[1], ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, lib.cc_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, expected, rtol=RTOL)
        assert np.all(got > 0)
        last = cur
    d.close()


def _call(lib, cur_d, last_d, n, out):
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.cc_residual_rms_noalloc(ctypes.c_void_p(cur_d.data_ptr()), ctypes.c_void_p(last_d.data_ptr()), n,
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.cc_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_ragged_multi_cta_size_matches_context_residual():
    """33^3 = 35,937 points: nine partial sums, the last of a ragged 3,073
    points, against the context's residual of the same step."""
    import torch

    lib = cc.load_library()
    n_side = 33
    case = cases.case_box(n_side, species=cases.synthetic_species(), seed=9)
    dims = (n_side,) * 3
    d = cc.Driver.from_case(case, "fp64")
    d.initialize_computation()
    last = _rho_vel_p_t(d.field[0].get_state()[0], dims)
    d.simulate(1, residual=True)
    expected = d.residual()
    cur = _rho_vel_p_t(d.field[0].get_state()[0], dims)
    d.close()
    assert cur.shape[1] == 35937
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    got = _call(lib, torch.from_numpy(cur).cuda(), torch.from_numpy(last).cuda(), cur.shape[1], out)
    np.testing.assert_allclose(got, expected, rtol=RTOL)


def _reference_rms(cur, last):
    d = cur - last
    return np.sqrt((d * d).sum(axis=1) / cur.shape[1])


def test_noalloc_grow_then_shrink_and_allocates_nothing():
    """A call over 70,000 points (18 partials, ragged tail) and then one over
    5,000 (2 partials): the second finds the first's partial sums in the
    shared scratch and must read only its own.  A warm call changes neither
    torch's allocation counters nor the device's free memory."""
    import torch

    lib = cc.load_library()
    rng = np.random.default_rng(3)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    bufs = {}
    for n in (70000, 5000):
        cur = rng.uniform(0.5, 2.0, (4, n))
        last = cur + rng.normal(0.0, 1e-3, (4, n))
        bufs[n] = (torch.from_numpy(cur).cuda(), torch.from_numpy(last).cuda(), cur, last)
    for n in (70000, 5000, 70000):
        cur_d, last_d, cur, last = bufs[n]
        got = _call(lib, cur_d, last_d, n, out)
        np.testing.assert_allclose(got, _reference_rms(cur, last), rtol=RTOL)
    # warm call: nothing allocated on the device
    cur_d, last_d, cur, last = bufs[5000]
    torch.cuda.synchronize()
    alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    free0, _ = torch.cuda.mem_get_info()
    got = _call(lib, cur_d, last_d, 5000, out)
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == reserved0
    assert free1 == free0
    np.testing.assert_allclose(got, _reference_rms(cur, last), rtol=RTOL)


def test_noalloc_near_maximum_size():
    """n = CC_NOALLOC_MAX_POINTS - 1,000 (2,048 partials, the last ragged):
    against a numpy FP64 reduction of the same arrays."""
    import torch

    lib = cc.load_library()
    n = 8388608 - 1000
    rng = np.random.default_rng(4)
    cur = rng.uniform(0.5, 2.0, (4, n))
    last = cur + rng.normal(0.0, 1e-3, (4, n))
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    got = _call(lib, torch.from_numpy(cur).cuda(), torch.from_numpy(last).cuda(), n, out)
    np.testing.assert_allclose(got, _reference_rms(cur, last), rtol=RTOL)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    lib = cc.load_library()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    rc = lib.cc_residual_rms_noalloc(p, p, 8388608 + 1, p, None)
    assert rc == -1
    assert b"8388608" in lib.cc_last_error()
