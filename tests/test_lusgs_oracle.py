"""The LU-SGS steady step of the CPU oracle (the implicit scheme the
reference declares as temporal_scheme 1, TemporalScheme.cuh:19-21 and
Driver.cu:318-321, without a body): its Jacobian-vector product against a
finite difference of the mixture's flux, its small-CFL limit (the explicit
step of the reference's loop) and its convergence on a steady channel."""
import copy

import numpy as np

from combustioncodegpu_b200 import cases
from oracle import oracle_py as op

R_U = 8314.462618


def _temperature(species, e, Y, t0=1000.0):
    """T of sum Y_k h_k(T) - R T = e, Newton to machine precision."""
    mw = np.asarray(species["mw"])
    R = R_U * float((Y / mw).sum())
    t = t0
    for _ in range(60):
        h, cp = op.kat_h_cp(species, t)
        f = float((Y * h).sum()) - R * t - e
        t_new = t - f / (float((Y * cp).sum()) - R)
        if abs(t_new - t) < 1e-13 * t:
            return t_new
        t = t_new
    return t


def _flux(species, Q, k):
    """k . F(Q) of the thermally perfect mixture (p = rho R T)."""
    rho = Q[0]
    u = Q[1:4] / rho
    Y = Q[5:] / rho
    e = Q[4] / rho - 0.5 * float(u @ u)
    t = _temperature(species, e, Y)
    p = rho * R_U * float((Y / np.asarray(species["mw"])).sum()) * t
    U = float(k @ u)
    return np.concatenate([[rho * U], Q[1:4] * U + k * p, [(Q[4] + p) * U], Q[5:] * U])


def test_jacobian_vector_product_matches_finite_difference(species):
    rng = np.random.default_rng(5)
    mw = np.asarray(species["mw"])
    for _ in range(4):
        rho, t = rng.uniform(0.3, 1.5), rng.uniform(400.0, 2200.0)
        u = rng.uniform(-80, 80, 3)
        Y = rng.dirichlet(np.ones(species["n_spec"]))
        h, cp = op.kat_h_cp(species, t)
        R = R_U * float((Y / mw).sum())
        e = float((Y * h).sum()) - R * t
        Q = np.concatenate([[rho], rho * u, [rho * (e + 0.5 * float(u @ u))], rho * Y])
        p = rho * R * t
        cp_mix = float((Y * cp).sum())
        gam = cp_mix / (cp_mix - R)
        psi = gam * (R_U / mw) * t - (gam - 1.0) * h
        k = rng.uniform(-1, 1, 3)
        dQ = rng.standard_normal(Q.size) * np.abs(Q).clip(1e-3) * 1e-2
        dF = op.kat_lusgs_jac_vec(Q, p, gam, psi, k, dQ)
        eps = 1e-4
        fd = (_flux(species, Q + eps * dQ, k) - _flux(species, Q - eps * dQ, k)) / (2 * eps)
        scale = np.abs(fd).max()
        np.testing.assert_allclose(dF, fd, rtol=0, atol=1e-6 * scale)


def test_jacobian_vector_product_air_model():
    """Calorically perfect air: dp = (gamma - 1)(dE - u.dm + |u|^2/2 drho), no species terms."""
    rho, u, p, gam = 1.2, np.array([30.0, -5.0, 2.0]), 1.0e5, 1.4
    E = p / (gam - 1) + 0.5 * rho * float(u @ u)
    Q = np.array([rho, *(rho * u), E])
    k = np.array([0.3, 0.9, -0.2])

    def flux(Q):
        r, m, E = Q[0], Q[1:4], Q[4]
        p = (gam - 1) * (E - 0.5 * float(m @ m) / r)
        U = float(k @ m) / r
        return np.concatenate([[r * U], m * U + k * p, [(E + p) * U]])

    dQ = np.array([0.01, 0.2, -0.3, 0.05, 800.0])
    dF = op.kat_lusgs_jac_vec(Q, p, gam, [], k, dQ)
    eps = 1e-5
    fd = (flux(Q + eps * dQ) - flux(Q - eps * dQ)) / (2 * eps)
    np.testing.assert_allclose(dF, fd, rtol=1e-7, atol=1e-9 * np.abs(fd).max())


def _with_cfl(case, cfl):
    c = copy.deepcopy(case)
    c["params"]["cfl"] = cfl
    return c


def test_small_cfl_limit_is_the_explicit_step(species):
    """As dt -> 0 the LU-SGS update tends to the explicit dq dt / J: the
    relative difference of the conserved change is O(CFL)."""
    base = cases.case_box(10, species=species, seed=8)
    dQ = []
    for scheme in ("steady", "lusgs"):
        o = op.Oracle(_with_cfl(base, 1e-4))
        o.init()
        q0 = o.state(0)[2].copy()
        getattr(o, scheme + "_step")(1)
        dQ.append(o.state(0)[2] - q0)
        o.close()
    rel = np.abs(dQ[1] - dQ[0]).max(axis=1) / np.abs(dQ[0]).max(axis=1)
    assert rel.max() < 1e-3, rel
    assert rel.max() > 0


def _interior_rhs(o, case):
    tot = 0.0
    for b, blk in enumerate(case["blocks"]):
        mx, my, mz = blk["dims"]
        d = o.dq(b).reshape(-1, mz, my, mx)[0, 1:-1, 1:-1, 1:-1]
        tot += float((d * d).sum())
    return np.sqrt(tot)


def test_lusgs_converges_faster_than_explicit(species):
    """Viscous channel (inflow, outflow, isothermal walls): after 1000 steps
    the interior continuity residual of LU-SGS at CFL 5 is well below that
    of the reference's explicit loop at CFL 0.5."""
    base = cases.case_channel((11, 8, 6), species=species)
    out = {}
    for scheme, cfl in (("steady", 0.5), ("lusgs", 5.0)):
        case = _with_cfl(base, cfl)
        o = op.Oracle(case)
        o.init()
        r0 = _interior_rhs(o, case)
        getattr(o, scheme + "_step")(1000)
        bv = o.state(0)[0]
        assert np.isfinite(bv).all() and o.newton_failures() == 0
        out[scheme] = _interior_rhs(o, case) / r0
        o.close()
    assert out["lusgs"] < 0.5 * out["steady"], out
