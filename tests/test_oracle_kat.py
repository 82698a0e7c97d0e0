"""Known-answer checks of the CPU oracle (the restatement of the reference's
thermo, transport, reconstruction, AUSM+ and Newton)."""
import math

import numpy as np
import pytest

from combustioncodegpu_b200 import cases
from oracle import oracle_py as op


def test_minmod_cases():
    # Limiter.cuh:13-16: 0.5 (sgn a + sgn b) min(|a|, |b|)
    assert op.kat_minmod(1.0, 2.0) == 1.0
    assert op.kat_minmod(-3.0, -0.5) == -0.5
    assert op.kat_minmod(1.0, -2.0) == 0.0
    assert op.kat_minmod(0.0, 5.0) == 0.0
    assert op.kat_minmod(0.0, 0.0) == 0.0


def test_nasa_h_derivative_is_cp(species):
    for T in (250.0, 600.0, 999.0, 1001.0, 2000.0, 3000.0):
        dT = 1e-3
        hp, _ = op.kat_h_cp(species, T + dT)
        hm, _ = op.kat_h_cp(species, T - dT)
        _, cp = op.kat_h_cp(species, T)
        np.testing.assert_allclose((hp - hm) / (2 * dT), cp, rtol=2e-6)


def test_nasa_below_t_low_is_linear(species):
    tl = species["t_low"][0]
    h0, cp0 = op.kat_h_cp(species, tl)
    h1, cp1 = op.kat_h_cp(species, tl - 50.0)
    np.testing.assert_allclose(cp1, cp0, rtol=0, atol=0)
    np.testing.assert_allclose(h1, h0 - 50.0 * cp0, rtol=1e-12)


def test_nasa_continuity_at_t_mid(species):
    tm = species["t_mid"][0]
    ha, cpa = op.kat_h_cp(species, tm * (1 - 1e-12))
    hb, cpb = op.kat_h_cp(species, tm)
    np.testing.assert_allclose(ha, hb, rtol=1e-6, atol=1.0)
    np.testing.assert_allclose(cpa, cpb, rtol=1e-7)


def test_newton_round_trip(species):
    rng = np.random.default_rng(5)
    ns = species["n_spec"]
    for _ in range(20):
        Y = rng.dirichlet(np.full(ns, 0.5))
        T = rng.uniform(300, 2500)
        rho = rng.uniform(0.1, 2.0)
        u, v, w = rng.normal(0, 50, 3)
        h, _ = op.kat_h_cp(species, T)
        R = cases.R_U * float((Y / species["mw"]).sum())
        e = float((h * Y).sum()) - R * T
        q5 = [rho, rho * u, rho * v, rho * w, rho * (e + 0.5 * (u * u + v * v + w * w))]
        t = op.kat_temperature(species, q5, Y, T * rng.uniform(0.9, 1.1))
        assert abs(t - T) / T < 1e-5


def test_wilke_single_species_gives_species_viscosity():
    sp = cases.synthetic_species()
    one = {k: (np.asarray(v)[:1] if k in ("mw", "t_low", "t_mid", "t_high", "LJ_potent_inv", "vis_coeff") else v)
           for k, v in sp.items()}
    one["n_spec"] = 1
    one["low_temp_coeff"] = sp["low_temp_coeff"][:1]
    one["high_temp_coeff"] = sp["high_temp_coeff"][:1]
    one["WjDivWi_to_One4th"] = sp["WjDivWi_to_One4th"][:1, :1]
    one["sqrt_WiDivWjPl1Mul8"] = sp["sqrt_WiDivWjPl1Mul8"][:1, :1]
    T = 800.0
    mu, lam, rd = op.kat_transport(one, T, np.array([1.0]))
    t_dl = T * one["LJ_potent_inv"][0]
    omega = 1.147 * t_dl ** -0.145 + (t_dl + 0.5) ** -2
    mu_k = one["vis_coeff"][0] * math.sqrt(T) / omega
    assert abs(mu - mu_k) / mu_k < 1e-14
    _, cp = op.kat_h_cp(one, T)
    lam_k = mu_k * (cp[0] + 1.25 * cases.R_U / one["mw"][0])
    assert abs(lam - lam_k) / lam_k < 1e-13
    # X = 1: constant Schmidt branch rho D = mu / Sc (Transport.cu:88-89)
    assert abs(rd[0] - mu / 0.9) / rd[0] < 1e-14


def _physical_flux(species, s, k):
    ns = 0 if species is None else species["n_spec"]
    rho, u, v, w, p = s[:5]
    Y = s[5:5 + ns]
    if ns:
        T = p / (rho * cases.R_U * (Y / species["mw"]).sum())
        h, _ = op.kat_h_cp(species, T)
        E = rho * ((h * Y).sum() + 0.5 * (u * u + v * v + w * w)) - p
    else:
        E = p / (cases.GAMMA_AIR - 1) + 0.5 * rho * (u * u + v * v + w * w)
    U = k[0] * u + k[1] * v + k[2] * w
    f = [rho * U, rho * u * U + p * k[0], rho * v * U + p * k[1], rho * w * U + p * k[2], (E + p) * U]
    return np.array(f + list(rho * Y * U))


@pytest.mark.parametrize("multispecies", [False, True])
@pytest.mark.parametrize("mach", [0.05, 0.7, 1.6, -0.4, -2.5])
def test_ausm_consistency(species, multispecies, mach):
    """AUSM+ with equal left and right states is the physical flux."""
    sp = species if multispecies else None
    ns = sp["n_spec"] if sp else 0
    Y = np.full(ns, 1.0 / ns) if ns else np.zeros(0)
    rho, p = 0.8, 9.0e4
    T = p / (rho * cases.R_U * ((Y / sp["mw"]).sum() if ns else 1.0 / cases.MW_AIR))
    if ns:
        h, cp = op.kat_h_cp(sp, T)
        cpm = (cp * Y).sum()
        R = cases.R_U * (Y / sp["mw"]).sum()
        c = math.sqrt(cpm / (cpm - R) * p / rho)
    else:
        c = math.sqrt(cases.GAMMA_AIR * p / rho)
    k = np.array([0.6, 0.0, 0.8]) * 1.3
    u = mach * c
    s = np.concatenate([[rho, u * 0.6, 0.0, u * 0.8, p], Y])
    fc = op.kat_face_inviscid(sp, np.stack([s, s, s, s]), k)
    np.testing.assert_allclose(fc, _physical_flux(sp, s, k), rtol=1e-11, atol=1e-9 * abs(p))


def test_muscl_exact_on_linear_data():
    """Linear primitive data: MUSCL face states equal the linear value at the
    face, so the flux equals the physical flux of that state."""
    k = np.array([1.0, 0.0, 0.0])
    base = np.array([1.0, 10.0, 0.0, 0.0, 1.0e5])
    slope = np.array([0.01, 0.5, 0.0, 0.0, 100.0])
    pv4 = np.stack([base + (t - 1.5) * slope for t in range(4)])
    fc = op.kat_face_inviscid(None, pv4, k)
    # the face state is `base`; AUSM+ of a subsonic state with L=R recovers F(base)
    np.testing.assert_allclose(fc, _physical_flux(None, base, k), rtol=1e-12)


def test_periodic_box_conserves(species):
    from oracle.oracle_py import Oracle
    c = cases.case_box(9, species=species, seed=21)
    o = Oracle(c)
    o.init()
    sl = (slice(None), slice(2, -3), slice(2, -3), slice(2, -3))  # unique points of the shared-layer box
    before = o.state(0)[2].reshape(14, 13, 13, 13)[sl].sum(axis=(1, 2, 3))
    o.rk3_step(2)
    after = o.state(0)[2].reshape(14, 13, 13, 13)[sl].sum(axis=(1, 2, 3))
    np.testing.assert_allclose(after, before, rtol=1e-13, atol=1e-13 * np.abs(before).max())


def test_renormalised_mass_fractions_sum_to_one(species):
    from oracle.oracle_py import Oracle
    c = cases.case_box(8, species=species, seed=22)
    o = Oracle(c)
    o.init()
    o.rk3_step(2, renorm_y=True)
    yk = o.state(0)[1]
    g = yk.reshape(species["n_spec"], 12, 12, 12)[:, 2:-2, 2:-2, 2:-2].sum(axis=0)
    np.testing.assert_allclose(g, 1.0, rtol=0, atol=1e-14)


def test_closure_mlp_oracle_gradient_by_finite_difference():
    """The oracle's backward pass (what the training kernels are tested against),
    without its BF16 rounding: central differences of the loss."""
    from oracle import closure_mlp as om

    rng = np.random.default_rng(4)
    n_in, H, n_out, B = 5, 7, 3, 9
    lay, n = om.layout(n_in, H, n_out)
    p = rng.standard_normal(n) * 0.5
    x, y = rng.standard_normal((B, n_in)), rng.standard_normal((B, n_out))
    scale = rng.uniform(0.5, 2.0, n_out)
    _, g = om.loss_and_grad(p, x, y, scale, n_in, H, n_out, quantized=False)
    for e in rng.choice(n, 25, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[e] += h
        pm[e] -= h
        fd = (om.loss_and_grad(pp, x, y, scale, n_in, H, n_out, quantized=False)[0]
              - om.loss_and_grad(pm, x, y, scale, n_in, H, n_out, quantized=False)[0]) / (2 * h)
        assert abs(fd - g[e]) <= 1e-6 * max(1.0, abs(g[e])), (e, fd, g[e])


def test_bf16_rounding_ties_to_even():
    from oracle import closure_mlp as om

    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 1.0 + 2 ** -9, 3.14159], dtype=np.float32)
    got = om.bf16(x)
    np.testing.assert_array_equal(got[:5], np.array([1.0, 1.0, 1.0 + 2 ** -6, -1.0, 1.0], dtype=np.float32))
    assert abs(got[5] - 3.140625) == 0.0
