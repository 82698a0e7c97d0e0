"""Exact solution of the 1D Riemann problem for a calorically perfect gas
(the two-wave pressure-function method of Toro, Riemann Solvers and
Numerical Methods for Fluid Dynamics, ch. 4), used as a known answer for the
Sod shock tube."""
import math

import numpy as np


def _f(p, rho, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1) * rho)
        B = (g - 1) / (g + 1) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1 - 0.5 * (p - pk) / (B + p))
    r = p / pk  # rarefaction
    return 2 * ck / (g - 1) * (r ** ((g - 1) / (2 * g)) - 1), 1.0 / (rho * ck) * r ** (-(g + 1) / (2 * g))


def star_state(L, R, g):
    rl, ul, pl = L
    rr, ur, pr = R
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p_new = max(1e-8, p - dp)
        if abs(p_new - p) < 1e-14 * p:
            p = p_new
            break
        p = p_new
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur + fr - fl)
    return p, u


def sample(L, R, g, xi):
    """(rho, u, p) at the similarity coordinates xi = (x - x0)/t."""
    rl, ul, pl = L
    rr, ur, pr = R
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    ps, us = star_state(L, R, g)
    out = np.zeros((3, len(xi)))
    for n, s in enumerate(xi):
        if s <= us:  # left of contact
            if ps > pl:
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    out[:, n] = (rl, ul, pl)
                else:
                    r = rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    out[:, n] = (r, us, ps)
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    out[:, n] = (rl, ul, pl)
                elif s >= stl:
                    out[:, n] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    r = rl * (c / cl) ** (2 / (g - 1))
                    out[:, n] = (r, u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:  # right of contact
            if ps > pr:
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    out[:, n] = (rr, ur, pr)
                else:
                    r = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    out[:, n] = (r, us, ps)
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    out[:, n] = (rr, ur, pr)
                elif s <= str_:
                    out[:, n] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    r = rr * (c / cr) ** (2 / (g - 1))
                    out[:, n] = (r, u, pr * (c / cr) ** (2 * g / (g - 1)))
    return out
