"""Exact solution of the 1D Riemann problem for an ideal gas (test infrastructure only).

Restates the exact solver of E. F. Toro, "Riemann Solvers and Numerical Methods for
Fluid Dynamics" (3rd ed., 2009), chapter 4: the star-region pressure is the root of
f(p) = f_L(p) + f_R(p) + (u_R - u_L), with f_K the shock (Rankine-Hugoniot) or
rarefaction (isentropic) branch, found by Newton iteration from the two-rarefaction
guess; the solution at x/t is sampled wave by wave (section 4.5).

It is the accuracy oracle of the Sod shock-tube case, standing in for the reference's
caseUtils/compressible/sod/sodSolution.py:200 (solve); tests/golden/sod_exact.npz, made
by tests/golden/make_sod_exact.py from that module, pins the two against each other.
"""
from __future__ import annotations

import numpy as np


def _fk(p, rho, pk, ck, g):
    """f_K(p) and its derivative (Toro eqs. 4.6, 4.7, 4.37)."""
    if p > pk:
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        s = np.sqrt(A / (p + B))
        return (p - pk) * s, s * (1.0 - 0.5 * (p - pk) / (B + p))
    e = (g - 1.0) / (2.0 * g)
    r = (p / pk) ** e
    return 2.0 * ck / (g - 1.0) * (r - 1.0), 1.0 / (rho * ck) * (p / pk) ** (-(g + 1.0) / (2.0 * g))


def star_state(left, right, gamma=1.4, tol=1e-14, max_iter=100):
    """(p*, u*) for left/right states given as (rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    g = gamma
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    if 2.0 * (cl + cr) / (g - 1.0) <= ur - ul:
        raise ValueError("the initial states generate a vacuum")
    e = (g - 1.0) / (2.0 * g)
    p = ((cl + cr - 0.5 * (g - 1.0) * (ur - ul)) / (cl / pl ** e + cr / pr ** e)) ** (1.0 / e)   # two-rarefaction guess
    p = max(p, tol)
    for _ in range(max_iter):
        fl, dl = _fk(p, rl, pl, cl, g)
        fr, dr = _fk(p, rr, pr, cr, g)
        pn = p - (fl + fr + ur - ul) / (dl + dr)
        pn = max(pn, tol)
        if abs(pn - p) <= tol * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _fk(p, rl, pl, cl, g)
    fr, _ = _fk(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(x, t, left, right, x0=0.0, gamma=1.4):
    """(rho, u, p) at positions x and time t > 0 for the discontinuity at x0."""
    rl, ul, pl = left
    rr, ur, pr = right
    g = gamma
    ps, us = star_state(left, right, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    S = (np.asarray(x, np.float64) - x0) / t
    rho = np.empty_like(S); u = np.empty_like(S); p = np.empty_like(S)
    gm = (g - 1.0) / (g + 1.0)
    for k, s in enumerate(S):
        if s <= us:                                   # left of the contact
            if ps > pl:                               # left shock
                SL = ul - cl * np.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                if s <= SL:
                    rho[k], u[k], p[k] = rl, ul, pl
                else:
                    rho[k], u[k], p[k] = rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps
            else:                                     # left rarefaction
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                shl, stl = ul - cl, us - csl
                if s <= shl:
                    rho[k], u[k], p[k] = rl, ul, pl
                elif s > stl:
                    rho[k], u[k], p[k] = rl * (ps / pl) ** (1.0 / g), us, ps
                else:
                    c = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * (ul - s))
                    rho[k] = rl * (c / cl) ** (2.0 / (g - 1.0))
                    u[k] = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + s)
                    p[k] = pl * (c / cl) ** (2.0 * g / (g - 1.0))
        else:                                         # right of the contact
            if ps > pr:                               # right shock
                SR = ur + cr * np.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                if s >= SR:
                    rho[k], u[k], p[k] = rr, ur, pr
                else:
                    rho[k], u[k], p[k] = rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps
            else:                                     # right rarefaction
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                shr, str_ = ur + cr, us + csr
                if s >= shr:
                    rho[k], u[k], p[k] = rr, ur, pr
                elif s < str_:
                    rho[k], u[k], p[k] = rr * (ps / pr) ** (1.0 / g), us, ps
                else:
                    c = 2.0 / (g + 1.0) * (cr - (g - 1.0) / 2.0 * (ur - s))
                    rho[k] = rr * (c / cr) ** (2.0 / (g - 1.0))
                    u[k] = 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + s)
                    p[k] = pr * (c / cr) ** (2.0 * g / (g - 1.0))
    return rho, u, p


def wave_positions(t, left, right, x0=0.0, gamma=1.4):
    """Head and tail of the left rarefaction, contact and right shock (Sod's wave pattern)."""
    rl, ul, pl = left
    rr, ur, pr = right
    g = gamma
    ps, us = star_state(left, right, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
    SR = ur + cr * np.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
    return dict(head=x0 + (ul - cl) * t, tail=x0 + (us - csl) * t, contact=x0 + us * t, shock=x0 + SR * t)
