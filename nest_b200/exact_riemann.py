"""Exact solution of the 1D Riemann problem for a gamma-law gas.

Used to report L1(rho) errors of the solver against the analytic Sod solution
(1D, and along the normal s = (x + y - 1)/sqrt(2) of the diagonal 2D problem).
nest has no exact solver; this follows the published method of
E. F. Toro, "Riemann Solvers and Numerical Methods for Fluid Dynamics",
3rd ed., Springer 2009, chapter 4: pressure functions f_K(p) for shocks
(Rankine-Hugoniot) and rarefactions (isentropic), Newton iteration for the
star pressure p* from the two-rarefaction guess, then sampling of the wave
pattern at x/t.  Vectorised over sample points with numpy (FP64).
"""
from __future__ import annotations

import math

import numpy as np


def _f_and_df(p, rho, pk, ck, g):
    """Toro (4.6)-(4.7): pressure function of one side and its derivative."""
    if p > pk:  # shock
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + B))
    r = p / pk  # rarefaction
    f = 2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rho * ck) * r ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g=1.4, tol=1e-14, itmax=100):
    """Star-region pressure and velocity (Toro section 4.3.1)."""
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    du = ur - ul
    if 2.0 * (cl + cr) / (g - 1.0) <= du:
        raise ValueError("initial data generate vacuum")
    z = (g - 1.0) / (2.0 * g)
    p = ((cl + cr - 0.5 * (g - 1.0) * du) / (cl / pl ** z + cr / pr ** z)) ** (1.0 / z)  # two-rarefaction guess
    p = max(p, tol)
    for _ in range(itmax):
        fl, dfl = _f_and_df(p, rl, pl, cl, g)
        fr, dfr = _f_and_df(p, rr, pr, cr, g)
        pn = max(p - (fl + fr + du) / (dfl + dfr), tol)
        if abs(pn - p) / (0.5 * (pn + p)) < tol:
            p = pn
            break
        p = pn
    fl, _ = _f_and_df(p, rl, pl, cl, g)
    fr, _ = _f_and_df(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(xi, rl, ul, pl, rr, ur, pr, g=1.4):
    """(rho, u, p) of the exact solution at similarity coordinates xi = x/t
    (Toro section 4.5, figure 4.14)."""
    xi = np.asarray(xi, dtype=np.float64)
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    gm, gp = g - 1.0, g + 1.0
    rho = np.empty_like(xi)
    u = np.empty_like(xi)
    p = np.empty_like(xi)
    left = xi <= us
    # ---- left of the contact
    if ps > pl:  # left shock
        rls = rl * ((ps / pl + gm / gp) / (gm / gp * ps / pl + 1.0))
        sl = ul - cl * math.sqrt(gp / (2 * g) * ps / pl + gm / (2 * g))
        m = left & (xi < sl)
        rho[m], u[m], p[m] = rl, ul, pl
        m = left & (xi >= sl)
        rho[m], u[m], p[m] = rls, us, ps
    else:  # left rarefaction
        rls = rl * (ps / pl) ** (1.0 / g)
        cls = cl * (ps / pl) ** (gm / (2 * g))
        shl, stl = ul - cl, us - cls
        m = left & (xi < shl)
        rho[m], u[m], p[m] = rl, ul, pl
        m = left & (xi >= shl) & (xi < stl)
        c = 2.0 / gp * (cl + gm / 2.0 * (ul - xi[m]))
        uu = 2.0 / gp * (cl + gm / 2.0 * ul + xi[m])
        rho[m] = rl * (c / cl) ** (2.0 / gm)
        u[m] = uu
        p[m] = pl * (c / cl) ** (2.0 * g / gm)
        m = left & (xi >= stl)
        rho[m], u[m], p[m] = rls, us, ps
    # ---- right of the contact
    right = ~left
    if ps > pr:  # right shock
        rrs = rr * ((ps / pr + gm / gp) / (gm / gp * ps / pr + 1.0))
        sr = ur + cr * math.sqrt(gp / (2 * g) * ps / pr + gm / (2 * g))
        m = right & (xi > sr)
        rho[m], u[m], p[m] = rr, ur, pr
        m = right & (xi <= sr)
        rho[m], u[m], p[m] = rrs, us, ps
    else:  # right rarefaction
        rrs = rr * (ps / pr) ** (1.0 / g)
        crs = cr * (ps / pr) ** (gm / (2 * g))
        shr, str_ = ur + cr, us + crs
        m = right & (xi > shr)
        rho[m], u[m], p[m] = rr, ur, pr
        m = right & (xi <= shr) & (xi > str_)
        c = 2.0 / gp * (cr - gm / 2.0 * (ur - xi[m]))
        rho[m] = rr * (c / cr) ** (2.0 / gm)
        u[m] = 2.0 / gp * (-cr + gm / 2.0 * ur + xi[m])
        p[m] = pr * (c / cr) ** (2.0 * g / gm)
        m = right & (xi <= str_)
        rho[m], u[m], p[m] = rrs, us, ps
    return rho, u, p


SOD = (1.0, 0.0, 1.0, 0.125, 0.0, 0.1)


def sod_density(x, t, x0=0.5, g=1.4):
    """Exact Sod density at positions x and time t > 0."""
    rho, _, _ = sample((np.asarray(x) - x0) / t, *SOD, g=g)
    return rho


def l1_rho_1d(rho_num, t, g=1.4):
    """L1 error (mean absolute difference, i.e. the integral over [0,1]) of a
    1D Sod density on N cell centres against the exact solution at the
    centres."""
    n = len(rho_num)
    x = (np.arange(n) + 0.5) / n
    return float(np.mean(np.abs(rho_num - sod_density(x, t, g=g))))


def l1_rho_diagonal(rho_num, t, g=1.4, margin=0.0):
    """L1 error of the diagonal 2D Riemann problem (discontinuity x + y = 1)
    against the 1D exact solution along s = (x + y - 1)/sqrt(2).  `margin`
    excludes cells within that distance of the domain boundary (where the
    outflow boundary and the corners perturb the planar solution)."""
    nx, ny = rho_num.shape
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    s = (X + Y - 1.0) / math.sqrt(2.0)
    ex = sod_density(s.ravel(), t, x0=0.0, g=g).reshape(nx, ny)
    m = (X > margin) & (X < 1 - margin) & (Y > margin) & (Y < 1 - margin)
    return float(np.abs(rho_num - ex)[m].mean())
