"""Tangent-linear restatement of the 1D stage -- TEST INFRASTRUCTURE ONLY.

Forward-mode differentiation of the oracle's 1D periodic Heun step
(oracle/euler_oracle.c: orc1d_stage / orc1d_rk2_step, which restate
examples/benchmark/benchmark_euler1d.cpp:113-209) with dual numbers.  Every
branch (minmod, HLLE regime, Davis min/max, p >= 0 clamp) is taken on the
value exactly as the forward takes it, so the result is the exact directional
derivative of the discrete map along the branches of the base point -- the
quantity a discrete adjoint must reproduce, free of the kink crossings that
limit finite differences.  Pure Python: small sizes only."""
from __future__ import annotations

import math


class D:
    __slots__ = ("v", "d")

    def __init__(self, v, d=0.0):
        self.v, self.d = float(v), float(d)

    def __add__(s, o):
        o = o if isinstance(o, D) else D(o)
        return D(s.v + o.v, s.d + o.d)
    __radd__ = __add__

    def __sub__(s, o):
        o = o if isinstance(o, D) else D(o)
        return D(s.v - o.v, s.d - o.d)

    def __rsub__(s, o):
        return D(o) - s

    def __mul__(s, o):
        o = o if isinstance(o, D) else D(o)
        return D(s.v * o.v, s.d * o.v + s.v * o.d)
    __rmul__ = __mul__

    def __truediv__(s, o):
        o = o if isinstance(o, D) else D(o)
        return D(s.v / o.v, (s.d * o.v - s.v * o.d) / (o.v * o.v))

    def __neg__(s):
        return D(-s.v, -s.d)


def dsqrt(x):
    r = math.sqrt(x.v)
    return D(r, x.d / (2.0 * r) if r > 0 else 0.0)


def dabs(x):
    return x if x.v >= 0 else -x


def smin(a, b):  # std::min
    return b if b.v < a.v else a


def smax(a, b):  # std::max
    return b if a.v < b.v else a


def minmod(a, b):  # euler1d.hpp:112-115
    if a.v * b.v <= 0.0:
        return D(0.0)
    return a if abs(a.v) < abs(b.v) else b


def pressure(g, r, m, e):  # euler1d.hpp:31-44
    u = m / r
    p = (g - 1.0) * (e - 0.5 * r * u * u)
    return D(0.0) if p.v < 0.0 else p


def hlle(g, WL, WR):  # euler1d.hpp:178-242
    rL, uL, pL = WL
    rR, uR, pR = WR
    cL, cR = dsqrt(g * pL / rL), dsqrt(g * pR / rR)
    EL = pL / (g - 1.0) + 0.5 * rL * uL * uL
    ER = pR / (g - 1.0) + 0.5 * rR * uR * uR
    SL = smin(uL - cL, uR - cR)
    SR = smax(uL + cL, uR + cR)
    FL = [rL * uL, rL * uL * uL + pL, (EL + pL) * uL]
    FR = [rR * uR, rR * uR * uR + pR, (ER + pR) * uR]
    UL = [rL, rL * uL, EL]
    UR = [rR, rR * uR, ER]
    if SL.v >= 0.0:
        return FL
    if SR.v <= 0.0:
        return FR
    return [(SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) / (SR - SL) for k in range(3)]


def stage(g, U, lam):
    """One forward-Euler stage on a periodic list of cells U[i] = [rho, m, E] (duals)."""
    n = len(U)
    W = []
    for r, m, e in U:
        W.append([r, m / r, pressure(g, r, m, e)])
    S = []
    for i in range(n):
        S.append([minmod(W[i][k] - W[i - 1][k], W[(i + 1) % n][k] - W[i][k]) for k in range(3)])
    F = []  # F[i] = flux through the left face of cell i
    for i in range(n):
        a = i - 1
        L = [W[a][k] + 0.5 * S[a][k] for k in range(3)]
        R = [W[i][k] - 0.5 * S[i][k] for k in range(3)]
        F.append(hlle(g, L, R))
    return [[U[i][k] - lam * (F[(i + 1) % n][k] - F[i][k]) for k in range(3)] for i in range(n)]


def heun(g, U, lam):
    U1 = stage(g, U, lam)
    U2 = stage(g, U1, lam)
    return [[0.5 * (U[i][k] + U2[i][k]) for k in range(3)] for i in range(len(U))]


def tangent_rollout(U0, dU0, dts, dx, gamma=1.4):
    """U0, dU0: arrays [3][n] (interior, periodic).  Returns (U_T, dU_T) as
    [3][n] nested lists of floats."""
    n = len(U0[0])
    U = [[D(U0[k][i], dU0[k][i]) for k in range(3)] for i in range(n)]
    for dt in dts:
        U = heun(gamma, U, dt / dx)
    return ([[U[i][k].v for i in range(n)] for k in range(3)], [[U[i][k].d for i in range(n)] for k in range(3)])


# ---------------------------------------------------------------------------
# 2D unsplit stage (oracle/euler_oracle.c: orc2d_stage / orc_hlle2d), periodic
# ---------------------------------------------------------------------------

def ke2(r, u, v):
    return 0.5 * r * u * u + 0.5 * r * v * v


def prim2(g, U):
    r, mu, mv, E = U
    u, v = mu / r, mv / r
    p = (g - 1.0) * (E - ke2(r, u, v))
    return [r, u, v, D(0.0) if p.v < 0.0 else p]


def hlle2(g, WL, WR):  # (rho, un, ut, p) -> (rho un, rho un un + p, rho un ut, (E + p) un)
    rL, nL, tL, pL = WL
    rR, nR, tR, pR = WR
    cL, cR = dsqrt(g * pL / rL), dsqrt(g * pR / rR)
    EL = pL / (g - 1.0) + ke2(rL, nL, tL)
    ER = pR / (g - 1.0) + ke2(rR, nR, tR)
    SL = smin(nL - cL, nR - cR)
    SR = smax(nL + cL, nR + cR)
    FL = [rL * nL, rL * nL * nL + pL, rL * nL * tL, (EL + pL) * nL]
    FR = [rR * nR, rR * nR * nR + pR, rR * nR * tR, (ER + pR) * nR]
    UL = [rL, rL * nL, rL * tL, EL]
    UR = [rR, rR * nR, rR * tR, ER]
    if SL.v >= 0.0:
        return FL
    if SR.v <= 0.0:
        return FR
    return [(SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) / (SR - SL) for k in range(4)]


def stage2d(g, U, lx, ly):
    """U[i][j] = [rho, mu, mv, E] duals on an nx x ny periodic grid."""
    nx, ny = len(U), len(U[0])
    W = [[prim2(g, U[i][j]) for j in range(ny)] for i in range(nx)]

    def face(a2, a, b, b2, xdir):
        perm = (lambda w: [w[0], w[1], w[2], w[3]]) if xdir else (lambda w: [w[0], w[2], w[1], w[3]])
        A2, A, B, B2 = perm(a2), perm(a), perm(b), perm(b2)
        L = [A[k] + 0.5 * minmod(A[k] - A2[k], B[k] - A[k]) for k in range(4)]
        R = [B[k] - 0.5 * minmod(B[k] - A[k], B2[k] - B[k]) for k in range(4)]
        f = hlle2(g, L, R)
        return [f[0], f[1], f[2], f[3]] if xdir else [f[0], f[2], f[1], f[3]]

    out = []
    for i in range(nx):
        row = []
        for j in range(ny):
            w = lambda a, b: W[a % nx][b % ny]
            fxm = face(w(i - 2, j), w(i - 1, j), w(i, j), w(i + 1, j), True)
            fxp = face(w(i - 1, j), w(i, j), w(i + 1, j), w(i + 2, j), True)
            fym = face(w(i, j - 2), w(i, j - 1), w(i, j), w(i, j + 1), False)
            fyp = face(w(i, j - 1), w(i, j), w(i, j + 1), w(i, j + 2), False)
            row.append([U[i][j][k] - (lx * (fxp[k] - fxm[k]) + ly * (fyp[k] - fym[k])) for k in range(4)])
        out.append(row)
    return out


def tangent_rollout_2d(U0, dU0, dts, dx, dy, gamma=1.4):
    """U0, dU0: arrays [4][nx][ny] (interior, periodic).  Heun steps with the
    given dts; returns (U_T, dU_T) as numpy-convertible nested lists [4][nx][ny]."""
    nx, ny = len(U0[0]), len(U0[0][0])
    U = [[[D(U0[k][i][j], dU0[k][i][j]) for k in range(4)] for j in range(ny)] for i in range(nx)]
    for dt in dts:
        lx, ly = dt / dx, dt / dy
        U1 = stage2d(gamma, U, lx, ly)
        U2 = stage2d(gamma, U1, lx, ly)
        U = [[[0.5 * (U[i][j][k] + U2[i][j][k]) for k in range(4)] for j in range(ny)] for i in range(nx)]
    val = [[[U[i][j][k].v for j in range(ny)] for i in range(nx)] for k in range(4)]
    der = [[[U[i][j][k].d for j in range(ny)] for i in range(nx)] for k in range(4)]
    return val, der
