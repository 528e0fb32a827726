"""Initial states of the benchmark workloads (synthetic, seeded).

All states are conserved SoA arrays in nest's extended layout: 1D
[var][n + 2h], 2D [var][nx + 4][ny + 4] with the y index fastest.  Ghost
cells are filled by the solver on upload.
"""
from __future__ import annotations

import numpy as np

GAMMA = 1.4


def sod_1d(n: int, h: int = 2, gamma: float = GAMMA, x_disc: float = 0.5) -> np.ndarray:
    """Sod shock tube on [0,1] (examples/benchmark/benchmark_euler1d.cpp:53-77):
    (1, 0, 1) for x < 0.5 else (0.125, 0, 0.1), cell centres (i - h + 0.5) dx."""
    dx = 1.0 / n
    i = np.arange(n + 2 * h)
    x = 0.0 + (i - h + 0.5) * dx
    left = x < x_disc
    rho = np.where(left, 1.0, 0.125)
    u = np.zeros_like(rho)
    p = np.where(left, 1.0, 0.1)
    U = np.empty((3, n + 2 * h))
    U[0] = rho
    U[1] = rho * u
    U[2] = p / (gamma - 1.0) + 0.5 * rho * u * u
    return U


def prim_to_cons_2d(rho, u, v, p, gamma: float = GAMMA) -> np.ndarray:
    """(rho, u, v, p) -> (rho, rho u, rho v, E) with E = p/(g-1) + ((0.5 rho) u) u + ((0.5 rho) v) v."""
    U = np.empty((4,) + np.shape(rho))
    U[0] = rho
    U[1] = rho * u
    U[2] = rho * v
    U[3] = p / (gamma - 1.0) + (0.5 * rho * u * u + 0.5 * rho * v * v)
    return U


def riemann_2d(nx: int, ny: int, gamma: float = GAMMA, rows: tuple[int, int] | None = None) -> np.ndarray:
    """Diagonal 2D Riemann problem on [0,1]^2: (1, 0, 0, 1) where x + y < 1 at
    cell centres, else (0.125, 0, 0, 0.1).  rows = (x0, n) returns only the
    extended rows of that x-slab ([4][n+4][ny+4])."""
    x0, n = rows if rows is not None else (0, nx)
    x = (np.arange(x0 - 2, x0 + n + 2) + 0.5) / nx
    y = (np.arange(-2, ny + 2) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    left = (X + Y) < 1.0
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros_like(rho)
    return prim_to_cons_2d(rho, z, z, p, gamma)


def kelvin_helmholtz(nx: int, ny: int, seed: int, gamma: float = GAMMA) -> np.ndarray:
    """Periodic Kelvin-Helmholtz layer on [0,1]^2: rho = 2, u = +0.5 where
    |y - 0.5| < 0.25, else rho = 1, u = -0.5; p = 2.5;
    v = 0.01 sin(4 pi x) + uniform noise of amplitude 1e-3 (numpy PCG64, `seed`)."""
    x = (np.arange(-2, nx + 2) + 0.5) / nx
    y = (np.arange(-2, ny + 2) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    band = np.abs(Y - 0.5) < 0.25
    rho = np.where(band, 2.0, 1.0)
    u = np.where(band, 0.5, -0.5)
    p = np.full_like(rho, 2.5)
    rng = np.random.default_rng(seed)
    v = 0.01 * np.sin(4.0 * np.pi * X) + rng.uniform(-1e-3, 1e-3, size=X.shape)
    return prim_to_cons_2d(rho, u, v, p, gamma)


def kh_sizes(count: int = 512, seed: int = 0, lo: int = 64, hi: int = 1024, step: int = 64):
    """Side lengths of the batched KH problems: nx, ny independent, uniform in
    {lo, lo+step, ..., hi} (numpy PCG64, `seed`)."""
    rng = np.random.default_rng(seed)
    choices = np.arange(lo, hi + 1, step)
    return rng.choice(choices, size=count), rng.choice(choices, size=count)


def fourier_fields_1d(n: int, seed: int, modes: int = 16):
    """Primitive fields of the 1D adjoint workload on [0,1) (periodic, n cells):
    f, g, h = sum_{k=1..modes} (a_k cos 2 pi k x + b_k sin 2 pi k x) with
    a, b ~ N(0, 1) (numpy PCG64, `seed`), scaled to rho = 1 + 0.5 f/max|f|,
    u = 0.3 g/max|g|, p = 1 + 0.5 h/max|h|."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    k = np.arange(1, modes + 1)[:, None]
    out = []
    for _ in range(3):
        a, b = rng.standard_normal((2, modes, 1))
        f = (a * np.cos(2 * np.pi * k * x) + b * np.sin(2 * np.pi * k * x)).sum(axis=0)
        out.append(f / np.abs(f).max())
    f, g, h = out
    return 1.0 + 0.5 * f, 0.3 * g, 1.0 + 0.5 * h


def fourier_fields_2d(nx: int, ny: int, seed: int, modes: int = 4, gamma: float = GAMMA) -> np.ndarray:
    """Smooth periodic conserved state [4][nx+4][ny+4] on [0,1)^2 (ghosts zero):
    rho, u, v, p each a random sum of modes (kx, ky) in [0, modes]^2 of
    a cos(2 pi (kx x + ky y) + phi), a ~ N(0, 1), phi ~ U(0, 2 pi) (numpy PCG64,
    `seed`), scaled to rho = 1 + 0.4 f, u = 0.3 g, v = 0.3 h, p = 1 + 0.4 q with
    max|f| = max|g| = max|h| = max|q| = 1.  No region is uniform, so no limiter
    slope sits at the minmod(0, 0) corner."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    out = []
    for _ in range(4):
        f = np.zeros((nx, ny))
        for kx in range(modes + 1):
            for ky in range(modes + 1):
                if kx == 0 and ky == 0:
                    continue
                a, phi = rng.standard_normal(), rng.uniform(0.0, 2.0 * np.pi)
                f += a * np.cos(2 * np.pi * (kx * X + ky * Y) + phi)
        out.append(f / np.abs(f).max())
    f, g, h, q = out
    U = np.zeros((4, nx + 4, ny + 4))
    U[:, 2:-2, 2:-2] = prim_to_cons_2d(1.0 + 0.4 * f, 0.3 * g, 0.3 * h, 1.0 + 0.4 * q, gamma)
    return U


def prim_to_cons_1d(rho, u, p, gamma: float = GAMMA, h: int = 2) -> np.ndarray:
    """(rho, u, p) interior fields -> conserved SoA [3][n + 2h] (ghosts zero;
    the solver fills them)."""
    n = len(rho)
    U = np.zeros((3, n + 2 * h))
    U[0, h:h + n] = rho
    U[1, h:h + n] = rho * u
    U[2, h:h + n] = p / (gamma - 1.0) + 0.5 * rho * u * u
    return U
