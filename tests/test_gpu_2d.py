"""2D unsplit scheme on the GPU.

FP64 plain form: bit for bit against the oracle on small grids (odd sizes,
all boundary combinations, several launch shapes) and through size-independent
properties at the full 4096^2 workload (mirror symmetry of the diagonal
Riemann problem; y-uniform runs equal to the 1D solver).  FP32 form: L1(rho)
against FP64, totals in FP64, positivity repair."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import BC_OUTFLOW, BC_PERIODIC
from nest_b200.problems import kelvin_helmholtz, riemann_2d, sod_1d

pytestmark = pytest.mark.gpu
G = 1.4


def gpu_run(gpu, U, nx, ny, bc, nsteps=0, t_final=0.0, prec=None, tiling=None, flags=0, cfl=0.4):
    s = gpu.Solver(2, nx, ny, bc=bc, precision=gpu.F64 if prec is None else prec, flags=flags)
    if tiling:
        s.set_tiling(*tiling)
    s.upload(U)
    if t_final > 0:
        s.run_to(t_final, cfl)
    else:
        s.step(nsteps, cfl)
    return s, s.download()


@pytest.mark.parametrize("nx,ny,bc,kind", [
    (64, 48, (BC_OUTFLOW, BC_OUTFLOW), "riemann"),
    (40, 72, (BC_PERIODIC, BC_PERIODIC), "kh"),
    (33, 37, (BC_PERIODIC, BC_OUTFLOW), "kh"),
    (29, 31, (BC_OUTFLOW, BC_PERIODIC), "riemann"),
])
@pytest.mark.parametrize("tiling", [None, (8, 1), (16, 2), (64, 8)])
def test_fp64_matches_oracle_bitwise(gpu, oracle, nx, ny, bc, kind, tiling):
    U = riemann_2d(nx, ny) if kind == "riemann" else kelvin_helmholtz(nx, ny, seed=nx)
    want = np.ascontiguousarray(U.copy())
    _, t, _ = oracle.run2d(want, nx, ny, 2, 1 / nx, 1 / ny, G, 0.4, nsteps=37, bc=bc)
    s, got = gpu_run(gpu, U, nx, ny, bc, nsteps=37, tiling=tiling)
    I = (slice(None), slice(2, -2), slice(2, -2))
    assert np.array_equal(got[I], want[I])
    assert s.time() == (t, 37)


def test_fp64_run_to_t_final(gpu, oracle):
    nx = ny = 48
    U = riemann_2d(nx, ny)
    want = U.copy()
    steps, t, _ = oracle.run2d(want, nx, ny, 2, 1 / nx, 1 / ny, G, 0.4, t_final=0.05, bc=BC_OUTFLOW)
    s, got = gpu_run(gpu, U, nx, ny, (BC_OUTFLOW, BC_OUTFLOW), t_final=0.05)
    assert s.time() == (t, steps)
    assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


def test_fp64_full_size_matches_oracle(gpu, oracle):
    """The benchmark workload itself (diagonal Riemann problem, 4096^2 as 16 x
    16 patches of 256^2, outflow, CFL 0.4, 200 RK2 steps) through
    nest_solver_step with the default launch shape: every cell of all four
    variables and the simulated time equal the oracle's bit for bit (the
    tolerance `north_star` allows is a relative 1e-12; the FP64 form has no
    FMA contraction, so it is exact).  The oracle runs on every host core."""
    import os
    n, steps = 4096, 200
    U = riemann_2d(n, n)
    s, got = gpu_run(gpu, U, n, n, (BC_OUTFLOW, BC_OUTFLOW), nsteps=steps)
    t_gpu, k = s.time()
    s.close()
    oracle.set_threads(len(os.sched_getaffinity(0)))
    want = np.ascontiguousarray(U)
    ksteps, t, _ = oracle.run2d(want, n, n, 2, 1 / n, 1 / n, G, 0.4, nsteps=steps, bc=BC_OUTFLOW)
    a, b = got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2]
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    assert rel.max() <= 1e-12, rel.max()
    assert np.array_equal(a, b)
    assert k == ksteps == steps and t_gpu == t


def test_fp64_full_size_mirror_symmetry(gpu):
    """Diagonal Riemann problem, 4096^2, 200 steps (the benchmark workload):
    the scheme is mirror symmetric about x = y, so rho(i,j) == rho(j,i) and
    (rho u)(i,j) == (rho v)(j,i) exactly."""
    n = 4096
    s, got = gpu_run(gpu, riemann_2d(n, n), n, n, (BC_OUTFLOW, BC_OUTFLOW), nsteps=200)
    I = got[:, 2:-2, 2:-2]
    assert np.array_equal(I[0], I[0].T)
    assert np.array_equal(I[1], I[2].T)
    assert np.array_equal(I[3], I[3].T)
    t, steps = s.time()
    assert steps == 200 and 0.01 < t < 0.03
    assert np.all(np.isfinite(I)) and I[0].min() > 0


def test_fp64_y_uniform_equals_1d_solver(gpu):
    """A y-uniform 2D run with the 1D solver's dt sequence reproduces the 1D
    GPU solver bit for bit (full length 4096)."""
    n, ny, steps = 4096, 8, 60
    s1 = gpu.Solver(1, n, bc=BC_OUTFLOW, flags=gpu.FLAG_NO_RESIDENT)
    s1.record_dts(steps)
    s1.upload(sod_1d(n))
    s1.step(steps, 0.4)
    dts = s1.recorded_dts(steps)
    want = s1.download()
    U0 = sod_1d(n)
    U2 = np.zeros((4, n + 4, ny + 4))
    U2[0], U2[1], U2[3] = U0[0][:, None], U0[1][:, None], U0[2][:, None]
    s2 = gpu.Solver(2, n, ny, dx=1.0 / n, dy=1.0 / ny, bc=BC_OUTFLOW)
    s2.freeze_dts(dts)
    s2.upload(U2)
    assert s2.run_to(10.0, 0.4) == steps
    got = s2.download()
    for j in range(2, ny + 2):
        assert np.array_equal(got[[0, 1, 3], 2:-2, j], want[:, 2:-2])


def test_fp32_close_to_fp64(gpu):
    nx = ny = 256
    U = riemann_2d(nx, ny)
    _, a64 = gpu_run(gpu, U, nx, ny, (BC_OUTFLOW, BC_OUTFLOW), nsteps=100)
    for flags in (0, gpu.FLAG_REPAIR):
        _, a32 = gpu_run(gpu, U.astype(np.float32), nx, ny, (BC_OUTFLOW, BC_OUTFLOW), nsteps=100,
                         prec=gpu.F32, flags=flags)
        r64 = a64[0, 2:-2, 2:-2]
        r32 = a32[0, 2:-2, 2:-2].astype(np.float64)
        l1 = np.abs(r32 - r64).mean()
        # FP32 rounding only: orders of magnitude below the scheme's truncation error
        assert l1 < 2e-6, l1


def test_fp32_totals_conserved_periodic(gpu, oracle):
    nx, ny = 200, 136
    U = kelvin_helmholtz(nx, ny, seed=11)
    oracle.fill_ghosts2d(U, nx, ny, 2, BC_PERIODIC)
    m0 = oracle.totals2d(U, nx, ny, 2, 1 / nx, 1 / ny)
    s, _ = gpu_run(gpu, U.astype(np.float32), nx, ny, (BC_PERIODIC, BC_PERIODIC), nsteps=64,
                   prec=gpu.F32, flags=gpu.FLAG_TOTALS | gpu.FLAG_REPAIR)
    tot = s.totals()
    got = s.download().astype(np.float64)
    direct = got[:, 2:-2, 2:-2].sum(axis=(1, 2)) / (nx * ny)
    assert np.allclose(tot, direct, rtol=1e-12, atol=1e-12)
    # mass and energy drift of the FP32 form stays at FP32 rounding level
    assert abs(tot[0] - m0[0]) < 1e-5 * m0[0]
    assert abs(tot[3] - m0[3]) < 1e-5 * m0[3]
    assert s.repairs() == 0


def test_fp32_repair_near_vacuum(gpu):
    """Two strong rarefactions (u = -/+ 2 away from x = 0.5) drive the
    centre toward vacuum; with repair the FP32 run stays finite and positive."""
    nx, ny = 128, 16
    x = (np.arange(-2, nx + 2) + 0.5) / nx
    X = np.repeat(x[:, None], ny + 4, axis=1)
    rho = np.full_like(X, 1.0)
    u = np.where(X < 0.5, -2.0, 2.0)
    p = np.full_like(X, 0.4)
    from nest_b200.problems import prim_to_cons_2d
    U = prim_to_cons_2d(rho, u, 0 * u, p).astype(np.float32)
    s, got = gpu_run(gpu, U, nx, ny, (BC_OUTFLOW, BC_OUTFLOW), nsteps=150, prec=gpu.F32, flags=gpu.FLAG_REPAIR)
    I = got[:, 2:-2, 2:-2].astype(np.float64)
    assert np.all(np.isfinite(I)) and I[0].min() > 0
    pr = 0.4 * (I[3] - 0.5 * (I[1] ** 2 + I[2] ** 2) / I[0])
    assert pr.min() > -1e-6


@pytest.mark.parametrize("nx,ny,bc", [(40, 5, (BC_OUTFLOW, BC_OUTFLOW)), (33, 59, (BC_PERIODIC, BC_PERIODIC)),
                                      (31, 60, (BC_OUTFLOW, BC_PERIODIC)), (29, 61, (BC_PERIODIC, BC_OUTFLOW)),
                                      (64, 121, (BC_OUTFLOW, BC_OUTFLOW)), (17, 64, (BC_PERIODIC, BC_PERIODIC))])
def test_fp32_packed_matches_fp64_and_scalar(gpu, nx, ny, bc):
    """The packed FP32x2 kernel (two columns per lane) on ragged widths around
    its 60-column strip, every boundary combination: close to FP64 and to the
    scalar FP32 kernel at FP32 rounding level."""
    U = kelvin_helmholtz(nx, ny, seed=nx + ny) if bc[1] == BC_PERIODIC else riemann_2d(nx, ny)
    _, a64 = gpu_run(gpu, U, nx, ny, bc, nsteps=30)
    _, ax2 = gpu_run(gpu, U.astype(np.float32), nx, ny, bc, nsteps=30, prec=gpu.F32)
    _, asc = gpu_run(gpu, U.astype(np.float32), nx, ny, bc, nsteps=30, prec=gpu.F32, flags=gpu.FLAG_FP32_SCALAR)
    I = (slice(None), slice(2, -2), slice(2, -2))
    ref = a64[I]
    scale = np.abs(ref).max(axis=(1, 2), keepdims=True) + 1e-30
    for got in (ax2[I].astype(np.float64), asc[I].astype(np.float64)):
        assert np.all(np.isfinite(got))
        assert (np.abs(got - ref) / scale).max() < 2e-4
        assert (np.abs(got - ref) / scale).mean() < 2e-6
    # ghost ring written by the packed kernel matches the boundary rule
    G = ax2
    if bc[0] == BC_OUTFLOW:
        assert np.array_equal(G[:, 0, 2:-2], G[:, 2, 2:-2]) and np.array_equal(G[:, -1, 2:-2], G[:, -3, 2:-2])
    else:
        assert np.array_equal(G[:, 0, 2:-2], G[:, nx, 2:-2]) and np.array_equal(G[:, -1, 2:-2], G[:, 3, 2:-2])
    if bc[1] == BC_OUTFLOW:
        assert np.array_equal(G[:, 2:-2, 0], G[:, 2:-2, 2]) and np.array_equal(G[:, 2:-2, -1], G[:, 2:-2, -3])
    else:
        assert np.array_equal(G[:, 2:-2, 0], G[:, 2:-2, ny]) and np.array_equal(G[:, 2:-2, -1], G[:, 2:-2, 3])


def test_split_compat_matches_nest_sweeps(gpu, oracle, ref):
    """nest's own 2D scheme on the device (NEST_FLAG_SPLIT_COMPAT): the sod2d
    configuration (200 x 20, 2 x 2 periodic patches, CFL 0.3, t = 0.2) equals
    nest's x_sweep_t / y_sweep_t run on the CPU bit for bit."""
    from test_oracle import sod2d_reference_run
    want, t_ref, steps_ref = sod2d_reference_run(ref, oracle)
    nx, ny = 200, 20
    from nest_b200.problems import prim_to_cons_2d
    x = (np.arange(-2, nx + 2) + 0.5) / nx
    X = np.repeat(x[:, None], ny + 4, axis=1)
    left = X < 0.5
    z = np.zeros_like(X)
    U = prim_to_cons_2d(np.where(left, 1.0, 0.125), z, z, np.where(left, 1.0, 0.1))
    s = gpu.Solver(2, nx, ny, dx=1.0 / nx, dy=0.1 / ny, bc=BC_PERIODIC, precision=gpu.F64,
                   flags=gpu.FLAG_SPLIT_COMPAT)
    s.upload(U)
    steps = s.run_to(0.2, 0.3)
    got = s.download()
    assert steps == steps_ref and s.time()[0] == t_ref
    assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])
