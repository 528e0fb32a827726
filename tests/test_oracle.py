"""The CPU oracle is pinned to nest's own code and golden vectors (CPU only).

Known answers restate tests/test_euler.cpp:54-237; full-run fixtures come
from nest's own programs (tests/golden/make_golden.py)."""
from __future__ import annotations

import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.oracle import BC_OUTFLOW, BC_PERIODIC, sod_ic_1d

G = 1.4


def test_known_answers_test_euler(oracle):
    L = oracle.L
    # eos_pressure, eos_total_energy, eos_sound_speed: test_euler.cpp:54-87
    assert abs(L.orc_pressure(G, 1.0, 0.0, 2.5) - 1.0) < 1e-10
    assert abs(L.orc_total_energy(G, 1.0, 1.0, 1.0) - 3.0) < 1e-10
    assert abs(L.orc_sound_speed(G, 1.0, 1.0) - math.sqrt(1.4)) < 1e-10
    # minmod cases: test_euler.cpp:133-146
    for a, b, want in [(1, 2, 1), (2, 1, 1), (-1, -2, -1), (1, -1, 0), (-1, 1, 0), (0, 1, 0), (1, 0, 0)]:
        assert L.orc_minmod(a, b) == want
    # HLLE stationary / supersonic: test_euler.cpp:180-211
    F = oracle.hlle1d(G, [1, 0, 1], [1, 0, 1])
    assert abs(F[0]) < 1e-10 and abs(F[1] - 1.0) < 1e-10 and abs(F[2]) < 1e-10
    F = oracle.hlle1d(G, [1, 10, 1], [1, 10, 1])
    assert abs(F[0] - 10.0) < 1e-8 and abs(F[1] - 101.0) < 1e-8


def test_plm_known_answers(oracle):
    # plm_reconstruction_flat / _monotone: test_euler.cpp:148-174
    import ctypes as C
    dp = C.POINTER(C.c_double)
    m, z, p = (np.array(v, dtype=np.float64) for v in ([1, 0, 1], [2, 0, 1], [3, 0, 1]))
    WL, WR = np.zeros(3), np.zeros(3)
    oracle.L.orc_plm(m.ctypes.data_as(dp), z.ctypes.data_as(dp), p.ctypes.data_as(dp), 3, 0,
                     WL.ctypes.data_as(dp), WR.ctypes.data_as(dp))
    assert WL[0] == 1.5 and WR[0] == 2.5


def test_hlle_matches_reference_golden(oracle):
    ka = json.loads((GOLDEN / "known_answers.json").read_text())
    assert oracle.hlle1d(G, [1, 0, 1], [1, 0, 1]).tolist() == ka["hlle_stationary"]
    assert oracle.hlle1d(G, [1, 10, 1], [1, 10, 1]).tolist() == ka["hlle_supersonic"]
    for c in ka["hlle_random"]:
        assert oracle.hlle1d(G, c["WL"], c["WR"]).tolist() == c["F"]  # bit for bit
    assert oracle.L.orc_pressure(G, 1.0, 0.0, 2.5) == ka["eos_pressure_1_0_2.5"]
    assert oracle.L.orc_sound_speed(G, 1.0, 1.0) == ka["eos_sound_speed_1_1"]


def test_run_matches_reference_test_fixture(oracle):
    """nest's CPU-vs-GPU test configuration (tests/test_euler_cuda.cpp:27-43):
    periodic Sod, N=100, t=0.1, CFL 0.3 -- oracle equals nest bit for bit."""
    want = np.load(GOLDEN / "sod100_periodic.npy")
    U = sod_ic_1d(100)
    steps, t, _ = oracle.run1d(U, 100, 2, 0.01, G, 0.3, t_final=0.1, bc=BC_PERIODIC)
    assert steps == 70 and t == pytest.approx(0.1, abs=0)
    assert np.array_equal(U[:, 2:-2], want[:, 2:-2])


def test_numerics_match_reference_library(oracle, ref):
    rng = np.random.default_rng(3)
    for _ in range(500):
        WL = np.array([rng.uniform(0.01, 3), rng.normal(0, 3), rng.uniform(0.0, 3)])
        WR = np.array([rng.uniform(0.01, 3), rng.normal(0, 3), rng.uniform(0.0, 3)])
        assert np.array_equal(oracle.hlle1d(G, WL, WR), ref.hlle_flux(G, WL, WR))
        a, b = rng.normal(size=2) * 10.0 ** rng.integers(-200, 200, size=2)
        assert oracle.L.orc_minmod(a, b) == ref.L.ref_minmod(a, b)
        assert oracle.L.orc_mc(a, b) == ref.L.ref_mc(a, b)
        rho, mom, erg = rng.uniform(0.01, 3), rng.normal(), rng.uniform(-1, 3)
        assert oracle.L.orc_pressure(G, rho, mom, erg) == ref.L.ref_pressure(G, rho, mom, erg)


def test_benchmark_loop_matches_reference_run(oracle, ref):
    for n, t_final, cfl in [(64, 0.05, 0.4), (257, 0.03, 0.8), (100, 0.1, 0.3)]:
        want = ref.run_cpu_sod(n, t_final, cfl)
        U = sod_ic_1d(n)
        oracle.run1d(U, n, 2, 1.0 / n, G, cfl, t_final=t_final, bc=BC_PERIODIC)
        assert np.array_equal(U[:, 2:-2], want[:, 2:-2])


def test_patch_stage_matches_euler_rhs(oracle, ref):
    """One-sided patch-edge stencil of euler_rhs_t (euler1d.hpp:337-346, 366-374)."""
    rng = np.random.default_rng(5)
    n, h = 37, 2
    W = np.stack([rng.uniform(0.2, 2, n + 4), rng.normal(0, 0.5, n + 4), rng.uniform(0.2, 2, n + 4)])
    U = np.stack([W[0], W[0] * W[1], W[2] / 0.4 + 0.5 * W[0] * W[1] * W[1]])
    got = oracle.patch_stage1d(np.ascontiguousarray(U), n, h, 1.0 / n, 1e-3, G)
    want = ref.patch_stage(np.ascontiguousarray(U).ravel(), n, h, 1.0 / n, 1e-3, G).reshape(3, n + 4)
    assert np.array_equal(got[:, 2:-2], want[:, 2:-2])


def test_sod1d_example_golden(oracle):
    """sod1d (4 periodic patches, one-sided patch edges, SSPRK2 combine
    0.5 U0 + 0.5 U2; examples/sod1d/sod1d.cpp:219-302) restated on the oracle's
    patch stage reproduces nest's own output file."""
    want = np.load(GOLDEN / "sod1d_final.npy")
    n, npatch, h = 400, 4, 2
    m = n // npatch
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    rho = np.where(x < 0.5, 1.0, 0.125)
    p = np.where(x < 0.5, 1.0, 0.1)
    Ug = np.stack([rho, 0 * rho, p / 0.4])  # global interior state

    def patches_of(U):
        out = []
        for k in range(npatch):
            idx = np.arange(k * m - h, (k + 1) * m + h) % n  # periodic exchange
            out.append(np.ascontiguousarray(U[:, idx]))
        return out

    t, tf = 0.0, 0.2
    while t < tf:
        ms = 0.0
        for i in range(n):
            r, mo, e = Ug[:, i]
            u = mo / r
            pp = oracle.L.orc_pressure(G, r, mo, e)
            ms = max(ms, abs(u) + math.sqrt(G * pp / r))
        dt = min(0.4 * dx / ms, tf - t)
        U0 = Ug.copy()
        U1 = np.concatenate([oracle.patch_stage1d(P, m, h, dx, dt, G)[:, h:-h] for P in patches_of(Ug)], axis=1)
        U2 = np.concatenate([oracle.patch_stage1d(P, m, h, dx, dt, G)[:, h:-h] for P in patches_of(U1)], axis=1)
        Ug = 0.5 * U0 + 0.5 * U2
        t += dt
    u = Ug[1] / Ug[0]
    pr = np.array([oracle.L.orc_pressure(G, *Ug[:, i]) for i in range(n)])
    # the .dat file holds 11 significant digits
    assert np.allclose(Ug[0], want[:, 1], rtol=2e-10, atol=0)
    assert np.allclose(u, want[:, 2], rtol=2e-10, atol=1e-14)
    assert np.allclose(pr, want[:, 3], rtol=2e-10, atol=0)


def test_2d_reduces_to_1d_bitwise(oracle):
    from nest_b200.problems import sod_1d
    n, ny = 64, 6
    U1 = sod_1d(n)
    _, _, dts = oracle.run1d(U1, n, 2, 1 / n, G, 0.4, nsteps=30, bc=BC_OUTFLOW, record_dts=True)
    U0 = sod_1d(n)
    U2 = np.zeros((4, n + 4, ny + 4))
    U2[0], U2[1], U2[3] = U0[0][:, None], U0[1][:, None], U0[2][:, None]
    oracle.run2d(U2, n, ny, 2, 1 / n, 1 / ny, G, 0.4, nsteps=30, bc=BC_OUTFLOW, dts_in=dts)
    for j in range(2, ny + 2):
        assert np.array_equal(U2[[0, 1, 3], 2:-2, j], U1[:, 2:-2])
    assert np.all(U2[2, 2:-2, 2:-2] == 0)


def test_2d_mirror_symmetry(oracle):
    from nest_b200.problems import riemann_2d
    N = 40
    U = riemann_2d(N, N)
    oracle.run2d(U, N, N, 2, 1 / N, 1 / N, G, 0.4, nsteps=50, bc=BC_OUTFLOW)
    I = U[:, 2:-2, 2:-2]
    assert np.array_equal(I[0], I[0].T) and np.array_equal(I[1], I[2].T) and np.array_equal(I[3], I[3].T)


def test_2d_cfl_matches_reference_compute_dt_2d(oracle, ref):
    import ctypes as C
    from nest_b200.problems import kelvin_helmholtz
    nx, ny = 24, 20
    U = np.ascontiguousarray(kelvin_helmholtz(nx, ny, seed=3))
    sx, sy = oracle.max_speeds2d(U, nx, ny, 2, G)
    got = oracle.dt2d(sx, sy, 1 / nx, 1 / ny, 0.4)
    want = ref.L.ref_compute_dt_2d(U.ctypes.data_as(C.POINTER(C.c_double)), nx, ny, 2, 1 / nx, 1 / ny, 0.4, G)
    assert got == want


def test_2d_periodic_conserves_mass(oracle):
    from nest_b200.problems import kelvin_helmholtz
    nx, ny = 32, 32
    U = kelvin_helmholtz(nx, ny, seed=1)
    oracle.fill_ghosts2d(U, nx, ny, 2, BC_PERIODIC)
    m0 = oracle.totals2d(U, nx, ny, 2, 1 / nx, 1 / ny)
    oracle.run2d(U, nx, ny, 2, 1 / nx, 1 / ny, G, 0.4, nsteps=40, bc=BC_PERIODIC)
    m1 = oracle.totals2d(U, nx, ny, 2, 1 / nx, 1 / ny)
    assert abs(m1[0] - m0[0]) < 1e-13 * abs(m0[0])
    assert abs(m1[3] - m0[3]) < 1e-13 * abs(m0[3])


def sod2d_reference_run(ref, oracle, lim=0):
    """nest's sod2d (examples/sod2d/sod2d.cpp:239-366) on one periodic domain
    with nest's own x_sweep_t / y_sweep_t / compute_dt_2d from oracle/_ref
    (lim: 0 minmod as in sod2d, 1 MC, 2 none)."""
    import ctypes as C
    nx, ny, tf, cfl = 200, 20, 0.2, 0.3
    dx, dy = 1.0 / nx, 0.1 / ny
    from nest_b200.problems import prim_to_cons_2d
    x = (np.arange(-2, nx + 2) + 0.5) * dx
    X = np.repeat(x[:, None], ny + 4, axis=1)
    left = X < 0.5
    z = np.zeros_like(X)
    U = np.ascontiguousarray(prim_to_cons_2d(np.where(left, 1.0, 0.125), z, z, np.where(left, 1.0, 0.1)))
    dp = C.POINTER(C.c_double)
    t, steps = 0.0, 0
    while t < tf:
        dt = ref.L.ref_compute_dt_2d(U.ctypes.data_as(dp), nx, ny, 2, dx, dy, cfl, G)
        dt = min(dt, tf - t)
        for sweep, d in ((ref.L.ref_x_sweep, dx), (ref.L.ref_y_sweep, dy)):
            oracle.fill_ghosts2d(U, nx, ny, 2, BC_PERIODIC)
            out = np.empty_like(U)
            sweep(U.ctypes.data_as(dp), out.ctypes.data_as(dp), nx, ny, 2, d, dt, G, lim)
            U = out
        t += dt
        steps += 1
    return U, t, steps


def test_sod2d_example_golden(oracle, ref):
    """nest's split 2D sweeps on one periodic domain reproduce nest's own
    patch-based sod2d output file (11 digits) -- the reference for the
    device compatibility mode."""
    U, t, steps = sod2d_reference_run(ref, oracle)
    g = np.load(GOLDEN / "sod2d_final.npz")
    i = np.rint(g["x"] * 200 - 0.5).astype(int)
    j = np.rint(g["y"] * 200 - 0.5).astype(int)
    rho = U[0, 2:-2, 2:-2][i, j]
    u = U[1, 2:-2, 2:-2][i, j] / rho
    assert abs(t - 0.2) < 1e-15
    assert np.allclose(rho, g["rho"], rtol=2e-10, atol=0)
    assert np.allclose(u, g["u"], rtol=2e-10, atol=1e-14)


def test_nest_pipeline_program_equals_oracle_patch_steps(oracle, ref):
    """nest::execute of (dt reduce, exchange, euler_rhs compute) on nest's own
    patches (oracle/ref_prog_pipeline.cpp) equals forward-Euler steps of the
    oracle's patch stage with the periodic exchange: pins the program the
    device pipeline is compared with."""
    n, npatch, h, nexec, cfl = 403, 5, 2, 12, 0.4
    rng = np.random.default_rng(3)
    x = (np.arange(n) + 0.5) / n
    rho = np.where(x < 0.5, 1.0, 0.125) + 0.01 * rng.random(n)
    u = 0.2 * np.sin(2 * np.pi * x)
    p = np.where(x < 0.5, 1.0, 0.1)
    U = np.stack([rho, rho * u, p / 0.4 + 0.5 * rho * u * u])
    got, dts = ref.pipeline_euler1d(U, npatch, h, G, cfl, nexec)
    bounds = [(k * (n // npatch) + min(k, n % npatch), n // npatch + (1 if k < n % npatch else 0))
              for k in range(npatch)]
    dx = 1.0 / n
    for e in range(nexec):
        ms = 0.0
        for i in range(n):
            r, mo, en = U[:, i]
            ms = max(ms, abs(mo / r) + math.sqrt(G * oracle.L.orc_pressure(G, r, mo, en) / r))
        dt = 0.4 * dx / ms
        assert dt == dts[e]
        new = U.copy()
        for s0, m in bounds:
            idx = np.arange(s0 - h, s0 + m + h) % n
            new[:, s0:s0 + m] = oracle.patch_stage1d(np.ascontiguousarray(U[:, idx]), m, h, dx, dt, G)[:, h:-h]
        U = new
    assert np.array_equal(got, U)
