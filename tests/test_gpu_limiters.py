"""Slope limiter options (nest's limiter_t: minmod, MC, none;
examples/sod1d/euler1d.hpp:106-137) on the device, FP64 bit for bit against
the oracle (1D, 2D unsplit) and against nest's own split sweeps (compat)."""
from __future__ import annotations

import contextlib

import numpy as np
import pytest

from oracle.oracle import BC_OUTFLOW, BC_PERIODIC, sod_ic_1d

pytestmark = pytest.mark.gpu
G = 1.4
LIMS = {"mc": 1, "none": 2}


@contextlib.contextmanager
def limiter(oracle, lim):
    oracle.set_limiter(lim)
    try:
        yield
    finally:
        oracle.set_limiter(0)


def flag(gpu, name):
    return gpu.FLAG_LIMITER_MC if name == "mc" else gpu.FLAG_LIMITER_NONE


@pytest.mark.parametrize("name", ["mc", "none"])
@pytest.mark.parametrize("resident", [True, False])
def test_1d_limiters_match_oracle(gpu, oracle, name, resident):
    n, tf = 400, 0.1
    U = sod_ic_1d(n)
    want = U.copy()
    with limiter(oracle, LIMS[name]):
        wsteps, wt, _ = oracle.run1d(want, n, 2, 1.0 / n, G, 0.4, t_final=tf, bc=BC_OUTFLOW)
    fl = flag(gpu, name) | (0 if resident else gpu.FLAG_NO_RESIDENT)
    s = gpu.Solver(1, n, bc=BC_OUTFLOW, flags=fl)
    s.upload(U)
    assert s.run_to(tf, 0.4) == wsteps
    assert np.array_equal(s.download()[:, 2:-2], want[:, 2:-2])
    # the limiter changes the answer
    base = gpu.Solver(1, n, bc=BC_OUTFLOW, flags=0 if resident else gpu.FLAG_NO_RESIDENT)
    base.upload(U)
    base.run_to(tf, 0.4)
    assert not np.array_equal(base.download(), s.download())


@pytest.mark.parametrize("name", ["mc", "none"])
def test_2d_limiters_match_oracle(gpu, oracle, name):
    from nest_b200.problems import kelvin_helmholtz
    nx, ny, nsteps = 70, 52, 12
    U = kelvin_helmholtz(nx, ny, seed=3)
    want = U.copy()
    with limiter(oracle, LIMS[name]):
        oracle.run2d(want, nx, ny, 2, 1.0 / nx, 1.0 / ny, G, 0.4, nsteps=nsteps, bc=BC_PERIODIC)
    s = gpu.Solver(2, nx, ny, bc=BC_PERIODIC, precision=gpu.F64, flags=flag(gpu, name))
    s.upload(U)
    s.step(nsteps, 0.4)
    assert np.array_equal(s.download()[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


@pytest.mark.parametrize("name", ["mc", "none"])
def test_2d_fp32_limiters_track_fp64(gpu, name):
    from nest_b200.problems import kelvin_helmholtz
    nx, ny = 64, 64
    U = kelvin_helmholtz(nx, ny, seed=5)
    out = {}
    for prec in (gpu.F64, gpu.F32):
        s = gpu.Solver(2, nx, ny, bc=BC_PERIODIC, precision=prec, flags=flag(gpu, name))
        s.upload(U.astype(np.float64 if prec == gpu.F64 else np.float32))
        s.step(20, 0.4)
        out[prec] = s.download()[:, 2:-2, 2:-2].astype(np.float64)
    err = np.abs(out[gpu.F32] - out[gpu.F64]).max()
    assert err < 1e-4, err


def test_split_compat_mc_matches_nest_sod2d(gpu, oracle, ref):
    from test_oracle import sod2d_reference_run
    from nest_b200.problems import prim_to_cons_2d
    want, t_ref, steps_ref = sod2d_reference_run(ref, oracle, LIMS["mc"])
    nx, ny = 200, 20
    x = (np.arange(-2, nx + 2) + 0.5) / nx
    X = np.repeat(x[:, None], ny + 4, axis=1)
    left = X < 0.5
    z = np.zeros_like(X)
    U = prim_to_cons_2d(np.where(left, 1.0, 0.125), z, z, np.where(left, 1.0, 0.1))
    s = gpu.Solver(2, nx, ny, dx=1.0 / nx, dy=0.1 / ny, bc=BC_PERIODIC, precision=gpu.F64,
                   flags=gpu.FLAG_SPLIT_COMPAT | gpu.FLAG_LIMITER_MC)
    s.upload(U)
    assert s.run_to(0.2, 0.3) == steps_ref
    assert np.array_equal(s.download()[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


@pytest.mark.parametrize("name", ["mc", "none"])
def test_split_compat_limiters_match_nest_smooth(gpu, oracle, ref, name):
    """Unlimited slopes oscillate at a shock (nest's sod2d with limiter_t::none
    blows up), so the limiter-none check runs a smooth periodic state."""
    import ctypes as C
    from nest_b200.problems import fourier_fields_2d
    nx, ny, nsteps, cfl = 48, 40, 10, 0.3
    dx, dy = 1.0 / nx, 1.0 / ny
    U0 = fourier_fields_2d(nx, ny, seed=6)
    U = np.ascontiguousarray(U0.copy())
    dp = C.POINTER(C.c_double)
    for _ in range(nsteps):
        oracle.fill_ghosts2d(U, nx, ny, 2, BC_PERIODIC)
        dt = ref.L.ref_compute_dt_2d(U.ctypes.data_as(dp), nx, ny, 2, dx, dy, cfl, G)
        for sweep, d in ((ref.L.ref_x_sweep, dx), (ref.L.ref_y_sweep, dy)):
            oracle.fill_ghosts2d(U, nx, ny, 2, BC_PERIODIC)
            out = np.empty_like(U)
            sweep(U.ctypes.data_as(dp), out.ctypes.data_as(dp), nx, ny, 2, d, dt, G, LIMS[name])
            U = out
    s = gpu.Solver(2, nx, ny, bc=BC_PERIODIC, precision=gpu.F64, flags=gpu.FLAG_SPLIT_COMPAT | flag(gpu, name))
    s.upload(U0)
    s.step(nsteps, cfl)
    assert np.array_equal(s.download()[:, 2:-2, 2:-2], U[:, 2:-2, 2:-2])


def test_limiter_rejections(gpu):
    from nest_b200.adjoint import Adjoint
    s = gpu.Solver(1, 64, bc=BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT | gpu.FLAG_LIMITER_MC)
    with pytest.raises(gpu.NestError):
        Adjoint(s, 4)
    with pytest.raises(gpu.NestError):
        gpu.Solver(1, 64, flags=gpu.FLAG_LIMITER_MC | gpu.FLAG_LIMITER_NONE)
