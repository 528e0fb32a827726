"""1D FP64 path on the GPU against the oracle: bit for bit.

Covers nest's drop-in ABI (euler1d_gpu_*), the resident single-CTA solver,
the tiled multi-CTA path, periodic and outflow boundaries, ragged sizes,
fixed-dt steps, compute_dt and frozen/recorded dt sequences."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.oracle import BC_OUTFLOW, BC_PERIODIC, sod_ic_1d

pytestmark = pytest.mark.gpu
G = 1.4


def test_dropin_matches_reference_test(gpu):
    """nest's own CPU-vs-GPU test (tests/test_euler_cuda.cpp:280-306): it
    allows 1e-8; the B200 path matches nest's CPU result exactly."""
    want = np.load(GOLDEN / "sod100_periodic.npy")
    s = gpu.Euler1DGPU(100, 2, 0.01, G)
    s.upload(sod_ic_1d(100))
    steps = s.run(0.1, 0.3)
    got = s.download()
    assert steps == 70
    assert np.array_equal(got[:, 2:-2], want[:, 2:-2])


# 257 / 1000 cells split unevenly over the resident solver's 16-CTA cluster
# (last chunk 2 / 55 cells); 3001 and 4080 cells only fit the cluster form
# (one CTA's shared memory holds up to about 2340), 4080 = 16 x 255 its largest
@pytest.mark.parametrize("n,bc,cfl,tf", [(1024, BC_OUTFLOW, 0.4, 0.2), (1024, BC_PERIODIC, 0.4, 0.2),
                                         (97, BC_OUTFLOW, 0.8, 0.1), (2300, BC_PERIODIC, 0.4, 0.05),
                                         (257, BC_PERIODIC, 0.5, 0.1), (1000, BC_OUTFLOW, 0.4, 0.1),
                                         (3001, BC_OUTFLOW, 0.4, 0.02), (4080, BC_PERIODIC, 0.4, 0.01)])
@pytest.mark.parametrize("resident", [True, False])
def test_run_to_matches_oracle(gpu, oracle, n, bc, cfl, tf, resident):
    U = sod_ic_1d(n)
    want = U.copy()
    wsteps, wt, _ = oracle.run1d(want, n, 2, 1.0 / n, G, cfl, t_final=tf, bc=bc)
    s = gpu.Solver(1, n, bc=bc, flags=0 if resident else gpu.FLAG_NO_RESIDENT)
    s.upload(U)
    steps = s.run_to(tf, cfl)
    t, total = s.time()
    got = s.download()
    assert steps == wsteps and total == wsteps and t == wt
    assert np.array_equal(got[:, 2:-2], want[:, 2:-2])


@pytest.mark.parametrize("n", [4, 255, 256, 257, 4099, 70001])
@pytest.mark.parametrize("bc", [BC_PERIODIC, BC_OUTFLOW])
def test_tiled_fixed_steps_ragged(gpu, oracle, n, bc):
    rng = np.random.default_rng(n)
    x = np.arange(n + 4)
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * x / max(n, 8)) + 0.05 * rng.random(n + 4)
    u = 0.2 * np.cos(2 * np.pi * x / max(n, 8))
    p = 1.0 + 0.2 * rng.random(n + 4)
    U = np.stack([rho, rho * u, p / 0.4 + 0.5 * rho * u * u])
    want = U.copy()
    oracle.run1d(want, n, 2, 1.0 / n, G, 0.5, nsteps=23, bc=bc)
    s = gpu.Solver(1, n, bc=bc, flags=gpu.FLAG_NO_RESIDENT)
    s.upload(U)
    s.step(23, 0.5)
    got = s.download()
    assert np.array_equal(got[:, 2:-2], want[:, 2:-2])


@pytest.mark.parametrize("bc", [BC_PERIODIC, BC_OUTFLOW])
def test_step_sequences_mix_launch_forms(gpu, oracle, bc):
    """Tiled steps go in pairs of one-launch steps (U -> U1 -> U, the stage-1
    halo recomputed per block) and an odd last step runs the two stage
    launches in place; any sequence of calls, with CFL dt from the wave
    speeds each form leaves behind, follows the oracle bit for bit."""
    n = 9001  # past the cluster form: tiled path
    U = sod_ic_1d(n)
    want = U.copy()
    s = gpu.Solver(1, n, bc=bc)
    s.upload(U)
    total = 0
    for k in [1, 2, 3, 16, 5, 33, 1]:
        s.step(k, 0.4)
        total += k
    wsteps, wt, _ = oracle.run1d(want, n, 2, 1.0 / n, G, 0.4, nsteps=total, bc=bc)
    t, steps = s.time()
    assert steps == wsteps == total and t == wt
    assert np.array_equal(s.download()[:, 2:-2], want[:, 2:-2])
    # a stopping time inside a pair: the finished step passes the state on unchanged
    tf = t + 2.5 * (wt / total)
    k = s.run_to(tf, 0.4)
    want = U.copy()
    wall, wtf, _ = oracle.run1d(want, n, 2, 1.0 / n, G, 0.4, t_final=tf, bc=bc)
    assert k == wall - total and s.time() == (wtf, wall)
    assert np.array_equal(s.download()[:, 2:-2], want[:, 2:-2])


def test_compute_dt_and_rk2_step(gpu, oracle):
    n = 300
    U = sod_ic_1d(n)
    s = gpu.Euler1DGPU(n, 2, 1.0 / n, G)
    s.upload(U)
    want = U.copy()
    for _ in range(5):
        dt = s.compute_dt(0.4)
        assert dt == 0.4 * (1.0 / n) / oracle.max_speed1d(want, n, 2, G)
        s.rk2_step(dt)
        oracle.run1d(want, n, 2, 1.0 / n, G, 0.4, nsteps=1, bc=BC_PERIODIC, dts_in=np.array([dt]))
    assert np.array_equal(s.download()[:, 2:-2], want[:, 2:-2])
    ms, steps = s.run_timed(0.01, 0.4)
    assert steps > 0 and ms > 0


def test_dts_record_then_freeze(gpu):
    n = 5000
    s = gpu.Solver(1, n, bc=BC_OUTFLOW, flags=gpu.FLAG_NO_RESIDENT)
    s.record_dts(64)
    s.upload(sod_ic_1d(n))
    s.step(40, 0.4)
    dts = s.recorded_dts(40)
    a = s.download()
    s2 = gpu.Solver(1, n, bc=BC_OUTFLOW)
    s2.freeze_dts(dts)
    s2.upload(sod_ic_1d(n))
    steps = s2.run_to(1.0, 0.4)  # ends when the frozen sequence runs out
    assert steps == 40
    assert np.array_equal(s2.download()[:, 2:-2], a[:, 2:-2])


@pytest.mark.parametrize("bc", [BC_OUTFLOW, BC_PERIODIC])
def test_fp32_form_close_to_fp64(gpu, bc):
    """The 1D FP32 form (tiled kernels, FP32 state and arithmetic, FP64 time
    and dt) tracks the FP64 plain form on Sod to FP32 rounding level; ghost
    cells follow the boundary rule."""
    n = 1000
    U = sod_ic_1d(n, 2)
    a64 = gpu.Solver(1, n, bc=bc, flags=gpu.FLAG_NO_RESIDENT)
    a64.upload(U)
    k64 = a64.run_to(0.1, 0.4)
    a32 = gpu.Solver(1, n, bc=bc, precision=gpu.F32)
    a32.upload(U.astype(np.float32))
    k32 = a32.run_to(0.1, 0.4)
    assert abs(k32 - k64) <= 1
    r64 = a64.download()[:, 2:-2]
    got = a32.download()
    r32 = got[:, 2:-2].astype(np.float64)
    assert np.all(np.isfinite(r32))
    scale = np.abs(r64).max(axis=1, keepdims=True)
    assert (np.abs(r32 - r64) / scale).mean() < 1e-5
    assert (np.abs(r32 - r64) / scale).max() < 2e-3
    if bc == BC_OUTFLOW:
        assert np.array_equal(got[:, 0], got[:, 2]) and np.array_equal(got[:, -1], got[:, -3])
    else:
        assert np.array_equal(got[:, 0], got[:, n]) and np.array_equal(got[:, -1], got[:, 3])
