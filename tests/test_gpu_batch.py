"""Batched independent problems (one persistent launch per stage over a work
list): FP64 bit for bit per problem against the oracle, for every launch
shape; FP32 (packed) against FP64; per-problem dt, time and totals."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import BC_OUTFLOW, BC_PERIODIC
from nest_b200.problems import kelvin_helmholtz, riemann_2d

pytestmark = pytest.mark.gpu
G = 1.4
SIZES = [(64, 128), (96, 64), (128, 192), (64, 64), (40, 72), (33, 61)]


def make_batch(gpu, prec, flags=0, tiling=None, bc=(BC_PERIODIC, BC_PERIODIC)):
    nx = [s[0] for s in SIZES]
    ny = [s[1] for s in SIZES]
    b = gpu.Batch(nx, ny, bc=bc, precision=prec, flags=flags)
    if tiling:
        b.set_tiling(*tiling)
    ics = []
    for p, (a, c) in enumerate(SIZES):
        U = kelvin_helmholtz(a, c, seed=1 + p)
        ics.append(U)
        b.upload(p, U if prec == gpu.F64 else U.astype(np.float32))
    return b, ics


@pytest.mark.parametrize("tiling", [None, (8, 1, 0), (16, 4, 1), (64, 2, 0)])
def test_batch_fp64_matches_oracle_per_problem(gpu, oracle, tiling):
    b, ics = make_batch(gpu, gpu.F64, tiling=tiling)
    b.step(21, 0.4)
    times, steps = b.times()
    for p, (nx, ny) in enumerate(SIZES):
        want = ics[p].copy()
        _, t, _ = oracle.run2d(want, nx, ny, 2, 1 / nx, 1 / ny, G, 0.4, nsteps=21, bc=BC_PERIODIC)
        got = b.download(p)
        assert steps[p] == 21 and times[p] == t
        assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2]), p


def test_batch_fp64_outflow_riemann(gpu, oracle):
    nx, ny = [48, 64, 37], [48, 40, 53]
    b = gpu.Batch(nx, ny, bc=(BC_OUTFLOW, BC_OUTFLOW), precision=gpu.F64)
    for p in range(3):
        b.upload(p, riemann_2d(nx[p], ny[p]))
    b.step(17, 0.4)
    for p in range(3):
        want = riemann_2d(nx[p], ny[p])
        oracle.run2d(want, nx[p], ny[p], 2, 1 / nx[p], 1 / ny[p], G, 0.4, nsteps=17, bc=BC_OUTFLOW)
        assert np.array_equal(b.download(p)[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


def test_batch_fp32_close_to_fp64_and_conserves(gpu):
    b64, _ = make_batch(gpu, gpu.F64, flags=gpu.FLAG_TOTALS)
    b32, ics = make_batch(gpu, gpu.F32, flags=gpu.FLAG_TOTALS | gpu.FLAG_REPAIR)
    b64.step(40, 0.4)
    b32.step(40, 0.4)
    t64, _ = b64.times()
    t32, _ = b32.times()
    assert np.allclose(t32, t64, rtol=1e-5)
    tot32 = b32.totals()
    for p, (nx, ny) in enumerate(SIZES):
        a = b64.download(p)[:, 2:-2, 2:-2]
        c = b32.download(p)[:, 2:-2, 2:-2].astype(np.float64)
        scale = np.abs(a).max(axis=(1, 2), keepdims=True)
        assert (np.abs(c - a) / scale).mean() < 2e-6
        direct = c.sum(axis=(1, 2)) / (nx * ny)
        assert np.allclose(tot32[p], direct, rtol=1e-12, atol=1e-12)
        m0 = ics[p][0, 2:-2, 2:-2].astype(np.float32).astype(np.float64).sum() / (nx * ny)
        assert abs(tot32[p][0] - m0) < 1e-5 * m0


def test_batch_info_and_uneven_sizes(gpu):
    from nest_b200.problems import kh_sizes
    nx, ny = kh_sizes(24, seed=0)
    b = gpu.Batch(nx, ny, precision=gpu.F32)
    cells, items, blocks = b.info()
    assert cells == int(np.sum(nx.astype(np.int64) * ny)) and items > 24 and blocks >= 148
    for p in range(24):
        b.upload(p, kelvin_helmholtz(int(nx[p]), int(ny[p]), seed=1 + p).astype(np.float32))
    b.step(20, 0.4)
    t, s = b.times()
    assert np.all(s == 20) and np.all(t > 0)
    # each problem has its own dt: different sizes give different times
    assert len(np.unique(np.round(t, 12))) > 1
    for p in (0, 7, 23):
        assert np.all(np.isfinite(b.download(p)))


@pytest.mark.parametrize("tiling", [(8, 2, 1), (8, 4, 1), (8, 4, 2)])
def test_batch_fp32_multiwarp_matches_single(gpu, tiling):
    """Persistent FP32 batch with several warps per block and several work
    items per warp (each warp stages the rows of one item after another
    through the same shared-memory ring slots) against the single-domain
    FP32 solver, bit for bit per problem."""
    sizes = [(256, 256), (192, 320), (128, 200), (300, 128)] * 6
    nx = [a for a, _ in sizes]
    ny = [c for _, c in sizes]
    flags = gpu.FLAG_TOTALS | gpu.FLAG_REPAIR
    b = gpu.Batch(nx, ny, precision=gpu.F32, flags=flags)
    b.set_tiling(*tiling)
    ics = [kelvin_helmholtz(a, c, seed=1 + p).astype(np.float32) for p, (a, c) in enumerate(sizes)]
    for p, U in enumerate(ics):
        b.upload(p, U)
    b.step(30, 0.4)
    _, items, blocks = b.info()
    assert items > 2 * blocks * tiling[1]  # several items per warp
    for p, (a, c) in enumerate(sizes):
        s = gpu.Solver(2, a, c, bc=gpu.BC_PERIODIC, precision=gpu.F32, flags=flags)
        s.upload(ics[p])
        s.step(30, 0.4)
        assert np.array_equal(b.download(p)[:, 2:-2, 2:-2], s.download()[:, 2:-2, 2:-2]), p
