"""Positivity and finiteness checks on the device (nest's check,
examples/sod1d/sod1d.cpp:279-301: rho <= 0 or p <= 0 in an interior cell
stops the run with an error naming the step and the cell).

A bad cell is planted in an otherwise smooth state and uploaded from the
host: a pressure deficit (E < 1/2 rho u^2, a finite state with p <= 0), a
negative density and a NaN.  The FP64 oracle, advanced one step at a time
from the same state, gives the first failing step and the set of failing
cells (the FP64 form follows it bit for bit, NaNs included); every entry
point must report NEST_ERR_NUMERIC with that step and one of those cells,
stop advancing, and run again after a good state is uploaded."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle.oracle import BC_PERIODIC, Oracle

pytestmark = pytest.mark.gpu
G = 1.4
KINDS = ["p", "rho", "nan"]


def smooth_1d(n):
    x = (np.arange(n + 4) - 2 + 0.5) / n
    rho = 1 + 0.2 * np.sin(2 * np.pi * x)
    u = 0.3 * np.cos(2 * np.pi * x)
    p = np.ones_like(x)
    return np.stack([rho, rho * u, p / (G - 1) + 0.5 * rho * u * u])


def smooth_2d(nx, ny):
    x = (np.arange(nx + 4) - 2 + 0.5)[:, None] / nx
    y = (np.arange(ny + 4) - 2 + 0.5)[None, :] / ny
    rho = 1 + 0.2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    u = 0.3 * np.cos(2 * np.pi * y) + 0 * x
    v = 0.2 * np.sin(2 * np.pi * x) + 0 * y
    p = np.ones_like(rho)
    return np.stack([rho, rho * u, rho * v, p / (G - 1) + (0.5 * rho * u * u + 0.5 * rho * v * v)])


def plant(U, kind, idx):
    """Bad cell at interior index idx (1D: (i,), 2D: (i, j))."""
    U = U.copy()
    e = tuple(k + 2 for k in idx)
    if kind == "p":      # |u| = 2, E = 1/5 of the kinetic energy: p < 0
        U[(1,) + e] = 2.0 * U[(0,) + e]
        U[(-1,) + e] = 0.2 * 0.5 * U[(0,) + e] * 4.0
    elif kind == "rho":
        U[(0,) + e] = -0.5
    else:
        U[(-1,) + e] = np.nan
    return U


def bad_cells(U):
    """Interior cells with !(rho > 0) or !(p > 0), the scheme's pressure."""
    with np.errstate(all="ignore"):
        if U.ndim == 2:
            r, m, E = U[0, 2:-2], U[1, 2:-2], U[2, 2:-2]
            u = m / r
            p = (G - 1) * (E - 0.5 * r * u * u)
        else:
            r, mu, mv, E = (U[k, 2:-2, 2:-2] for k in range(4))
            u, v = mu / r, mv / r
            p = (G - 1) * (E - (0.5 * r * u * u + 0.5 * r * v * v))
        b = ~(r > 0) | ~(p > 0)
    return {tuple(int(c) for c in t) for t in zip(*np.nonzero(b))}


def expected(U, steps=6):
    """(first failing step, failing cells, NaN at that step?) of the FP64 oracle."""
    orc = Oracle()
    W = U.copy()
    for s in range(1, steps + 1):
        if W.ndim == 2:
            n = W.shape[1] - 4
            orc.run1d(W, n, 2, 1.0 / n, G, 0.4, nsteps=1, bc=BC_PERIODIC)
        else:
            nx, ny = W.shape[1] - 4, W.shape[2] - 4
            orc.run2d(W, nx, ny, 2, 1.0 / nx, 1.0 / ny, G, 0.4, nsteps=1, bc=BC_PERIODIC)
        b = bad_cells(W)
        if b:
            return s, b
    raise AssertionError("planted cell never failed in the oracle")


def parse(msg):
    """(kind, step, cell) from the error text."""
    import re
    m = re.search(r"(positivity violation|non-finite state).* at step (\d+) in cell \((-?\d+), (-?\d+)\)", msg)
    assert m, msg
    return ("p" if m.group(1).startswith("positivity") else "nan"), int(m.group(2)), (int(m.group(3)), int(m.group(4)))


def check_report(err, kind, step, cells, dim):
    from nest_b200 import _capi as A
    assert err.status == A.NEST_ERR_NUMERIC, str(err)
    what, s, cell = parse(str(err))
    assert s == step, (str(err), step)
    assert (cell[:1] if dim == 1 else cell) in cells, (str(err), sorted(cells)[:8])
    assert what == ("p" if kind == "p" else "nan"), str(err)


# 1D: resident single CTA (200 cells), 16-CTA cluster (1024), tiled stages (1000), FP32 form (1000)
PATHS_1D = {"resident": (200, "F64", 0), "cluster": (1024, "F64", 0), "tiled": (1000, "F64", "NO_RESIDENT"),
            "f32": (1000, "F32", 0)}


@pytest.mark.parametrize("path", list(PATHS_1D))
@pytest.mark.parametrize("kind", KINDS)
def test_1d_reports_and_stops(gpu, path, kind):
    n, prec, flag = PATHS_1D[path]
    prec = getattr(gpu, prec)
    flags = gpu.FLAG_NO_RESIDENT if flag == "NO_RESIDENT" else 0
    k = n // 3
    U = plant(smooth_1d(n), kind, (k,))
    step, cells = expected(U)
    s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, precision=prec, flags=flags)
    s.upload(U)
    s.step(8, 0.4)
    with pytest.raises(gpu.NestError) as ei:
        s.sync()
    if prec == gpu.F64:
        check_report(ei.value, kind, step, cells, 1)
    else:  # FP32 rounding: same step, a cell the planted one reaches in a step (two stages, +-4)
        what, st, cell = parse(str(ei.value))
        assert st == step and abs(cell[0] - k) <= 5, str(ei.value)
        assert what == "p" if kind == "p" else kind == "rho" or what == "nan", str(ei.value)
    # the solver stops at the failing step: more steps leave the state alone
    frozen = s.download()
    s.step(4, 0.4)
    with pytest.raises(gpu.NestError):
        s.sync()
    assert np.array_equal(s.download(), frozen, equal_nan=True)
    # a good state clears the record and runs (the clock keeps counting)
    s.upload(smooth_1d(n))
    k0 = s.time()[1]
    s.step(3, 0.4)
    s.sync()
    assert s.time()[1] == k0 + 3
    s.close()


# 2D: FP64 plain form, packed FP32 (plain), one-column-per-lane FP32
FORMS_2D = {"f64": ("F64", 0), "f32x2": ("F32", 0), "f32scalar": ("F32", "FP32_SCALAR")}


@pytest.mark.parametrize("form", list(FORMS_2D))
@pytest.mark.parametrize("kind", KINDS)
def test_2d_reports_and_stops(gpu, form, kind):
    nx, ny = 70, 66
    prec, flag = FORMS_2D[form]
    prec = getattr(gpu, prec)
    flags = gpu.FLAG_FP32_SCALAR if flag == "FP32_SCALAR" else 0
    ij = (31, 17)
    U = plant(smooth_2d(nx, ny), kind, ij)
    step, cells = expected(U)
    s = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=prec, flags=flags)
    s.upload(U)
    s.step(5, 0.4)
    with pytest.raises(gpu.NestError) as ei:
        s.sync()
    if prec == gpu.F64:
        check_report(ei.value, kind, step, cells, 2)
    else:
        # the FP32 sound speed stays finite at rho < 0, so a negative density
        # can remain a finite positivity violation where FP64 turns it into NaN
        what, st, cell = parse(str(ei.value))
        assert st == step and abs(cell[0] - ij[0]) <= 5 and abs(cell[1] - ij[1]) <= 5, str(ei.value)
        assert what == "p" if kind == "p" else kind == "rho" or what == "nan", str(ei.value)
    frozen = s.download()
    s.step(3, 0.4)
    with pytest.raises(gpu.NestError):
        s.sync()
    assert np.array_equal(s.download(), frozen, equal_nan=True)
    s.upload(smooth_2d(nx, ny))
    s.step(2, 0.4)
    s.sync()
    s.close()


@pytest.mark.parametrize("kind", KINDS)
def test_2d_fp32_repair_fixes_positivity_and_reports_nan(gpu, kind):
    """The FP32 form with FP64 repair raises rho and p near vacuum instead of
    failing; a NaN still stops it."""
    nx, ny = 70, 66
    U = plant(smooth_2d(nx, ny), kind, (31, 17))
    s = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=gpu.F32, flags=gpu.FLAG_REPAIR | gpu.FLAG_TOTALS)
    s.upload(U)
    s.step(5, 0.4)
    if kind == "nan":
        with pytest.raises(gpu.NestError) as ei:
            s.sync()
        assert parse(str(ei.value))[0] == "nan"
    else:
        s.sync()
        assert s.repairs() > 0
        assert np.all(np.isfinite(s.download()))
    s.close()


@pytest.mark.parametrize("prec", ["F64", "F32"])
def test_batch_names_the_problem(gpu, prec):
    nx, ny = np.array([40, 70, 64]), np.array([48, 66, 64])
    b = gpu.Batch(nx, ny, precision=getattr(gpu, prec))
    for p in range(3):
        U = smooth_2d(int(nx[p]), int(ny[p]))
        if p == 1:
            U = plant(U, "p", (31, 17))
            step, cells = expected(U)
        b.upload(p, U)
    b.step(4, 0.4)
    with pytest.raises(gpu.NestError) as ei:
        b.times()
    msg = str(ei.value)
    assert "problem 1:" in msg, msg
    what, st, cell = parse(msg)
    assert what == "p" and st == step
    if prec == "F64":
        assert cell in cells, msg
    b.close()


def test_noalloc_and_dropin_report(gpu):
    import torch
    from nest_b200 import _capi as A
    n = 1000
    U = plant(smooth_1d(n), "p", (400,))
    step, cells = expected(U)
    state = torch.from_numpy(U.copy()).cuda()
    nsteps, t = C.c_int(0), C.c_double(0.0)
    st = A.lib.nest_euler1d_run_noalloc(C.c_void_p(state.data_ptr()), n, 2, 1.0 / n, G, A.BC_PERIODIC, 0.05, 0.4,
                                        C.byref(nsteps), C.byref(t), None)
    assert st == A.NEST_ERR_NUMERIC
    what, s, cell = parse(A.last_error())
    assert what == "p" and s == step and cell[:1] in cells

    g = gpu.Euler1DGPU(n, 2, 1.0 / n, G)
    g.upload(U)
    assert A.lib.euler1d_gpu_run(g._h, 0.05, 0.4) == -1  # nest's ABI: the step count, -1 on error
    assert A.lib.euler1d_gpu_status(g._h) == A.NEST_ERR_NUMERIC
    what, s, cell = parse(A.last_error())
    assert what == "p" and s == step and cell[:1] in cells
