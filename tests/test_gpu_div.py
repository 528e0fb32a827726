"""The FP64 stage kernels' checked division (nest_b200/csrc/f64div.cuh)
against IEEE division.

The FP64 plain form's staged row march divides with a branch-free quotient
and keeps it only where an exact residual test shows it is the correctly
rounded IEEE quotient; everything else goes back to the IEEE division.  So
every quotient the test accepts (ok = 1) must equal numpy's a / b (correctly
rounded) bit for bit, zero signs included.  Cases: operands spread over 60
decades, quotients within a few ulps of a rounding midpoint (the hard cases
of the rounding test), quotients at and around powers of two, and every
pair of special values (zeros, subnormals, huge, infinite, NaN);
well-scaled operands must almost all be accepted."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(lib, a, b):
    import torch
    da = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    dq = torch.empty_like(da)
    dok = torch.zeros(da.numel(), dtype=torch.int32, device="cuda")
    st = lib.nest_selftest_div_f64(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), C.c_void_p(dq.data_ptr()),
                                   C.c_void_p(dok.data_ptr()), da.numel())
    return st, dq.cpu().numpy(), dok.cpu().numpy().astype(bool)


def bits(x):
    return np.asarray(x, dtype=np.float64).view(np.int64)


def check(lib, a, b):
    from nest_b200 import _capi as A
    st, q, ok = run(lib, a, b)
    assert st == A.NEST_OK, A.last_error()
    with np.errstate(all="ignore"):
        want = a / b
    bad = ok & (bits(q) != bits(want))
    assert not bad.any(), list(zip(a[bad][:5], b[bad][:5], q[bad][:5], want[bad][:5]))
    return ok


def test_wide_range(gpu):
    from nest_b200 import _capi as A
    rng = np.random.default_rng(7)
    n = 2_000_000
    a = rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)
    b = rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)
    ok = check(A.lib, a, b)
    assert ok.mean() > 0.999, ok.mean()


def test_quotients_near_midpoints(gpu):
    """a = RN(m b) for the midpoint m of two neighbouring doubles (formed in
    extended precision): a / b lies within about an ulp of m, where a wrong
    rounding decision would show."""
    from nest_b200 import _capi as A
    rng = np.random.default_rng(11)
    n = 2_000_000
    x = rng.uniform(1.0, 2.0, n) * 2.0 ** rng.integers(-40, 40, n)
    b = rng.uniform(1.0, 2.0, n) * 2.0 ** rng.integers(-20, 20, n)
    mid = x.astype(np.longdouble) + np.spacing(x).astype(np.longdouble) / 2
    a = (mid * b.astype(np.longdouble)).astype(np.float64)
    ok = check(A.lib, a, b)
    assert ok.mean() > 0.9, ok.mean()


def test_quotients_near_powers_of_two(gpu):
    """Below a power of two the doubles are twice as dense: quotients just
    under and just over 2^k, and exactly 2^k, from both sides."""
    from nest_b200 import _capi as A
    rng = np.random.default_rng(13)
    n = 1_000_000
    p2 = 2.0 ** rng.integers(-30, 30, n)
    b = rng.uniform(1.0, 2.0, n) * 2.0 ** rng.integers(-20, 20, n)
    k = rng.integers(-6, 7, n).astype(np.longdouble)  # quarter-ulp steps around 2^k
    q = p2.astype(np.longdouble) * (1 + k * np.longdouble(2.0 ** -55))
    a = (q * b.astype(np.longdouble)).astype(np.float64)
    a[: n // 10] = p2[: n // 10] * b[: n // 10]  # exact quotients 2^k where representable
    ok = check(A.lib, a, b)
    assert ok.mean() > 0.9, ok.mean()


def test_tiny_numerators(gpu):
    """Numerators down to the subnormals (the decaying tail of a wave): every
    kept quotient equals the IEEE one; numerators and quotients at or above
    2^-959 are kept."""
    from nest_b200 import _capi as A
    rng = np.random.default_rng(17)
    n = 1_000_000
    a = rng.uniform(1.0, 2.0, n) * 2.0 ** rng.integers(-1074, -900, n).astype(np.float64)
    b = rng.uniform(0.1, 4.0, n)
    ok = check(A.lib, a, b)
    with np.errstate(all="ignore"):
        in_range = (np.abs(a) >= 2.0 ** -959) & (np.abs(a / b) >= 2.0 ** -959)
    assert in_range.sum() > 1000 and ok[in_range].mean() > 0.999, ok[in_range].mean()


def test_special_values(gpu):
    from nest_b200 import _capi as A
    vals = np.array([0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 3.0, -7.25, 1e-300, -1e-300, 5e-324, 2.2e-308, 1e300, -1e300,
                     1.7e308, np.inf, -np.inf, np.nan, 0.1, 0.4, 1.4])
    a, b = np.meshgrid(vals, vals, indexing="ij")
    a, b = a.ravel(), b.ravel()
    ok = check(A.lib, a, b)
    # zero numerators over well-scaled divisors and ordinary quotients are kept
    keep = (a == 0) & (np.abs(b) > 1e-30) & (np.abs(b) < 1e30)
    assert ok[keep].all()
    assert ok[(a == 0.1) & (b == 3.0)].all() and ok[(a == 1.4) & (b == 3.0)].all()
    assert ok[(a == 0.1) & (b == 0.4)].all() and ok[(a == 3.0) & (b == 3.0)].all()  # exact quotients 0.25 and 1
    # nothing non-finite, zero-divisor or subnormal is accepted
    assert not ok[~np.isfinite(a) | ~np.isfinite(b) | (b == 0)].any()
