"""The acceptance rule of the checked FP64 division (nest_b200/csrc/f64div.cuh),
restated on the host with exact rational arithmetic.

The device kernels keep a fast quotient q of a / b only when the rule accepts
it and recompute the row with IEEE division otherwise, so their bit-for-bit
parity rests on the rule accepting nothing but RN(a / b).  Here the rule is
applied to the correctly rounded quotient and to its neighbours up to three
ulps away, for operands across the range where it is trusted, near powers of
two, for exact quotients and outside the range:
  * soundness: an accepted candidate is RN(a / b);
  * the correctly rounded quotient is accepted whenever |a| and |q| lie in
    the range;
  * a quotient of two doubles is either a power of two p or at least half
    the spacing above p away from it (write a = p b (1 + e): a lies on the
    grid of p b's binade or of a neighbouring one, which puts |e| at 2^-53 or
    more).  So a correctly rounded power-of-two quotient is exact, and the
    rule's narrower interval at powers of two turns nothing correct away;
    the full-width test would be just as sound there.
The fused multiply-add is an exact product and sum rounded once; Python's
float(Fraction) rounds to nearest even, as the device does.  The device's own
arithmetic is checked against IEEE division in tests/test_gpu_div.py.
"""
from __future__ import annotations

import math
import random
import struct
from fractions import Fraction


def _bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _hi(x: float) -> int:
    return _bits(x) >> 32


def _lo(x: float) -> int:
    return _bits(x) & 0xFFFFFFFF


def _from_hilo(h: int, lo: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", ((h & 0xFFFFFFFF) << 32) | lo))[0]


def _fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _exp_safe(ex: int) -> bool:
    return ((ex - 64) & 0xFFFFFFFF) < 1920


def accepted(a: float, b: float, q: float, narrow_pow2: bool = True) -> bool:
    """The rule of div_rn_checked for a candidate q that carries the sign of
    a / b (the device sets it), with the same operations in the same order;
    narrow_pow2=False drops the narrower interval at powers of two."""
    r = _fma(-b, q, a)
    hq = _hi(q)
    exq = (hq >> 20) & 0x7FF
    hu = _from_hilo((hq & 0x7FF00000) - (53 << 20), 0)
    pow2 = narrow_pow2 and ((hq & 0xFFFFF) | _lo(q)) == 0
    thr = abs(b) * (0.5 * hu if pow2 else hu)
    aok = _exp_safe((_hi(a) >> 20) & 0x7FF)
    return (aok and _exp_safe(exq) and abs(r) < thr) or (r == 0.0 and (aok or a == 0.0))


def rn_div(a: float, b: float) -> float:
    try:
        return float(Fraction(a) / Fraction(b))
    except OverflowError:
        return math.copysign(math.inf, a) * math.copysign(1.0, b)


def candidates(q: float):
    out, lo, hi = [q], q, q
    for _ in range(3):
        lo, hi = math.nextafter(lo, -math.inf), math.nextafter(hi, math.inf)
        out += [lo, hi]
    return out


def is_pow2(x: float) -> bool:
    return x != 0.0 and math.isfinite(x) and math.frexp(abs(x))[0] == 0.5


def in_range(x: float) -> bool:
    return 2.0 ** -959 <= abs(x) < 2.0 ** 961


def check_pair(a: float, b: float):
    """Soundness for every candidate; acceptance of RN(a / b) where the rule
    promises it.  Returns whether RN(a / b) was accepted."""
    q = rn_div(a, b)
    for c in candidates(q):
        for narrow in (True, False):
            if accepted(a, b, c, narrow):
                assert c == q, (a, b, c, q, narrow)
    ok = accepted(a, b, q)
    if in_range(a) and in_range(q):
        assert ok, (a, b, q)
    if is_pow2(q):
        assert Fraction(a) / Fraction(b) == Fraction(q), (a, b)
    return ok


def rand_double(rng: random.Random, lo_exp: int, hi_exp: int) -> float:
    m = rng.getrandbits(52) | (1 << 52)
    return math.ldexp(m, rng.randint(lo_exp, hi_exp) - 52) * rng.choice((-1.0, 1.0))


def test_random_operands_in_range():
    rng = random.Random(7)
    for _ in range(3000):
        a = rand_double(rng, -900, 900)
        b = rand_double(rng, -60, 60)
        check_pair(a, b)


def test_quotients_next_to_powers_of_two():
    rng = random.Random(8)
    for _ in range(1500):
        b = rand_double(rng, -20, 20)
        p = math.ldexp(1.0, rng.randint(-40, 40)) * (1.0 if b > 0 else -1.0)
        # a / b within a few ulps of the power of two p, on either side,
        # including numerators one step into the binade below p b
        if rng.random() < 0.5:
            a = float(Fraction(p) * Fraction(b) * (1 + Fraction(rng.randint(-6, 6), 2 ** 54)))
        else:
            b = math.ldexp(1.0 + rng.randint(0, 8) * 2.0 ** -52, rng.randint(-20, 20)) * math.copysign(1.0, b)
            a = Fraction(p) * Fraction(b)
            a = float(a)
            for _ in range(rng.randint(0, 4)):
                a = math.nextafter(a, 0.0)
        check_pair(a, b)
        dist = abs(Fraction(a) / Fraction(b) - Fraction(p))
        assert dist == 0 or dist >= Fraction(math.ulp(p)) / 2, (a, b, p)


def test_exact_and_zero_quotients():
    for a, b in [(6.0, 3.0), (-6.0, 3.0), (1.0, 0.25), (0.75, 3.0), (5.0, -0.5), (1.0, 1.0)]:
        assert accepted(a, b, rn_div(a, b)), (a, b)
    for a, b in [(0.0, 3.0), (-0.0, 3.0), (0.0, -2.5), (0.0, 1e-300), (0.0, 1e300)]:
        assert accepted(a, b, math.copysign(0.0, a) * math.copysign(1.0, b))


def test_out_of_range_operands_are_refused():
    rng = random.Random(9)
    for _ in range(300):
        b = rand_double(rng, -10, 10)
        # numerators under 2^-959 (and subnormals), quotients at the top of the range
        for a in (rand_double(rng, -1070, -960), rand_double(rng, 962, 1020)):
            q = rn_div(a, b)
            if math.isinf(q) or q == 0.0:
                continue
            for c in candidates(q):
                r = _fma(-b, c, a)
                if accepted(a, b, c):
                    # only an exact quotient may pass outside the range
                    assert r == 0.0 and c == q, (a, b, c)
