// Correctly rounded FP64 division without a slow-path branch in the common
// case, for the FP64 plain form's row marches (sm_100a; compiled with
// -fmad=false, every fused multiply-add below is an explicit fma()).
//
// Method (textbook, not a restatement of any library routine):
//   * y ~ 1/b from the hardware approximation (PTX rcp.approx.ftz.f64),
//     refined by two Newton-Raphson steps y <- y + y (1 - b y), each of which
//     roughly doubles the number of correct bits;
//   * q0 = a y, then one residual correction q = q0 + (a - b q0) y, with the
//     residual formed exactly by a fused multiply-add (P. Markstein,
//     "Computation of elementary functions on the IBM RISC System/6000
//     processor", IBM J. Res. Dev. 34(1), 1990);
//   * a rounding test on the exact residual r = a - b q: q is the correctly
//     rounded quotient RN(a/b) if |a/b - q| < ulp(q)/2, i.e. |r| < |b| ulp(q)/2
//     (a quotient of two doubles is never exactly halfway between two
//     doubles, so no tie arises), provided r is exact, which holds when q is
//     within an ulp of a/b and nothing under- or overflows (J.-M. Muller et
//     al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018, ch. 4).  A q
//     further than an ulp from a/b gives |r| >= |b| ulp(q) and fails the
//     test, so an accepted q is always RN(a/b).
// The test is only trusted inside a safe range: |a| and |q| in
// [2^-959, 2^961).  There ulp(q)/2 >= 2^-1012 and the threshold
// |b| ulp(q)/2 ~ |a| 2^-53 are normal, nothing overflows, and a - b q is a
// multiple of ulp(b) ulp(q) >= 2^-1074 smaller than 2^53 of them, so the
// fused multiply-add forms it exactly.  Where |q| is a power of two the
// spacing below it is half the spacing above, and the test takes the
// narrower interval on both sides.  That refuses nothing correct: a quotient
// of two doubles is a power of two p or at least half the spacing above p
// away from it, so a correct power-of-two quotient is exact (r = 0), and the
// full-width test would be as sound there.
// r = 0 is an exact quotient; with a = 0 and b finite and nonzero that is
// the zero of sign(a) xor sign(b), the sign every quotient is given.
// Everything else, and any q the test does not accept, clears `ok`; the
// caller then recomputes with the IEEE division.  (Scaling numerators under
// 2^-959 by a power of two to keep them on the fast path measured slower than
// recomputing the few rows that meet them.)
#pragma once

#include <cuda_runtime.h>

namespace nestb {

__device__ __forceinline__ unsigned f64_biased_exp(double x) { return ((unsigned)__double2hiint(x) >> 20) & 0x7ffu; }

// Whether a biased exponent lies in [64, 1983] (|x| in [2^-959, 2^961)).
__device__ __forceinline__ bool f64_exp_safe(unsigned ex) { return ex - 64u < 1920u; }

__device__ __forceinline__ double div_rn_checked(double a, double b, bool& ok) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    y = fma(y, fma(-b, y, 1.0), y);
    y = fma(y, fma(-b, y, 1.0), y);
    const double q0 = a * y;
    const double qm = fma(fma(-b, q0, a), y, q0);
    const int ha = __double2hiint(a), hb = __double2hiint(b);
    // the IEEE quotient's sign is sign(a) xor sign(b); setting it also gives
    // a zero quotient its sign
    const double q = __hiloint2double((__double2hiint(qm) & 0x7fffffff) | ((ha ^ hb) & (int)0x80000000u),
                                      __double2loint(qm));
    const double r = fma(-b, q, a);
    const int hq = __double2hiint(q);
    const unsigned exq = ((unsigned)hq >> 20) & 0x7ffu;
    // ulp(q)/2 = 2^(e(q) - 53): q's exponent field lowered by 53, mantissa 0
    const double hu = __hiloint2double((int)((unsigned)hq & 0x7ff00000u) - (53 << 20), 0);
    // |q| a power of two: the spacing below it is half, so the narrower
    // interval is used on both sides there
    const bool pow2 = (((unsigned)hq & 0xfffffu) | (unsigned)__double2loint(q)) == 0u;
    const double thr = fabs(b) * (pow2 ? 0.5 * hu : hu);
    const bool aok = f64_exp_safe(f64_biased_exp(a));
    // r = 0: an exact quotient (a = 0 included, b finite and nonzero: else r is NaN)
    ok = ok && ((aok && f64_exp_safe(exq) && fabs(r) < thr) || (r == 0.0 && (aok || a == 0.0)));
    return q;
}

}  // namespace nestb
