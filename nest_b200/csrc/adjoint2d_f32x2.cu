// FP32 discrete adjoint of the unsplit 2D stage as a packed FP32x2 row march
// (sm_100a; compiled with -use_fast_math).
//
// Same map as the tile kernel of adjoint2d.cuh:
//   Lin = alpha * S'(U)^T Lout + beta * Extra,
//   S(U) = U - lx (F_{i+1/2} - F_{i-1/2}) - ly (G_{j+1/2} - G_{j-1/2}),
// periodic on both axes, with the same subgradient choices: minmod's active
// argument (the second difference on a tie, none at a sign change or a
// zero), the HLLE regime and the active argument of each Davis min / max.
//
// Each warp owns a strip of 64 columns c0 .. c0+63, two adjacent columns
// per lane kept as a float2 pair, writes the 56 columns c0+4 .. c0+59
// (lanes 2..29), and marches down a segment of rows.  Step a of the march:
//   * primitives of row a+2 (the conserved rows, Lout and Extra arrive
//     through per-warp shared-memory rings filled by cp.async one step
//     ahead), x-slope of row a+1 and the masks of its active minmod argument,
//   * reverse HLLE of x-face a+1/2 with flux adjoint lx (Lout_{a+1} -
//     Lout_a): face-state adjoints to rows a and a+1, the now complete
//     x-slope adjoint of row a to rows a-1 .. a+1,
//   * the y-direction part of row a: y-slopes, the lane's two y-faces
//     (a|b and b|a'), their reverse HLLE and the y-slope scatter, with
//     shuffles for the neighbouring columns,
//   * row a-1 has all its contributions:
//     Lin = alpha (Lout + (dW/dU)^T Wbar) + beta Extra.
// Every x-face is reversed once per strip and every y-face once (the tile
// kernel reverses 2.4 faces per cell and converts 2 cells' primitives per
// cell); nothing but the rings goes through shared memory.
#include "euler2d_kernels.cuh"
#include "f2ops.cuh"
#include "kernels.h"

#include <algorithm>
#include <mutex>

namespace nestb {
namespace {

// Launch shape and register budget, measured on the 2048^2 FP32 KH adjoint
// (200 steps, backward ms): 2 warps per CTA at 200 registers (198 used, no
// spills, 10 warps per SM) 75.7; 2 or 4 warps at 168 (16 bytes spilled, 12
// warps per SM) 76.1 / 77.2; 144 registers 84.3; 128 registers 94.7; the
// march unrolled by 2 / 3 76.4 / 84.0.
#ifndef NEST_ADJX2_WARPS
#define NEST_ADJX2_WARPS 2
#define NEST_ADJX2_REGS 200
#define NEST_ADJX2_UNROLL 1
#endif
constexpr int ASTRIP = 56;                // output columns per warp
constexpr int AWARPS = NEST_ADJX2_WARPS;  // warps per CTA (strips side by side)
constexpr int AUNROLL = NEST_ADJX2_UNROLL;
// ring slots per warp: conserved rows (2), Lout rows (4), Extra rows (2),
// each [4 variables][32 lanes] float2
constexpr int RU = 2, RL = 4, RE = 2;
constexpr int RING_F2 = (RU + RL + RE) * 4 * 32;
extern __shared__ __align__(16) F2 adj_ring[];

struct Q4 { F2 a, b, c, d; };

// Asynchronous global -> shared copy of 8 bytes (one column pair).
__device__ __forceinline__ void cp8(F2* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ float mm(float a, float b) {
    float t;
    asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(t) : "f"(a), "f"(b));
    return copysignf(fmaxf(t, 0.f), a);
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float t;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(t) : "f"(a), "f"(b), "f"(c));
    return t;
}

// Minmod slope of a pair and the masks of its active argument: mz = 1 where
// the slope is not 0, me = 1 where it equals the second difference (the
// second argument is active where mz me = 1, exact ties included; the first
// where mz (1 - me) = 1), me = 1/2 at a near-tie (tie_mask).  A slope adjoint sb then scatters as t2 = me (mz sb) to
// the second difference and t1 = mz sb - t2 to the first.
// Near-ties of minmod: where |d1| and |d2| differ by no more than 2^-19 |w|
// (w the cell's primitive), which of the two is the smaller is decided by the
// rounding of the FP32 primitives (approximate reciprocal, cancellation in the
// pressure), not by the flow; the mask then splits the slope adjoint half and
// half between the two differences (the mean of the two one-sided
// derivatives).  Taking either one instead sent an O(1) share of the slope
// adjoint to a neighbour chosen by rounding in many cells of a rolled-up
// Kelvin-Helmholtz layer: after 4000 steps of the 2048^2 periodic KH problem the
// FP32 gradient had a relative L2 distance 12.8 from the FP64 one (cosine
// 0.08) while finite differences of the FP32 forward map agreed with the FP64
// map's to 1e-4; with the split it is 0.011 (cosine 0.99994) and its
// directional derivatives match those finite differences to about 1 %.
// Where the slope is not zero d1 and d2 have one sign, so ||d1| - |d2|| is
// |d1 - d2|: one packed subtraction and one packed product per pair.  Where
// it is zero the mask is not used.
__device__ __forceinline__ float tie_mask(float s, float d2, float dd, float tol) {
    // (where the slope is zero the mask is not used: mz = 0)
    return fabsf(dd) <= fabsf(tol) ? 0.5f : (s == d2 ? 1.f : 0.f);
}
__device__ __forceinline__ F2 mm_mask(F2 d1, F2 d2, F2& mz, F2& me, F2 w) {
    F2 s = make_float2(mm(d1.x, d2.x), mm(d1.y, d2.y));
    const F2 dd = sub2(d1, d2), tol = mul2(sp(1.9073486e-06f), w);  // 2^-19 w
    mz = make_float2(s.x != 0.f ? 1.f : 0.f, s.y != 0.f ? 1.f : 0.f);
    me = make_float2(tie_mask(s.x, d2.x, dd.x, tol.x), tie_mask(s.y, d2.y, dd.y, tol.y));
    return s;
}

__device__ __forceinline__ Q4 prim2(const Q4& U, float gm1) {
    Q4 w;
    F2 ir = rcp2(U.a);
    w.a = U.a;
    w.b = mul2(U.b, ir);
    w.c = mul2(U.c, ir);
    F2 ke = mul2(mul2(sp(0.5f), U.a), fma2(w.c, w.c, mul2(w.b, w.b)));
    w.d = max2(mul2(sp(gm1), sub2(U.d, ke)), 0.f);
    return w;
}

// Reverse of the four-variable HLLE with Davis speeds (euler1d.hpp:178-242)
// along a normal, on a pair of faces: states (r, n, t, p) per side, flux
// adjoint (f0, f1, f2, f3) in the order (mass, normal momentum, transverse
// momentum, energy); the face-state adjoints are added to Lb and Rb.
// Written in the relative-flux form of the forward kernel, with
// sl = min(S_L, 0) = -nsl and sr = max(S_R, 0):
//   F = wL (F_L - sl U_L) + wR (F_R - sr U_R),
//   wL = sr / (sr - sl), wR = -sl / (sr - sl),
// which is the HLLE average in the subsonic regime and F_L (wL = 1) or F_R
// (wR = 1) in the supersonic ones, without branches.  With
// X = f0 + f1 n + f2 t, Y = f1 + f3 n, k = (n^2 + t^2) / 2 and
// g = wS (n - s) (s = sl on the left, sr on the right), the side adjoints are
//   rb = g (X + f3 k),  nb = wS (r X + f3 (E + p)) + g r Y,
//   tb = g r (f2 + f3 t),  pb = wS Y + g f3 / (gamma - 1),
// plus the sound-speed terms dc/dp = gamma / (2 r c), dc/dr = -c / (2 r).
// The speed adjoints are
//   dF/dsl . fb = sr / (sr - sl)^2 (fb . (G_L(sr) - G_R(sr))),
//   dF/dsr . fb = sl / (sr - sl)^2 (fb . (G_R(sl) - G_L(sl))),
// with fb . G_S(s) = (n - s) (r X + f3 E) + p Y for G_S(s) = F_S - s U_S;
// each applies only where its clamp is open (S_L < 0, S_R > 0).
__device__ __forceinline__ void hlle2_adj(float gamma, float igm1, const Q4& L, const Q4& R, F2 f0, F2 f1, F2 f2,
                                          F2 f3, Q4& Lb, Q4& Rb) {
    const F2 g = sp(gamma), h = sp(0.5f);
    const F2 rL = L.a, nL = L.b, tL = L.c, pL = L.d;
    const F2 rR = R.a, nR = R.b, tR = R.c, pR = R.d;
    F2 gpL = mul2(g, pL), gpR = mul2(g, pR);
    F2 qL = rsq2(max2(mul2(gpL, rL), 1e-37f)), qR = rsq2(max2(mul2(gpR, rR), 1e-37f));
    F2 cL = mul2(gpL, qL), cR = mul2(gpR, qR);
    F2 kL = mul2(h, fma2(tL, tL, mul2(nL, nL))), kR = mul2(h, fma2(tR, tR, mul2(nR, nR)));
    F2 EL = fma2(pL, sp(igm1), mul2(rL, kL)), ER = fma2(pR, sp(igm1), mul2(rR, kR));
    F2 aL = sub2(cL, nL), aR = sub2(cR, nR), bL = add2(nL, cL), bR = add2(nR, cR);
    F2 nsl = make_float2(max3f(aL.x, aR.x, 0.f), max3f(aL.y, aR.y, 0.f));
    F2 sr = make_float2(max3f(bL.x, bR.x, 0.f), max3f(bL.y, bR.y, 0.f));
    F2 inv = rcp2(max2(add2(sr, nsl), 1e-30f));
    F2 wL = mul2(sr, inv), wR = mul2(nsl, inv);
    F2 gL = mul2(wL, add2(nL, nsl)), gR = mul2(wR, sub2(nR, sr));
    F2 XL = fma2(f2, tL, fma2(f1, nL, f0)), XR = fma2(f2, tR, fma2(f1, nR, f0));
    F2 YL = fma2(f3, nL, f1), YR = fma2(f3, nR, f1);
    F2 ZL = fma2(rL, XL, mul2(f3, EL)), ZR = fma2(rR, XR, mul2(f3, ER));
    F2 D = sub2(mul2(pL, YL), mul2(pR, YR));
    F2 s1 = add2(fma2(sub2(nL, sr), ZL, D), mul2(sub2(sr, nR), ZR));
    F2 s2 = sub2(fma2(add2(nR, nsl), ZR, mul2(sp(-1.f), D)), mul2(add2(nL, nsl), ZL));
    // the speed adjoints apply only where both clamps are open (subsonic):
    // in the supersonic regimes one of nsl, sr is 0 and the other adjoint is
    // 0 by its own factor, so one mask serves both
    F2 i2 = mul2(mul2(inv, inv), make_float2(nsl.x * sr.x > 0.f ? 1.f : 0.f, nsl.y * sr.y > 0.f ? 1.f : 0.f));
    F2 Slb = mul2(mul2(sr, i2), s1);               // adjoint of S_L
    F2 Srb = mul2(mul2(sp(-1.f), mul2(nsl, i2)), s2);  // adjoint of S_R
    // active arguments (S_L = min(nL - cL, nR - cR), S_R = max(nL + cL, nR + cR);
    // the right argument only where strictly smaller / larger; nR - cR < nL - cL
    // <=> cR - nR > cL - nL, exact negations)
    F2 mL = make_float2(aR.x > aL.x ? 1.f : 0.f, aR.y > aL.y ? 1.f : 0.f);
    F2 mR = make_float2(bL.x < bR.x ? 1.f : 0.f, bL.y < bR.y ? 1.f : 0.f);
    F2 sl_R = mul2(mL, Slb), sl_L = sub2(Slb, sl_R);
    F2 sr_R = mul2(mR, Srb), sr_L = sub2(Srb, sr_R);
    F2 nbL = add2(sl_L, sr_L), cbL = sub2(sr_L, sl_L);
    F2 nbR = add2(sl_R, sr_R), cbR = sub2(sr_R, sl_R);
    // sound-speed derivatives, zero where p = 0 (c = 0)
    F2 hL = make_float2(pL.x > 0.f ? 0.5f * qL.x : 0.f, pL.y > 0.f ? 0.5f * qL.y : 0.f);
    F2 hR = make_float2(pR.x > 0.f ? 0.5f * qR.x : 0.f, pR.y > 0.f ? 0.5f * qR.y : 0.f);
    auto side = [&](F2 w, F2 gs, F2 r, F2 n, F2 t, F2 p, F2 E, F2 k, F2 X, F2 Y, F2 c, F2 hh, F2 nb0, F2 cb,
                    Q4& out) {
        F2 rb = mul2(gs, fma2(f3, k, X));
        rb = fma2(mul2(sp(-1.f), mul2(cb, c)), mul2(c, hh), rb);
        F2 nb = fma2(w, fma2(r, X, mul2(f3, add2(E, p))), fma2(mul2(gs, r), Y, nb0));
        F2 tb = mul2(mul2(gs, r), fma2(f3, t, f2));
        F2 pb = fma2(w, Y, fma2(mul2(gs, f3), sp(igm1), mul2(mul2(cb, g), hh)));
        out.a = add2(out.a, rb);
        out.b = add2(out.b, nb);
        out.c = add2(out.c, tb);
        out.d = add2(out.d, pb);
    };
    side(wL, gL, rL, nL, tL, pL, EL, kL, XL, YL, cL, hL, nbL, cbL, Lb);
    side(wR, gR, rR, nR, tR, pR, ER, kR, XR, YR, cR, hR, nbR, cbR, Rb);
}

struct AdjX2Args {
    const float* U;
    const float* Lout;
    const float* Extra;
    float* Lin;
    Geo2D g;
    const double* dtp;
    float alpha, beta;
    int seg_rows;  // rows per warp segment
};

__global__ void __maxnreg__(NEST_ADJX2_REGS) k2d_adjoint_x2(AdjX2Args A) {
    const Geo2D& g = A.g;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = blockIdx.x * AWARPS + warp;
    const int nx = g.nx, ny = g.ny, pitch = g.pitch;
    const int j0 = strip * ASTRIP;
    if (j0 >= ny) return;
    const int r0 = blockIdx.y * A.seg_rows;
    if (r0 >= nx) return;
    const int rows = min(A.seg_rows, nx - r0);
    const long long vs = g.vstride;
    const double dt = *A.dtp;
    const F2 lx = sp((float)(dt / g.dx)), ly = sp((float)(dt / g.dy));
    const float gamma = (float)g.gamma, gm1 = (float)(g.gamma - 1.0), igm1 = (float)(1.0 / (g.gamma - 1.0));
    const F2 half = sp(0.5f), mhalf = sp(-0.5f);

    // the lane's column pair (even first column; ny is even, so a wrapped
    // pair stays adjacent)
    const int ca = j0 - 4 + 2 * lane;
    int cw = ca % ny;
    if (cw < 0) cw += ny;
    const long long coff = cw + 2;
    const bool out_a = lane >= 2 && lane <= 29 && ca < ny;
    const bool out_b = lane >= 2 && lane <= 29 && ca + 1 < ny;
    auto wrapr = [&](int i) {
        int r = i % nx;
        return r < 0 ? r + nx : r;
    };
    auto rowoff = [&](int i) { return (long long)(wrapr(i) + 2) * pitch + coff; };
    // wrapped rows of the three streams issued at march step a (conserved
    // row a+3, Lout row a+2, Extra row a), advanced by one per step
    auto next_row = [&](int& r) { r = (r + 1 == nx) ? 0 : r + 1; };
    int ru = wrapr(r0 + 1), rl = wrapr(r0), re = wrapr(r0 - 2);

    F2* const ring = adj_ring + warp * RING_F2 + lane;
    F2* const ringU = ring;
    F2* const ringL = ring + RU * 128;
    F2* const ringE = ring + (RU + RL) * 128;
    auto issue_row = [&](const float* base, int r, F2* slot) {  // r: wrapped row
        const float* q = base + (long long)(r + 2) * pitch + coff;
        cp8(slot, q);
        cp8(slot + 32, q + vs);
        cp8(slot + 64, q + 2 * vs);
        cp8(slot + 96, q + 3 * vs);
    };
    auto rd = [&](const F2* slot) {
        Q4 q;
        q.a = slot[0]; q.b = slot[32]; q.c = slot[64]; q.d = slot[96];
        return q;
    };
    auto ld = [&](const float* base, int i) {
        const long long o = rowoff(i);
        Q4 q;
        q.a = __ldg(reinterpret_cast<const F2*>(base + o));
        q.b = __ldg(reinterpret_cast<const F2*>(base + vs + o));
        q.c = __ldg(reinterpret_cast<const F2*>(base + 2 * vs + o));
        q.d = __ldg(reinterpret_cast<const F2*>(base + 3 * vs + o));
        return q;
    };
    const bool has_extra = A.Extra != nullptr;

    // prologue: primitives of rows r0-3 .. r0-1, x-slope of row r0-2; rings:
    // conserved row r0, Lout rows r0-2 and r0-1
    Q4 Wm, W0, W1;  // rows a-1, a, a+1 at step a
    Q4 P0;          // upper face state of row a
    Q4 m1, m2;      // minmod masks of row a's x-slope
    {
        Wm = prim2(ld(A.U, r0 - 3), gm1);
        W0 = prim2(ld(A.U, r0 - 2), gm1);
        W1 = prim2(ld(A.U, r0 - 1), gm1);
        Q4 s;
        s.a = mm_mask(sub2(W0.a, Wm.a), sub2(W1.a, W0.a), m1.a, m2.a, W0.a);
        s.b = mm_mask(sub2(W0.b, Wm.b), sub2(W1.b, W0.b), m1.b, m2.b, W0.b);
        s.c = mm_mask(sub2(W0.c, Wm.c), sub2(W1.c, W0.c), m1.c, m2.c, W0.c);
        s.d = mm_mask(sub2(W0.d, Wm.d), sub2(W1.d, W0.d), m1.d, m2.d, W0.d);
        P0 = { fma2(half, s.a, W0.a), fma2(half, s.b, W0.b), fma2(half, s.c, W0.c), fma2(half, s.d, W0.d) };
        issue_row(A.U, wrapr(r0), ringU + (r0 & (RU - 1)) * 128);
        issue_row(A.Lout, wrapr(r0 - 2), ringL + ((r0 - 2) & (RL - 1)) * 128);
        issue_row(A.Lout, wrapr(r0 - 1), ringL + ((r0 - 1) & (RL - 1)) * 128);
        cp_commit();
    }
    const F2 z = sp(0.f);
    Q4 Bm = { z, z, z, z }, B0 = { z, z, z, z };  // primitive adjoints of rows a-1, a
    Q4 Sp = { z, z, z, z };                       // x-slope adjoint of row a so far

#pragma unroll AUNROLL
    for (int a = r0 - 2; a <= r0 + rows; ++a) {
        issue_row(A.U, ru, ringU + ((a + 3) & (RU - 1)) * 128);
        issue_row(A.Lout, rl, ringL + ((a + 2) & (RL - 1)) * 128);
        if (has_extra) issue_row(A.Extra, re, ringE + (a & (RE - 1)) * 128);
        next_row(ru);
        next_row(rl);
        next_row(re);
        cp_commit();
        cp_wait1();

        // row a+2, x-slope of row a+1
        Q4 W2 = prim2(rd(ringU + ((a + 2) & (RU - 1)) * 128), gm1);
        Q4 n1, n2, s1;
        s1.a = mm_mask(sub2(W1.a, W0.a), sub2(W2.a, W1.a), n1.a, n2.a, W1.a);
        s1.b = mm_mask(sub2(W1.b, W0.b), sub2(W2.b, W1.b), n1.b, n2.b, W1.b);
        s1.c = mm_mask(sub2(W1.c, W0.c), sub2(W2.c, W1.c), n1.c, n2.c, W1.c);
        s1.d = mm_mask(sub2(W1.d, W0.d), sub2(W2.d, W1.d), n1.d, n2.d, W1.d);

        // x-face a+1/2: left P0, right W1 - s1/2 (normal u, transverse v)
        Q4 L0 = rd(ringL + (a & (RL - 1)) * 128);
        Q4 L1 = rd(ringL + ((a + 1) & (RL - 1)) * 128);
        Q4 B1 = { z, z, z, z };
        {
            Q4 M1 = { fma2(mhalf, s1.a, W1.a), fma2(mhalf, s1.b, W1.b), fma2(mhalf, s1.c, W1.c),
                      fma2(mhalf, s1.d, W1.d) };
            Q4 wl = { z, z, z, z }, wr = { z, z, z, z };
            hlle2_adj(gamma, igm1, P0, M1, mul2(lx, sub2(L1.a, L0.a)), mul2(lx, sub2(L1.b, L0.b)),
                      mul2(lx, sub2(L1.c, L0.c)), mul2(lx, sub2(L1.d, L0.d)), wl, wr);
            // slope adjoint of row a is complete: sbar = wl/2 + Sp; scatter by the masks
            Q4 sb = { fma2(half, wl.a, Sp.a), fma2(half, wl.b, Sp.b), fma2(half, wl.c, Sp.c),
                      fma2(half, wl.d, Sp.d) };
            auto scat = [&](F2 s, F2 kz, F2 ke, F2& bm, F2& b0, F2& b1, F2 wl_, F2 wr_) {
                F2 u = mul2(kz, s), t2 = mul2(ke, u), t1 = sub2(u, t2);
                bm = sub2(bm, t1);
                b0 = add2(b0, add2(wl_, sub2(t1, t2)));
                b1 = add2(wr_, t2);
            };
            scat(sb.a, m1.a, m2.a, Bm.a, B0.a, B1.a, wl.a, wr.a);
            scat(sb.b, m1.b, m2.b, Bm.b, B0.b, B1.b, wl.b, wr.b);
            scat(sb.c, m1.c, m2.c, Bm.c, B0.c, B1.c, wl.c, wr.c);
            scat(sb.d, m1.d, m2.d, Bm.d, B0.d, B1.d, wl.d, wr.d);
            Sp = { mul2(mhalf, wr.a), mul2(mhalf, wr.b), mul2(mhalf, wr.c), mul2(mhalf, wr.d) };
        }

        // y-direction part of row a (only output rows need it)
        if (a >= r0 && a < r0 + rows) {
            Q4 ym1, ym2, P, R;
            Q4 Lr;  // Lout of the next lane's first column
            auto yvar = [&](F2 w, F2& k1, F2& k2, F2& p, F2& rr) {
                float lb = __shfl_up_sync(0xffffffffu, w.y, 1);
                float ra = __shfl_down_sync(0xffffffffu, w.x, 1);
                F2 s = mm_mask(sub2(w, make_float2(lb, w.x)), sub2(make_float2(w.y, ra), w), k1, k2, w);
                p = fma2(half, s, w);
                F2 m = fma2(mhalf, s, w);
                rr = make_float2(m.y, __shfl_down_sync(0xffffffffu, m.x, 1));
            };
            yvar(W0.a, ym1.a, ym2.a, P.a, R.a);
            yvar(W0.b, ym1.b, ym2.b, P.b, R.b);
            yvar(W0.c, ym1.c, ym2.c, P.c, R.c);
            yvar(W0.d, ym1.d, ym2.d, P.d, R.d);
            Lr.a = make_float2(L0.a.y, __shfl_down_sync(0xffffffffu, L0.a.x, 1));
            Lr.b = make_float2(L0.b.y, __shfl_down_sync(0xffffffffu, L0.b.x, 1));
            Lr.c = make_float2(L0.c.y, __shfl_down_sync(0xffffffffu, L0.c.x, 1));
            Lr.d = make_float2(L0.d.y, __shfl_down_sync(0xffffffffu, L0.d.x, 1));
            // faces (a|b, b|a'): normal v, transverse u; flux order (mass, mv, mu, E)
            Q4 PL = { P.a, P.c, P.b, P.d }, RR = { R.a, R.c, R.b, R.d };
            Q4 wl = { z, z, z, z }, wr = { z, z, z, z };
            hlle2_adj(gamma, igm1, PL, RR, mul2(ly, sub2(Lr.a, L0.a)), mul2(ly, sub2(Lr.c, L0.c)),
                      mul2(ly, sub2(Lr.b, L0.b)), mul2(ly, sub2(Lr.d, L0.d)), wl, wr);
            // back to (rho, u, v, p): wl/wr .b is the normal (v), .c the transverse (u)
            auto ycell = [&](F2 l, F2 r, F2 k1, F2 k2, F2& b) {
                // right-state adjoint of the face on the cell's left: for the
                // first column from the left lane's second face
                F2 q = make_float2(__shfl_up_sync(0xffffffffu, r.y, 1), r.x);
                F2 sb = mul2(half, sub2(l, q));
                F2 u = mul2(k1, sb), t2 = mul2(k2, u), t1 = sub2(u, t2);
                F2 t1n = make_float2(t1.y, __shfl_down_sync(0xffffffffu, t1.x, 1));
                F2 t2p = make_float2(__shfl_up_sync(0xffffffffu, t2.y, 1), t2.x);
                b = add2(b, add2(add2(l, q), add2(sub2(t1, t2), sub2(t2p, t1n))));
            };
            ycell(wl.a, wr.a, ym1.a, ym2.a, B0.a);
            ycell(wl.c, wr.c, ym1.b, ym2.b, B0.b);
            ycell(wl.b, wr.b, ym1.c, ym2.c, B0.c);
            ycell(wl.d, wr.d, ym1.d, ym2.d, B0.d);
        }

        // row a-1 is complete
        if (a - 1 >= r0 && out_a) {
            Q4 Lm = rd(ringL + ((a - 1) & (RL - 1)) * 128);
            F2 ir = rcp2(Wm.a);
            F2 u = Wm.b, v = Wm.c;
            F2 g3 = mul2(sp(gm1), Bm.d);
            g3 = make_float2(Wm.d.x > 0.f ? g3.x : 0.f, Wm.d.y > 0.f ? g3.y : 0.f);
            F2 q2 = mul2(half, fma2(v, v, mul2(u, u)));
            Q4 o;
            o.a = fma2(g3, q2, sub2(Bm.a, mul2(fma2(Bm.c, v, mul2(Bm.b, u)), ir)));
            o.b = sub2(mul2(Bm.b, ir), mul2(g3, u));
            o.c = sub2(mul2(Bm.c, ir), mul2(g3, v));
            o.d = g3;
            const F2 al = sp(A.alpha);
            o.a = mul2(al, add2(Lm.a, o.a));
            o.b = mul2(al, add2(Lm.b, o.b));
            o.c = mul2(al, add2(Lm.c, o.c));
            o.d = mul2(al, add2(Lm.d, o.d));
            if (has_extra) {
                Q4 E = rd(ringE + ((a - 1) & (RE - 1)) * 128);
                const F2 be = sp(A.beta);
                o.a = fma2(be, E.a, o.a);
                o.b = fma2(be, E.b, o.b);
                o.c = fma2(be, E.c, o.c);
                o.d = fma2(be, E.d, o.d);
            }
            const long long off = (long long)(a - 1 + 2) * pitch + ca + 2;
            if (out_b) {
                *reinterpret_cast<F2*>(A.Lin + off) = o.a;
                *reinterpret_cast<F2*>(A.Lin + vs + off) = o.b;
                *reinterpret_cast<F2*>(A.Lin + 2 * vs + off) = o.c;
                *reinterpret_cast<F2*>(A.Lin + 3 * vs + off) = o.d;
            } else {
                A.Lin[off] = o.a.x;
                A.Lin[vs + off] = o.b.x;
                A.Lin[2 * vs + off] = o.c.x;
                A.Lin[3 * vs + off] = o.d.x;
            }
        }

        // advance the window
        Wm = W0; W0 = W1; W1 = W2;
        P0 = { fma2(half, s1.a, W0.a), fma2(half, s1.b, W0.b), fma2(half, s1.c, W0.c), fma2(half, s1.d, W0.d) };
        m1 = n1; m2 = n2;
        Bm = B0; B0 = B1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

}  // namespace

// Packed row-march form of the FP32 2D adjoint stage; cudaErrorNotSupported
// (nothing launched) for an odd ny, whose wrapped column pairs would not be
// adjacent: the caller then uses the tile kernel.
cudaError_t launch_2d_adjoint_stage_f32x2(const float* U, const float* Lout, const float* Extra, float* Lin,
                                          const Geo2D& g, const double* dtp, double alpha, double beta,
                                          cudaStream_t st) {
    if ((g.ny & 1) || g.pitch % 2 != 0) return cudaErrorNotSupported;
    const size_t smem = sizeof(F2) * RING_F2 * AWARPS;
    // per-device launch facts, looked up once (SM count, resident CTAs)
    constexpr int MAXDEV = 64;
    static std::mutex mu;
    static int dev_sms[MAXDEV] = {}, dev_per_sm[MAXDEV] = {};
    int dev = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    int sms = 0, per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < MAXDEV && dev_sms[dev] > 0) {
            sms = dev_sms[dev];
            per_sm = dev_per_sm[dev];
        } else {
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k2d_adjoint_x2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
                return e;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2d_adjoint_x2, 32 * AWARPS, smem)) !=
                cudaSuccess)
                return e;
            if (per_sm < 1) per_sm = 1;
            if (dev < MAXDEV) {
                dev_sms[dev] = sms;
                dev_per_sm[dev] = per_sm;
            }
        }
    }
    const int strips = (g.ny + ASTRIP - 1) / ASTRIP;
    const int cx = (strips + AWARPS - 1) / AWARPS;
    // enough row segments for one wave of resident warps, at least 16 rows each
    const long long slots = (long long)sms * per_sm * AWARPS;
    int segs = (int)std::max<long long>(1, slots / ((long long)cx * AWARPS));
    int seg_rows = (g.nx + segs - 1) / segs;
    if (seg_rows < 16) seg_rows = 16;
    segs = (g.nx + seg_rows - 1) / seg_rows;
    AdjX2Args a{ U, Lout, Extra, Lin, g, dtp, (float)alpha, (float)beta, seg_rows };
    k2d_adjoint_x2<<<dim3(cx, segs), 32 * AWARPS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace nestb
