// FP32 form of the 2D stage kernels with packed FP32x2 arithmetic (sm_100a).
//
// Each lane owns two adjacent columns (a, b) and keeps every quantity as a
// float2 pair, so the reconstruction, both HLLE fluxes and the update run on
// the FFMA2/FADD2/FMUL2 instructions of sm_100 (one issue slot per two
// cells).  A warp covers 64 columns j0-2 .. j0+61 and writes 60 of them
// (lanes 1..30; lanes 0 and 31 only feed their neighbours), marching down a
// tile of rows with a three-row register window exactly like the scalar
// kernel in euler2d_kernels.cuh.  Per lane and row:
//   * 64-bit loads/stores of the (a, b) pair of each variable,
//   * x-faces: one packed HLLE for the faces under columns a and b,
//   * y-faces: one packed HLLE for the faces a|b and b|a' (a' = next lane's
//     first column), with 2 + 1 + 1 shuffles per variable.
// Minmod is median(0, a, b) = max(min(a, b), min(max(a, b), 0)), which equals
// nest's minmod (euler1d.hpp:112-115) without a multiply or branch.
// Compiled with -use_fast_math: reciprocal and rsqrt are single MUFU ops.
#include "euler2d_kernels.cuh"
#include "kernels.h"

namespace nestb {
namespace {

constexpr int STRIP2 = 60;  // output columns per warp

using F2 = float2;

__device__ __forceinline__ F2 sp(float a) { return make_float2(a, a); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 sub2(F2 a, F2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ F2 rcp2(F2 a) { return make_float2(__fdividef(1.f, a.x), __fdividef(1.f, a.y)); }
__device__ __forceinline__ F2 rsq2(F2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ F2 max2(F2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }
__device__ __forceinline__ F2 min2(F2 a, float b) { return make_float2(fminf(a.x, b), fminf(a.y, b)); }
__device__ __forceinline__ F2 vmax2(F2 a, F2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ F2 vmin2(F2 a, F2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }

__device__ __forceinline__ float mm(float a, float b) { return fmaxf(fminf(a, b), fminf(fmaxf(a, b), 0.f)); }
__device__ __forceinline__ F2 mm2(F2 a, F2 b) { return make_float2(mm(a.x, b.x), mm(a.y, b.y)); }

struct Q4 { F2 a, b, c, d; };  // four variables, each a column pair

// cons -> prim on a pair: (rho, mu, mv, E) -> (rho, u, v, p), p >= 0.
template <bool REPAIR>
__device__ __forceinline__ Q4 prim2(const Q4& U, float gm1) {
    Q4 w;
    F2 ir = rcp2(U.a);
    w.a = U.a;
    w.b = mul2(U.b, ir);
    w.c = mul2(U.c, ir);
    F2 ke = mul2(mul2(sp(0.5f), U.a), fma2(w.c, w.c, mul2(w.b, w.b)));
    w.d = max2(mul2(sp(gm1), sub2(U.d, ke)), 0.f);
    if (REPAIR) {
        const float fl = 1e-10f;
        if (!(w.a.x >= fl) || !(w.d.x >= fl) || !(w.a.y >= fl) || !(w.d.y >= fl)) {
            Prim4<float> p0 = cons2prim<float, true>(U.a.x, U.b.x, U.c.x, U.d.x, gm1);
            Prim4<float> p1 = cons2prim<float, true>(U.a.y, U.b.y, U.c.y, U.d.y, gm1);
            w.a = make_float2(p0.r, p1.r); w.b = make_float2(p0.u, p1.u);
            w.c = make_float2(p0.v, p1.v); w.d = make_float2(p0.p, p1.p);
        }
    }
    return w;
}

// Packed four-variable HLLE along the normal (states (rho, un, ut, p)),
// branchless form of euler1d.hpp:178-242 with Davis speeds.
__device__ __forceinline__ void hlle2(float gamma, float igm1,
                                      F2 rL, F2 nL, F2 tL, F2 pL, F2 rR, F2 nR, F2 tR, F2 pR,
                                      F2& f0, F2& f1, F2& f2, F2& f3) {
    F2 g = sp(gamma), h = sp(0.5f);
    F2 gpL = mul2(g, pL), gpR = mul2(g, pR);
    F2 cL = mul2(gpL, rsq2(max2(mul2(gpL, rL), 1e-37f)));
    F2 cR = mul2(gpR, rsq2(max2(mul2(gpR, rR), 1e-37f)));
    F2 EL = fma2(pL, sp(igm1), mul2(mul2(h, rL), fma2(tL, tL, mul2(nL, nL))));
    F2 ER = fma2(pR, sp(igm1), mul2(mul2(h, rR), fma2(tR, tR, mul2(nR, nR))));
    F2 SL = vmin2(sub2(nL, cL), sub2(nR, cR));
    F2 SR = vmax2(add2(nL, cL), add2(nR, cR));
    F2 mL = mul2(rL, nL), mR = mul2(rR, nR);
    F2 sl = min2(SL, 0.f), sr = max2(SR, 0.f);
    F2 inv = rcp2(max2(sub2(sr, sl), 1e-30f));
    F2 A = mul2(sr, inv);
    F2 B = mul2(make_float2(-sl.x, -sl.y), inv);  // -sl / (sr - sl)
    F2 Cc = mul2(mul2(sl, sr), inv);
    // f = A FL + B FR + Cc (UR - UL)
    f0 = fma2(Cc, sub2(rR, rL), fma2(A, mL, mul2(B, mR)));
    f1 = fma2(Cc, sub2(mR, mL), fma2(A, fma2(mL, nL, pL), mul2(B, fma2(mR, nR, pR))));
    f2 = fma2(Cc, sub2(mul2(rR, tR), mul2(rL, tL)), fma2(A, mul2(mL, tL), mul2(B, mul2(mR, tR))));
    f3 = fma2(Cc, sub2(ER, EL), fma2(A, mul2(add2(EL, pL), nL), mul2(B, mul2(add2(ER, pR), nR))));
}

__device__ __forceinline__ Q4 minmod_pair(const Q4& m, const Q4& o, const Q4& p) {
    return { mm2(sub2(o.a, m.a), sub2(p.a, o.a)), mm2(sub2(o.b, m.b), sub2(p.b, o.b)),
             mm2(sub2(o.c, m.c), sub2(p.c, o.c)), mm2(sub2(o.d, m.d), sub2(p.d, o.d)) };
}

// y-slopes of the lane's pair (a, b) from the left neighbour's b and the right
// neighbour's a.
__device__ __forceinline__ F2 yslope(F2 w) {
    float lb = __shfl_up_sync(0xffffffffu, w.y, 1);
    float ra = __shfl_down_sync(0xffffffffu, w.x, 1);
    F2 e = sub2(w, make_float2(lb, w.x));  // (a - left, b - a)
    return make_float2(mm(e.x, e.y), mm(e.y, ra - w.y));
}

// One warp's work: the rows of tile `tile_row` under column strip `strip`.
// The warp owning strip 0 / tile 0 publishes the step's dt for the domain.
template <int STAGE, bool REPAIR>
__device__ __forceinline__ void x2_body(const StageArgs<float>& a, int strip, int tile_row) {
    const Geo2D& g = a.g;
    const int lane = threadIdx.x & 31;
    const float gamma = (float)g.gamma;
    const float gm1 = (float)(g.gamma - 1.0);
    const float igm1 = (float)(1.0 / (g.gamma - 1.0));

    double dt;
    if (STAGE == 1) {
        bool done = step_is_done(a.ctrl, a.p, a.lp);
        double pd = done ? -1.0 : prescribed_dt(a.ctrl, a.p, a.lp);
        if (pd > 0.0) {
            dt = pd;
        } else {
            dt = dt_from_speeds(bits_speed(a.ctrl->maxs[a.p][0]), bits_speed(a.ctrl->maxs[a.p][1]),
                                g.dx, g.dy, a.lp.cfl);
            if (a.lp.t_final > 0.0) dt = smin(dt, a.lp.t_final - a.ctrl->time[a.p]);
        }
        if (strip == 0 && tile_row == 0 && lane == 0) publish_step(a.ctrl, a.p, a.lp, done, dt);
        if (done) return;
    } else {
        if (!a.ctrl->active[a.p]) return;
        dt = a.ctrl->dt[a.p];
    }
    const float dtdx = (float)(dt / g.dx);
    const float dtdy = (float)(dt / g.dy);

    const int j0 = strip * STRIP2;
    if (j0 >= g.ny) return;  // whole warp idle
    const int ca = j0 - 2 + 2 * lane;  // first of the lane's two columns
    // element offset of the pair within a row; pairs past the ghost ring read
    // the row padding (finite, discarded)
    const int coff = min(ca + 2, g.pitch - 2);
    const bool lane_out = lane >= 1 && lane <= 30;
    const bool out_a = lane_out && ca < g.ny;
    const bool out_b = lane_out && ca + 1 < g.ny;
    const int i0 = tile_row * a.tx;
    if (i0 >= g.nx) return;
    const int rows = min(a.tx, g.nx - i0);
    const long long vs = g.vstride;
    const float* __restrict__ Ui = a.Uin;

    auto load = [&](int i, Q4& q) {
        const long long o = (long long)(i + 2) * g.pitch + coff;
        q.a = __ldg(reinterpret_cast<const F2*>(Ui + o));
        q.b = __ldg(reinterpret_cast<const F2*>(Ui + vs + o));
        q.c = __ldg(reinterpret_cast<const F2*>(Ui + 2 * vs + o));
        q.d = __ldg(reinterpret_cast<const F2*>(Ui + 3 * vs + o));
    };

    // Window entering iteration r: W0 = W(r-2), W1 = W(r-1) (primitives),
    // P0 = W(r-2) + S(r-2)/2 (upper x-face state of row r-2), Fp = x-flux of
    // face r-5/2.  The conserved values of the row being updated are re-read
    // from L1 (they were loaded two iterations earlier); stage 2's U^n row is
    // requested at the top of the iteration, ahead of the flux work.
    Q4 W0, W1, P0, Fp, nxt, un;
    float smx = 0.f, smy = 0.f;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    const F2 half = sp(0.5f), mhalf = sp(-0.5f);
    const float* Unp = a.Un;
    auto load_un = [&](int i, Q4& q) {
        const long long o = (long long)(i + 2) * g.pitch + coff;
        q.a = *reinterpret_cast<const F2*>(Unp + o);
        q.b = *reinterpret_cast<const F2*>(Unp + vs + o);
        q.c = *reinterpret_cast<const F2*>(Unp + 2 * vs + o);
        q.d = *reinterpret_cast<const F2*>(Unp + 3 * vs + o);
    };

    load(i0 - 2, nxt);
    for (int r = -2; r <= rows + 1; ++r) {
        Q4 cur = nxt;
        if (r + 1 <= rows + 1) load(i0 + r + 1, nxt);
        Q4 C0;
        if (r >= 2) {
            load(i0 + r - 2, C0);  // L1 hit: loaded as `cur` two iterations ago
            if (STAGE == 2) load_un(i0 + r - 2, un);  // used after this iteration's flux work
        }
        Q4 W2 = prim2<REPAIR>(cur, gm1);
        Q4 P1, M1;
        if (r >= 0) {
            Q4 S1 = minmod_pair(W0, W1, W2);  // x-slope of row r-1
            P1 = { fma2(half, S1.a, W1.a), fma2(half, S1.b, W1.b), fma2(half, S1.c, W1.c), fma2(half, S1.d, W1.d) };
            M1 = { fma2(mhalf, S1.a, W1.a), fma2(mhalf, S1.b, W1.b), fma2(mhalf, S1.c, W1.c), fma2(mhalf, S1.d, W1.d) };
        }
        if (r >= 1) {
            // x-faces between rows r-2 and r-1 under both columns
            Q4 Fc;
            hlle2(gamma, igm1, P0.a, P0.b, P0.c, P0.d, M1.a, M1.b, M1.c, M1.d, Fc.a, Fc.b, Fc.c, Fc.d);
            if (r >= 2) {
                const int i = i0 + r - 2;
                // y-faces on row i: (a|b, b|a') with normal v, transverse u
                Q4 sy = { yslope(W0.a), yslope(W0.b), yslope(W0.c), yslope(W0.d) };
                Q4 M = { fma2(mhalf, sy.a, W0.a), fma2(mhalf, sy.b, W0.b), fma2(mhalf, sy.c, W0.c), fma2(mhalf, sy.d, W0.d) };
                Q4 R;
                R.a = make_float2(M.a.y, __shfl_down_sync(0xffffffffu, M.a.x, 1));
                R.b = make_float2(M.b.y, __shfl_down_sync(0xffffffffu, M.b.x, 1));
                R.c = make_float2(M.c.y, __shfl_down_sync(0xffffffffu, M.c.x, 1));
                R.d = make_float2(M.d.y, __shfl_down_sync(0xffffffffu, M.d.x, 1));
                Q4 G;  // G.b = mu flux (transverse), G.c = mv flux (normal)
                hlle2(gamma, igm1,
                      fma2(half, sy.a, W0.a), fma2(half, sy.c, W0.c), fma2(half, sy.b, W0.b), fma2(half, sy.d, W0.d),
                      R.a, R.c, R.b, R.d,
                      G.a, G.c, G.b, G.d);
                // G(face a-1/2) from the left lane's G(b+1/2)
                Q4 dG;
                dG.a = sub2(G.a, make_float2(__shfl_up_sync(0xffffffffu, G.a.y, 1), G.a.x));
                dG.b = sub2(G.b, make_float2(__shfl_up_sync(0xffffffffu, G.b.y, 1), G.b.x));
                dG.c = sub2(G.c, make_float2(__shfl_up_sync(0xffffffffu, G.c.y, 1), G.c.x));
                dG.d = sub2(G.d, make_float2(__shfl_up_sync(0xffffffffu, G.d.y, 1), G.d.x));
                if (out_a) {
                    const F2 fx = sp(dtdx), fy = sp(dtdy);
                    Q4 s;
                    s.a = sub2(C0.a, fma2(fx, sub2(Fc.a, Fp.a), mul2(fy, dG.a)));
                    s.b = sub2(C0.b, fma2(fx, sub2(Fc.b, Fp.b), mul2(fy, dG.b)));
                    s.c = sub2(C0.c, fma2(fx, sub2(Fc.c, Fp.c), mul2(fy, dG.c)));
                    s.d = sub2(C0.d, fma2(fx, sub2(Fc.d, Fp.d), mul2(fy, dG.d)));
                    const long long o = (long long)(i + 2) * g.pitch + (ca + 2);
                    if (STAGE == 2) {
                        const F2 n0 = un.a, n1 = un.b, n2 = un.c, n3 = un.d;
                        s.a = mul2(half, add2(n0, s.a));
                        s.b = mul2(half, add2(n1, s.b));
                        s.c = mul2(half, add2(n2, s.c));
                        s.d = mul2(half, add2(n3, s.d));
                        if (REPAIR) {
                            // FP64 positivity repair, element by element (rare)
                            auto fix = [&](float& r0, float& m1, float& m2, float& e3) {
                                const double fl = 1e-10;
                                double r_ = (double)r0, rr = smax(r_, fl);
                                double u_ = (double)m1 / rr, v_ = (double)m2 / rr;
                                double keD = 0.5 * rr * (u_ * u_ + v_ * v_);
                                double pD = (g.gamma - 1.0) * ((double)e3 - keD);
                                if (!(r_ >= fl) || !(pD >= fl)) {
                                    r0 = (float)rr;
                                    e3 = (float)smax((double)e3, keD + fl / (g.gamma - 1.0));
                                    atomicAdd(&a.ctrl->repairs, 1u);
                                }
                            };
                            fix(s.a.x, s.b.x, s.c.x, s.d.x);
                            if (out_b) fix(s.a.y, s.b.y, s.c.y, s.d.y);
                        }
                        // wave speeds |u|+c, |v|+c with the floors of compute_dt_2d
                        F2 rho = max2(s.a, 1e-10f);
                        F2 ir = rcp2(rho);
                        F2 u = mul2(s.b, ir), v = mul2(s.c, ir);
                        F2 ke = mul2(mul2(half, rho), fma2(v, v, mul2(u, u)));
                        F2 pp = max2(mul2(sp(gm1), sub2(s.d, ke)), 1e-10f);
                        F2 gp = mul2(sp(gamma), pp);
                        F2 c = mul2(gp, rsq2(mul2(gp, rho)));
                        smx = fmaxf(smx, fabsf(u.x) + c.x);
                        smy = fmaxf(smy, fabsf(v.x) + c.x);
                        if (out_b) {
                            smx = fmaxf(smx, fabsf(u.y) + c.y);
                            smy = fmaxf(smy, fabsf(v.y) + c.y);
                        }
                        if (a.partials) {
                            t0 += (double)s.a.x; t1 += (double)s.b.x; t2 += (double)s.c.x; t3 += (double)s.d.x;
                            if (out_b) {
                                t0 += (double)s.a.y; t1 += (double)s.b.y; t2 += (double)s.c.y; t3 += (double)s.d.y;
                            }
                        }
                    }
                    float* Uo = a.Uout;
                    if (out_b) {
                        *reinterpret_cast<F2*>(Uo + o) = s.a;
                        *reinterpret_cast<F2*>(Uo + vs + o) = s.b;
                        *reinterpret_cast<F2*>(Uo + 2 * vs + o) = s.c;
                        *reinterpret_cast<F2*>(Uo + 3 * vs + o) = s.d;
                    } else {
                        Uo[o] = s.a.x; Uo[vs + o] = s.b.x; Uo[2 * vs + o] = s.c.x; Uo[3 * vs + o] = s.d.x;
                    }
                    if (i < 2 || i >= g.nx - 2 || ca < 2 || ca + 1 >= g.ny - 2) {
                        store_ghosts(Uo, g, 0, i, ca, s.a.x); store_ghosts(Uo, g, 1, i, ca, s.b.x);
                        store_ghosts(Uo, g, 2, i, ca, s.c.x); store_ghosts(Uo, g, 3, i, ca, s.d.x);
                        if (out_b) {
                            store_ghosts(Uo, g, 0, i, ca + 1, s.a.y); store_ghosts(Uo, g, 1, i, ca + 1, s.b.y);
                            store_ghosts(Uo, g, 2, i, ca + 1, s.c.y); store_ghosts(Uo, g, 3, i, ca + 1, s.d.y);
                        }
                    }
                }
            }
            Fp = Fc;
        }
        W0 = W1; W1 = W2; P0 = P1;
    }
    if (STAGE == 2) {
        double mx = warp_max((double)smx), my = warp_max((double)smy);
        if (lane == 0) {
            if (!(mx == mx) || !(my == my) || mx > 1.79e308 || my > 1.79e308) atomicOr(&a.ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][0], mx);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][1], my);
        }
        if (a.partials) {
            t0 = warp_sum(t0); t1 = warp_sum(t1); t2 = warp_sum(t2); t3 = warp_sum(t3);
            if (lane == 0) {
                long long wid = ((long long)tile_row * ((g.ny + STRIP2 - 1) / STRIP2) + strip) * 4;  // per-domain slot
                a.partials[wid + 0] = t0; a.partials[wid + 1] = t1;
                a.partials[wid + 2] = t2; a.partials[wid + 3] = t3;
            }
        }
    }
}

// Register budgets of the plain (no repair) stage kernels, from a sweep at
// 4096^2 (B200, 16-row tiles, one warp per block): stage 2 under
// __launch_bounds__(256) alone measured 0.341 ms per launch; with an explicit
// budget of 120-128 it measured 0.243-0.247 ms, and 0.35 ms again at 118 and
// below.  Stage 1 measured 0.218-0.220 ms for every budget from 116 to 128.
#ifndef NEST_X2_REGS1
#define NEST_X2_REGS1 128
#endif
#ifndef NEST_X2_REGS2
#define NEST_X2_REGS2 124
#endif

__global__ void __maxnreg__(NEST_X2_REGS1) k2d_f32x2_1(StageArgs<float> a) {
    x2_body<1, false>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}
__global__ void __maxnreg__(NEST_X2_REGS2) k2d_f32x2_2(StageArgs<float> a) {
    x2_body<2, false>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

// Positivity-repair variants (FP64 repair branch; rarely taken).
template <int STAGE>
__global__ void __launch_bounds__(256) k2d_f32x2_repair(StageArgs<float> a) {
    x2_body<STAGE, true>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

// Out-of-line copy of the per-warp body for the batched loop: keeping the
// work-list loop's state out of the body's register allocation halves the
// batched kernel's register count (about 128 instead of about 195).
template <int STAGE, bool REPAIR>
__device__ __noinline__ void x2_body_call(const StageArgs<float>& a, int strip, int tile_row) {
    x2_body<STAGE, REPAIR>(a, strip, tile_row);
}

// Persistent batched stage: every warp walks the work list (problem, strip,
// tile row) with a stride of the whole grid's warp count.
template <int STAGE, bool REPAIR>
__global__ void __launch_bounds__(256) kbatch_f32x2(BatchArgs<float> b) {
    const int nw = gridDim.x * blockDim.y;
    for (int it = blockIdx.x * blockDim.y + threadIdx.y; it < b.nitems; it += nw) {
        const int4 w = b.items[it];
        const BatchProblem& P = b.probs[w.x];
        StageArgs<float> a{STAGE == 1 ? b.U + P.off : b.U1 + P.off, STAGE == 2 ? b.U + P.off : nullptr,
                           STAGE == 1 ? b.U1 + P.off : b.U + P.off, P.g, b.lp, b.ctrls + w.x,
                           (STAGE == 2 && b.partials) ? b.partials + 4ll * P.item0 : nullptr, b.p, b.tx};
        x2_body_call<STAGE, REPAIR>(a, w.y, w.z);
    }
}

}  // namespace

int strips_f32x2(int ny) { return (ny + STRIP2 - 1) / STRIP2; }

cudaError_t launch_batch_f32x2(const BatchArgs<float>& b, bool repair, int which, int blocks, int warps,
                               cudaStream_t st) {
    dim3 blk(32, warps);
    BatchArgs<float> b1 = b, b2 = b;
    if (repair) {
        if (which & 1) kbatch_f32x2<1, true><<<blocks, blk, 0, st>>>(b1);
        if (which & 2) kbatch_f32x2<2, true><<<blocks, blk, 0, st>>>(b2);
    } else {
        if (which & 1) kbatch_f32x2<1, false><<<blocks, blk, 0, st>>>(b1);
        if (which & 2) kbatch_f32x2<2, false><<<blocks, blk, 0, st>>>(b2);
    }
    return cudaGetLastError();
}

int batch_max_blocks_f32x2(int warps) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kbatch_f32x2<2, false>, 32 * warps, 0);
    return nb;
}

cudaError_t launch_2d_step_f32x2(float* U, float* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl,
                                 double* partials, int p, int tx, int warps, bool repair, int which,
                                 cudaStream_t st, float* Uout) {
    int nstrips = strips_f32x2(g.ny);
    dim3 b(32, warps), gr((nstrips + warps - 1) / warps, (g.nx + tx - 1) / tx);
    StageArgs<float> a1{U, nullptr, U1, g, lp, ctrl, nullptr, p, tx};
    StageArgs<float> a2{U1, U, Uout ? Uout : U, g, lp, ctrl, partials, p, tx};
    if (repair) {
        if (which & 1) k2d_f32x2_repair<1><<<gr, b, 0, st>>>(a1);
        if (which & 2) k2d_f32x2_repair<2><<<gr, b, 0, st>>>(a2);
    } else {
        if (which & 1) k2d_f32x2_1<<<gr, b, 0, st>>>(a1);
        if (which & 2) k2d_f32x2_2<<<gr, b, 0, st>>>(a2);
    }
    return cudaGetLastError();
}

}  // namespace nestb
