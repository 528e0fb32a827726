// FP32 form of the 2D stage kernels with packed FP32x2 arithmetic (sm_100a).
//
// Each lane owns two adjacent columns (a, b) and keeps every quantity as a
// float2 pair, so the reconstruction, both HLLE fluxes and the update run on
// the FFMA2/FADD2/FMUL2 instructions of sm_100 (one issue slot per two
// cells).  A warp covers 64 columns j0-2 .. j0+61 and writes 60 of them
// (lanes 1..30; lanes 0 and 31 only feed their neighbours), marching down a
// tile of rows with a three-row register window like the scalar kernel in
// euler2d_kernels.cuh.  Per lane and row:
//   * input rows staged through shared memory by 16-byte cp.async copies
//     (see x2_body), read back and stored as the lane's 64-bit (a, b) pair of
//     each variable,
//   * x-faces: one packed HLLE for the faces under columns a and b,
//   * y-faces: one packed HLLE for the faces a|b and b|a' (a' = next lane's
//     first column), with 2 + 1 + 1 shuffles per variable.
// Minmod takes three ALU operations (min.xorsign.abs, max, copysign) and the
// HLLE flux is written in relative-flux form with dt/dx folded into its
// weights (hlle2 below).
// Compiled with -use_fast_math: reciprocal and rsqrt are single MUFU ops.
#include "euler2d_kernels.cuh"
#include "f2ops.cuh"
#include "kernels.h"

namespace nestb {
namespace {

constexpr int STRIP2 = 60;  // output columns per warp

// nest's minmod (euler1d.hpp:112-115) in three ALU operations:
// min.xorsign.abs gives min(|a|, |b|) carrying the sign sign(a) xor sign(b),
// negative exactly when the signs differ; max(., 0) zeroes that case and
// copysign restores sign(a).  Only the sign of a zero result can differ.
__device__ __forceinline__ float mm(float a, float b) {
    float t;
    asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(t) : "f"(a), "f"(b));
    return copysignf(fmaxf(t, 0.f), a);
}
__device__ __forceinline__ F2 mm2(F2 a, F2 b) { return make_float2(mm(a.x, b.x), mm(a.y, b.y)); }

// Three-input max (sm_100).
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float t;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(t) : "f"(a), "f"(b), "f"(c));
    return t;
}

struct Q4 { F2 a, b, c, d; };  // four variables, each a column pair

__device__ __forceinline__ Q4 q_fma(F2 h, const Q4& s, const Q4& w) {
    return { fma2(h, s.a, w.a), fma2(h, s.b, w.b), fma2(h, s.c, w.c), fma2(h, s.d, w.d) };
}

// Asynchronous global -> shared copy of 16 bytes (cp.async, L2 only): four
// consecutive columns of one variable.  A copy holds no registers while in
// flight.
__device__ __forceinline__ void cp16(F2* smem_dst, const float* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared-memory row rings of one warp: RING_U slots of the stage input and,
// in stage 2, RING_N slots of U^n; a slot holds the warp's 64-column row
// segment of the four variables, [var][64 columns], filled by 16-byte copies
// (two per lane) and read as one column pair per lane.
// LOOK: rows of the stage input in flight ahead of the row march (the row
// issued at iteration i is consumed at iteration i + LOOK - 2); U^n runs
// LOOK - 2 rows ahead.  Measured at 4096^2: LOOK 3 0.386 ms per step, 4 and
// 5 (8-slot rings) 0.437 / 0.443 ms (the larger rings cost warps per SM).
constexpr int LOOK = 3;
constexpr int RING_U = 4, RING_N = 2;
static_assert(RING_U >= LOOK + 1 && RING_N >= LOOK - 1, "ring too small for the lookahead");
__host__ __device__ constexpr int ring_f2_per_warp(int stage) { return (RING_U + (stage == 2 ? RING_N : 0)) * 4 * 32; }
extern __shared__ __align__(16) F2 x2_ring[];

// 1/x for a positive double x that is an FP32 value of at least 1e-10:
// Newton-Raphson iteration y <- y + y (1 - x y), which doubles the number of
// correct bits per step, from the ~22-bit FP32 approximate reciprocal; two
// steps reach double precision (to within an ulp or two).  Unlike a
// division it needs no out-of-line slow path, so the rare FP64 branches
// below leave the row loop free of calls.
__device__ __forceinline__ double rcp_nr(double x) {
    double y = (double)__fdividef(1.0f, (float)x);
    y = fma(y, fma(-x, y, 1.0), y);
    return fma(y, fma(-x, y, 1.0), y);
}

// FP64 primitives of one cell with the 1e-10 floors on rho and p (the FP32
// form's near-vacuum path).
__device__ __forceinline__ Prim4<float> prim_floor64(float U0, float U1, float U2, float U3, float gm1) {
    const double fl = 1e-10;
    double r = smax((double)U0, fl), ir = rcp_nr(r);
    double u = (double)U1 * ir, v = (double)U2 * ir;
    double pd = (double)gm1 * ((double)U3 - (0.5 * r * u * u + 0.5 * r * v * v));
    return { (float)r, (float)u, (float)v, (float)smax(pd, fl) };
}

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
        // one compare on the smallest of the four (min.NaN keeps a NaN); the
        // vote over the active lanes keeps the rare FP64 path a real branch
        float m;
        asm("min.NaN.f32 %0, %1, %2, %3;" : "=f"(m) : "f"(w.a.x), "f"(w.a.y), "f"(w.d.x));
        asm("min.NaN.f32 %0, %1, %2;" : "=f"(m) : "f"(m), "f"(w.d.y));
        const bool need = !(m >= fl);
        if (__any_sync(__activemask(), need) && need) {
            Prim4<float> p0 = prim_floor64(U.a.x, U.b.x, U.c.x, U.d.x, gm1);
            Prim4<float> p1 = prim_floor64(U.a.y, U.b.y, U.c.y, U.d.y, gm1);
            w.a = make_float2(p0.r, p1.r); w.b = make_float2(p0.u, p1.u);
            w.c = make_float2(p0.v, p1.v); w.d = make_float2(p0.p, p1.p);
        }
    }
    return w;
}

// Packed four-variable HLLE along the normal (states (rho, un, ut, p)) with
// Davis speeds, euler1d.hpp:178-242, returning the flux times `scale`.
// Written in relative-flux form: with sl = min(S_L, 0), sr = max(S_R, 0),
//   F = [sr (F_L - sl U_L) - sl (F_R - sr U_R)] / (sr - sl),
// which is the HLLE average in the subsonic case and reduces to F_L
// (sl = 0) or F_R (sr = 0) in the supersonic ones, and
//   F - s U = (q, q un + p, q ut, (un - s) E + p un),  q = rho (un - s).
__device__ __forceinline__ void hlle2(float gamma, float igm1, F2 scale,
                                      F2 rL, F2 nL, F2 tL, F2 pL, F2 rR, F2 nR, F2 tR, F2 pR,
                                      F2& f0, F2& f1, F2& f2, F2& f3) {
    F2 g = sp(gamma), h = sp(0.5f), tiny = sp(1e-37f);
    F2 gpL = mul2(g, pL), gpR = mul2(g, pR);
    // c = g p / sqrt(g p rho + 1e-37): the added 1e-37 keeps p = 0 finite
    // (c = 0) and is below the rounding of any state with p, rho >= 1e-15
    F2 cL = mul2(gpL, rsq2(fma2(gpL, rL, tiny)));
    F2 cR = mul2(gpR, rsq2(fma2(gpR, rR, tiny)));
    // nsl = -min(S_L, 0) = max(c_L - u_L, c_R - u_R, 0), sr = max(S_R, 0);
    // nsl is floored at 1e-30 instead of 0, which keeps sr + nsl > 0 (a
    // vacuum at rest) and gives the supersonic-right flux an extra weight
    // 1e-30 / sr on F_R - sr U_R, far below the rounding of F_L
    F2 aL = sub2(cL, nL), aR = sub2(cR, nR), bL = add2(nL, cL), bR = add2(nR, cR);
    F2 nsl = make_float2(max3f(aL.x, aR.x, 1e-30f), max3f(aL.y, aR.y, 1e-30f));
    F2 sr = make_float2(max3f(bL.x, bR.x, 0.f), max3f(bL.y, bR.y, 0.f));
    F2 inv = mul2(scale, rcp2(add2(sr, nsl)));
    F2 A = mul2(sr, inv);   //  scale sr / (sr - sl)
    F2 B = mul2(nsl, inv);  // -scale sl / (sr - sl)
    F2 dL = add2(nL, nsl), dR = sub2(nR, sr);
    F2 qL = mul2(rL, dL), qR = mul2(rR, dR);
    F2 EL = fma2(pL, sp(igm1), mul2(mul2(h, rL), fma2(tL, tL, mul2(nL, nL))));
    F2 ER = fma2(pR, sp(igm1), mul2(mul2(h, rR), fma2(tR, tR, mul2(nR, nR))));
    f0 = fma2(A, qL, mul2(B, qR));
    f1 = fma2(A, fma2(qL, nL, pL), mul2(B, fma2(qR, nR, pR)));
    f2 = fma2(A, mul2(qL, tL), mul2(B, mul2(qR, tR)));
    f3 = fma2(A, fma2(dL, EL, mul2(pL, nL)), mul2(B, fma2(dR, ER, mul2(pR, nR))));
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

// Element offset of a work item's arrays from the argument bases: zero for a
// single domain, the problem's offset in a batch.
__device__ __forceinline__ long long view_offset(const StageArgs<float>&) { return 0; }
template <class A>
__device__ __forceinline__ long long view_offset(const A& a) { return a.off; }

// One warp's work: the rows of tile `tile_row` under column strip `strip`.
// The warp owning strip 0 / tile 0 publishes the step's dt for the domain.
//
// Row march: before the loop the window holds the primitives of rows q and
// q+1, the upper x-face state P of row q and the x-flux of face q-1/2 (all
// for q = the tile's first row); iteration q adds row q+2, computes the
// x-flux of face q+1/2 and the y-fluxes of row q, and updates row q.  Fluxes
// come out of hlle2 already multiplied by dt/dx (dt/dy), and by 1/2 in stage
// 2, where the Heun average is folded into the update.
template <int STAGE, bool REPAIR, bool TOT, bool GHOST, class A>
__device__ __forceinline__ void x2_body(const A& a, int strip, int tile_row) {
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
    const double gmd = g.gamma - 1.0, igmd = 1.0 / gmd;  // FP64 repair constants
    const double hs = STAGE == 2 ? 0.5 : 1.0;
    const float dtdx = (float)(hs * dt / g.dx);
    const float dtdy = (float)(hs * dt / g.dy);
    const F2 sx = sp(dtdx), sy_ = sp(dtdy);

    // geometry used inside the row loop, held in registers (in the batched
    // kernel `g` lives in global memory)
    const int nx = g.nx, ny = g.ny, pitch = g.pitch;
    const int j0 = strip * STRIP2;
    if (j0 >= ny) return;  // whole warp idle
    const int ca = j0 - 2 + 2 * lane;  // first of the lane's two columns
    // element offset of the pair within a row (plus the problem's offset in a
    // batch); pairs past the ghost ring read the row padding (finite, discarded)
    const long long coff = view_offset(a) + min(ca + 2, pitch - 2);
    const bool lane_out = lane >= 1 && lane <= 30;
    const bool out_a = lane_out && ca < ny;
    const bool out_b = lane_out && ca + 1 < ny;
    const bool edge_col = ca < 2 || ca + 1 >= ny - 2;
    const int i0 = tile_row * a.tx;
    if (i0 >= nx) return;
    const int rows = min(a.tx, nx - i0);
    const int last_row = nx + 1;  // last ghost row: loads past it are clamped to it
    const long long vs = g.vstride;
    const float* __restrict__ Ui = a.Uin;
    const float* Unp = a.Un;
    float* const Uo = a.Uout;

    auto load = [&](int i, Q4& q) {
        const long long o = (long long)(min(i, last_row) + 2) * pitch + coff;
        q.a = __ldg(reinterpret_cast<const F2*>(Ui + o));
        q.b = __ldg(reinterpret_cast<const F2*>(Ui + vs + o));
        q.c = __ldg(reinterpret_cast<const F2*>(Ui + 2 * vs + o));
        q.d = __ldg(reinterpret_cast<const F2*>(Ui + 3 * vs + o));
    };
    const F2 half = sp(0.5f), mhalf = sp(-0.5f);

    // Input rows are staged through this warp's shared-memory rings (row r of
    // the stage input in slot r & 3, row r of U^n in slot r & 1), issued
    // three rows (U^n: one row) ahead of their use.  Before staging (loads
    // into registers one row ahead, the update's re-read of its own row from
    // L1) ncu measured a 10 % L1 hit rate on that re-read and long-scoreboard
    // waits as the top stall, at 0.434 ms per 4096^2 step against 0.386.
    F2* const ringw = x2_ring + threadIdx.y * ring_f2_per_warp(STAGE);  // this warp's rings
    F2* const ring = ringw + lane;                                       // this lane's column pair
    // 16-byte chunk copies: lane l moves column chunk l & 15 (columns
    // j0 - 2 + 4 (l & 15) .. + 3) of variables l >> 4 and (l >> 4) + 2.  Chunk
    // starts are 16-byte aligned (j0 = 60 strip, pitch a multiple of 32); a
    // chunk past the row end re-reads the row's last four columns, which feed
    // only discarded lanes.
    const int part = lane & 15, cvar = lane >> 4;
    const long long cseg = view_offset(a) + min(j0 + 4 * part, pitch - 4) + (long long)cvar * vs;
    const int cofs = cvar * 32 + 2 * part;  // F2 index of the chunk in a slot
    auto stage_rows = [&](const float* base, int i, F2* slot) {
        const float* q = base + (long long)(min(i, last_row) + 2) * pitch + cseg;
        cp16(slot + cofs, q);
        cp16(slot + cofs + 64, q + 2 * vs);
    };
    auto stage_row = [&](int i) { stage_rows(Ui, i, ringw + (i & (RING_U - 1)) * 128); };
    auto stage_un = [&](int i) { stage_rows(Unp, i, ringw + RING_U * 128 + (i & (RING_N - 1)) * 128); };
    auto ring_row = [&](int i, Q4& q) {
        const F2* d = ring + (i & (RING_U - 1)) * 128;
        q.a = d[0]; q.b = d[32]; q.c = d[64]; q.d = d[96];
    };
    auto ring_un = [&](int i, Q4& q) {
        const F2* d = ring + RING_U * 128 + (i & (RING_N - 1)) * 128;
        q.a = d[0]; q.b = d[32]; q.c = d[64]; q.d = d[96];
    };

    // prologue: rows i0-2 .. i0+1, x-flux of face i0-1/2
    Q4 Wq, Wq1, Pq, Fm;
    {
        Q4 c0, c1, c2, c3;
        load(i0 - 2, c0); load(i0 - 1, c1);
        for (int r = 0; r < LOOK; ++r) stage_row(i0 + r);
        if (STAGE == 2)
            for (int r = 0; r < LOOK - 2; ++r) stage_un(i0 + r);
        cp_commit();
        cp_wait<0>();
        __syncwarp();
        ring_row(i0, c2); ring_row(i0 + 1, c3);
        Q4 Wa = prim2<REPAIR>(c0, gm1), Wb = prim2<REPAIR>(c1, gm1);
        Wq = prim2<REPAIR>(c2, gm1); Wq1 = prim2<REPAIR>(c3, gm1);
        Q4 Sb = minmod_pair(Wa, Wb, Wq), Sq = minmod_pair(Wb, Wq, Wq1);
        Q4 Pb = q_fma(half, Sb, Wb), Mq = q_fma(mhalf, Sq, Wq);
        hlle2(gamma, igm1, sx, Pb.a, Pb.b, Pb.c, Pb.d, Mq.a, Mq.b, Mq.c, Mq.d, Fm.a, Fm.b, Fm.c, Fm.d);
        Pq = q_fma(half, Sq, Wq);
    }

    float smx = 0.f, smy = 0.f;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    // Unrolled by 2 in the plain kernels only (the unroll removes part of the
    // window rotation's register copies).  Measured at 4096^2 (ms per step,
    // stage 1 + stage 2): plain 0.3823 -> 0.3627 with the unroll; with
    // repair + totals 0.4086 -> 0.4211 (stage 2 +5 %, near the 128-register
    // budget); unrolls of 3 and 4 lost 12-25 %.
    constexpr int kUnroll = (!REPAIR && !TOT) ? 2 : 1;
#pragma unroll kUnroll
    for (int k = 0; k < rows; ++k) {
        const int i = i0 + k;
        Q4 cur;
        // A lane reads its column pair from chunks that other lanes copied, so
        // the warp synchronises twice per row: before the copies that refill
        // the slots of rows i-1 (every lane has finished reading them) and
        // after the wait (every lane's copies of row i+2 and U^n row i have
        // landed).  Measured at 4096^2 against the same loop without the two
        // barriers: 0.4088 / 0.4094 ms per step with totals + repair, 0.3828 /
        // 0.3761 plain; one barrier with the wait moved before the refill,
        // 0.4085 / 0.3910.
        __syncwarp();
        stage_row(i + LOOK);
        if (STAGE == 2) stage_un(i + LOOK - 2);
        cp_commit();
        cp_wait<LOOK - 2>();
        __syncwarp();
        ring_row(i + 2, cur);

        // x-face i+1/2 from rows i .. i+2
        Q4 W2 = prim2<REPAIR>(cur, gm1);
        Q4 S1 = minmod_pair(Wq, Wq1, W2);
        Q4 M1 = q_fma(mhalf, S1, Wq1);
        Q4 Fc;
        hlle2(gamma, igm1, sx, Pq.a, Pq.b, Pq.c, Pq.d, M1.a, M1.b, M1.c, M1.d, Fc.a, Fc.b, Fc.c, Fc.d);

        // The conserved values of row i and, in stage 2, its U^n are read from
        // the rings between the two flux computations in stage 2 and after
        // them in stage 1 (the faster placement of each, measured at 4096^2).
        Q4 C0, un;
        if (STAGE == 2) {
            ring_row(i, C0);
            ring_un(i, un);
        }
        // y-faces on row i: (a|b, b|a') with normal v, transverse u
        Q4 sy = { yslope(Wq.a), yslope(Wq.b), yslope(Wq.c), yslope(Wq.d) };
        Q4 Py = q_fma(half, sy, Wq), My = q_fma(mhalf, sy, Wq);
        Q4 R;
        R.a = make_float2(My.a.y, __shfl_down_sync(0xffffffffu, My.a.x, 1));
        R.b = make_float2(My.b.y, __shfl_down_sync(0xffffffffu, My.b.x, 1));
        R.c = make_float2(My.c.y, __shfl_down_sync(0xffffffffu, My.c.x, 1));
        R.d = make_float2(My.d.y, __shfl_down_sync(0xffffffffu, My.d.x, 1));
        Q4 G;  // G.b = mu flux (transverse), G.c = mv flux (normal)
        hlle2(gamma, igm1, sy_, Py.a, Py.c, Py.b, Py.d, R.a, R.c, R.b, R.d, G.a, G.c, G.b, G.d);
        // G(face a-1/2) from the left lane's G(b+1/2)
        Q4 dG;
        dG.a = sub2(G.a, make_float2(__shfl_up_sync(0xffffffffu, G.a.y, 1), G.a.x));
        dG.b = sub2(G.b, make_float2(__shfl_up_sync(0xffffffffu, G.b.y, 1), G.b.x));
        dG.c = sub2(G.c, make_float2(__shfl_up_sync(0xffffffffu, G.c.y, 1), G.c.x));
        dG.d = sub2(G.d, make_float2(__shfl_up_sync(0xffffffffu, G.d.y, 1), G.d.x));

        if (STAGE == 1) ring_row(i, C0);
        if (out_a) {
            Q4 s;
            if (STAGE == 1) {  // U1 = U - (dF + dG)
                s.a = sub2(add2(C0.a, Fm.a), add2(Fc.a, dG.a));
                s.b = sub2(add2(C0.b, Fm.b), add2(Fc.b, dG.b));
                s.c = sub2(add2(C0.c, Fm.c), add2(Fc.c, dG.c));
                s.d = sub2(add2(C0.d, Fm.d), add2(Fc.d, dG.d));
            } else {  // U^{n+1} = (U^n + U1)/2 - (dF + dG)/2, fluxes already halved
                s.a = fma2(half, add2(un.a, C0.a), sub2(sub2(Fm.a, Fc.a), dG.a));
                s.b = fma2(half, add2(un.b, C0.b), sub2(sub2(Fm.b, Fc.b), dG.b));
                s.c = fma2(half, add2(un.c, C0.c), sub2(sub2(Fm.c, Fc.c), dG.c));
                s.d = fma2(half, add2(un.d, C0.d), sub2(sub2(Fm.d, Fc.d), dG.d));
            }
            const long long o = (long long)(i + 2) * pitch + coff;  // = ca + 2 on output lanes
            if (STAGE == 2) {
                // wave speeds |u|+c, |v|+c of the new state with the floors of compute_dt_2d
                F2 rho = max2(s.a, 1e-10f);
                F2 ir = rcp2(rho);
                F2 u = mul2(s.b, ir), v = mul2(s.c, ir);
                F2 ke = mul2(mul2(half, rho), fma2(v, v, mul2(u, u)));
                F2 pr = mul2(sp(gm1), sub2(s.d, ke));
                if (REPAIR) {
                    // FP64 positivity repair: a cell with rho < 1e-10 or an FP64
                    // pressure below 1e-10 gets rho >= 1e-10 and E raised to
                    // ke + 1e-10/(gamma-1).  The FP32 pressure differs from the
                    // FP64 one by far less than 1e-5 (gamma-1)(|E| + ke), so only
                    // cells under that bound (near vacuum) take the FP64 path.
                    auto fix = [&](float& r0, float& m1, float& m2, float& e3) {
                        const double fl = 1e-10;
                        double r_ = (double)r0, rr = smax(r_, fl), irr = rcp_nr(rr);
                        double u_ = (double)m1 * irr, v_ = (double)m2 * irr;
                        double keD = 0.5 * rr * (u_ * u_ + v_ * v_);
                        double pD = gmd * ((double)e3 - keD);
                        if (!(r_ >= fl) || !(pD >= fl)) {
                            r0 = (float)rr;
                            e3 = (float)smax((double)e3, keD + fl * igmd);
                            atomicAdd(&a.ctrl->repairs, 1u);
                        }
                    };
                    F2 tol = fma2(sp(1e-5f * gm1), add2(make_float2(fabsf(s.d.x), fabsf(s.d.y)), ke), sp(1e-10f));
                    const bool near_x = !(s.a.x >= 1e-10f) || !(pr.x >= tol.x);
                    const bool near_y = out_b && (!(s.a.y >= 1e-10f) || !(pr.y >= tol.y));
                    if (__any_sync(__activemask(), near_x || near_y) && (near_x || near_y)) {
                        if (near_x) fix(s.a.x, s.b.x, s.c.x, s.d.x);
                        if (near_y) fix(s.a.y, s.b.y, s.c.y, s.d.y);
                        rho = max2(s.a, 1e-10f);
                        ir = rcp2(rho);
                        u = mul2(s.b, ir); v = mul2(s.c, ir);
                        ke = mul2(mul2(half, rho), fma2(v, v, mul2(u, u)));
                        pr = mul2(sp(gm1), sub2(s.d, ke));
                    }
                }
                {
                    // positivity (with REPAIR: NaN only, the repair keeps rho and p positive in FP64)
                    const bool bx = REPAIR ? (!(s.a.x == s.a.x) || !(pr.x == pr.x)) : (!(s.a.x > 0.f) || !(pr.x > 0.f));
                    const bool by = out_b && (REPAIR ? (!(s.a.y == s.a.y) || !(pr.y == pr.y))
                                                     : (!(s.a.y > 0.f) || !(pr.y > 0.f)));
                    if (bx) flag_cell(a.ctrl, a.ctrl->step[a.p] + 1, s.a.x, pr.x, i, ca);
                    if (by) flag_cell(a.ctrl, a.ctrl->step[a.p] + 1, s.a.y, pr.y, i, ca + 1);
                }
                F2 pp = max2(pr, 1e-10f);
                F2 gp = mul2(sp(gamma), pp);
                F2 c = mul2(gp, rsq2(mul2(gp, rho)));
                F2 au = add2(make_float2(fabsf(u.x), fabsf(u.y)), c);
                F2 av = add2(make_float2(fabsf(v.x), fabsf(v.y)), c);
                if (!out_b) { au.y = 0.f; av.y = 0.f; }
                smx = max3f(smx, au.x, au.y);
                smy = max3f(smy, av.x, av.y);
                if (TOT) {
                    t0 += (double)s.a.x; t1 += (double)s.b.x; t2 += (double)s.c.x; t3 += (double)s.d.x;
                    if (out_b) {
                        t0 += (double)s.a.y; t1 += (double)s.b.y; t2 += (double)s.c.y; t3 += (double)s.d.y;
                    }
                }
            }
            if (out_b) {
                *reinterpret_cast<F2*>(Uo + o) = s.a;
                *reinterpret_cast<F2*>(Uo + vs + o) = s.b;
                *reinterpret_cast<F2*>(Uo + 2 * vs + o) = s.c;
                *reinterpret_cast<F2*>(Uo + 3 * vs + o) = s.d;
            } else {
                Uo[o] = s.a.x; Uo[vs + o] = s.b.x; Uo[2 * vs + o] = s.c.x; Uo[3 * vs + o] = s.d.x;
            }
            if (GHOST && (edge_col || i < 2 || i >= nx - 2)) {
                store_ghosts(Uo + view_offset(a), g, 0, i, ca, s.a.x); store_ghosts(Uo + view_offset(a), g, 1, i, ca, s.b.x);
                store_ghosts(Uo + view_offset(a), g, 2, i, ca, s.c.x); store_ghosts(Uo + view_offset(a), g, 3, i, ca, s.d.x);
                if (out_b) {
                    store_ghosts(Uo + view_offset(a), g, 0, i, ca + 1, s.a.y); store_ghosts(Uo + view_offset(a), g, 1, i, ca + 1, s.b.y);
                    store_ghosts(Uo + view_offset(a), g, 2, i, ca + 1, s.c.y); store_ghosts(Uo + view_offset(a), g, 3, i, ca + 1, s.d.y);
                }
            }
        }
        Fm = Fc;
        Pq = q_fma(half, S1, Wq1);
        Wq = Wq1;
        Wq1 = W2;
    }
    // Drain the copies still in flight (rows staged past the tile): the
    // batched kernel's next work item stages its first rows into the same
    // slots, and two copies into one slot are not ordered.
    cp_wait<0>();
    __syncwarp();
    if (STAGE == 2) {
        double mx = warp_max((double)smx), my = warp_max((double)smy);
        if (lane == 0) {
            if (!(mx == mx) || !(my == my) || mx > 1.79e308 || my > 1.79e308) atomicOr(&a.ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][0], mx);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][1], my);
        }
        if (TOT) {
            t0 = warp_sum(t0); t1 = warp_sum(t1); t2 = warp_sum(t2); t3 = warp_sum(t3);
            if (lane == 0) {
                long long wid = ((long long)tile_row * ((ny + STRIP2 - 1) / STRIP2) + strip) * 4;  // per-domain slot
                a.partials[wid + 0] = t0; a.partials[wid + 1] = t1;
                a.partials[wid + 2] = t2; a.partials[wid + 3] = t3;
            }
        }
    }
}

// Single-domain stage kernels: STAGE 1 or 2, REPAIR = FP64 positivity repair,
// TOT = per-warp FP64 totals (stage 2).  All run under a 128-register budget
// (16 warps per SM): from sweeps at 4096^2 (B200, 16-row tiles, one warp per
// block), budgets of 104-120 (17-19 warps) ran 7-18 % slower and 144 (14
// warps) 15 % slower in stage 1.
template <int STAGE, bool REPAIR, bool TOT>
__global__ void __maxnreg__(128) k2d_f32x2(StageArgs<float> a) {
    x2_body<STAGE, REPAIR, TOT, true>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

// Arguments of one batched work item: the array bases are the batch's (kernel
// parameters), `off` is the problem's element offset, and the problem's
// geometry stays in global memory (the body copies the few fields its row
// loop needs).
struct X2View {
    const float* Uin;
    const float* Un;
    float* Uout;
    long long off;
    const Geo2D& g;
    const LoopParams& lp;
    StepCtrl* ctrl;
    double* partials;
    int p;
    int tx;
};

// Persistent batched stage: every warp walks the work list (problem, strip,
// tile row) with a stride of the whole grid's warp count.  The 128-register
// budget matches the single-domain kernels (16 warps per SM).  The ghost rings
// are filled afterwards by kbatch_ghosts: with many small problems a large
// share of the warps sit on a domain edge, and one copy pass over all rings
// costs less than the edge branch inside the row loop.
template <int STAGE, bool REPAIR, bool TOT>
__global__ void __maxnreg__(128) kbatch_f32x2(BatchArgs<float> b) {
    const int nw = gridDim.x * blockDim.y;
    for (int it = blockIdx.x * blockDim.y + threadIdx.y; it < b.nitems; it += nw) {
        const int4 w = b.items[it];
        const BatchProblem& P = b.probs[w.x];
        const long long off = P.off;
        X2View v{STAGE == 1 ? b.U : b.U1, STAGE == 2 ? b.U : nullptr, STAGE == 1 ? b.U1 : b.U, off, P.g, b.lp,
                 b.ctrls + w.x,
                 TOT ? b.partials + 4ll * P.item0 : nullptr, b.p, b.tx};
        x2_body<STAGE, REPAIR, TOT, false>(v, w.y, w.z);
    }
}

// Ghost rings of every problem of a batch (block row y = problem): rows -2,
// -1, nx, nx+1 under the interior columns and columns -2, -1, ny, ny+1 beside
// the interior rows, copied from the cells nest's periodic copy or the
// zero-gradient copy name (the corners are never read: the stencil is a
// cross).  Rows filled by a halo exchange are left alone.
__global__ void __launch_bounds__(256) kbatch_ghosts(float* base, const BatchProblem* probs, int nprobs) {
  for (int pb = blockIdx.y; pb < nprobs; pb += gridDim.y) {
    const BatchProblem& P = probs[pb];
    const Geo2D& g = P.g;
    float* U = base + P.off;
    const int nx = g.nx, ny = g.ny;
    const long long vs = g.vstride;
    const int nrow = 4 * ny, ntot = nrow + 4 * nx;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += gridDim.x * blockDim.x) {
        int di, dj, si, sj;
        if (t < nrow) {  // ghost rows, consecutive threads along a row
            const int r = t / ny;
            dj = sj = t - r * ny;
            di = r < 2 ? r - 2 : nx + r - 2;
            if ((di < 0 && g.xlo_ex) || (di >= nx && g.xhi_ex)) continue;
            si = g.bcx == BC_PERIODIC ? (di < 0 ? di + nx : di - nx) : (di < 0 ? 0 : nx - 1);
        } else {  // ghost columns, four consecutive threads per row
            const int u = t - nrow, c = u & 3;
            di = si = u >> 2;
            dj = c < 2 ? c - 2 : ny + c - 2;
            sj = g.bcy == BC_PERIODIC ? (dj < 0 ? dj + ny : dj - ny) : (dj < 0 ? 0 : ny - 1);
        }
        const long long d = g.at(di, dj), s = g.at(si, sj);
        U[d] = U[s];
        U[vs + d] = U[vs + s];
        U[2 * vs + d] = U[2 * vs + s];
        U[3 * vs + d] = U[3 * vs + s];
    }
  }
}

// Dynamic shared memory of a stage launch: the row rings of its warps.
size_t ring_bytes(int stage, int warps) {
    return (size_t)warps * ring_f2_per_warp(stage) * sizeof(F2);
}

}  // namespace

int strips_f32x2(int ny) { return (ny + STRIP2 - 1) / STRIP2; }

cudaError_t launch_batch_f32x2(const BatchArgs<float>& b, bool repair, int which, int blocks, int warps,
                               cudaStream_t st) {
    dim3 blk(32, warps);
    const bool tot = b.partials != nullptr;
    const size_t sm1 = ring_bytes(1, warps), sm2 = ring_bytes(2, warps);
    // ghost-ring pass: enough 256-thread blocks per problem for its largest ring
    const dim3 ggrid(b.ghost_blocks, b.nprobs < 65535 ? b.nprobs : 65535);
    if (which & 1) {
        if (repair) kbatch_f32x2<1, true, false><<<blocks, blk, sm1, st>>>(b);
        else kbatch_f32x2<1, false, false><<<blocks, blk, sm1, st>>>(b);
        kbatch_ghosts<<<ggrid, 256, 0, st>>>(b.U1, b.probs, b.nprobs);
    }
    if (which & 2) {
        if (repair && tot) kbatch_f32x2<2, true, true><<<blocks, blk, sm2, st>>>(b);
        else if (repair) kbatch_f32x2<2, true, false><<<blocks, blk, sm2, st>>>(b);
        else if (tot) kbatch_f32x2<2, false, true><<<blocks, blk, sm2, st>>>(b);
        else kbatch_f32x2<2, false, false><<<blocks, blk, sm2, st>>>(b);
        kbatch_ghosts<<<ggrid, 256, 0, st>>>(b.U, b.probs, b.nprobs);
    }
    return cudaGetLastError();
}

int batch_max_blocks_f32x2(int warps) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kbatch_f32x2<2, true, true>, 32 * warps, ring_bytes(2, warps));
    return nb;
}

cudaError_t launch_2d_step_f32x2(float* U, float* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl,
                                 double* partials, int p, int tx, int warps, bool repair, int which,
                                 cudaStream_t st, float* Uout) {
    int nstrips = strips_f32x2(g.ny);
    dim3 b(32, warps), gr((nstrips + warps - 1) / warps, (g.nx + tx - 1) / tx);
    StageArgs<float> a1{U, nullptr, U1, g, lp, ctrl, nullptr, p, tx};
    StageArgs<float> a2{U1, U, Uout ? Uout : U, g, lp, ctrl, partials, p, tx};
    const bool tot = partials != nullptr;
    const size_t sm1 = ring_bytes(1, warps), sm2 = ring_bytes(2, warps);
    if (which & 1) {
        if (repair) k2d_f32x2<1, true, false><<<gr, b, sm1, st>>>(a1);
        else k2d_f32x2<1, false, false><<<gr, b, sm1, st>>>(a1);
    }
    if (which & 2) {
        if (repair && tot) k2d_f32x2<2, true, true><<<gr, b, sm2, st>>>(a2);
        else if (repair) k2d_f32x2<2, true, false><<<gr, b, sm2, st>>>(a2);
        else if (tot) k2d_f32x2<2, false, true><<<gr, b, sm2, st>>>(a2);
        else k2d_f32x2<2, false, false><<<gr, b, sm2, st>>>(a2);
    }
    return cudaGetLastError();
}

}  // namespace nestb
