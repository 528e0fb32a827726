// FP64 plain form of the 2D stage kernels as a staged row march (sm_100a).
//
// Same scheme, operation order and results (bit for bit) as stage2d_body in
// euler2d_kernels.cuh, compiled with -fmad=false; what changes is how a warp
// keeps its work fed:
//   * input rows reach the warp through shared-memory rings filled by 16-byte
//     cp.async copies issued three rows ahead (U^n one row ahead in stage 2),
//     so loads in flight hold no registers and the update's re-read of its
//     own row is a shared-memory hit;
//   * the row window is the primitives of rows q and q+1, the upper x-face
//     state of row q and the x-flux of face q-1/2 (16 doubles), and the first
//     rows of the tile are computed before the loop, so the loop body is one
//     block with the x-face and the y-face fluxes of a row side by side,
//     free to interleave their division and square-root chains.
// A warp owns a strip of 32 columns j0-2 .. j0+29 (j0 = 28 strip) and
// writes lanes 2..29, like stage2d_body.
#include "euler2d_kernels.cuh"
#include "f64div.cuh"
#include "kernels.h"

#include <algorithm>
#include <cstdlib>
#include <string>

namespace nestb {
namespace {

#ifndef NEST_F64R_UNROLL
#define NEST_F64R_UNROLL 1
#endif
constexpr int kUnrollD = NEST_F64R_UNROLL;  // row-loop unroll
constexpr int LOOKD = 3;                   // stage-input rows in flight ahead of the march
constexpr int RING_UD = 4, RING_ND = 2;    // ring slots: stage input, U^n (stage 2)
__host__ __device__ constexpr int ring_d_per_warp(int stage) { return (RING_UD + (stage == 2 ? RING_ND : 0)) * 4 * 32; }
extern __shared__ __align__(16) double f64r_ring[];

__device__ __forceinline__ void cp16d(double* smem_dst, const double* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpd_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpd_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

using W4 = Win4<double>;

__device__ __forceinline__ W4 half_step(const W4& w, const W4& s, double h) {
    return { w.a + h * s.a, w.b + h * s.b, w.c + h * s.c, w.d + h * s.d };
}
__device__ __forceinline__ W4 half_back(const W4& w, const W4& s) {
    return { w.a - 0.5 * s.a, w.b - 0.5 * s.b, w.c - 0.5 * s.c, w.d - 0.5 * s.d };
}

// Division policies of a row: the IEEE division, or the checked fast
// division of f64div.cuh, which returns the same value whenever it leaves
// `ok` set (a row with any cleared flag in the warp is recomputed with the
// IEEE policy before anything of it is stored).
struct DivIeee {
    __device__ __forceinline__ double div(double x, double y) { return x / y; }
};
struct DivChecked {
    bool ok = true;
    __device__ __forceinline__ double div(double x, double y) { return div_rn_checked(x, y, ok); }
};

// cons2prim, hlle4 and cell_speeds_p of euler2d_kernels.cuh for the FP64
// plain form (the same expressions in the same order, so the same values),
// with their divisions taken from a policy.
template <class D>
__device__ __forceinline__ W4 prim_d(D& d, const W4& c, double gm1) {
    const double u = d.div(c.b, c.a), v = d.div(c.c, c.a);
    const double p = gm1 * (c.d - ke2(c.a, u, v));
    return { c.a, u, v, smax(p, 0.0) };
}

template <class D>
__device__ __forceinline__ void hlle4_d(D& d, double gamma, double gm1, double rL, double nL, double tL, double pL,
                                        double rR, double nR, double tR, double pR, double& f0, double& f1,
                                        double& f2, double& f3) {
    const double cL = sqrt(d.div(gamma * pL, rL));
    const double cR = sqrt(d.div(gamma * pR, rR));
    const double EL = d.div(pL, gm1) + ke2(rL, nL, tL);
    const double ER = d.div(pR, gm1) + ke2(rR, nR, tR);
    const double SL = smin(nL - cL, nR - cR);
    const double SR = smax(nL + cL, nR + cR);
    const double mL = rL * nL, mR = rR * nR;
    const double FL0 = mL, FL1 = mL * nL + pL, FL2 = mL * tL, FL3 = (EL + pL) * nL;
    const double FR0 = mR, FR1 = mR * nR + pR, FR2 = mR * tR, FR3 = (ER + pR) * nR;
    if (SL >= 0.0) {
        f0 = FL0; f1 = FL1; f2 = FL2; f3 = FL3;
    } else if (SR <= 0.0) {
        f0 = FR0; f1 = FR1; f2 = FR2; f3 = FR3;
    } else {
        const double SLR = SL * SR, dS = SR - SL;
        f0 = d.div(SR * FL0 - SL * FR0 + SLR * (rR - rL), dS);
        f1 = d.div(SR * FL1 - SL * FR1 + SLR * (mR - mL), dS);
        f2 = d.div(SR * FL2 - SL * FR2 + SLR * (rR * tR - rL * tL), dS);
        f3 = d.div(SR * FL3 - SL * FR3 + SLR * (ER - EL), dS);
    }
}

template <class D>
__device__ __forceinline__ double speeds_d(D& d, double U0, double U1, double U2, double U3, double gamma,
                                           double gm1, double& sx, double& sy) {
    const double rho = smax(U0, 1e-10);
    const double u = d.div(U1, rho), v = d.div(U2, rho);
    const double ke = 0.5 * rho * (u * u + v * v);
    const double p = smax(gm1 * (U3 - ke), 1e-10);
    const double c = sqrt(d.div(gamma * p, rho));
    sx = fabs(u) + c;
    sy = fabs(v) + c;
    return gm1 * (U3 - ke2(rho, u, v));
}

// LIM: the slope limiter fixed at compile time (LIM_MINMOD, nest's default),
// or -1 to read it from the loop parameters; a fixed limiter leaves no
// limiter branch in the row loop.
template <int STAGE, bool TOT, int LIM>
__device__ __forceinline__ void f64r_body(const StageArgs<double>& a, int strip, int tile_row) {
    const Geo2D& g = a.g;
    const int lane = threadIdx.x & 31;
    const double gamma = g.gamma;
    const double gm1 = g.gamma - 1.0;

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
    const double dtdx = dt / g.dx;
    const double dtdy = dt / g.dy;
    const int lim = LIM >= 0 ? LIM : a.lp.lim;

    const int nx = g.nx, ny = g.ny, pitch = g.pitch;
    const int j0 = strip * STRIP;
    if (j0 >= ny) return;                  // whole warp idle
    const int j = j0 - 2 + lane;           // this lane's column
    const bool out_col = lane >= 2 && lane < 30 && j < ny;
    const bool edge_col = j < 2 || j >= ny - 2;
    const int i0 = tile_row * a.tx;
    if (i0 >= nx) return;
    const int rows = min(a.tx, nx - i0);
    const int last_row = nx + 1;           // staged rows past it are clamped to it
    const long long vs = g.vstride;
    const double* __restrict__ Ui = a.Uin;
    const double* Unp = a.Un;
    double* const Uo = a.Uout;

    // this warp's rings: RING_UD slots of the stage input, then RING_ND of U^n;
    // a slot is [var][32 columns]
    double* const ringw = f64r_ring + threadIdx.y * ring_d_per_warp(STAGE);
    // 16-byte chunk copies: lane l moves columns j0-2+2(l & 15) .. +1 of
    // variables l >> 4 and (l >> 4) + 2.  Chunk starts are 16-byte aligned
    // (j0 = 28 strip, pitch a multiple of 16); chunks past the row end re-read
    // the row's last two columns, which feed only discarded lanes.
    const int part = lane & 15, cvar = lane >> 4;
    const long long cseg = min(j0 + 2 * part, pitch - 2) + (long long)cvar * vs;
    const int cofs = cvar * 32 + 2 * part;
    auto stage_rows = [&](const double* base, int i, double* slot) {
        const double* q = base + (long long)(min(i, last_row) + 2) * pitch + cseg;
        cp16d(slot + cofs, q);
        cp16d(slot + cofs + 64, q + 2 * vs);
    };
    auto stage_row = [&](int i) { stage_rows(Ui, i, ringw + (i & (RING_UD - 1)) * 128); };
    auto stage_un = [&](int i) { stage_rows(Unp, i, ringw + RING_UD * 128 + (i & (RING_ND - 1)) * 128); };
    auto ring_row = [&](int i) -> W4 {
        const double* d = ringw + (i & (RING_UD - 1)) * 128 + lane;
        return { d[0], d[32], d[64], d[96] };
    };
    auto ring_un = [&](int i) -> W4 {
        const double* d = ringw + RING_UD * 128 + (i & (RING_ND - 1)) * 128 + lane;
        return { d[0], d[32], d[64], d[96] };
    };
    auto load = [&](int i) -> W4 {
        const long long o = g.at(i, min(j, ny + 1));
        return { __ldg(Ui + o), __ldg(Ui + vs + o), __ldg(Ui + 2 * vs + o), __ldg(Ui + 3 * vs + o) };
    };

    // prologue: rows i0-2 .. i0+1, the x-flux of face i0-1/2 and the upper
    // x-face state of row i0
    W4 Wq, Wq1, Pq, Fm;
    {
        const W4 c0 = load(i0 - 2), c1 = load(i0 - 1);
        for (int r = 0; r < LOOKD; ++r) stage_row(i0 + r);
        if (STAGE == 2)
            for (int r = 0; r < LOOKD - 2; ++r) stage_un(i0 + r);
        cpd_commit();
        cpd_wait<0>();
        __syncwarp();
        // with the checked divisions, again with IEEE ones if a lane up to the
        // last ghost column failed one (as in the row loop below)
        auto pro = [&](auto& d) {
            const W4 Wa = prim_d(d, c0, gm1), Wb = prim_d(d, c1, gm1);
            Wq = prim_d(d, ring_row(i0), gm1);
            Wq1 = prim_d(d, ring_row(i0 + 1), gm1);
            const W4 Sb = limit4(Wa, Wb, Wq, lim), Sq = limit4(Wb, Wq, Wq1, lim);
            const W4 L = half_step(Wb, Sb, 0.5), R = half_back(Wq, Sq);
            hlle4_d(d, gamma, gm1, L.a, L.b, L.c, L.d, R.a, R.b, R.c, R.d, Fm.a, Fm.b, Fm.c, Fm.d);
            Pq = half_step(Wq, Sq, 0.5);
        };
        DivChecked dpro;
        pro(dpro);
        if (__any_sync(0xffffffffu, !dpro.ok && j <= ny + 1)) {
            DivIeee di;
            pro(di);
        }
    }

    double smx = 0.0, smy = 0.0;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll kUnrollD
    for (int k = 0; k < rows; ++k) {
        const int i = i0 + k;
        // refill the slots of row i-1 once every lane has read them; then
        // wait for rows up to i+2 (and U^n row i)
        __syncwarp();
        stage_row(i + LOOKD);
        if (STAGE == 2) stage_un(i + LOOKD - 2);
        cpd_commit();
        cpd_wait<LOOKD - 2>();
        __syncwarp();

        // The row's arithmetic, with the divisions of a policy: the x-face
        // i+1/2 from rows i .. i+2, the y-faces of row i (face j+1/2, normal v,
        // transverse u; the left face from the left neighbour), the update of
        // every lane's cell of row i and, in stage 2, its wave speeds.
        struct RowOut {
            W4 W2, S1, Fc, s;
            double sx, sy, pc;
        };
        auto row = [&](auto& dp, auto& dv) {
            RowOut o;
            o.W2 = prim_d(dp, ring_row(i + 2), gm1);
            o.S1 = limit4(Wq, Wq1, o.W2, lim);
            const W4 M1 = half_back(Wq1, o.S1);
            hlle4_d(dv, gamma, gm1, Pq.a, Pq.b, Pq.c, Pq.d, M1.a, M1.b, M1.c, M1.d, o.Fc.a, o.Fc.b, o.Fc.c, o.Fc.d);
            const W4 sy = limit4(shfl_up4(Wq), Wq, shfl_dn4(Wq), lim);
            const W4 Rq = shfl_dn4(half_back(Wq, sy));
            const W4 Ly = half_step(Wq, sy, 0.5);
            W4 Gy;
            hlle4_d(dv, gamma, gm1, Ly.a, Ly.c, Ly.b, Ly.d, Rq.a, Rq.c, Rq.b, Rq.d, Gy.a, Gy.c, Gy.b, Gy.d);
            const W4 Gl = shfl_up4(Gy);
            const W4 C0 = ring_row(i);
            o.s.a = C0.a - (dtdx * (o.Fc.a - Fm.a) + dtdy * (Gy.a - Gl.a));
            o.s.b = C0.b - (dtdx * (o.Fc.b - Fm.b) + dtdy * (Gy.b - Gl.b));
            o.s.c = C0.c - (dtdx * (o.Fc.c - Fm.c) + dtdy * (Gy.c - Gl.c));
            o.s.d = C0.d - (dtdx * (o.Fc.d - Fm.d) + dtdy * (Gy.d - Gl.d));
            if (STAGE == 2) {
                const W4 N0 = ring_un(i);
                o.s.a = 0.5 * (N0.a + o.s.a);
                o.s.b = 0.5 * (N0.b + o.s.b);
                o.s.c = 0.5 * (N0.c + o.s.c);
                o.s.d = 0.5 * (N0.d + o.s.d);
                o.pc = speeds_d(dv, o.s.a, o.s.b, o.s.c, o.s.d, gamma, gm1, o.sx, o.sy);
            }
            return o;
        };
        // The checked divisions first; if one of them that can reach an
        // output could not be shown to be correctly rounded, the whole row
        // again with IEEE divisions.  Either way the stored values are those
        // of the IEEE arithmetic.  What reaches an output: the primitives of
        // every lane up to the last ghost column (y-slopes of the lanes two
        // away), and the fluxes and wave speeds of lanes 1..29 inside the
        // domain (lane j-1's y-face is lane j's left face); lanes past the
        // ghost columns read the row padding.
        DivChecked dp, dc;
        RowOut o = row(dp, dc);
        const bool need = (!dp.ok && j <= ny + 1) || (!dc.ok && lane >= 1 && lane < 30 && j < ny);
        if (__any_sync(0xffffffffu, need)) {
            DivIeee di;
            o = row(di, di);
        }

        if (out_col) {
            const double s0 = o.s.a, s1 = o.s.b, s2 = o.s.c, s3 = o.s.d;
            if (STAGE == 2) {
                const double pc = o.pc;
                if (!(s0 >= 1e-10) || !(pc > 0.0)) {
                    double pe = pc;
                    if (s0 > 0.0 && s0 < 1e-10) pe = gm1 * (s3 - ke2(s0, s1 / s0, s2 / s0));
                    if (!(s0 > 0.0) || !(pe > 0.0) || !(pe == pe))
                        flag_cell(a.ctrl, a.ctrl->step[a.p] + 1, s0, pe, i, j);
                }
                smx = smax(smx, o.sx);
                smy = smax(smy, o.sy);
                if (TOT) { t0 += s0; t1 += s1; t2 += s2; t3 += s3; }
            }
            const long long oo = g.at(i, j);
            Uo[oo] = s0; Uo[vs + oo] = s1; Uo[2 * vs + oo] = s2; Uo[3 * vs + oo] = s3;
            if (edge_col || i < 2 || i >= nx - 2) {
                store_ghosts(Uo, g, 0, i, j, s0);
                store_ghosts(Uo, g, 1, i, j, s1);
                store_ghosts(Uo, g, 2, i, j, s2);
                store_ghosts(Uo, g, 3, i, j, s3);
            }
        }
        Fm = o.Fc;
        Pq = half_step(Wq1, o.S1, 0.5);
        Wq = Wq1;
        Wq1 = o.W2;
    }
    // no copy may land in shared memory after the warp has left
    cpd_wait<0>();
    __syncwarp();
    if (STAGE == 2) {
        smx = warp_max(smx);
        smy = warp_max(smy);
        if (lane == 0) {
            if (!(smx == smx) || !(smy == smy) || smx > 1.79e308 || smy > 1.79e308)
                atomicOr(&a.ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][0], smx);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][1], smy);
        }
        if (TOT) {
            t0 = warp_sum(t0); t1 = warp_sum(t1); t2 = warp_sum(t2); t3 = warp_sum(t3);
            if (lane == 0) {
                long long wid = ((long long)tile_row * ((ny + STRIP - 1) / STRIP) + strip) * 4;
                a.partials[wid + 0] = t0; a.partials[wid + 1] = t1;
                a.partials[wid + 2] = t2; a.partials[wid + 3] = t3;
            }
        }
    }
}

// Row-loop unroll and register budget (0: ptxas's choice).
#ifndef NEST_F64R_REGS
#define NEST_F64R_REGS 0
#endif
#if NEST_F64R_REGS > 0
#define NEST_F64R_ATTR __maxnreg__(NEST_F64R_REGS)
#else
#define NEST_F64R_ATTR __launch_bounds__(256)
#endif

template <int STAGE, bool TOT, int LIM>
__global__ void NEST_F64R_ATTR k2d_f64r(StageArgs<double> a) {
    f64r_body<STAGE, TOT, LIM>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

template <int LIM>
void launch_f64r_lim(const StageArgs<double>& a1, const StageArgs<double>& a2, dim3 gr, dim3 b, size_t sm1,
                     size_t sm2, int which, bool tot, cudaStream_t st) {
    if (which & 1) k2d_f64r<1, false, LIM><<<gr, b, sm1, st>>>(a1);
    if (which & 2) {
        if (tot) k2d_f64r<2, true, LIM><<<gr, b, sm2, st>>>(a2);
        else k2d_f64r<2, false, LIM><<<gr, b, sm2, st>>>(a2);
    }
}

size_t f64r_ring_bytes(int stage, int warps) { return (size_t)warps * ring_d_per_warp(stage) * sizeof(double); }

}  // namespace

cudaError_t launch_2d_step_f64r(double* U, double* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl,
                                double* partials, int p, int tx, int warps, int which, cudaStream_t st,
                                double* Uout) {
    const int nstrips = (g.ny + STRIP - 1) / STRIP;
    dim3 b(32, warps), gr((nstrips + warps - 1) / warps, (g.nx + tx - 1) / tx);
    StageArgs<double> a1{U, nullptr, U1, g, lp, ctrl, nullptr, p, tx};
    StageArgs<double> a2{U1, U, Uout ? Uout : U, g, lp, ctrl, partials, p, tx};
    const size_t sm1 = f64r_ring_bytes(1, warps), sm2 = f64r_ring_bytes(2, warps);
    if (lp.lim == LIM_MINMOD) launch_f64r_lim<LIM_MINMOD>(a1, a2, gr, b, sm1, sm2, which, partials != nullptr, st);
    else launch_f64r_lim<-1>(a1, a2, gr, b, sm1, sm2, which, partials != nullptr, st);
    return cudaGetLastError();
}

namespace {
__global__ void k_div_selftest(const double* a, const double* b, double* q, int* ok, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        bool k = true;
        q[t] = div_rn_checked(a[t], b[t], k);
        ok[t] = k ? 1 : 0;
    }
}
}  // namespace

}  // namespace nestb

extern "C" nest_status nest_selftest_div_f64(const double* d_a, const double* d_b, double* d_q, int* d_ok, int n) {
    if (!d_a || !d_b || !d_q || !d_ok || n < 0) return nestb::record_error(NEST_ERR_INVALID, "null array or n < 0");
    if (n == 0) return NEST_OK;
    nestb::k_div_selftest<<<(n + 255) / 256, 256>>>(d_a, d_b, d_q, d_ok, n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        return nestb::record_error(NEST_ERR_CUDA, std::string("division self-test: ") + cudaGetErrorString(e));
    return NEST_OK;
}
