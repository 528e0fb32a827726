// 2D unsplit Euler stage kernels for sm_100a (template; instantiated in
// euler2d_f64.cu with -fmad=false and in euler2d_f32.cu with fast FP32 math).
//
// Scheme (one forward-Euler stage, both axes at once):
//   U_out = U_in - (dt/dx (F_{i+1/2} - F_{i-1/2}) + dt/dy (G_{j+1/2} - G_{j-1/2}))
// with PLM-minmod on (rho, u, v, p) along each axis and a four-variable HLLE
// flux with Davis speeds; the per-face arithmetic restates nest's 1D
// interface work (examples/benchmark/benchmark_euler1d.cpp:145-158,
// examples/sod1d/euler1d.hpp:178-242) along the face normal.
//
// HBM layout: one SoA array per solver, plane v at v*vstride, row x = i (slow
// axis, i in [-2, nx+2)), column y = j (fast axis, contiguous), pitch >= ny+4.
// This is nest's field_t row-major order with idx[1] fastest
// (include/nest/core.hpp:206-215) for the whole domain; patches are index
// ranges of it, so faces between patches are read directly and only the
// domain boundary needs ghost cells.
//
// Work decomposition: a warp owns a strip of 28 output columns.  Its 32 lanes
// cover columns j0-2 .. j0+29 (lanes 0,1,30,31 are halo lanes whose results
// are discarded) and march down TX rows keeping a three-row register window,
// so every x-face is computed once from registers; y-neighbours come from
// warp shuffles.  There is no shared memory and no block-wide barrier.
#pragma once

#include "common.cuh"

namespace nestb {

constexpr int STRIP = 28;  // output columns per warp

template <typename T> struct Pol;

// FP64 plain form: IEEE division and square root in nest's operation order.
template <> struct Pol<double> {
    static constexpr bool exact = true;
    __device__ static __forceinline__ double div(double a, double b) { return a / b; }
    __device__ static __forceinline__ double rcp(double b) { return 1.0 / b; }
    __device__ static __forceinline__ double sound(double gamma, double p, double rho) { return sqrt(gamma * p / rho); }
};

// FP32 form: approximate reciprocal / reciprocal square root (one MUFU each).
template <> struct Pol<float> {
    static constexpr bool exact = false;
    __device__ static __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    __device__ static __forceinline__ float rcp(float b) { return __fdividef(1.0f, b); }
    // c = sqrt(g p / rho) = g p / sqrt(g p rho); the clamp keeps p = 0 finite (c = 0).
    __device__ static __forceinline__ float sound(float gamma, float p, float rho) {
        float gp = gamma * p;
        return gp * rsqrtf(fmaxf(gp * rho, 1e-37f));
    }
};

struct Geo2D {
    int nx, ny;           // interior cells
    int pitch;            // elements per row
    long long vstride;    // elements per variable plane
    int bcx, bcy;         // boundary condition along x (rows) and y (columns)
    double dx, dy, gamma;
    int xlo_ex, xhi_ex;   // 1: that x side's ghost rows are filled by a halo exchange (sharded domain)
    __device__ __forceinline__ long long at(int i, int j) const {
        return (long long)(i + 2) * pitch + (j + 2);
    }
};

template <typename T>
struct Prim4 { T r, u, v, p; };

// ((0.5 rho) u) u + ((0.5 rho) v) v: with v = 0 this is bit for bit the 1D
// kinetic energy of euler1d.hpp:33/:48.
template <typename T>
__device__ __forceinline__ T ke2(T r, T u, T v) {
    return T(0.5) * r * u * u + T(0.5) * r * v * v;
}

// cons -> prim with the p >= 0 clamp of euler1d.hpp:43.  REPAIR (FP32 form)
// recomputes rho and p in FP64 with floors when FP32 gives rho or p below
// them (near vacuum the cancellation E - ke loses all FP32 digits).
template <typename T, bool REPAIR>
__device__ __forceinline__ Prim4<T> cons2prim(T U0, T U1, T U2, T U3, T gm1) {
    Prim4<T> w;
    w.r = U0;
    if (Pol<T>::exact) {
        w.u = Pol<T>::div(U1, U0);
        w.v = Pol<T>::div(U2, U0);
    } else {
        T ir = Pol<T>::rcp(U0);
        w.u = U1 * ir;
        w.v = U2 * ir;
    }
    T p = gm1 * (U3 - ke2(w.r, w.u, w.v));
    w.p = smax(p, T(0));
    if (REPAIR) {
        const double floor_ = 1e-10;
        if (!(w.r >= T(floor_)) || !(w.p >= T(floor_))) {
            double r = smax((double)U0, floor_);
            double u = (double)U1 / r, v = (double)U2 / r;
            double pd = (double)gm1 * ((double)U3 - (0.5 * r * u * u + 0.5 * r * v * v));
            w.r = (T)r; w.u = (T)u; w.v = (T)v; w.p = (T)smax(pd, floor_);
        }
    }
    return w;
}

// Four-variable HLLE along the normal: states are (rho, un, ut, p); the flux
// returns (rho un, rho un un + p, rho un ut, (E + p) un).  Operation order
// and branches follow hlle_flux, euler1d.hpp:178-242.
template <typename T>
__device__ __forceinline__ void hlle4(T gamma, T gm1, T igm1,
                                      T rL, T nL, T tL, T pL, T rR, T nR, T tR, T pR,
                                      T& f0, T& f1, T& f2, T& f3) {
    T cL = Pol<T>::sound(gamma, pL, rL);
    T cR = Pol<T>::sound(gamma, pR, rR);
    T EL = (Pol<T>::exact ? Pol<T>::div(pL, gm1) : pL * igm1) + ke2(rL, nL, tL);
    T ER = (Pol<T>::exact ? Pol<T>::div(pR, gm1) : pR * igm1) + ke2(rR, nR, tR);
    T SL = smin(nL - cL, nR - cR);
    T SR = smax(nL + cL, nR + cR);
    T mL = rL * nL, mR = rR * nR;
    T FL0 = mL, FL1 = mL * nL + pL, FL2 = mL * tL, FL3 = (EL + pL) * nL;
    T FR0 = mR, FR1 = mR * nR + pR, FR2 = mR * tR, FR3 = (ER + pR) * nR;
    if (Pol<T>::exact) {
        if (SL >= T(0)) {
            f0 = FL0; f1 = FL1; f2 = FL2; f3 = FL3;
        } else if (SR <= T(0)) {
            f0 = FR0; f1 = FR1; f2 = FR2; f3 = FR3;
        } else {
            T SLR = SL * SR, dS = SR - SL;
            f0 = Pol<T>::div(SR * FL0 - SL * FR0 + SLR * (rR - rL), dS);
            f1 = Pol<T>::div(SR * FL1 - SL * FR1 + SLR * (mR - mL), dS);
            f2 = Pol<T>::div(SR * FL2 - SL * FR2 + SLR * (rR * tR - rL * tL), dS);
            f3 = Pol<T>::div(SR * FL3 - SL * FR3 + SLR * (ER - EL), dS);
        }
    } else {
        // Branchless HLLE: with sl = min(SL, 0) and sr = max(SR, 0) the
        // average formula reduces to F_L when SL >= 0 and to F_R when SR <= 0.
        T sl = fmin(SL, T(0)), sr = fmax(SR, T(0));
        T inv = Pol<T>::rcp(fmax(sr - sl, T(1e-30)));
        T a = sr * inv, b = sl * inv, c = sl * sr * inv;
        f0 = a * FL0 - b * FR0 + c * (rR - rL);
        f1 = a * FL1 - b * FR1 + c * (mR - mL);
        f2 = a * FL2 - b * FR2 + c * (rR * tR - rL * tL);
        f3 = a * FL3 - b * FR3 + c * (ER - EL);
    }
}

// Wave speeds |u|+c, |v|+c of a conserved state with the 1e-10 floors of
// compute_dt_2d (examples/sod2d/euler2d.hpp:254-263).  Returns the pressure
// of cons2prim before its clamp, (gamma-1) (E - ke2(rho, u, v)), for the
// positivity check: for rho >= 1e-10 (no floor) u and v are cons2prim's, so
// this is the scheme's own pressure.
template <typename T>
__device__ __forceinline__ T cell_speeds_p(T U0, T U1, T U2, T U3, T gamma, T gm1, T& sx, T& sy) {
    T rho = smax(U0, T(1e-10));
    T u, v;
    if (Pol<T>::exact) {
        u = Pol<T>::div(U1, rho);
        v = Pol<T>::div(U2, rho);
    } else {
        T ir = Pol<T>::rcp(rho);
        u = U1 * ir;
        v = U2 * ir;
    }
    T ke = T(0.5) * rho * (u * u + v * v);
    T p = smax(gm1 * (U3 - ke), T(1e-10));
    T c = Pol<T>::sound(gamma, p, rho);
    sx = fabs(u) + c;
    sy = fabs(v) + c;
    return gm1 * (U3 - ke2(rho, u, v));
}

template <typename T>
__device__ __forceinline__ void cell_speeds(T U0, T U1, T U2, T U3, T gamma, T gm1, T& sx, T& sy) {
    (void)cell_speeds_p<T>(U0, U1, U2, U3, gamma, gm1, sx, sy);
}

// dt = cfl * min(dx / max(|u|+c), dy / max(|v|+c)), euler2d.hpp:249-270.
__device__ __forceinline__ double dt_from_speeds(double sx, double sy, double dx, double dy, double cfl) {
    double dtx = 1e10, dty = 1e10;
    if (sx > 0.0) dtx = smin(dtx, dx / sx);
    if (sy > 0.0) dty = smin(dty, dy / sy);
    return cfl * smin(dtx, dty);
}

template <typename T>
__device__ __forceinline__ void store_ghosts(T* Uo, const Geo2D& g, int k, int i, int j, T v) {
    T* p = Uo + (long long)k * g.vstride;
    if (g.bcy == BC_PERIODIC) {
        if (j < 2) p[g.at(i, j + g.ny)] = v;
        if (j >= g.ny - 2) p[g.at(i, j - g.ny)] = v;
    } else {
        if (j == 0) { p[g.at(i, -1)] = v; p[g.at(i, -2)] = v; }
        if (j == g.ny - 1) { p[g.at(i, g.ny)] = v; p[g.at(i, g.ny + 1)] = v; }
    }
    if (g.bcx == BC_PERIODIC) {
        if (i < 2 && !g.xhi_ex) p[g.at(i + g.nx, j)] = v;
        if (i >= g.nx - 2 && !g.xlo_ex) p[g.at(i - g.nx, j)] = v;
    } else {
        if (i == 0 && !g.xlo_ex) { p[g.at(-1, j)] = v; p[g.at(-2, j)] = v; }
        if (i == g.nx - 1 && !g.xhi_ex) { p[g.at(g.nx, j)] = v; p[g.at(g.nx + 1, j)] = v; }
    }
}

template <typename T>
struct Win4 { T a, b, c, d; };

template <typename T>
__device__ __forceinline__ Win4<T> shfl_up4(const Win4<T>& x) {
    return { __shfl_up_sync(0xffffffffu, x.a, 1), __shfl_up_sync(0xffffffffu, x.b, 1),
             __shfl_up_sync(0xffffffffu, x.c, 1), __shfl_up_sync(0xffffffffu, x.d, 1) };
}
template <typename T>
__device__ __forceinline__ Win4<T> shfl_dn4(const Win4<T>& x) {
    return { __shfl_down_sync(0xffffffffu, x.a, 1), __shfl_down_sync(0xffffffffu, x.b, 1),
             __shfl_down_sync(0xffffffffu, x.c, 1), __shfl_down_sync(0xffffffffu, x.d, 1) };
}

template <typename T>
__device__ __forceinline__ Win4<T> prim_win(const Prim4<T>& w) { return { w.r, w.u, w.v, w.p }; }

template <typename T>
__device__ __forceinline__ Win4<T> limit4(const Win4<T>& m, const Win4<T>& o, const Win4<T>& p, int lim) {
    return { limit(o.a - m.a, p.a - o.a, lim), limit(o.b - m.b, p.b - o.b, lim),
             limit(o.c - m.c, p.c - o.c, lim), limit(o.d - m.d, p.d - o.d, lim) };
}

// Per-launch arguments of a stage kernel.
template <typename T>
struct StageArgs {
    const T* __restrict__ Uin;  // stage input with filled ghost ring
    const T* Un;                // stage 2: U^n (own cell only)
    T* Uout;                    // output (stage 2 may alias Un)
    Geo2D g;
    LoopParams lp;
    StepCtrl* ctrl;
    double* partials;           // per-warp FP64 totals (stage 2, may be null)
    int p;                      // step parity
    int tx;                     // rows per tile
};

// One stage.  STAGE 1: U1 = U + dt L(U).  STAGE 2: U = 0.5 (U + U1 + dt L(U1)),
// plus the max wave speeds of the new state (next dt) and optional totals.
template <typename T, int STAGE, bool REPAIR>
__device__ __forceinline__ void stage2d_body(const StageArgs<T>& a, int strip, int tile_row) {
    const Geo2D& g = a.g;
    const int lane = threadIdx.x & 31;
    const T gamma = (T)g.gamma;
    const T gm1 = (T)(g.gamma - 1.0);
    const T igm1 = (T)(1.0 / (g.gamma - 1.0));

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
    const T dtdx = (T)(dt / g.dx);
    const T dtdy = (T)(dt / g.dy);

    const int j0 = strip * STRIP;          // first output column of the strip
    if (j0 >= g.ny) return;                // whole warp idle (uniform)
    const int j = j0 - 2 + lane;           // this lane's column
    const int jc = min(j, g.ny + 1);       // clamped for loads
    const bool out_col = (lane >= 2) && (lane < 30) && (j < g.ny);
    const int i0 = tile_row * a.tx;
    if (i0 >= g.nx) return;
    const int rows = min(a.tx, g.nx - i0);
    const long long vs = g.vstride;
    const T* __restrict__ Ui = a.Uin;

    auto load = [&](int i, T& u0, T& u1, T& u2, T& u3) {
        long long o = g.at(i, jc);
        u0 = __ldg(Ui + o); u1 = __ldg(Ui + vs + o); u2 = __ldg(Ui + 2 * vs + o); u3 = __ldg(Ui + 3 * vs + o);
    };

    // Window: rows r-2, r-1, r (W0, W1, W2); slopes of rows r-2, r-1 (S0, S1);
    // conserved values of rows r-2, r-1, r (C0, C1, C2); x-flux of face (r-3)+1/2.
    Win4<T> W0, W1, W2, S0, S1, Fp;
    Win4<T> nxt, C0, N0;
    double smx = 0.0, smy = 0.0;
    double tot0 = 0.0, tot1 = 0.0, tot2 = 0.0, tot3 = 0.0;

    load(i0 - 2, nxt.a, nxt.b, nxt.c, nxt.d);
    for (int r = -2; r <= rows + 1; ++r) {
        Win4<T> cur = nxt;
        if (r + 1 <= rows + 1) load(i0 + r + 1, nxt.a, nxt.b, nxt.c, nxt.d);
        if (r >= 2) {
            // conserved values of the row to update (an L1 hit: loaded as
            // `cur` two iterations ago) and, for stage 2, its U^n, requested
            // ahead of this iteration's flux work
            load(i0 + r - 2, C0.a, C0.b, C0.c, C0.d);
            if (STAGE == 2) {
                long long o = g.at(i0 + r - 2, jc);
                N0.a = a.Un[o]; N0.b = a.Un[vs + o]; N0.c = a.Un[2 * vs + o]; N0.d = a.Un[3 * vs + o];
            }
        }
        Prim4<T> w = cons2prim<T, REPAIR>(cur.a, cur.b, cur.c, cur.d, gm1);
        W0 = W1; W1 = W2; W2 = prim_win(w);
        if (r >= 0) {
            S0 = S1;
            S1 = limit4(W0, W1, W2, a.lp.lim);  // slope of row r-1
        }
        if (r >= 1) {
            // x-face between rows r-2 and r-1 (normal u, transverse v)
            Win4<T> Fc;
            hlle4<T>(gamma, gm1, igm1,
                     W0.a + T(0.5) * S0.a, W0.b + T(0.5) * S0.b, W0.c + T(0.5) * S0.c, W0.d + T(0.5) * S0.d,
                     W1.a - T(0.5) * S1.a, W1.b - T(0.5) * S1.b, W1.c - T(0.5) * S1.c, W1.d - T(0.5) * S1.d,
                     Fc.a, Fc.b, Fc.c, Fc.d);
            if (r >= 2) {
                // update row q = r - 2 with x-faces q-1/2 (Fp) and q+1/2 (Fc)
                const int i = i0 + r - 2;
                // y-direction on row q (window W0): slopes, faces, neighbours
                Win4<T> Wl = shfl_up4(W0), Wr = shfl_dn4(W0);
                Win4<T> sy = limit4(Wl, W0, Wr, a.lp.lim);
                Win4<T> Mq = { W0.a - T(0.5) * sy.a, W0.b - T(0.5) * sy.b, W0.c - T(0.5) * sy.c, W0.d - T(0.5) * sy.d };
                Win4<T> Rq = shfl_dn4(Mq);
                Win4<T> Gy;  // face j+1/2: normal v, transverse u
                hlle4<T>(gamma, gm1, igm1,
                         W0.a + T(0.5) * sy.a, W0.c + T(0.5) * sy.c, W0.b + T(0.5) * sy.b, W0.d + T(0.5) * sy.d,
                         Rq.a, Rq.c, Rq.b, Rq.d,
                         Gy.a, Gy.c, Gy.b, Gy.d);
                Win4<T> Gl = shfl_up4(Gy);
                if (out_col) {
                    T s0 = C0.a - (dtdx * (Fc.a - Fp.a) + dtdy * (Gy.a - Gl.a));
                    T s1 = C0.b - (dtdx * (Fc.b - Fp.b) + dtdy * (Gy.b - Gl.b));
                    T s2 = C0.c - (dtdx * (Fc.c - Fp.c) + dtdy * (Gy.c - Gl.c));
                    T s3 = C0.d - (dtdx * (Fc.d - Fp.d) + dtdy * (Gy.d - Gl.d));
                    if (STAGE == 2) {
                        s0 = T(0.5) * (N0.a + s0);
                        s1 = T(0.5) * (N0.b + s1);
                        s2 = T(0.5) * (N0.c + s2);
                        s3 = T(0.5) * (N0.d + s3);
                        // FP32 form: the FP64 repair below can only trigger for cells
                        // whose FP32 pressure is under 1e-5 (gamma-1)(|E| + ke) (the
                        // FP32 rounding error is far smaller), so other cells skip it.
                        bool near = true;
                        if (REPAIR && !Pol<T>::exact) {
                            T r32 = smax(s0, T(1e-10)), ir32 = Pol<T>::rcp(r32);
                            T u32 = s1 * ir32, v32 = s2 * ir32;
                            T ke32 = ke2(r32, u32, v32);
                            T p32 = gm1 * (s3 - ke32);
                            near = !(s0 >= T(1e-10)) || !(p32 >= T(1e-10) + T(1e-5) * gm1 * (fabs(s3) + ke32));
                        }
                        if (REPAIR && near) {
                            // positivity repair of the new state in FP64
                            const double fl = 1e-10;
                            double r_ = (double)s0;
                            double u_ = (double)s1 / smax(r_, fl), v_ = (double)s2 / smax(r_, fl);
                            double keD = 0.5 * smax(r_, fl) * (u_ * u_ + v_ * v_);
                            double pD = (g.gamma - 1.0) * ((double)s3 - keD);
                            if (!(r_ >= fl) || !(pD >= fl)) {
                                r_ = smax(r_, fl);
                                double e_ = keD + fl / (g.gamma - 1.0);
                                s0 = (T)r_;
                                s3 = (T)smax((double)s3, e_);
                                atomicAdd(&a.ctrl->repairs, 1u);
                            }
                        }
                        T sx, syv;
                        const T pc = cell_speeds_p<T>(s0, s1, s2, s3, gamma, gm1, sx, syv);
                        // positivity (REPAIR: NaN only, the repair keeps rho and p positive in FP64)
                        if (REPAIR ? (!(s0 == s0) || !(pc == pc)) : (!(s0 >= T(1e-10)) || !(pc > T(0)))) {
                            T pe = pc;
                            if (s0 > T(0) && s0 < T(1e-10)) {  // rho under the speed floor: unfloored pressure
                                T ue = Pol<T>::div(s1, s0), ve = Pol<T>::div(s2, s0);
                                pe = gm1 * (s3 - ke2(s0, ue, ve));
                            }
                            if (!(s0 > T(0)) || !(pe > T(0)) || !(pe == pe))
                                flag_cell(a.ctrl, a.ctrl->step[a.p] + 1, (double)s0, (double)pe, i, j);
                        }
                        smx = smax(smx, (double)sx);
                        smy = smax(smy, (double)syv);
                        tot0 += (double)s0; tot1 += (double)s1; tot2 += (double)s2; tot3 += (double)s3;
                    }
                    {
                        long long o = g.at(i, j);
                        a.Uout[o] = s0; a.Uout[vs + o] = s1; a.Uout[2 * vs + o] = s2; a.Uout[3 * vs + o] = s3;
                    }
                    if (i < 2 || i >= g.nx - 2 || j < 2 || j >= g.ny - 2) {
                        store_ghosts(a.Uout, g, 0, i, j, s0);
                        store_ghosts(a.Uout, g, 1, i, j, s1);
                        store_ghosts(a.Uout, g, 2, i, j, s2);
                        store_ghosts(a.Uout, g, 3, i, j, s3);
                    }
                }
            }
            Fp = Fc;
        }
    }
    if (STAGE == 2) {
        smx = warp_max(smx);
        smy = warp_max(smy);
        if (lane == 0) {
            if (!(smx == smx) || !(smy == smy) || smx > 1.79e308 || smy > 1.79e308)
                atomicOr(&a.ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][0], smx);
            atomic_max_speed(&a.ctrl->maxs[a.p ^ 1][1], smy);
        }
        if (a.partials) {
            tot0 = warp_sum(tot0); tot1 = warp_sum(tot1); tot2 = warp_sum(tot2); tot3 = warp_sum(tot3);
            if (lane == 0) {
                long long wid = ((long long)tile_row * ((g.ny + STRIP - 1) / STRIP) + strip) * 4;
                a.partials[wid + 0] = tot0; a.partials[wid + 1] = tot1;
                a.partials[wid + 2] = tot2; a.partials[wid + 3] = tot3;
            }
        }
    }
}

// One problem of a batch: its geometry, the offset of its arrays inside the
// batch buffers, and the index of its first work item (its totals slots).
struct BatchProblem {
    Geo2D g;
    long long off;
    int item0;
    int pad;
};

// Arguments of a persistent batched stage launch.
template <typename T>
struct BatchArgs {
    T* U;                       // all problems' states, problem p at U + probs[p].off
    T* U1;                      // stage buffers, same offsets
    const BatchProblem* probs;
    const int4* items;          // (problem, strip, tile row, 0)
    int nitems;
    StepCtrl* ctrls;            // one control block per problem
    double* partials;           // per-item FP64 totals (stage 2) or null
    LoopParams lp;
    int p;
    int tx;
    int nprobs;                 // number of problems
    int ghost_blocks;           // FP32 ghost-ring pass: blocks per problem
};

// Ghost ring (faces and corners) and wave-speed maxima of the current state
// into slot p.  Run once after an upload or an external state change.
template <typename T>
__device__ __forceinline__ void prepare2d_body(T* U, const Geo2D& g, StepCtrl* ctrl, int p) {
    // Blocks of 32 x 8 threads: columns across a warp, rows strided by the grid's
    // row extent, so each warp folds many cells before the block's one atomic pair.
    const T gamma = (T)g.gamma;
    const T gm1 = (T)(g.gamma - 1.0);
    const int j = blockIdx.x * blockDim.x + threadIdx.x - 2;  // column in [-2, ny+2)
    double smx = 0.0, smy = 0.0;
    for (int i = blockIdx.y * blockDim.y + threadIdx.y - 2; i < g.nx + 2; i += gridDim.y * blockDim.y) {
        bool in = (j >= -2 && j < g.ny + 2);
        if ((i < 0 && g.xlo_ex) || (i >= g.nx && g.xhi_ex)) in = false;  // filled by the halo exchange
        if (!in) continue;
        // source cell: wrap (periodic) or clamp (outflow) each axis
        int si = i, sj = j;
        if (i < 0 || i >= g.nx) si = (g.bcx == BC_PERIODIC) ? ((i + g.nx) % g.nx) : (i < 0 ? 0 : g.nx - 1);
        if (j < 0 || j >= g.ny) sj = (g.bcy == BC_PERIODIC) ? ((j + g.ny) % g.ny) : (j < 0 ? 0 : g.ny - 1);
        if (si != i || sj != j) {
            for (int k = 0; k < 4; ++k) U[k * g.vstride + g.at(i, j)] = U[k * g.vstride + g.at(si, sj)];
        } else {
            T sx, sy;
            long long o = g.at(i, j);
            cell_speeds<T>(U[o], U[g.vstride + o], U[2 * g.vstride + o], U[3 * g.vstride + o], gamma, gm1, sx, sy);
            smx = smax(smx, (double)sx);
            smy = smax(smy, (double)sy);
        }
    }
    smx = warp_max(smx);
    smy = warp_max(smy);
    __shared__ double red[2][32];
    const int w = (threadIdx.y * blockDim.x + threadIdx.x) >> 5, nw = (blockDim.x * blockDim.y) >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = smx; red[1][w] = smy; }
    __syncthreads();
    if (w == 0) {
        const int l = threadIdx.x & 31;
        smx = l < nw ? red[0][l] : 0.0;
        smy = l < nw ? red[1][l] : 0.0;
        smx = warp_max(smx);
        smy = warp_max(smy);
        if (l == 0) {
            atomic_max_speed(&ctrl->maxs[p][0], smx);
            atomic_max_speed(&ctrl->maxs[p][1], smy);
        }
    }
}

}  // namespace nestb
