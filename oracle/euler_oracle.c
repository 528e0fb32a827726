/*
 * CPU oracle for the nest Euler hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * and the CPU-baseline leg of bench.py load it.  The product path (the CUDA
 * library under nest_b200/) never links, loads or calls anything here.
 *
 * It is a plain-C restatement of nest's OpenMP CPU algorithm with the exact
 * operation order of the reference, so that a non-contracting FP64 GPU kernel
 * can be compared bit for bit.  Build with -ffp-contract=off and without
 * -ffast-math (oracle/Makefile).  Every function names the reference lines it
 * restates (paths relative to the nest source tree).
 *
 * Layouts
 *   1D: SoA U[var * n_total + i], n_total = n + 2h, interior i in [h, h+n)
 *       (src/backend_cuda/euler1d_solver.hpp:38-40).
 *   2D: SoA U[var * (nx+2h)*(ny+2h) + (i+h)*(ny+2h) + (j+h)], x index i is the
 *       slow axis and y index j the fast axis, as nest's row-major
 *       linear_index with idx[1] fastest (include/nest/core.hpp:206-215);
 *       one array for the whole domain with a ghost ring of width h.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NCONS1 3
#define NCONS2 4

enum { ORC_BC_PERIODIC = 0, ORC_BC_OUTFLOW = 1 };
enum { ORC_LIM_MINMOD = 0, ORC_LIM_MC = 1, ORC_LIM_NONE = 2 };

/* std::min / std::max semantics (first argument wins ties and NaN compares). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------------------
 * Gamma-law EOS -- examples/sod1d/euler1d.hpp:27-62
 * ------------------------------------------------------------------------- */

/* eos_t::pressure, euler1d.hpp:31-44 (clamp p >= 0 at :43). */
double orc_pressure(double gamma, double rho, double mom, double erg) {
    double u = mom / rho;
    double ke = 0.5 * rho * u * u;
    double p = (gamma - 1.0) * (erg - ke);
    return smax(p, 0.0);
}

/* eos_t::total_energy, euler1d.hpp:47-51. */
double orc_total_energy(double gamma, double rho, double u, double p) {
    double ke = 0.5 * rho * u * u;
    double ie = p / (gamma - 1.0);
    return ie + ke;
}

/* eos_t::sound_speed, euler1d.hpp:54-56. */
double orc_sound_speed(double gamma, double rho, double p) {
    return sqrt(gamma * p / rho);
}

/* cons_to_prim, euler1d.hpp:69-84. */
void orc_cons_to_prim(double gamma, const double* U, double* W) {
    double rho = U[0], mom = U[1], erg = U[2];
    double u = mom / rho;
    double p = orc_pressure(gamma, rho, mom, erg);
    W[0] = rho; W[1] = u; W[2] = p;
}

/* prim_to_cons, euler1d.hpp:87-100. */
void orc_prim_to_cons(double gamma, const double* W, double* U) {
    double rho = W[0], u = W[1], p = W[2];
    U[0] = rho;
    U[1] = rho * u;
    U[2] = orc_total_energy(gamma, rho, u, p);
}

/* ---------------------------------------------------------------------------
 * Limiters and PLM -- euler1d.hpp:106-171
 * ------------------------------------------------------------------------- */

/* minmod, euler1d.hpp:112-115. */
double orc_minmod(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    return (fabs(a) < fabs(b)) ? a : b;
}

/* mc_limiter via minmod3, euler1d.hpp:117-125. */
double orc_mc(double a, double b) {
    double c = 0.5 * (a + b);
    return orc_minmod(2.0 * a, orc_minmod(c, 2.0 * b));
}

/* apply_limiter, euler1d.hpp:127-137. */
double orc_limit(double left, double right, int lim) {
    switch (lim) {
        case ORC_LIM_MINMOD: return orc_minmod(left, right);
        case ORC_LIM_MC: return orc_mc(left, right);
        case ORC_LIM_NONE: return 0.5 * (left + right);
    }
    return 0.0;
}

/* plm_reconstruct, euler1d.hpp:149-171 (nvar components). */
void orc_plm(const double* Wm, const double* W0, const double* Wp, int nvar,
             int lim, double* WL, double* WR) {
    for (int k = 0; k < nvar; ++k) {
        double dl = W0[k] - Wm[k];
        double dr = Wp[k] - W0[k];
        double s = orc_limit(dl, dr, lim);
        WL[k] = W0[k] - 0.5 * s;
        WR[k] = W0[k] + 0.5 * s;
    }
}

/* ---------------------------------------------------------------------------
 * HLLE flux -- euler1d.hpp:178-242
 * ------------------------------------------------------------------------- */

/* hlle_flux, euler1d.hpp:178-242: Davis speeds, three branches. */
void orc_hlle1d(double gamma, const double* WL, const double* WR, double* F) {
    double rL = WL[0], uL = WL[1], pL = WL[2];
    double cL = orc_sound_speed(gamma, rL, pL);
    double EL = orc_total_energy(gamma, rL, uL, pL);
    double rR = WR[0], uR = WR[1], pR = WR[2];
    double cR = orc_sound_speed(gamma, rR, pR);
    double ER = orc_total_energy(gamma, rR, uR, pR);

    double SL = smin(uL - cL, uR - cR);
    double SR = smax(uL + cL, uR + cR);

    double FL[3] = { rL * uL, rL * uL * uL + pL, (EL + pL) * uL };
    double FR[3] = { rR * uR, rR * uR * uR + pR, (ER + pR) * uR };
    double UL[3] = { rL, rL * uL, EL };
    double UR[3] = { rR, rR * uR, ER };

    if (SL >= 0.0) {
        for (int k = 0; k < 3; ++k) F[k] = FL[k];
    } else if (SR <= 0.0) {
        for (int k = 0; k < 3; ++k) F[k] = FR[k];
    } else {
        for (int k = 0; k < 3; ++k)
            F[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) / (SR - SL);
    }
}

/* ---------------------------------------------------------------------------
 * 1D solver on one SoA array with a ghost ring of width h
 * ------------------------------------------------------------------------- */

/* Ghost fill.  Periodic: the benchmark's fill_halos lambda,
 * examples/benchmark/benchmark_euler1d.cpp:102-110.  Outflow (zero-gradient
 * copy of the nearest interior cell) has no counterpart in nest
 * (docs/EULER_SOLVER.md:249 lists only periodic). */
void orc1d_fill_ghosts(double* U, int n, int h, int bc) {
    int nt = n + 2 * h;
    for (int k = 0; k < NCONS1; ++k) {
        double* u = U + (size_t)k * nt;
        for (int g = 0; g < h; ++g) {
            if (bc == ORC_BC_PERIODIC) {
                u[g] = u[n + g];
                u[h + n + g] = u[h + g];
            } else {
                u[g] = u[h];
                u[h + n + g] = u[h + n - 1];
            }
        }
    }
}

/* Slope limiter of the stage functions below (minmod unless set; the
 * OpenMP path of benchmark_euler1d.cpp:145-154 is minmod, nest's sweeps and
 * plm_reconstruct take any limiter_t).  Process-wide: not for concurrent use
 * with different limiters. */
static int g_lim = ORC_LIM_MINMOD;
void orc_set_limiter(int lim) { g_lim = lim; }

/* One forward-Euler stage U_out = U_in - dt/dx (F_{i+1/2} - F_{i-1/2}) on
 * the interior: the compute_rhs lambda, benchmark_euler1d.cpp:113-165
 * (cons->prim over n_total 116-125, PLM 145-154, two HLLE 156-158,
 * update 160-163).  W is caller scratch of 3*n_total. */
void orc1d_stage(const double* Uin, double* Uout, double* W, int n, int h,
                 double dx, double dt, double gamma) {
    int nt = n + 2 * h;
    for (int i = 0; i < nt; ++i) {
        double Ul[3] = { Uin[i], Uin[nt + i], Uin[2 * nt + i] }, Wl[3];
        orc_cons_to_prim(gamma, Ul, Wl);
        W[i] = Wl[0]; W[nt + i] = Wl[1]; W[2 * nt + i] = Wl[2];
    }
    #pragma omp parallel for schedule(static)
    for (int i = h; i < h + n; ++i) {
        double Wm2[3], Wm1[3], W0[3], Wp1[3], Wp2[3];
        for (int k = 0; k < 3; ++k) {
            Wm2[k] = W[k * nt + i - 2]; Wm1[k] = W[k * nt + i - 1];
            W0[k] = W[k * nt + i];      Wp1[k] = W[k * nt + i + 1];
            Wp2[k] = W[k * nt + i + 2];
        }
        double WLm[3], WRm[3], WLp[3], WRp[3];
        for (int k = 0; k < 3; ++k) {
            double s_im1 = orc_limit(Wm1[k] - Wm2[k], W0[k] - Wm1[k], g_lim);
            double s_i = orc_limit(W0[k] - Wm1[k], Wp1[k] - W0[k], g_lim);
            double s_ip1 = orc_limit(Wp1[k] - W0[k], Wp2[k] - Wp1[k], g_lim);
            WLm[k] = Wm1[k] + 0.5 * s_im1;
            WRm[k] = W0[k] - 0.5 * s_i;
            WLp[k] = W0[k] + 0.5 * s_i;
            WRp[k] = Wp1[k] - 0.5 * s_ip1;
        }
        double FLf[3], FRf[3];
        orc_hlle1d(gamma, WLm, WRm, FLf);
        orc_hlle1d(gamma, WLp, WRp, FRf);
        for (int k = 0; k < 3; ++k)
            Uout[k * nt + i] = Uin[k * nt + i] - (dt / dx) * (FRf[k] - FLf[k]);
    }
}

/* Max |u|+c over the interior: compute_dt lambda,
 * benchmark_euler1d.cpp:168-180 (without the final cfl*dx/ division). */
double orc1d_max_speed(const double* U, int n, int h, double gamma) {
    int nt = n + 2 * h;
    double ms = 0.0;
    for (int i = h; i < h + n; ++i) {
        double rho = U[i], mom = U[nt + i], erg = U[2 * nt + i];
        double u = mom / rho;
        double p = orc_pressure(gamma, rho, mom, erg);
        double c = orc_sound_speed(gamma, rho, p);
        ms = smax(ms, fabs(u) + c);
    }
    return ms;
}

/* One Heun step: benchmark_euler1d.cpp:192-205.  The average
 * U = 0.5 (U + U*) touches the interior only (:201-205). */
void orc1d_rk2_step(double* U, double* Utmp, double* Ustar, double* W, int n,
                    int h, double dx, double dt, double gamma, int bc) {
    int nt = n + 2 * h;
    orc1d_fill_ghosts(U, n, h, bc);
    orc1d_stage(U, Utmp, W, n, h, dx, dt, gamma);
    orc1d_fill_ghosts(Utmp, n, h, bc);
    orc1d_stage(Utmp, Ustar, W, n, h, dx, dt, gamma);
    for (int k = 0; k < NCONS1; ++k)
        for (int i = h; i < h + n; ++i)
            U[k * nt + i] = 0.5 * (U[k * nt + i] + Ustar[k * nt + i]);
}

/* Time loop: benchmark_euler1d.cpp:185-209.
 *   t_final > 0 : run while time < t_final, dt = min(dt, t_final - time)
 *   nsteps  > 0 : stop after nsteps steps (also with t_final > 0)
 *   dts_in      : if non-NULL, use these dt values (frozen sequence)
 *   dts_out     : if non-NULL, record the dt of every step
 * Returns the number of steps; *t_out receives the final time. */
int orc1d_run(double* U, int n, int h, double dx, double gamma, double cfl,
              double t_final, int nsteps, int bc, const double* dts_in,
              double* dts_out, double* t_out) {
    size_t bytes = (size_t)NCONS1 * (n + 2 * h) * sizeof(double);
    double* Utmp = (double*)calloc(1, bytes);
    double* Ustar = (double*)calloc(1, bytes);
    double* W = (double*)calloc(1, bytes);
    double time = 0.0;
    int step = 0;
    for (;;) {
        if (t_final > 0.0 && !(time < t_final)) break;
        if (nsteps > 0 && step >= nsteps) break;
        if (t_final <= 0.0 && nsteps <= 0) break;
        double dt;
        if (dts_in) {
            dt = dts_in[step];
        } else {
            dt = cfl * dx / orc1d_max_speed(U, n, h, gamma);
            if (t_final > 0.0) dt = smin(dt, t_final - time);
        }
        if (dts_out) dts_out[step] = dt;
        orc1d_rk2_step(U, Utmp, Ustar, W, n, h, dx, dt, gamma, bc);
        time += dt;
        ++step;
    }
    free(Utmp); free(Ustar); free(W);
    if (t_out) *t_out = time;
    return step;
}

/* ---------------------------------------------------------------------------
 * Patch form of the 1D right-hand side (sod1d path)
 * ------------------------------------------------------------------------- */

/* euler_rhs_t::operator(), euler1d.hpp:297-396, on one patch stored with its
 * own ghost ring (extended space n_p + 2h).  The first and last interior
 * cells of every patch replace the i-2 / i+2 neighbour by i-1 / i+1
 * (:337-346, :366-374). */
void orc1d_patch_stage(const double* Uin, double* Uout, double* W, int n, int h,
                       double dx, double dt, double gamma) {
    int nt = n + 2 * h;
    for (int i = 0; i < nt; ++i) {
        double Ul[3] = { Uin[i], Uin[nt + i], Uin[2 * nt + i] }, Wl[3];
        orc_cons_to_prim(gamma, Ul, Wl);
        W[i] = Wl[0]; W[nt + i] = Wl[1]; W[2 * nt + i] = Wl[2];
    }
    for (int i = h; i < h + n; ++i) {
        double Wim1[3], Wi[3], Wip1[3], Wim2[3], Wip2[3];
        for (int k = 0; k < 3; ++k) {
            Wim1[k] = W[k * nt + i - 1]; Wi[k] = W[k * nt + i]; Wip1[k] = W[k * nt + i + 1];
            Wim2[k] = (i >= h + 1) ? W[k * nt + i - 2] : Wim1[k];
            Wip2[k] = (i < h + n - 1) ? W[k * nt + i + 2] : Wip1[k];
        }
        double a_L[3], a_R[3], b_L[3], b_R[3], c_L[3], c_R[3];
        orc_plm(Wim2, Wim1, Wi, 3, ORC_LIM_MINMOD, a_L, a_R);
        orc_plm(Wim1, Wi, Wip1, 3, ORC_LIM_MINMOD, b_L, b_R);
        orc_plm(Wi, Wip1, Wip2, 3, ORC_LIM_MINMOD, c_L, c_R);
        double fl[3], fr[3];
        orc_hlle1d(gamma, a_R, b_L, fl);
        orc_hlle1d(gamma, b_R, c_L, fr);
        for (int k = 0; k < 3; ++k)
            Uout[k * nt + i] = Uin[k * nt + i] - (dt / dx) * (fr[k] - fl[k]);
    }
}

/* ---------------------------------------------------------------------------
 * 2D unsplit scheme (no 2D RK2 exists in nest; built from its 1D pieces)
 *
 * Primitives W = (rho, u, v, p).  Kinetic energy is written
 * ((0.5 rho) u) u + ((0.5 rho) v) v so that with v = 0 every operation is the
 * 1D operation of euler1d.hpp:33 and :48 and a y-uniform 2D run reproduces
 * the 1D scheme bit for bit.
 * ------------------------------------------------------------------------- */

static inline double ke2(double rho, double u, double v) {
    return 0.5 * rho * u * u + 0.5 * rho * v * v;
}

/* cons->prim in 2D with the p >= 0 clamp of euler1d.hpp:43. */
void orc_cons_to_prim2d(double gamma, const double* U, double* W) {
    double rho = U[0];
    double u = U[1] / rho;
    double v = U[2] / rho;
    double p = (gamma - 1.0) * (U[3] - ke2(rho, u, v));
    W[0] = rho; W[1] = u; W[2] = v; W[3] = smax(p, 0.0);
}

void orc_prim_to_cons2d(double gamma, const double* W, double* U) {
    double rho = W[0], u = W[1], v = W[2], p = W[3];
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = p / (gamma - 1.0) + ke2(rho, u, v);
}

/* Four-variable HLLE with Davis speeds along the normal direction.
 * Face states are (rho, un, ut, p); the flux is returned in the order
 * (rho, rho*un, rho*ut, E) and mapped to (rho, mu, mv, E) by the caller.
 * Branch structure and operation order follow hlle_flux,
 * euler1d.hpp:178-242; the transverse flux is (rho un) ut. */
void orc_hlle2d(double gamma, const double* WL, const double* WR, double* F) {
    double rL = WL[0], nL = WL[1], tL = WL[2], pL = WL[3];
    double rR = WR[0], nR = WR[1], tR = WR[2], pR = WR[3];
    double cL = sqrt(gamma * pL / rL);
    double cR = sqrt(gamma * pR / rR);
    double EL = pL / (gamma - 1.0) + ke2(rL, nL, tL);
    double ER = pR / (gamma - 1.0) + ke2(rR, nR, tR);
    double SL = smin(nL - cL, nR - cR);
    double SR = smax(nL + cL, nR + cR);
    double FL[4] = { rL * nL, rL * nL * nL + pL, rL * nL * tL, (EL + pL) * nL };
    double FR[4] = { rR * nR, rR * nR * nR + pR, rR * nR * tR, (ER + pR) * nR };
    double UL[4] = { rL, rL * nL, rL * tL, EL };
    double UR[4] = { rR, rR * nR, rR * tR, ER };
    if (SL >= 0.0) {
        for (int k = 0; k < 4; ++k) F[k] = FL[k];
    } else if (SR <= 0.0) {
        for (int k = 0; k < 4; ++k) F[k] = FR[k];
    } else {
        for (int k = 0; k < 4; ++k)
            F[k] = (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k])) / (SR - SL);
    }
}

#define IX2(i, j) ((size_t)((i) + h) * (size_t)(ny + 2 * h) + (size_t)((j) + h))

/* Ghost ring of the whole domain (faces only; corners are never read by the
 * 5-point cross stencil).  Periodic wrap follows build_periodic_mesh_2d,
 * include/nest/patch.hpp:207-326; outflow is zero-gradient. */
void orc2d_fill_ghosts(double* U, int nx, int ny, int h, int bcx, int bcy) {
    size_t plane = (size_t)(nx + 2 * h) * (size_t)(ny + 2 * h);
    for (int k = 0; k < NCONS2; ++k) {
        double* u = U + k * plane;
        for (int g = 1; g <= h; ++g) {
            for (int j = 0; j < ny; ++j) {
                if (bcx == ORC_BC_PERIODIC) {
                    u[IX2(-g, j)] = u[IX2(nx - g, j)];
                    u[IX2(nx - 1 + g, j)] = u[IX2(g - 1, j)];
                } else {
                    u[IX2(-g, j)] = u[IX2(0, j)];
                    u[IX2(nx - 1 + g, j)] = u[IX2(nx - 1, j)];
                }
            }
            for (int i = 0; i < nx; ++i) {
                if (bcy == ORC_BC_PERIODIC) {
                    u[IX2(i, -g)] = u[IX2(i, ny - g)];
                    u[IX2(i, ny - 1 + g)] = u[IX2(i, g - 1)];
                } else {
                    u[IX2(i, -g)] = u[IX2(i, 0)];
                    u[IX2(i, ny - 1 + g)] = u[IX2(i, ny - 1)];
                }
            }
        }
    }
}

/* Load primitives of cell (i, j) into (rho, un, ut, p) order. */
static inline void w_at(const double* W, size_t plane, size_t idx, int xdir, double* out) {
    out[0] = W[idx];
    out[1] = W[(xdir ? 1 : 2) * plane + idx];
    out[2] = W[(xdir ? 2 : 1) * plane + idx];
    out[3] = W[3 * plane + idx];
}

/* Flux through the face between cells a (left/bottom) and b, with a2 the
 * cell before a and b2 the cell after b along the normal. */
static void face_flux(const double* W, size_t plane, size_t a2, size_t a, size_t b,
                      size_t b2, int xdir, double gamma, double* F) {
    double Wa2[4], Wa[4], Wb[4], Wb2[4], WLf[4], WRf[4];
    w_at(W, plane, a2, xdir, Wa2); w_at(W, plane, a, xdir, Wa);
    w_at(W, plane, b, xdir, Wb);   w_at(W, plane, b2, xdir, Wb2);
    for (int k = 0; k < 4; ++k) {
        double sa = orc_limit(Wa[k] - Wa2[k], Wb[k] - Wa[k], g_lim);
        double sb = orc_limit(Wb[k] - Wa[k], Wb2[k] - Wb[k], g_lim);
        WLf[k] = Wa[k] + 0.5 * sa;
        WRf[k] = Wb[k] - 0.5 * sb;
    }
    double f[4];
    orc_hlle2d(gamma, WLf, WRf, f);
    /* map (rho, rho un, rho ut, E) -> (rho, mu, mv, E) */
    F[0] = f[0];
    F[1] = xdir ? f[1] : f[2];
    F[2] = xdir ? f[2] : f[1];
    F[3] = f[3];
}

/* One forward-Euler stage of the unsplit scheme on the interior:
 *   U_out = U_in - (dt/dx (F_{i+1/2} - F_{i-1/2}) + dt/dy (G_{j+1/2} - G_{j-1/2}))
 * The per-face arithmetic is the per-interface work of
 * benchmark_euler1d.cpp:145-158 applied along each axis.  W is caller
 * scratch of 4 planes. */
void orc2d_stage(const double* Uin, double* Uout, double* W, int nx, int ny, int h,
                 double dtdx, double dtdy, double gamma) {
    size_t plane = (size_t)(nx + 2 * h) * (size_t)(ny + 2 * h);
    int nxt = nx + 2 * h;
    #pragma omp parallel for schedule(static)
    for (int ii = 0; ii < nxt; ++ii) {
        for (int jj = 0; jj < ny + 2 * h; ++jj) {
            size_t idx = (size_t)ii * (size_t)(ny + 2 * h) + (size_t)jj;
            double U[4] = { Uin[idx], Uin[plane + idx], Uin[2 * plane + idx], Uin[3 * plane + idx] };
            double Wl[4];
            orc_cons_to_prim2d(gamma, U, Wl);
            for (int k = 0; k < 4; ++k) W[k * plane + idx] = Wl[k];
        }
    }
    size_t sx = (size_t)(ny + 2 * h);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            size_t c = IX2(i, j);
            double fxm[4], fxp[4], fym[4], fyp[4];
            face_flux(W, plane, c - 2 * sx, c - sx, c, c + sx, 1, gamma, fxm);
            face_flux(W, plane, c - sx, c, c + sx, c + 2 * sx, 1, gamma, fxp);
            face_flux(W, plane, c - 2, c - 1, c, c + 1, 0, gamma, fym);
            face_flux(W, plane, c - 1, c, c + 1, c + 2, 0, gamma, fyp);
            for (int k = 0; k < 4; ++k)
                Uout[k * plane + c] = Uin[k * plane + c] -
                    (dtdx * (fxp[k] - fxm[k]) + dtdy * (fyp[k] - fym[k]));
        }
    }
}

/* Max of |u|+c and |v|+c over the interior with the 1e-10 floors of
 * compute_dt_2d, examples/sod2d/euler2d.hpp:242-271. */
void orc2d_max_speeds(const double* U, int nx, int ny, int h, double gamma,
                      double* sx_out, double* sy_out) {
    size_t plane = (size_t)(nx + 2 * h) * (size_t)(ny + 2 * h);
    double msx = 0.0, msy = 0.0;
    #pragma omp parallel for reduction(max:msx, msy) schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            size_t c = IX2(i, j);
            double rho = smax(U[c], 1e-10);
            double u = U[plane + c] / rho;
            double v = U[2 * plane + c] / rho;
            double ke = 0.5 * rho * (u * u + v * v);
            double p = smax((gamma - 1.0) * (U[3 * plane + c] - ke), 1e-10);
            double cs = sqrt(gamma * p / rho);
            double a = fabs(u) + cs, b = fabs(v) + cs;
            if (a > msx) msx = a;
            if (b > msy) msy = b;
        }
    }
    *sx_out = msx; *sy_out = msy;
}

/* dt = cfl * min(dx / max(|u|+c), dy / max(|v|+c)), euler2d.hpp:249-270.
 * min over cells of dx/s equals dx/max(s) for correctly rounded division. */
double orc2d_dt_from_speeds(double sx, double sy, double dx, double dy, double cfl) {
    double dt_x = 1e10, dt_y = 1e10;
    if (sx > 0.0) dt_x = smin(dt_x, dx / sx);
    if (sy > 0.0) dt_y = smin(dt_y, dy / sy);
    return cfl * smin(dt_x, dt_y);
}

/* One Heun step of the unsplit scheme (U1 = U + dt L(U), U** = U1 + dt L(U1),
 * U = 0.5 (U + U**)), the 2D analogue of benchmark_euler1d.cpp:192-205. */
void orc2d_rk2_step(double* U, double* U1, double* Us, double* W, int nx, int ny,
                    int h, double dx, double dy, double dt, double gamma, int bcx, int bcy) {
    size_t plane = (size_t)(nx + 2 * h) * (size_t)(ny + 2 * h);
    double dtdx = dt / dx, dtdy = dt / dy;
    orc2d_fill_ghosts(U, nx, ny, h, bcx, bcy);
    orc2d_stage(U, U1, W, nx, ny, h, dtdx, dtdy, gamma);
    orc2d_fill_ghosts(U1, nx, ny, h, bcx, bcy);
    orc2d_stage(U1, Us, W, nx, ny, h, dtdx, dtdy, gamma);
    for (int k = 0; k < NCONS2; ++k) {
        #pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                size_t c = k * plane + IX2(i, j);
                U[c] = 0.5 * (U[c] + Us[c]);
            }
    }
}

/* 2D time loop with the same stopping rules as orc1d_run. */
int orc2d_run(double* U, int nx, int ny, int h, double dx, double dy, double gamma,
              double cfl, double t_final, int nsteps, int bcx, int bcy, const double* dts_in,
              double* dts_out, double* t_out) {
    size_t bytes = (size_t)NCONS2 * (nx + 2 * h) * (ny + 2 * h) * sizeof(double);
    double* U1 = (double*)calloc(1, bytes);
    double* Us = (double*)calloc(1, bytes);
    double* W = (double*)calloc(1, bytes);
    double time = 0.0;
    int step = 0;
    for (;;) {
        if (t_final > 0.0 && !(time < t_final)) break;
        if (nsteps > 0 && step >= nsteps) break;
        if (t_final <= 0.0 && nsteps <= 0) break;
        double dt;
        if (dts_in) {
            dt = dts_in[step];
        } else {
            double sx, sy;
            orc2d_max_speeds(U, nx, ny, h, gamma, &sx, &sy);
            dt = orc2d_dt_from_speeds(sx, sy, dx, dy, cfl);
            if (t_final > 0.0) dt = smin(dt, t_final - time);
        }
        if (dts_out) dts_out[step] = dt;
        orc2d_rk2_step(U, U1, Us, W, nx, ny, h, dx, dy, dt, gamma, bcx, bcy);
        time += dt;
        ++step;
    }
    free(U1); free(Us); free(W);
    if (t_out) *t_out = time;
    return step;
}

/* Conserved totals over the interior times the cell area (the FP64 totals of
 * the FP32 form are checked against this). */
void orc2d_totals(const double* U, int nx, int ny, int h, double dx, double dy, double* out) {
    size_t plane = (size_t)(nx + 2 * h) * (size_t)(ny + 2 * h);
    for (int k = 0; k < NCONS2; ++k) {
        double s = 0.0;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) s += U[k * plane + IX2(i, j)];
        out[k] = s * dx * dy;
    }
}
