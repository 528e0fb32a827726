// nest's own 2D scheme on the device (compatibility mode), FP64.
//
// nest's 2D CPU path (examples/sod2d/euler2d.hpp:67-271, driven by
// examples/sod2d/sod2d.cpp:318-366) is dimensionally split forward Euler:
// an x-sweep then a y-sweep per step, each updating (rho, rho u_n, E) with
// nest's 1D HLLE on (rho, u_n, p) -- kinetic energy of the normal velocity
// only -- and the transverse momentum as a passive scalar upwinded by the
// HLLE interface velocity; primitives carry the 1e-10 floors of
// get_prim_2d (euler2d.hpp:36-64).  These kernels restate that arithmetic
// in the same operation order (compiled with -fmad=false), so a device run
// equals nest's sod2d bit for bit.  One thread per cell: this mode exists for
// parity with nest, the unsplit RK2 kernels are the fast path.
//
// A step reuses the StepCtrl protocol of the RK2 kernels: "stage 1" is the
// x-sweep (it derives dt from the wave-speed maxima, compute_dt_2d,
// euler2d.hpp:242-271), "stage 2" the y-sweep, which also reduces the wave
// speeds of the new state for the next dt.
#include "euler2d_kernels.cuh"
#include "kernels.h"

namespace nestb {
namespace {

struct P3 { double r, u, p; double q; };  // (rho, u_normal, p) + transverse momentum

// get_prim_2d, euler2d.hpp:36-64.
__device__ __forceinline__ P3 prim_compat(const double* U, long long vs, long long o, bool xdir, double gm1) {
    double rho = smax(U[o], 1e-10);
    double ru = U[vs + o], rv = U[2 * vs + o], E = U[3 * vs + o];
    double u = ru / rho, v = rv / rho;
    double ke = 0.5 * rho * (u * u + v * v);
    double p = smax(gm1 * (E - ke), 1e-10);
    P3 w;
    w.r = rho;
    w.p = p;
    w.u = xdir ? u : v;
    w.q = xdir ? rv : ru;
    return w;
}

// compute_interface_velocity, euler2d.hpp:20-28.
__device__ __forceinline__ double iface_velocity(double uL, double uR, double cL, double cR) {
    double SL = smin(uL - cL, uR - cR);
    double SR = smax(uL + cL, uR + cR);
    if (SL >= 0.0) return uL;
    if (SR <= 0.0) return uR;
    return (SR * uL - SL * uR) / (SR - SL);
}

// passive_flux, euler2d.hpp:31-33.
__device__ __forceinline__ double passive(double qL, double qR, double u) { return (u >= 0.0) ? u * qL : u * qR; }

// Flux of one face from the four cells m2, m1 | p0, p1 (plm_reconstruct with
// nest's limiter choice,
// euler1d.hpp:149-171, then hlle_flux, euler1d.hpp:178-242, and the passive
// transverse flux).  f[0..2]: (rho, normal momentum, E); f[3]: transverse.
__device__ __forceinline__ void compat_face(const P3& m2, const P3& m1, const P3& p0, const P3& p1, double gamma,
                                            double gm1, int lim, double f[4]) {
    double sa0 = limit(m1.r - m2.r, p0.r - m1.r, lim), sa1 = limit(m1.u - m2.u, p0.u - m1.u, lim),
           sa2 = limit(m1.p - m2.p, p0.p - m1.p, lim);
    double sb0 = limit(p0.r - m1.r, p1.r - p0.r, lim), sb1 = limit(p0.u - m1.u, p1.u - p0.u, lim),
           sb2 = limit(p0.p - m1.p, p1.p - p0.p, lim);
    double rL = m1.r + 0.5 * sa0, uL = m1.u + 0.5 * sa1, pL = m1.p + 0.5 * sa2;
    double rR = p0.r - 0.5 * sb0, uR = p0.u - 0.5 * sb1, pR = p0.p - 0.5 * sb2;
    hlle1d(gamma, gm1, rL, uL, pL, rR, uR, pR, f[0], f[1], f[2]);
    double cL = sqrt(gamma * pL / rL), cR = sqrt(gamma * pR / rR);
    double ui = iface_velocity(uL, uR, cL, cR);
    double qL = m1.q + 0.5 * limit(m1.q - m2.q, p0.q - m1.q, lim);
    double qR = p0.q - 0.5 * limit(p0.q - m1.q, p1.q - p0.q, lim);
    f[3] = passive(qL, qR, ui);
}

// XDIR: x-sweep (stage 1 of a step), else y-sweep (stage 2).
template <bool XDIR>
__global__ void __launch_bounds__(256) k2d_compat_sweep(const double* __restrict__ Uin, double* Uout, Geo2D g,
                                                        LoopParams lp, StepCtrl* ctrl, int p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const bool lead = (blockIdx.x | blockIdx.y | threadIdx.x | threadIdx.y) == 0;
    const double gamma = g.gamma, gm1 = g.gamma - 1.0;
    double dt;
    if (XDIR) {
        bool done = step_is_done(ctrl, p, lp);
        double pd = done ? -1.0 : prescribed_dt(ctrl, p, lp);
        if (pd > 0.0) {
            dt = pd;
        } else {
            dt = dt_from_speeds(bits_speed(ctrl->maxs[p][0]), bits_speed(ctrl->maxs[p][1]), g.dx, g.dy, lp.cfl);
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - ctrl->time[p]);
        }
        if (lead) publish_step(ctrl, p, lp, done, dt);
        if (done) return;
    } else {
        if (!ctrl->active[p]) return;
        dt = ctrl->dt[p];
    }
    double smx = 0.0, smy = 0.0;
    if (i < g.nx && j < g.ny) {
        const long long vs = g.vstride;
        const long long st = XDIR ? (long long)g.pitch : 1;
        const long long o = g.at(i, j);
        P3 w[5];
        for (int k = 0; k < 5; ++k) w[k] = prim_compat(Uin, vs, o + (k - 2) * st, XDIR, gm1);
        double fL[4], fR[4];
        compat_face(w[0], w[1], w[2], w[3], gamma, gm1, lp.lim, fL);
        compat_face(w[1], w[2], w[3], w[4], gamma, gm1, lp.lim, fR);
        double dtd = dt / (XDIR ? g.dx : g.dy);
        double v0 = Uin[o] - dtd * (fR[0] - fL[0]);
        double vn = Uin[(XDIR ? 1 : 2) * vs + o] - dtd * (fR[1] - fL[1]);
        double vt = Uin[(XDIR ? 2 : 1) * vs + o] - dtd * (fR[3] - fL[3]);
        double vE = Uin[3 * vs + o] - dtd * (fR[2] - fL[2]);
        double v1 = XDIR ? vn : vt, v2 = XDIR ? vt : vn;
        Uout[o] = v0; Uout[vs + o] = v1; Uout[2 * vs + o] = v2; Uout[3 * vs + o] = vE;
        if (i < 2 || i >= g.nx - 2 || j < 2 || j >= g.ny - 2) {
            store_ghosts(Uout, g, 0, i, j, v0); store_ghosts(Uout, g, 1, i, j, v1);
            store_ghosts(Uout, g, 2, i, j, v2); store_ghosts(Uout, g, 3, i, j, vE);
        }
        if (!XDIR) {
            double sx, sy;
            cell_speeds<double>(v0, v1, v2, vE, gamma, gm1, sx, sy);
            smx = sx; smy = sy;
        }
    }
    if (!XDIR) {
        smx = warp_max(smx);
        smy = warp_max(smy);
        if ((threadIdx.x & 31) == 0) {
            if (!(smx == smx) || !(smy == smy) || smx > 1.79e308) atomicOr(&ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&ctrl->maxs[p ^ 1][0], smx);
            atomic_max_speed(&ctrl->maxs[p ^ 1][1], smy);
        }
    }
}

}  // namespace

// One split step: x-sweep U -> U1, y-sweep U1 -> U (sod2d.cpp:331-362 with
// the patch copies folded into the ghost push).
cudaError_t launch_2d_compat_step(double* U, double* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl, int p,
                                  int which, cudaStream_t st) {
    dim3 b(32, 8), gr((g.ny + 31) / 32, (g.nx + 7) / 8);
    if (which & 1) k2d_compat_sweep<true><<<gr, b, 0, st>>>(U, U1, g, lp, ctrl, p);
    if (which & 2) k2d_compat_sweep<false><<<gr, b, 0, st>>>(U1, U, g, lp, ctrl, p);
    return cudaGetLastError();
}

}  // namespace nestb
