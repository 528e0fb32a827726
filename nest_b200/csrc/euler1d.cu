// 1D Euler hot path for sm_100a: fused PLM-minmod + HLLE + flux divergence +
// RK2 stage, on-device ghost fill and CFL max-speed reduction.
//
// Compiled with -fmad=false: the FP64 arithmetic keeps the operation order
// of nest's OpenMP path (examples/benchmark/benchmark_euler1d.cpp:113-209)
// and matches it bit for bit.
//
// Two execution shapes:
//   * resident: one CTA holds the whole domain in shared memory and runs the
//     complete time loop (dt, ghost fill, both stages, Heun average) with no
//     kernel boundary and no host round-trip per step.  Used while
//     12 * (n + 4) doubles fit in shared memory.
//   * tiled: stage kernels over 256-cell tiles; stage 2 fuses the Heun
//     average, the ghost fill of the new state and the max-wave-speed
//     reduction; dt is derived on the device from that maximum, so a step is
//     two launches and no host synchronisation (steps are captured in CUDA
//     graphs by the host code).
#include "common.cuh"
#include "kernels.h"

namespace nestb {

// ---------------------------------------------------------------------------
// Resident single-CTA solver
// ---------------------------------------------------------------------------

__device__ __forceinline__ int ghost_src_1d(int e, int n, int h, int bc) {
    // extended index e of a ghost cell -> extended index of its source
    if (e < h) return bc == BC_PERIODIC ? n + e : h;
    return bc == BC_PERIODIC ? e - n : h + n - 1;
}

__device__ double block_max_1d(double v, double* red) {
    v = warp_max(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double x = (l < nw) ? red[l] : 0.0;
        x = warp_max(x);
        if (l == 0) red[32] = x;
    }
    __syncthreads();
    double r = red[32];
    __syncthreads();
    return r;
}

// One stage inside the resident kernel.  Uin/Uout are shared-memory SoA
// arrays of 3*nt; W scratch 3*nt; F scratch 3*(n+1).  If avg != nullptr the
// result is 0.5*(avg + stage) (second Heun stage, written into avg).
__device__ void resident_stage(const double* Uin, double* Uout, double* avg, double* W, double* F,
                               int n, int h, double dtdx, double gamma, double gm1, int lim) {
    int nt = n + 2 * h;
    for (int f = threadIdx.x; f <= n; f += blockDim.x) {
        // face between extended cells a = h+f-1 and b = h+f
        int a = h + f - 1, b = h + f;
        double sa[3], sb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double* w = W + k * nt;
            sa[k] = limit(w[a] - w[a - 1], w[b] - w[a], lim);
            sb[k] = limit(w[b] - w[a], w[b + 1] - w[b], lim);
        }
        double rL = W[a] + 0.5 * sa[0], uL = W[nt + a] + 0.5 * sa[1], pL = W[2 * nt + a] + 0.5 * sa[2];
        double rR = W[b] - 0.5 * sb[0], uR = W[nt + b] - 0.5 * sb[1], pR = W[2 * nt + b] - 0.5 * sb[2];
        double f0, f1, f2;
        hlle1d(gamma, gm1, rL, uL, pL, rR, uR, pR, f0, f1, f2);
        F[f] = f0; F[(n + 1) + f] = f1; F[2 * (n + 1) + f] = f2;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int e = h + c;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = Uin[k * nt + e] - dtdx * (F[k * (n + 1) + c + 1] - F[k * (n + 1) + c]);
            if (avg) avg[k * nt + e] = 0.5 * (avg[k * nt + e] + v);
            else Uout[k * nt + e] = v;
        }
    }
    __syncthreads();
}

// Primitive pass over the extended array (cons_to_prim, euler1d.hpp:69-84),
// returning this thread's max |u|+c over interior cells (benchmark_euler1d.cpp:168-180).
__device__ double resident_prims(const double* U, double* W, int n, int h, double gamma, double gm1) {
    int nt = n + 2 * h;
    double ms = 0.0;
    for (int e = threadIdx.x; e < nt; e += blockDim.x) {
        double rho = U[e], mom = U[nt + e], erg = U[2 * nt + e];
        double u = mom / rho;
        double p = eos_pressure(gm1, rho, mom, erg);
        W[e] = rho; W[nt + e] = u; W[2 * nt + e] = p;
        if (e >= h && e < h + n) {
            double c = sqrt(gamma * p / rho);
            ms = smax(ms, fabs(u) + c);
        }
    }
    return ms;
}

__device__ void resident_ghosts(double* U, int n, int h, int bc) {
    int nt = n + 2 * h;
    for (int t = threadIdx.x; t < 3 * 2 * h; t += blockDim.x) {
        int k = t / (2 * h), g = t % (2 * h);
        int e = (g < h) ? g : h + n + (g - h);
        U[k * nt + e] = U[k * nt + ghost_src_1d(e, n, h, bc)];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(1024)
k1d_resident(double* __restrict__ Ug, int n, int h, double dx, double gamma, int bc,
             LoopParams lp, StepCtrl* ctrl, int p) {
    extern __shared__ double sm[];
    int nt = n + 2 * h;
    double* U = sm;
    double* U1 = U + 3 * nt;
    double* W = U1 + 3 * nt;
    double* F = W + 3 * nt;
    double* red = F + 3 * (n + 1);
    double gm1 = gamma - 1.0;
    for (int i = threadIdx.x; i < 3 * nt; i += blockDim.x) { U[i] = Ug[i]; U1[i] = 0.0; }
    __syncthreads();
    double time = ctrl->time[p];
    int step = ctrl->step[p];
    for (int it = 0;; ++it) {
        if (lp.step_budget > 0 && it >= lp.step_budget) break;
        if (lp.t_final > 0.0 && !(time < lp.t_final)) break;
        if (lp.max_steps > 0 && step >= lp.max_steps) break;
        if (lp.dts_in && step >= lp.dts_cap) break;
        // Stage 1: ghost fill of U, primitives (+ CFL max over the interior).
        resident_ghosts(U, n, h, bc);
        double ms = block_max_1d(resident_prims(U, W, n, h, gamma, gm1), red);
        double dt;
        if (lp.fixed_dt > 0.0) {
            dt = lp.fixed_dt;
        } else if (lp.dts_in) {
            dt = lp.dts_in[step];
        } else {
            dt = lp.cfl * dx / ms;
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - time);
        }
        if (!(ms == ms) || ms > 1.79e308) { if (threadIdx.x == 0) atomicOr(&ctrl->err, ERRW_NONFINITE); break; }
        if (threadIdx.x == 0 && lp.dts_out && step < lp.dts_cap) lp.dts_out[step] = dt;
        double dtdx = dt / dx;
        resident_stage(U, U1, nullptr, W, F, n, h, dtdx, gamma, gm1, lp.lim);
        // Stage 2 on U1, averaged into U.
        resident_ghosts(U1, n, h, bc);
        resident_prims(U1, W, n, h, gamma, gm1);
        __syncthreads();
        resident_stage(U1, nullptr, U, W, F, n, h, dtdx, gamma, gm1, lp.lim);
        time += dt;
        ++step;
    }
    resident_ghosts(U, n, h, bc);
    for (int i = threadIdx.x; i < 3 * nt; i += blockDim.x) Ug[i] = U[i];
    if (threadIdx.x == 0) {
        ctrl->time[p] = time; ctrl->step[p] = step;
        ctrl->time[p ^ 1] = time; ctrl->step[p ^ 1] = step;
    }
}

size_t resident_smem_bytes(int n, int h) {
    int nt = n + 2 * h;
    return sizeof(double) * (size_t)(9 * nt + 3 * (n + 1) + 33);
}

cudaError_t launch_1d_resident(double* U, int n, int h, double dx, double gamma, int bc,
                               const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st) {
    size_t smem = resident_smem_bytes(n, h);
    cudaError_t e = cudaFuncSetAttribute(k1d_resident, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int nt = n + 2 * h;
    int threads = nt >= 1024 ? 1024 : ((nt + 31) / 32) * 32;
    k1d_resident<<<1, threads, smem, st>>>(U, n, h, dx, gamma, bc, lp, ctrl, p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Tiled multi-CTA stage kernels
// ---------------------------------------------------------------------------

constexpr int T1 = 256;  // cells per tile = threads per block

// Max |u|+c of one cell (benchmark_euler1d.cpp:170-178).
__device__ __forceinline__ double cell_speed_1d(double rho, double mom, double erg, double gamma, double gm1) {
    double u = mom / rho;
    double p = eos_pressure(gm1, rho, mom, erg);
    double c = sqrt(gamma * p / rho);
    return fabs(u) + c;
}

// Writes the ghost copies that the value of interior cell c (0-based) feeds.
__device__ __forceinline__ void push_ghosts_1d(double* U, int nt, int k, int c, int n, int h, int bc, double v) {
    if (bc == BC_PERIODIC) {
        if (c < h) U[k * nt + h + n + c] = v;
        if (c >= n - h) U[k * nt + (c - (n - h))] = v;
    } else {
        if (c == 0) for (int g = 0; g < h; ++g) U[k * nt + g] = v;
        if (c == n - 1) for (int g = 0; g < h; ++g) U[k * nt + h + n + g] = v;
    }
}

template <int STAGE>
__global__ void __launch_bounds__(T1)
k1d_stage(const double* __restrict__ Uin, const double* Un, double* Uout,
          int n, int h, double dx, double gamma, int bc, LoopParams lp, StepCtrl* ctrl, int p) {
    __shared__ double W[3][T1 + 4];
    __shared__ double F[3][T1 + 1];
    __shared__ double red[33];
    int nt = n + 2 * h;
    double gm1 = gamma - 1.0;
    double dt;
    if (STAGE == 1) {
        bool done = step_is_done(ctrl, p, lp);
        double ms = bits_speed(ctrl->maxs[p][0]);
        double pd = done ? -1.0 : prescribed_dt(ctrl, p, lp);
        if (pd > 0.0) dt = pd;
        else {
            dt = lp.cfl * dx / ms;
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - ctrl->time[p]);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) publish_step(ctrl, p, lp, done, dt);
        if (done) return;
    } else {
        if (!ctrl->active[p]) return;
        dt = ctrl->dt[p];
    }
    double dtdx = dt / dx;
    int c0 = blockIdx.x * T1;  // first interior cell of the tile
    // primitives of extended cells c0-2 .. c0+T1+1 (clamped at the array end)
    for (int t = threadIdx.x; t < T1 + 4; t += T1) {
        int e = min(h + c0 - 2 + t, nt - 1);
        double rho = Uin[e], mom = Uin[nt + e], erg = Uin[2 * nt + e];
        W[0][t] = rho;
        W[1][t] = mom / rho;
        W[2][t] = eos_pressure(gm1, rho, mom, erg);
    }
    __syncthreads();
    int nf = min(T1, n - c0) + 1;  // faces of this tile
    for (int f = threadIdx.x; f < nf; f += T1) {
        int a = f + 1, b = f + 2;  // tile-local W indices around the face
        double sa[3], sb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            sa[k] = limit(W[k][a] - W[k][a - 1], W[k][b] - W[k][a], lp.lim);
            sb[k] = limit(W[k][b] - W[k][a], W[k][b + 1] - W[k][b], lp.lim);
        }
        double f0, f1, f2;
        hlle1d(gamma, gm1, W[0][a] + 0.5 * sa[0], W[1][a] + 0.5 * sa[1], W[2][a] + 0.5 * sa[2],
               W[0][b] - 0.5 * sb[0], W[1][b] - 0.5 * sb[1], W[2][b] - 0.5 * sb[2], f0, f1, f2);
        F[0][f] = f0; F[1][f] = f1; F[2][f] = f2;
    }
    __syncthreads();
    int c = c0 + threadIdx.x;
    double ms = 0.0;
    if (c < n) {
        int e = h + c;
        double v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double s = Uin[k * nt + e] - dtdx * (F[k][threadIdx.x + 1] - F[k][threadIdx.x]);
            v[k] = (STAGE == 1) ? s : 0.5 * (Un[k * nt + e] + s);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Uout[k * nt + e] = v[k];
            push_ghosts_1d(Uout, nt, k, c, n, h, bc, v[k]);
        }
        if (STAGE == 2) ms = cell_speed_1d(v[0], v[1], v[2], gamma, gm1);
    }
    if (STAGE == 2) {
        ms = warp_max(ms);
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) red[w] = ms;
        __syncthreads();
        if (w == 0) {
            double x = (l < T1 / 32) ? red[l] : 0.0;
            x = warp_max(x);
            if (l == 0) {
                if (!(x == x) || x > 1.79e308) atomicOr(&ctrl->err, ERRW_NONFINITE);
                atomic_max_speed(&ctrl->maxs[p ^ 1][0], x);
            }
        }
    }
}

// Ghost fill + max |u|+c of the current state into slot p (used once after
// an upload, and by the standalone compute_dt entry point).
__global__ void __launch_bounds__(T1)
k1d_prepare(double* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p, int reset) {
    __shared__ double red[33];
    int nt = n + 2 * h;
    double gm1 = gamma - 1.0;
    int c = blockIdx.x * T1 + threadIdx.x;
    double ms = 0.0;
    if (c < n) {
        int e = h + c;
        double v0 = U[e], v1 = U[nt + e], v2 = U[2 * nt + e];
        push_ghosts_1d(U, nt, 0, c, n, h, bc, v0);
        push_ghosts_1d(U, nt, 1, c, n, h, bc, v1);
        push_ghosts_1d(U, nt, 2, c, n, h, bc, v2);
        ms = cell_speed_1d(v0, v1, v2, gamma, gm1);
    }
    ms = warp_max(ms);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = ms;
    __syncthreads();
    if (w == 0) {
        double x = (l < T1 / 32) ? red[l] : 0.0;
        x = warp_max(x);
        if (l == 0) atomic_max_speed(&ctrl->maxs[p][0], x);
    }
    (void)reset;
}

cudaError_t launch_1d_prepare(double* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p,
                              cudaStream_t st) {
    int blocks = (n + T1 - 1) / T1;
    k1d_prepare<<<blocks, T1, 0, st>>>(U, n, h, gamma, bc, ctrl, p, 0);
    return cudaGetLastError();
}

cudaError_t launch_1d_step(double* U, double* U1, int n, int h, double dx, double gamma, int bc,
                           const LoopParams& lp, StepCtrl* ctrl, int p, int which, cudaStream_t st, double* Uout) {
    int blocks = (n + T1 - 1) / T1;
    if (which & 1) k1d_stage<1><<<blocks, T1, 0, st>>>(U, nullptr, U1, n, h, dx, gamma, bc, lp, ctrl, p);
    if (which & 2) k1d_stage<2><<<blocks, T1, 0, st>>>(U1, U, Uout ? Uout : U, n, h, dx, gamma, bc, lp, ctrl, p);
    return cudaGetLastError();
}

}  // namespace nestb
