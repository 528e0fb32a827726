// Tiled multi-CTA 1D stage kernels, templated on the arithmetic type:
// instantiated for double in euler1d.cu (-fmad=false, nest's operation order,
// bit for bit with the OpenMP path) and for float in euler1d_f32.cu (the FP32
// form, fast reciprocal / square root).  Time, dt and the wave-speed maximum
// stay FP64 in both.
//
// One CTA of T1 + 32 threads owns T1 cells: primitives of its cells and a 2-cell
// halo into shared memory, one HLLE per face, the update with the ghost
// copies it feeds; stage 2 fuses the Heun average and the block's max
// |u|+c (one atomic per block).  dt is derived on the device from that
// maximum by the next stage 1, so a step is two launches and no host
// synchronisation.  k1d_step runs a whole step in one launch (out of place),
// recomputing the stage-1 halo per CTA.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace nestb {
namespace {

// cells per tile: 224 puts at most 448 cells on an SM at 65536 cells (293
// tiles over 148 SMs; 256 gave 512 on most SMs): FP64 step 8.76 -> 8.46 us
constexpr int T1 = 224;
// threads per block: at least one per extended cell (T1 + 4), so that no
// phase loops twice, in whole warps (the stage-2 reduction shuffles over
// full warps)
constexpr int NT1 = T1 + 32;

// Max |u|+c of one cell (benchmark_euler1d.cpp:170-178); p receives the
// cell's pressure (eos_t::pressure, clamped at 0) for the positivity check.
template <typename T>
__device__ __forceinline__ T cell_speed_1d(T rho, T mom, T erg, T gamma, T gm1, T& p) {
    T u = mom / rho;
    p = eos_pressure(gm1, rho, mom, erg);
    T c = sqrt(gamma * p / rho);
    return fabs(u) + c;
}

// Writes the ghost copies that the value of interior cell c (0-based) feeds.
template <typename T>
__device__ __forceinline__ void push_ghosts_1d(T* U, int nt, int k, int c, int n, int h, int bc, T v) {
    if (bc == BC_PERIODIC) {
        if (c < h) U[k * nt + h + n + c] = v;
        if (c >= n - h) U[k * nt + (c - (n - h))] = v;
    } else {
        if (c == 0) for (int g = 0; g < h; ++g) U[k * nt + g] = v;
        if (c == n - 1) for (int g = 0; g < h; ++g) U[k * nt + h + n + g] = v;
    }
}

// LIM (both kernels): the slope limiter fixed at compile time (LIM_MINMOD,
// nest's default) or -1 to read it from the loop parameters.
template <typename T, int STAGE, int LIM>
__global__ void __launch_bounds__(NT1)
k1d_stage(const T* __restrict__ Uin, const T* Un, T* Uout,
          int n, int h, double dx, double gamma_d, int bc, LoopParams lp, StepCtrl* ctrl, int p) {
    __shared__ T W[3][T1 + 4];
    __shared__ T F[3][T1 + 1];
    __shared__ double red[33];
    pdl_wait();
    pdl_trigger();
    int nt = n + 2 * h;
    const T gamma = (T)gamma_d;
    const T gm1 = (T)(gamma_d - 1.0);
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
    const T dtdx = (T)(dt / dx);
    int c0 = blockIdx.x * T1;  // first interior cell of the tile
    // primitives of extended cells c0-2 .. c0+T1+1 (clamped at the array end)
    for (int t = threadIdx.x; t < T1 + 4; t += NT1) {
        int e = min(h + c0 - 2 + t, nt - 1);
        T rho = Uin[e], mom = Uin[nt + e], erg = Uin[2 * nt + e];
        W[0][t] = rho;
        W[1][t] = mom / rho;
        W[2][t] = eos_pressure(gm1, rho, mom, erg);
    }
    __syncthreads();
    int nf = min(T1, n - c0) + 1;  // faces of this tile
    for (int f = threadIdx.x; f < nf; f += NT1) {
        int a = f + 1, b = f + 2;  // tile-local W indices around the face
        T sa[3], sb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            sa[k] = limit(W[k][a] - W[k][a - 1], W[k][b] - W[k][a], LIM >= 0 ? LIM : lp.lim);
            sb[k] = limit(W[k][b] - W[k][a], W[k][b + 1] - W[k][b], LIM >= 0 ? LIM : lp.lim);
        }
        T f0, f1, f2;
        hlle1d(gamma, gm1, W[0][a] + T(0.5) * sa[0], W[1][a] + T(0.5) * sa[1], W[2][a] + T(0.5) * sa[2],
               W[0][b] - T(0.5) * sb[0], W[1][b] - T(0.5) * sb[1], W[2][b] - T(0.5) * sb[2], f0, f1, f2);
        F[0][f] = f0; F[1][f] = f1; F[2][f] = f2;
    }
    __syncthreads();
    int c = c0 + threadIdx.x;
    double ms = 0.0;
    if (threadIdx.x < T1 && c < n) {
        int e = h + c;
        T v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            T s = Uin[k * nt + e] - dtdx * (F[k][threadIdx.x + 1] - F[k][threadIdx.x]);
            v[k] = (STAGE == 1) ? s : T(0.5) * (Un[k * nt + e] + s);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Uout[k * nt + e] = v[k];
            push_ghosts_1d(Uout, nt, k, c, n, h, bc, v[k]);
        }
        if (STAGE == 2) {
            T pr;
            ms = (double)cell_speed_1d(v[0], v[1], v[2], gamma, gm1, pr);
            if (!(v[0] > T(0)) || !(pr > T(0))) flag_cell(ctrl, ctrl->step[p] + 1, (double)v[0], (double)pr, c, 0);
        }
    }
    if (STAGE == 2) {
        ms = warp_max(ms);
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) red[w] = ms;
        __syncthreads();
        if (w == 0) {
            double x = (l < (NT1 + 31) / 32) ? red[l] : 0.0;
            x = warp_max(x);
            if (l == 0) {
                if (!(x == x) || x > 1.79e308) atomicOr(&ctrl->err, ERRW_NONFINITE);
                atomic_max_speed(&ctrl->maxs[p ^ 1][0], x);
            }
        }
    }
}

// Interior cell whose value cell c holds (any c, ghost cells and beyond
// included): nest's periodic copy, or the zero-gradient copy of the nearest
// end cell.
__device__ __forceinline__ int source_cell_1d(int c, int n, int bc) {
    if (bc == BC_PERIODIC) {
        c %= n;
        return c < 0 ? c + n : c;
    }
    return min(max(c, 0), n - 1);
}

// One whole RK2 (Heun) step in one launch, out of place (Un -> Unext; the
// caller alternates two buffers).  A CTA owns T1 cells and keeps everything
// of its step in shared memory:
//   U^n and its primitives over the cells c0-4 .. c0+T1+3,
//   the stage-1 faces and U1 over c0-2 .. c0+T1+1 (the 2-cell halo of U1 is
//   recomputed here instead of being exchanged through global memory),
//   the primitives of U1, the stage-2 faces and the Heun update of the T1
//   cells, the new state's ghost copies, positivity check and max |u|+c.
// Every value is computed by the same expression, on the same operands, as in
// the two stage kernels (and nest's loop): U1 of a ghost cell is U1 of the
// cell it copies, which the periodic wrap of the primitives gives directly
// and the zero-gradient case takes from that cell's faces.  The wave-speed
// maximum is reduced into maxs[q][1]; the last block to finish moves it to
// maxs[q][0] (block 0 cannot clear a slot at its start that other blocks may
// already be adding to).  U1out (optional) receives U1 of the step with its
// ghosts.  A finished step (time, step count or error) copies Un to Unext so
// that the state ends in the buffer the caller expects.
template <typename T, int LIM>
__global__ void __launch_bounds__(NT1)
k1d_step(const T* __restrict__ Un, T* __restrict__ Unext, T* __restrict__ U1out, int n, int h, double dx,
         double gamma_d, int bc, LoopParams lp, StepCtrl* ctrl, int p) {
    __shared__ T Q[3][T1 + 8];  // U^n, cells c0-4 ..
    __shared__ T W[3][T1 + 8];  // primitives of U^n (cells c0-4 ..), then of U1 (cells c0-2 ..)
    __shared__ T F[3][T1 + 5];  // faces of the stage
    __shared__ T V[3][T1 + 4];  // U1, cells c0-2 ..
    __shared__ double red[NT1 / 32];
    pdl_wait();
    pdl_trigger();
    const int nt = n + 2 * h;
    const T gamma = (T)gamma_d;
    const T gm1 = (T)(gamma_d - 1.0);
    const int c0 = blockIdx.x * T1;
    if (step_is_done(ctrl, p, lp)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) publish_step(ctrl, p, lp, true, 0.0, false);
        for (int t = threadIdx.x; t < T1; t += NT1) {
            const int c = c0 + t;
            if (c < n)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const T v = Un[k * nt + h + c];
                    Unext[k * nt + h + c] = v;
                    push_ghosts_1d(Unext, nt, k, c, n, h, bc, v);
                }
        }
        return;
    }
    double dt;
    {
        const double pd = prescribed_dt(ctrl, p, lp);
        if (pd > 0.0) {
            dt = pd;
        } else {
            dt = lp.cfl * dx / bits_speed(ctrl->maxs[p][0]);
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - ctrl->time[p]);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) publish_step(ctrl, p, lp, false, dt, false);
    const T dtdx = (T)(dt / dx);

    // U^n and its primitives, cells c0-4+t (read from the interior cell each copies)
    for (int t = threadIdx.x; t < T1 + 8; t += NT1) {
        const int e = h + source_cell_1d(c0 - 4 + t, n, bc);
        const T rho = Un[e], mom = Un[nt + e], erg = Un[2 * nt + e];
        Q[0][t] = rho; Q[1][t] = mom; Q[2][t] = erg;
        W[0][t] = rho;
        W[1][t] = mom / rho;
        W[2][t] = eos_pressure(gm1, rho, mom, erg);
    }
    __syncthreads();
    // face f between the cells of W slots f+1 and f+2
    auto faces = [&](int nf) {
        for (int f = threadIdx.x; f < nf; f += NT1) {
            const int a = f + 1, b = f + 2;
            T sa[3], sb[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sa[k] = limit(W[k][a] - W[k][a - 1], W[k][b] - W[k][a], LIM >= 0 ? LIM : lp.lim);
                sb[k] = limit(W[k][b] - W[k][a], W[k][b + 1] - W[k][b], LIM >= 0 ? LIM : lp.lim);
            }
            T f0, f1, f2;
            hlle1d(gamma, gm1, W[0][a] + T(0.5) * sa[0], W[1][a] + T(0.5) * sa[1], W[2][a] + T(0.5) * sa[2],
                   W[0][b] - T(0.5) * sb[0], W[1][b] - T(0.5) * sb[1], W[2][b] - T(0.5) * sb[2], f0, f1, f2);
            F[0][f] = f0; F[1][f] = f1; F[2][f] = f2;
        }
    };
    faces(T1 + 5);  // stage 1: faces between cells c0-3+f and c0-2+f
    __syncthreads();
    // U1 of cells c0-2+u (faces u, u+1; U^n slot u+2) and its primitives into W slot u
    for (int u = threadIdx.x; u < T1 + 4; u += NT1) {
        // zero-gradient ghost: the value of the end cell it copies, which lies
        // in this window whenever the window reaches past the domain
        const int us = bc == BC_PERIODIC ? u : source_cell_1d(c0 - 2 + u, n, bc) - c0 + 2;
        T v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = Q[k][us + 2] - dtdx * (F[k][us + 1] - F[k][us]);
            V[k][u] = v[k];
        }
        W[0][u] = v[0];
        W[1][u] = v[1] / v[0];
        W[2][u] = eos_pressure(gm1, v[0], v[1], v[2]);
    }
    __syncthreads();
    faces(T1 + 1);  // stage 2: faces between cells c0-1+f and c0+f
    __syncthreads();
    const int t = threadIdx.x, c = c0 + t;
    double ms = 0.0;
    if (t < T1 && c < n) {
        const int e = h + c;
        T v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const T s = V[k][t + 2] - dtdx * (F[k][t + 1] - F[k][t]);
            v[k] = T(0.5) * (Q[k][t + 4] + s);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Unext[k * nt + e] = v[k];
            push_ghosts_1d(Unext, nt, k, c, n, h, bc, v[k]);
            if (U1out) {
                U1out[k * nt + e] = V[k][t + 2];
                push_ghosts_1d(U1out, nt, k, c, n, h, bc, V[k][t + 2]);
            }
        }
        T pr;
        ms = (double)cell_speed_1d(v[0], v[1], v[2], gamma, gm1, pr);
        if (!(v[0] > T(0)) || !(pr > T(0))) flag_cell(ctrl, ctrl->step[p] + 1, (double)v[0], (double)pr, c, 0);
    }
    ms = warp_max(ms);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = ms;
    __syncthreads();
    if (w == 0) {
        double x = (l < NT1 / 32) ? red[l] : 0.0;
        x = warp_max(x);
        if (l == 0) {
            const int q = p ^ 1;
            if (!(x == x) || x > 1.79e308) atomicOr(&ctrl->err, ERRW_NONFINITE);
            atomic_max_speed(&ctrl->maxs[q][1], x);
            __threadfence();
            if (atomicAdd(&ctrl->blocks_done, 1u) == gridDim.x - 1) {
                // every block has added its maximum
                __threadfence();
                ctrl->maxs[q][0] = atomicExch(&ctrl->maxs[q][1], 0ull);
                ctrl->blocks_done = 0u;
            }
        }
    }
}

// Ghost fill + max |u|+c of the current state into slot p (used once after
// an upload, and by the standalone compute_dt entry point).
template <typename T>
__global__ void __launch_bounds__(T1)
k1d_prepare(T* U, int n, int h, double gamma_d, int bc, StepCtrl* ctrl, int p) {
    __shared__ double red[33];
    pdl_wait();
    pdl_trigger();
    int nt = n + 2 * h;
    const T gamma = (T)gamma_d;
    const T gm1 = (T)(gamma_d - 1.0);
    int c = blockIdx.x * T1 + threadIdx.x;
    double ms = 0.0;
    if (c < n) {
        int e = h + c;
        T v0 = U[e], v1 = U[nt + e], v2 = U[2 * nt + e];
        push_ghosts_1d(U, nt, 0, c, n, h, bc, v0);
        push_ghosts_1d(U, nt, 1, c, n, h, bc, v1);
        push_ghosts_1d(U, nt, 2, c, n, h, bc, v2);
        T pr;
        ms = (double)cell_speed_1d(v0, v1, v2, gamma, gm1, pr);
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
}

template <typename T>
cudaError_t launch_1d_prepare_t(T* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p, cudaStream_t st) {
    int blocks = (n + T1 - 1) / T1;
    return launch_pdl(k1d_prepare<T>, dim3(blocks), dim3(T1), 0, st, U, n, h, gamma, bc, ctrl, p);
}

template <typename T>
cudaError_t launch_1d_step_t(T* U, T* U1, int n, int h, double dx, double gamma, int bc, const LoopParams& lp,
                             StepCtrl* ctrl, int p, int which, cudaStream_t st, T* Uout) {
    int blocks = (n + T1 - 1) / T1;
    const bool mm = lp.lim == LIM_MINMOD;
    cudaError_t e = cudaSuccess;
    if (which & 1)
        e = launch_pdl(mm ? k1d_stage<T, 1, LIM_MINMOD> : k1d_stage<T, 1, -1>, dim3(blocks), dim3(NT1), 0, st,
                       (const T*)U, (const T*)nullptr, U1, n, h, dx, gamma, bc, lp, ctrl, p);
    if ((which & 2) && e == cudaSuccess)
        e = launch_pdl(mm ? k1d_stage<T, 2, LIM_MINMOD> : k1d_stage<T, 2, -1>, dim3(blocks), dim3(NT1), 0, st,
                       (const T*)U1, (const T*)U, Uout ? Uout : U, n, h, dx, gamma, bc, lp, ctrl, p);
    return e;
}

template <typename T>
cudaError_t launch_1d_fused_t(const T* Un, T* Unext, T* U1out, int n, int h, double dx, double gamma, int bc,
                              const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st) {
    int blocks = (n + T1 - 1) / T1;
    return launch_pdl(lp.lim == LIM_MINMOD ? k1d_step<T, LIM_MINMOD> : k1d_step<T, -1>, dim3(blocks), dim3(NT1), 0, st,
                      Un, Unext, U1out, n, h, dx, gamma, bc, lp, ctrl, p);
}

}  // namespace
}  // namespace nestb
