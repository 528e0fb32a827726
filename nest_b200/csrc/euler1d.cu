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
//   * tiled (euler1d_tiled.cuh): a whole step per launch over 224-cell tiles
//     (the stage-1 halo recomputed per CTA), or the two stage kernels; stage
//     2 fuses the Heun average, the ghost fill of the new state and the
//     max-wave-speed reduction; dt is derived on the device from that
//     maximum, so steps need no host synchronisation (they are captured in
//     CUDA graphs by the host code).
#include <cooperative_groups.h>

#include <map>
#include <mutex>

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

// Ghost copies fed by interior cell c (0-based) of a 3-variable SoA array
// over the extended range: nest's periodic copy or the zero-gradient copy.
__device__ __forceinline__ void ghost_copies_1d(double* A, int nt, int n, int h, int bc, int c, double v0, double v1,
                                                double v2) {
    auto put = [&](int e) { A[e] = v0; A[nt + e] = v1; A[2 * nt + e] = v2; };
    if (bc == BC_PERIODIC) {
        if (c >= n - h) put(c + h - n);
        if (c < h) put(h + n + c);
    } else {
        if (c == 0) for (int e = 0; e < h; ++e) put(e);
        if (c == n - 1) for (int e = h + n; e < nt; ++e) put(e);
    }
}

// Resident single-CTA solver: the whole extended domain lives in shared
// memory (U, U1, primitives W, face fluxes F) and the CTA runs the complete
// time loop.  A step is four phases separated by four barriers:
//   faces of stage 1 (PLM + HLLE from W)        | update U1, its primitives and ghost copies |
//   faces of stage 2 (from the primitives of U1) | Heun update of U, its primitives, ghost copies and max |u|+c
// Each thread handles K faces / cells per phase (K >= 2: independent
// chains of FP64 division / square root interleave).  The arithmetic of
// every face and cell is that of nest's OpenMP loop
// (examples/benchmark/benchmark_euler1d.cpp:113-209); primitives of a ghost
// cell are the primitives of its source cell, which is what nest computes
// from the copied conserved values.
// LIM (both resident kernels): the slope limiter fixed at compile time
// (LIM_MINMOD, nest's default) or -1 to read it from the loop parameters.
template <int K, int MAXT, int LIM>
__global__ void __launch_bounds__(MAXT)
k1d_resident(double* __restrict__ Ug, int n, int h, double dx, double gamma, int bc, LoopParams lp, StepCtrl* ctrl,
             int p) {
    extern __shared__ double sm[];
    const int nt = n + 2 * h, T = blockDim.x, tid = threadIdx.x;
    double* U = sm;
    double* U1 = U + 3 * nt;
    double* W = U1 + 3 * nt;
    double* F = W + 3 * nt;
    double* red = F + 3 * (n + 1);
    const double gm1 = gamma - 1.0;
    const int nw = (T + 31) >> 5;

    // primitives of cell value (r, m, e): u, p (cons_to_prim, euler1d.hpp:69-84)
    auto prims_of = [&](int c, double r, double m, double e, double* Wd) {
        const double u = m / r;
        const double pr = eos_pressure(gm1, r, m, e);
        const int x = h + c;
        Wd[x] = r; Wd[nt + x] = u; Wd[2 * nt + x] = pr;
        ghost_copies_1d(Wd, nt, n, h, bc, c, r, u, pr);
    };
    // max |u| + c over this thread's cells of A (benchmark_euler1d.cpp:168-180), warp maxima to red.
    // step_done > 0: the state after that step, checked for positivity; a
    // failing cell makes the maximum infinite, which ends the loop for the CTA
    auto speeds = [&](int step_done) {
        double ms = 0.0;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int c = tid + q * T;
            if (c < n) {
                const int x = h + c;
                const double u = W[nt + x], pr = W[2 * nt + x], r = W[x];
                const double cs = sqrt(gamma * pr / r);
                ms = smax(ms, fabs(u) + cs);
                if (step_done > 0 && (!(r > 0.0) || !(pr > 0.0))) {
                    flag_cell(ctrl, step_done, r, pr, c, 0);
                    ms = __longlong_as_double(0x7ff0000000000000ll);
                }
            }
        }
        ms = warp_max(ms);
        if ((tid & 31) == 0) red[tid >> 5] = ms;
    };
    auto reduce_red = [&]() {
        double ms = 0.0;
        for (int w = 0; w < nw; ++w) ms = smax(ms, red[w]);
        return ms;
    };
    // face fluxes of the stage whose primitives are in W
    auto faces = [&]() {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int f = tid + q * T;
            if (f <= n) {
                // face between extended cells a = h+f-1 and b = h+f
                const int a = h + f - 1, b = h + f;
                double sa[3], sb[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double* w = W + k * nt;
                    sa[k] = limit(w[a] - w[a - 1], w[b] - w[a], LIM >= 0 ? LIM : lp.lim);
                    sb[k] = limit(w[b] - w[a], w[b + 1] - w[b], LIM >= 0 ? LIM : lp.lim);
                }
                const double rL = W[a] + 0.5 * sa[0], uL = W[nt + a] + 0.5 * sa[1], pL = W[2 * nt + a] + 0.5 * sa[2];
                const double rR = W[b] - 0.5 * sb[0], uR = W[nt + b] - 0.5 * sb[1], pR = W[2 * nt + b] - 0.5 * sb[2];
                double f0, f1, f2;
                hlle1d(gamma, gm1, rL, uL, pL, rR, uR, pR, f0, f1, f2);
                F[f] = f0; F[(n + 1) + f] = f1; F[2 * (n + 1) + f] = f2;
            }
        }
    };
    // stage update of this thread's cells: out = in - dtdx (F_{c+1} - F_c),
    // or U = 0.5 (U + that) in stage 2; then the new state's primitives and ghosts
    auto update = [&](const double* Uin, double* Uout, bool heun, double dtdx) {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const int c = tid + q * T;
            if (c < n) {
                const int x = h + c;
                double v[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    v[k] = Uin[k * nt + x] - dtdx * (F[k * (n + 1) + c + 1] - F[k * (n + 1) + c]);
                    if (heun) v[k] = 0.5 * (Uout[k * nt + x] + v[k]);
                    Uout[k * nt + x] = v[k];
                }
                ghost_copies_1d(Uout, nt, n, h, bc, c, v[0], v[1], v[2]);
                prims_of(c, v[0], v[1], v[2], W);
            }
        }
    };

    // prologue: state, ghosts, primitives and the first max wave speed
    for (int i = tid; i < 3 * nt; i += T) { U[i] = Ug[i]; U1[i] = 0.0; }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const int c = tid + q * T;
        if (c < n) {
            const int x = h + c;
            const double r = U[x], m = U[nt + x], e = U[2 * nt + x];
            ghost_copies_1d(U, nt, n, h, bc, c, r, m, e);
            prims_of(c, r, m, e, W);
        }
    }
    __syncthreads();
    speeds(0);
    __syncthreads();
    double ms = reduce_red();

    double time = ctrl->time[p];
    int step = ctrl->step[p];
    const bool stopped = (ctrl->err & ERRW_STOP) != 0;  // an earlier step failed: run nothing
    for (int it = 0;; ++it) {
        if (stopped) break;
        if (lp.step_budget > 0 && it >= lp.step_budget) break;
        if (lp.t_final > 0.0 && !(time < lp.t_final)) break;
        if (lp.max_steps > 0 && step >= lp.max_steps) break;
        if (lp.dts_in && step >= lp.dts_cap) break;
        double dt;
        if (lp.fixed_dt > 0.0) {
            dt = lp.fixed_dt;
        } else if (lp.dts_in) {
            dt = lp.dts_in[step];
        } else {
            dt = lp.cfl * dx / ms;
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - time);
        }
        if (!(ms == ms) || ms > 1.79e308) { if (tid == 0) atomicOr(&ctrl->err, ERRW_NONFINITE); break; }
        if (tid == 0 && lp.dts_out && step < lp.dts_cap) lp.dts_out[step] = dt;
        const double dtdx = dt / dx;
        faces();                        // stage 1 fluxes from W = prims(U)
        __syncthreads();
        update(U, U1, false, dtdx);     // U1, W = prims(U1), ghosts
        __syncthreads();
        faces();                        // stage 2 fluxes
        __syncthreads();
        update(U1, U, true, dtdx);      // U = (U + U1 - dt L(U1)) / 2, W = prims(U), ghosts
        speeds(step + 1);
        __syncthreads();
        ms = reduce_red();
        time += dt;
        ++step;
    }
    for (int i = tid; i < 3 * nt; i += T) Ug[i] = U[i];
    if (tid == 0) {
        ctrl->time[p] = time; ctrl->step[p] = step;
        ctrl->time[p ^ 1] = time; ctrl->step[p ^ 1] = step;
    }
}

// Cluster form of the resident solver: a thread-block cluster of NC CTAs
// (one per SM) splits the cells into NC contiguous chunks and every CTA runs
// the complete time loop on its chunk in its own shared memory.  A CTA holds
// its chunk's U and U1, the primitives W of its cells plus two halo cells on
// each side, and its face fluxes.  Right after computing the primitives of
// its first two and last two cells it stores them into the halo slots of the
// neighbouring CTAs (distributed shared memory); W is double-buffered by
// stage, so one cluster barrier per stage orders those stores against the
// neighbours' reads.  The wave-speed maximum for dt is reduced over the
// cluster by reading every CTA's warp maxima after the stage-2 barrier, so
// all CTAs derive the same dt.  The per-face and per-cell arithmetic is the
// single-CTA kernel's (nest's OpenMP loop), so the result is the same bit for
// bit; spreading the FP64 division / square-root work over NC SMs is the gain.
template <int LIM>
__global__ void __launch_bounds__(256)
k1d_cluster(double* __restrict__ Ug, int n, int h, int m, double dx, double gamma, int bc, LoopParams lp,
            StepCtrl* ctrl, int p) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double sm[];
    const int NC = (int)cl.num_blocks();
    const int r = (int)cl.block_rank();
    const int tid = threadIdx.x, T = blockDim.x, nw = (T + 31) >> 5;
    const int nt = n + 2 * h;
    const int c_lo = r * m, mloc = min(n, c_lo + m) - c_lo;  // this CTA's cells [c_lo, c_lo + mloc)
    const int mw = m + 4;                                     // W row: 2 halo slots each side
    double* U = sm;                  // [3][m]
    double* U1 = U + 3 * m;          // [3][m]
    double* W = U1 + 3 * m;          // [2][3][mw]: buffer b, variable k, local cell l at 2 + l
    double* F = W + 6 * mw;          // [3][m + 1]
    double* red = F + 3 * (m + 1);   // [32] warp maxima
    const double gm1 = gamma - 1.0;
    const int left = (r + NC - 1) % NC, right = (r + 1) % NC;
    const int mloc_left = min(n, left * m + m) - left * m;
    auto Wb = [&](int b) { return W + b * 3 * mw; };
    // W buffer b of CTA `rank`, variable k, local slot s (halo slots 0, 1 and mloc + 2, mloc + 3)
    auto peerW = [&](int rank, int b, int k, int slot) {
        return cl.map_shared_rank(W, rank) + b * 3 * mw + k * mw + slot;
    };
    // primitives of local cell l into buffer b, plus the halo copies it feeds
    auto prims_of = [&](int l, double rr, double mm, double ee, int b) {
        const double u = mm / rr;
        const double pr = eos_pressure(gm1, rr, mm, ee);
        const double v[3] = { rr, u, pr };
        double* w = Wb(b);
#pragma unroll
        for (int k = 0; k < 3; ++k) w[k * mw + 2 + l] = v[k];
        const int c = c_lo + l;
        if (bc == BC_PERIODIC) {
            // first two cells -> right halo of the left neighbour; last two -> left halo of the right neighbour
            if (l < 2)
#pragma unroll
                for (int k = 0; k < 3; ++k) *peerW(left, b, k, mloc_left + 2 + l) = v[k];
            if (l >= mloc - 2)
#pragma unroll
                for (int k = 0; k < 3; ++k) *peerW(right, b, k, l - (mloc - 2)) = v[k];
        } else {
            if (l < 2 && r > 0)
#pragma unroll
                for (int k = 0; k < 3; ++k) *peerW(left, b, k, mloc_left + 2 + l) = v[k];
            if (l >= mloc - 2 && r < NC - 1)
#pragma unroll
                for (int k = 0; k < 3; ++k) *peerW(right, b, k, l - (mloc - 2)) = v[k];
            if (c == 0)  // zero-gradient ghosts of the domain's first cell
#pragma unroll
                for (int k = 0; k < 3; ++k) { w[k * mw + 0] = v[k]; w[k * mw + 1] = v[k]; }
            if (c == n - 1)
#pragma unroll
                for (int k = 0; k < 3; ++k) { w[k * mw + mloc + 2] = v[k]; w[k * mw + mloc + 3] = v[k]; }
        }
    };
    auto speeds = [&](int b) {
        double ms = 0.0;
        for (int l = tid; l < mloc; l += T) {
            const double* w = Wb(b);
            const double rr = w[2 + l], u = w[mw + 2 + l], pr = w[2 * mw + 2 + l];
            const double cs = sqrt(gamma * pr / rr);
            ms = smax(ms, fabs(u) + cs);
        }
        ms = warp_max(ms);
        if ((tid & 31) == 0) red[tid >> 5] = ms;
    };
    // max over every CTA's warp maxima: each lane reads its share of the
    // NC * nw values (remote loads in parallel), then a warp max; every warp
    // computes the same value, so all threads hold the same dt
    auto cluster_max = [&]() {
        double ms = 0.0;
        const int lane = tid & 31, total = NC * nw;
        for (int q = lane; q < total; q += 32) ms = smax(ms, cl.map_shared_rank(red, q / nw)[q % nw]);
        return warp_max(ms);
    };
    auto faces = [&](int b) {
        const double* Wc = Wb(b);
        for (int f = tid; f <= mloc; f += T) {
            // face between local cells f-1 and f: W slots a = f + 1, b = f + 2
            const int a = f + 1, bb = f + 2;
            double sa[3], sb[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double* w = Wc + k * mw;
                sa[k] = limit(w[a] - w[a - 1], w[bb] - w[a], LIM >= 0 ? LIM : lp.lim);
                sb[k] = limit(w[bb] - w[a], w[bb + 1] - w[bb], LIM >= 0 ? LIM : lp.lim);
            }
            const double rL = Wc[a] + 0.5 * sa[0], uL = Wc[mw + a] + 0.5 * sa[1], pL = Wc[2 * mw + a] + 0.5 * sa[2];
            const double rR = Wc[bb] - 0.5 * sb[0], uR = Wc[mw + bb] - 0.5 * sb[1], pR = Wc[2 * mw + bb] - 0.5 * sb[2];
            double f0, f1, f2;
            hlle1d(gamma, gm1, rL, uL, pL, rR, uR, pR, f0, f1, f2);
            F[f] = f0; F[(m + 1) + f] = f1; F[2 * (m + 1) + f] = f2;
        }
    };
    // stage update of this CTA's cells; in stage 2 (heun) also the max |u|+c
    // of the new state (same formulas as `speeds`) into red and the
    // positivity check of step `step_done`: a failing cell makes the maximum
    // infinite, which ends the loop on every CTA of the cluster
    auto update = [&](const double* Uin, double* Uout, bool heun, double dtdx, int bnext, int step_done) {
        double ms = 0.0;
        for (int l = tid; l < mloc; l += T) {
            double v[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                v[k] = Uin[k * m + l] - dtdx * (F[k * (m + 1) + l + 1] - F[k * (m + 1) + l]);
                if (heun) v[k] = 0.5 * (Uout[k * m + l] + v[k]);
                Uout[k * m + l] = v[k];
            }
            prims_of(l, v[0], v[1], v[2], bnext);
            if (heun) {
                const double* w = Wb(bnext);
                const double rr = w[2 + l], u = w[mw + 2 + l], pr = w[2 * mw + 2 + l];
                const double cs = sqrt(gamma * pr / rr);
                ms = smax(ms, fabs(u) + cs);
                if (!(rr > 0.0) || !(pr > 0.0)) {
                    flag_cell(ctrl, step_done, rr, pr, c_lo + l, 0);
                    ms = __longlong_as_double(0x7ff0000000000000ll);
                }
            }
        }
        if (heun) {
            ms = warp_max(ms);
            if ((tid & 31) == 0) red[tid >> 5] = ms;
        }
    };

    // prologue: this CTA's cells, their primitives (buffer 0) and the first dt
    for (int i = tid; i < 3 * m; i += T) {
        const int k = i / m, l = i - k * m;
        U[i] = l < mloc ? Ug[k * nt + h + c_lo + l] : 0.0;
        U1[i] = 0.0;
    }
    __syncthreads();
    for (int l = tid; l < mloc; l += T) prims_of(l, U[l], U[m + l], U[2 * m + l], 0);
    cl.sync();
    speeds(0);
    cl.sync();

    double time = ctrl->time[p];
    int step = ctrl->step[p];
    const bool stopped = (ctrl->err & ERRW_STOP) != 0;  // an earlier step failed: run nothing
    for (int it = 0;; ++it) {
        if (stopped) break;
        if (lp.step_budget > 0 && it >= lp.step_budget) break;
        if (lp.t_final > 0.0 && !(time < lp.t_final)) break;
        if (lp.max_steps > 0 && step >= lp.max_steps) break;
        if (lp.dts_in && step >= lp.dts_cap) break;
        // the stage-1 fluxes do not depend on dt: compute them while the
        // cluster-wide maximum (remote loads) and dt are in flight
        faces(0);
        const double ms = cluster_max();
        double dt;
        if (lp.fixed_dt > 0.0) {
            dt = lp.fixed_dt;
        } else if (lp.dts_in) {
            dt = lp.dts_in[step];
        } else {
            dt = lp.cfl * dx / ms;
            if (lp.t_final > 0.0) dt = smin(dt, lp.t_final - time);
        }
        if (!(ms == ms) || ms > 1.79e308) { if (r == 0 && tid == 0) atomicOr(&ctrl->err, ERRW_NONFINITE); break; }
        if (r == 0 && tid == 0 && lp.dts_out && step < lp.dts_cap) lp.dts_out[step] = dt;
        const double dtdx = dt / dx;
        __syncthreads();                // stage 1 fluxes (from W0 = prims(U)) complete
        update(U, U1, false, dtdx, 1, 0);  // U1, W1 = prims(U1) and the neighbours' halos
        cl.sync();
        faces(1);                       // stage 2 fluxes
        __syncthreads();
        update(U1, U, true, dtdx, 0, step + 1);  // U = (U + U1 - dt L(U1)) / 2, W0 = prims(U), max |u|+c
        cl.sync();
        time += dt;
        ++step;
    }
    // state and the domain's ghost cells back to global memory
    for (int i = tid; i < 3 * mloc; i += T) {
        const int k = i / mloc, l = i - k * mloc;
        const double v = U[k * m + l];
        const int c = c_lo + l;
        Ug[k * nt + h + c] = v;
        if (bc == BC_PERIODIC) {
            if (c >= n - h) Ug[k * nt + c + h - n] = v;
            if (c < h) Ug[k * nt + h + n + c] = v;
        } else {
            if (c == 0) for (int e = 0; e < h; ++e) Ug[k * nt + e] = v;
            if (c == n - 1) for (int e = h + n; e < nt; ++e) Ug[k * nt + e] = v;
        }
    }
    if (r == 0 && tid == 0) {
        ctrl->time[p] = time; ctrl->step[p] = step;
        ctrl->time[p ^ 1] = time; ctrl->step[p ^ 1] = step;
    }
    cl.sync();  // no CTA leaves while a neighbour may still read its shared memory
}

size_t resident_smem_bytes(int n, int h) {
    int nt = n + 2 * h;
    return sizeof(double) * (size_t)(9 * nt + 3 * (n + 1) + 33);
}

// Cluster launch of the resident solver with NC CTAs; returns
// cudaErrorNotSupported (nothing launched) when the chunk sizes or the
// device's cluster occupancy do not allow that cluster size.
static cudaError_t launch_1d_cluster(double* U, int n, int h, double dx, double gamma, int bc, const LoopParams& lp,
                                     StepCtrl* ctrl, int p, cudaStream_t st, int NC) {
    const int m = (n + NC - 1) / NC;
    if (m < 2 || n - (NC - 1) * m < 2) return cudaErrorNotSupported;  // every CTA needs two cells for the halos
    const int threads = (m + 1 + 31) / 32 * 32;
    if (threads > 256) return cudaErrorNotSupported;
    const size_t smem = sizeof(double) * (size_t)(3 * m + 3 * m + 6 * (m + 4) + 3 * (m + 1) + 32);
    auto kern = lp.lim == LIM_MINMOD ? k1d_cluster<LIM_MINMOD> : k1d_cluster<-1>;
    cudaError_t e;
    if (NC > 8 && (e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(NC, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = NC;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if ((e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg)) != cudaSuccess) {
        cudaGetLastError();
        return cudaErrorNotSupported;
    }
    if (clusters < 1) return cudaErrorNotSupported;
    return cudaLaunchKernelEx(&cfg, kern, U, n, h, m, dx, gamma, bc, lp, ctrl, p);
}

// Whether launch_1d_cluster can place a cluster of 16 or 8 CTAs for n cells
// on the current device (the chunk-size rules and the cluster occupancy query
// of launch_1d_cluster, with nothing launched); remembered per device and n.
bool cluster_1d_available(int n, int h) {
    if (n < 256) return false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    static std::mutex mu;
    static std::map<std::pair<int, int>, bool> known;
    std::lock_guard<std::mutex> lk(mu);
    auto it = known.find({dev, n});
    if (it != known.end()) return it->second;
    bool ok = false;
    for (int NC : {16, 8}) {
        const int m = (n + NC - 1) / NC;
        if (m < 2 || n - (NC - 1) * m < 2) continue;
        const int threads = (m + 1 + 31) / 32 * 32;
        if (threads > 256) continue;
        const size_t smem = sizeof(double) * (size_t)(3 * m + 3 * m + 6 * (m + 4) + 3 * (m + 1) + 32);
        // both limiter instances use the same threads and shared memory; the
        // minmod one stands for both
        if (NC > 8 && cudaFuncSetAttribute(k1d_cluster<LIM_MINMOD>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (cudaFuncSetAttribute(k1d_cluster<LIM_MINMOD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(NC, 1, 1);
        cfg.blockDim = dim3(threads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = NC;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k1d_cluster<LIM_MINMOD>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (clusters >= 1) { ok = true; break; }
    }
    known[{dev, n}] = ok;
    return ok;
}

cudaError_t launch_1d_resident(double* U, int n, int h, double dx, double gamma, int bc,
                               const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st) {
    // 256 cells or more: a cluster of 16 (else 8) CTAs, one per SM
    if (n >= 256) {
        for (int NC : {16, 8}) {
            cudaError_t e = launch_1d_cluster(U, n, h, dx, gamma, bc, lp, ctrl, p, st, NC);
            if (e != cudaErrorNotSupported) return e;
        }
    }
    size_t smem = resident_smem_bytes(n, h);
    // K faces per thread: at least two (independent FP64 chains per thread),
    // more when n + 1 faces exceed 2 * 1024
    const int K = (n + 1 <= 2048) ? 2 : 3;
    if (n + 1 > 3 * 1024) return cudaErrorInvalidValue;
    int threads = ((n + 1 + K - 1) / K + 31) / 32 * 32;
    cudaError_t e;
    // the thread bound sets the register budget: 640 threads (n < 1280, up to
    // 102 registers) or 1024 (64 registers)
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) kern<<<1, threads, smem, st>>>(U, n, h, dx, gamma, bc, lp, ctrl, p);
    };
    const bool mm = lp.lim == LIM_MINMOD;
    if (K == 2 && threads <= 640) mm ? go(k1d_resident<2, 640, LIM_MINMOD>) : go(k1d_resident<2, 640, -1>);
    else if (K == 2) mm ? go(k1d_resident<2, 1024, LIM_MINMOD>) : go(k1d_resident<2, 1024, -1>);
    else mm ? go(k1d_resident<3, 1024, LIM_MINMOD>) : go(k1d_resident<3, 1024, -1>);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace nestb

// Tiled multi-CTA stage kernels (FP64 instantiation; euler1d_f32.cu holds the
// FP32 one).
#include "euler1d_tiled.cuh"

namespace nestb {

cudaError_t launch_1d_prepare(double* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p,
                              cudaStream_t st) {
    return launch_1d_prepare_t<double>(U, n, h, gamma, bc, ctrl, p, st);
}

cudaError_t launch_1d_step(double* U, double* U1, int n, int h, double dx, double gamma, int bc,
                           const LoopParams& lp, StepCtrl* ctrl, int p, int which, cudaStream_t st, double* Uout) {
    return launch_1d_step_t<double>(U, U1, n, h, dx, gamma, bc, lp, ctrl, p, which, st, Uout);
}

cudaError_t launch_1d_fused(const double* Un, double* Unext, double* U1out, int n, int h, double dx, double gamma,
                            int bc, const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st) {
    return launch_1d_fused_t<double>(Un, Unext, U1out, n, h, dx, gamma, bc, lp, ctrl, p, st);
}

}  // namespace nestb
