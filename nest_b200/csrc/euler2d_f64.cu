// FP64 instantiation of the 2D stage kernels (the plain form).  Compiled with
// -fmad=false and IEEE division / square root so that it reproduces the CPU
// restatement of the scheme bit for bit.
#include <algorithm>
#include <cstdlib>

#include "euler2d_kernels.cuh"
#include "kernels.h"

namespace nestb {

// Register budgets of the two stage kernels (0: ptxas's choice, 124 and 152
// registers).  A sweep at 4096^2 (B200, 32-row tiles) measured stage 2 at
// 1.83 ms with 152 registers and 1.61 ms with a budget of 128 (small spill,
// 16 instead of 13 warps per SM); stage 1 was fastest as chosen by ptxas.
#ifndef NEST_F64_REGS1
#define NEST_F64_REGS1 0
#endif
#ifndef NEST_F64_REGS2
#define NEST_F64_REGS2 128
#endif
#if NEST_F64_REGS1 > 0
#define NEST_F64_ATTR1 __maxnreg__(NEST_F64_REGS1)
#else
#define NEST_F64_ATTR1 __launch_bounds__(256)
#endif
#if NEST_F64_REGS2 > 0
#define NEST_F64_ATTR2 __maxnreg__(NEST_F64_REGS2)
#else
#define NEST_F64_ATTR2 __launch_bounds__(256)
#endif

__global__ void NEST_F64_ATTR1 k2d_f64_1(StageArgs<double> a) {
    stage2d_body<double, 1, false>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}
__global__ void NEST_F64_ATTR2 k2d_f64_2(StageArgs<double> a) {
    stage2d_body<double, 2, false>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

__global__ void __launch_bounds__(256) k2d_prepare_f64(double* U, Geo2D g, StepCtrl* ctrl, int p) {
    prepare2d_body<double>(U, g, ctrl, p);
}

cudaError_t launch_2d_prepare_f64(double* U, const Geo2D& g, StepCtrl* ctrl, int p, cudaStream_t st) {
    // rows folded per thread: about 16 (grid rows capped at 32 blocks)
    dim3 b(32, 8), gr((g.ny + 4 + 31) / 32, std::min((g.nx + 4 + 7) / 8, 32));
    k2d_prepare_f64<<<gr, b, 0, st>>>(U, g, ctrl, p);
    return cudaGetLastError();
}

cudaError_t launch_2d_step_f64(double* U, double* U1, const Geo2D& g, const LoopParams& lp,
                               StepCtrl* ctrl, double* partials, int p, int tx, int warps,
                               int which, cudaStream_t st, double* Uout) {
    // the staged row march (euler2d_f64r.cu) is the default; the environment
    // variable NEST_F64_KERNEL=register selects this file's register-window
    // march (same results bit for bit).  4096^2 diagonal Riemann problem, ms
    // per step: 2.77 staged (16-row tiles) against 3.01 (32-row tiles).
    static const int staged = [] {
        const char* e = std::getenv("NEST_F64_KERNEL");
        return (e && e[0] == 'r' && e[1] == 'e') ? 0 : 1;
    }();
    if (staged) return launch_2d_step_f64r(U, U1, g, lp, ctrl, partials, p, tx, warps, which, st, Uout);
    int nstrips = (g.ny + STRIP - 1) / STRIP;
    dim3 b(32, warps), gr((nstrips + warps - 1) / warps, (g.nx + tx - 1) / tx);
    StageArgs<double> a1{U, nullptr, U1, g, lp, ctrl, nullptr, p, tx};
    if (which & 1) k2d_f64_1<<<gr, b, 0, st>>>(a1);
    StageArgs<double> a2{U1, U, Uout ? Uout : U, g, lp, ctrl, partials, p, tx};
    if (which & 2) k2d_f64_2<<<gr, b, 0, st>>>(a2);
    return cudaGetLastError();
}

template <int STAGE>
__device__ __noinline__ void f64_body_call(const StageArgs<double>& a, int strip, int tile_row) {
    stage2d_body<double, STAGE, false>(a, strip, tile_row);
}

// Persistent batched FP64 stage (bit-exact per problem).
template <int STAGE>
__global__ void __launch_bounds__(256) kbatch_f64(BatchArgs<double> b) {
    const int nw = gridDim.x * blockDim.y;
    for (int it = blockIdx.x * blockDim.y + threadIdx.y; it < b.nitems; it += nw) {
        const int4 w = b.items[it];
        const BatchProblem& P = b.probs[w.x];
        StageArgs<double> a{STAGE == 1 ? b.U + P.off : b.U1 + P.off, STAGE == 2 ? b.U + P.off : nullptr,
                            STAGE == 1 ? b.U1 + P.off : b.U + P.off, P.g, b.lp, b.ctrls + w.x,
                            (STAGE == 2 && b.partials) ? b.partials + 4ll * P.item0 : nullptr, b.p, b.tx};
        f64_body_call<STAGE>(a, w.y, w.z);
    }
}

cudaError_t launch_batch_f64(const BatchArgs<double>& b, int which, int blocks, int warps, cudaStream_t st) {
    dim3 blk(32, warps);
    if (which & 1) kbatch_f64<1><<<blocks, blk, 0, st>>>(b);
    if (which & 2) kbatch_f64<2><<<blocks, blk, 0, st>>>(b);
    return cudaGetLastError();
}

int batch_max_blocks_f64(int warps) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kbatch_f64<2>, 32 * warps, 0);
    return nb;
}

// Per-problem deterministic sums of the per-item totals: block p sums items
// [first[p], first[p+1]) in a fixed order.
__global__ void __launch_bounds__(256) k_sum_batch(const double* part, const int* first, double* out) {
    __shared__ double s[4][256];
    int p = blockIdx.x;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (long long r = first[p] + threadIdx.x; r < first[p + 1]; r += 256) {
        a0 += part[4 * r]; a1 += part[4 * r + 1]; a2 += part[4 * r + 2]; a3 += part[4 * r + 3];
    }
    s[0][threadIdx.x] = a0; s[1][threadIdx.x] = a1; s[2][threadIdx.x] = a2; s[3][threadIdx.x] = a3;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 4; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[4 * p + threadIdx.x] = s[threadIdx.x][0];
}

cudaError_t launch_sum_batch(const double* partials, const int* first, int count, double* out, cudaStream_t st) {
    k_sum_batch<<<count, 256, 0, st>>>(partials, first, out);
    return cudaGetLastError();
}

// Deterministic sum of per-warp totals: one block, fixed strided order, fixed tree.
__global__ void __launch_bounds__(256) k_sum_partials(const double* part, long long nrec, double* out) {
    __shared__ double s[4][256];
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (long long r = threadIdx.x; r < nrec; r += 256) {
        a0 += part[4 * r]; a1 += part[4 * r + 1]; a2 += part[4 * r + 2]; a3 += part[4 * r + 3];
    }
    s[0][threadIdx.x] = a0; s[1][threadIdx.x] = a1; s[2][threadIdx.x] = a2; s[3][threadIdx.x] = a3;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 4; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

cudaError_t launch_sum_partials(const double* partials, long long nrec, double* out4, cudaStream_t st) {
    k_sum_partials<<<1, 256, 0, st>>>(partials, nrec, out4);
    return cudaGetLastError();
}

}  // namespace nestb
