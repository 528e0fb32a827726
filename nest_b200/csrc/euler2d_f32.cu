// FP32 instantiation of the 2D stage kernels (the FP32 form: reconstruction,
// Riemann solve and update in FP32; wave-speed maxima, totals, time and
// positivity repair in FP64).  Compiled with FMA contraction and fast FP32
// division / square root.
#include <algorithm>

#include "euler2d_kernels.cuh"
#include "kernels.h"

namespace nestb {

template <int STAGE, bool REPAIR>
__global__ void __launch_bounds__(256) k2d_f32(StageArgs<float> a) {
    stage2d_body<float, STAGE, REPAIR>(a, blockIdx.x * blockDim.y + threadIdx.y, blockIdx.y);
}

__global__ void __launch_bounds__(256) k2d_prepare_f32(float* U, Geo2D g, StepCtrl* ctrl, int p) {
    prepare2d_body<float>(U, g, ctrl, p);
}

cudaError_t launch_2d_prepare_f32(float* U, const Geo2D& g, StepCtrl* ctrl, int p, cudaStream_t st) {
    // rows folded per thread: about 16 (grid rows capped at 32 blocks)
    dim3 b(32, 8), gr((g.ny + 4 + 31) / 32, std::min((g.nx + 4 + 7) / 8, 32));
    k2d_prepare_f32<<<gr, b, 0, st>>>(U, g, ctrl, p);
    return cudaGetLastError();
}

cudaError_t launch_2d_step_f32(float* U, float* U1, const Geo2D& g, const LoopParams& lp,
                               StepCtrl* ctrl, double* partials, int p, int tx, int warps,
                               bool repair, int which, cudaStream_t st) {
    int nstrips = (g.ny + STRIP - 1) / STRIP;
    dim3 b(32, warps), gr((nstrips + warps - 1) / warps, (g.nx + tx - 1) / tx);
    StageArgs<float> a1{U, nullptr, U1, g, lp, ctrl, nullptr, p, tx};
    StageArgs<float> a2{U1, U, U, g, lp, ctrl, partials, p, tx};
    if (repair) {
        if (which & 1) k2d_f32<1, true><<<gr, b, 0, st>>>(a1);
        if (which & 2) k2d_f32<2, true><<<gr, b, 0, st>>>(a2);
    } else {
        if (which & 1) k2d_f32<1, false><<<gr, b, 0, st>>>(a1);
        if (which & 2) k2d_f32<2, false><<<gr, b, 0, st>>>(a2);
    }
    return cudaGetLastError();
}

}  // namespace nestb
