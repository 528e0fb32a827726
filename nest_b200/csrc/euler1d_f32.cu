// FP32 form of the tiled 1D stage kernels (compiled with -use_fast_math):
// state, reconstruction, Riemann solve and update in FP32; time, dt and the
// wave-speed maximum in FP64.
#include "euler1d_tiled.cuh"

namespace nestb {

cudaError_t launch_1d_prepare_f32(float* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p,
                                  cudaStream_t st) {
    return launch_1d_prepare_t<float>(U, n, h, gamma, bc, ctrl, p, st);
}

cudaError_t launch_1d_step_f32(float* U, float* U1, int n, int h, double dx, double gamma, int bc,
                               const LoopParams& lp, StepCtrl* ctrl, int p, int which, cudaStream_t st, float* Uout) {
    return launch_1d_step_t<float>(U, U1, n, h, dx, gamma, bc, lp, ctrl, p, which, st, Uout);
}

cudaError_t launch_1d_fused_f32(const float* Un, float* Unext, float* U1out, int n, int h, double dx, double gamma,
                               int bc, const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st) {
    return launch_1d_fused_t<float>(Un, Unext, U1out, n, h, dx, gamma, bc, lp, ctrl, p, st);
}

}  // namespace nestb
