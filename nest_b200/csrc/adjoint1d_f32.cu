// FP32 instantiation of the 1D reverse step (adjoint1d.cuh), compiled with
// -use_fast_math like the FP32 forward kernels.
#include "adjoint1d.cuh"

namespace nestb {

cudaError_t launch_1d_adjoint_step_f32(const float* Un, const float* U1, const float* lam, float* lam_new, int n,
                                       int h, const double* dtp, double dx, double gamma, cudaStream_t st) {
    return launch_1d_adjoint_step_t<float>(Un, U1, lam, lam_new, n, h, dtp, dx, gamma, st);
}

}  // namespace nestb
