// FP64 instantiation of the 1D reverse step (adjoint1d.cuh).
#include "adjoint1d.cuh"

namespace nestb {

cudaError_t launch_1d_adjoint_step(const double* Un, const double* U1, const double* lam, double* lam_new, int n,
                                   int h, const double* dtp, double dx, double gamma, cudaStream_t st) {
    return launch_1d_adjoint_step_t<double>(Un, U1, lam, lam_new, n, h, dtp, dx, gamma, st);
}

}  // namespace nestb
