// FP32 instantiation of the 2D adjoint stage (compiled with -use_fast_math).
#include "adjoint2d_launch.cuh"

namespace nestb {

cudaError_t launch_2d_adjoint_stage_f32(const float* U, const float* Lout, const float* Extra, float* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st) {
    return adjoint2d_launch<float>(U, Lout, Extra, Lin, g, dtp, alpha, beta, st);
}

}  // namespace nestb
