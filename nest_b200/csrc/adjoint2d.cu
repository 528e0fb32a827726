// Instantiations and launchers of the 2D adjoint stage.  Each precision is
// compiled in its own translation unit: this one (FP64, IEEE arithmetic) and
// adjoint2d_f32.cu (FP32 with fast reciprocal / square root).
#include "adjoint2d_launch.cuh"

namespace nestb {

cudaError_t launch_2d_adjoint_stage_f64(const double* U, const double* Lout, const double* Extra, double* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st) {
    return adjoint2d_launch<double>(U, Lout, Extra, Lin, g, dtp, alpha, beta, st);
}

}  // namespace nestb
