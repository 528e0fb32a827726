// Instantiations and launchers of the 2D adjoint stage (FP32 and FP64).
#include "adjoint2d.cuh"
#include "kernels.h"

namespace nestb {
namespace {

template <typename T>
__global__ void __launch_bounds__(AT * AT) k2d_adjoint(const T* U, const T* Lout, const T* Extra, T* Lin, Geo2D g,
                                                       const double* dtp, T alpha, T beta) {
    const double dt = *dtp;
    adjoint2d_tile<T>(U, Lout, Extra, Lin, g, (T)(dt / g.dx), (T)(dt / g.dy), alpha, beta);
}

template <typename T>
cudaError_t launch(const T* U, const T* Lout, const T* Extra, T* Lin, const Geo2D& g, const double* dtp,
                   double alpha, double beta, cudaStream_t st) {
    size_t smem = sizeof(AdjSmem<T>);
    cudaError_t e = cudaFuncSetAttribute(k2d_adjoint<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 gr((g.ny + AT - 1) / AT, (g.nx + AT - 1) / AT);
    k2d_adjoint<T><<<gr, AT * AT, smem, st>>>(U, Lout, Extra, Lin, g, dtp, (T)alpha, (T)beta);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_2d_adjoint_stage_f64(const double* U, const double* Lout, const double* Extra, double* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st) {
    return launch<double>(U, Lout, Extra, Lin, g, dtp, alpha, beta, st);
}

cudaError_t launch_2d_adjoint_stage_f32(const float* U, const float* Lout, const float* Extra, float* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st) {
    return launch<float>(U, Lout, Extra, Lin, g, dtp, alpha, beta, st);
}

}  // namespace nestb
