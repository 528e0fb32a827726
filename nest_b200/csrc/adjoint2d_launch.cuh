// Kernel and launcher template of the 2D adjoint stage (one tile per CTA).
#pragma once

#include "adjoint2d.cuh"
#include "kernels.h"

namespace nestb {
namespace {

template <typename T>
__global__ void __launch_bounds__(ANT) k2d_adjoint(const T* U, const T* Lout, const T* Extra, T* Lin, Geo2D g,
                                                   const double* dtp, T alpha, T beta) {
    const double dt = *dtp;
    adjoint2d_tile<T>(U, Lout, Extra, Lin, g, (T)(dt / g.dx), (T)(dt / g.dy), alpha, beta);
}

template <typename T>
cudaError_t adjoint2d_launch(const T* U, const T* Lout, const T* Extra, T* Lin, const Geo2D& g, const double* dtp,
                             double alpha, double beta, cudaStream_t st) {
    size_t smem = sizeof(AdjSmem<T>);
    cudaError_t e = cudaFuncSetAttribute(k2d_adjoint<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 gr((g.ny + ATY - 1) / ATY, (g.nx + ATX - 1) / ATX);
    k2d_adjoint<T><<<gr, ANT, smem, st>>>(U, Lout, Extra, Lin, g, dtp, (T)alpha, (T)beta);
    return cudaGetLastError();
}

}  // namespace
}  // namespace nestb
