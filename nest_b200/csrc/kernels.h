// Internal launcher declarations shared by the kernel translation units and
// the host runtime (capi.cpp).  Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <string>

#include "../../include/nest_b200.h"

#include "common.cuh"

namespace nestb {

struct Geo2D;

// 1D plain form (FP64, bit-exact with nest's OpenMP path)
size_t resident_smem_bytes(int n, int h);
// The resident solver's cluster form can run n cells here (16 or 8 CTAs).
bool cluster_1d_available(int n, int h);
cudaError_t launch_1d_resident(double* U, int n, int h, double dx, double gamma, int bc,
                               const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st);
cudaError_t launch_1d_prepare(double* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p,
                              cudaStream_t st);
// Stage 1 reads U and writes U1; stage 2 reads U1 and U and writes Uout
// (null: U, in place).
cudaError_t launch_1d_step(double* U, double* U1, int n, int h, double dx, double gamma, int bc,
                           const LoopParams& lp, StepCtrl* ctrl, int p, int which, cudaStream_t st,
                           double* Uout = nullptr);
// One whole step in one launch, out of place: Un -> Unext (distinct buffers;
// the caller alternates them), U1 of the step into U1out when not null.  The
// same values as the two stage launches, bit for bit.
cudaError_t launch_1d_fused(const double* Un, double* Unext, double* U1out, int n, int h, double dx, double gamma,
                            int bc, const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st);
// 1D FP32 form (tiled kernels only; time, dt and wave speeds in FP64).
cudaError_t launch_1d_prepare_f32(float* U, int n, int h, double gamma, int bc, StepCtrl* ctrl, int p,
                                  cudaStream_t st);
cudaError_t launch_1d_step_f32(float* U, float* U1, int n, int h, double dx, double gamma, int bc,
                               const LoopParams& lp, StepCtrl* ctrl, int p, int which, cudaStream_t st,
                               float* Uout = nullptr);
cudaError_t launch_1d_fused_f32(const float* Un, float* Unext, float* U1out, int n, int h, double dx, double gamma,
                               int bc, const LoopParams& lp, StepCtrl* ctrl, int p, cudaStream_t st);

// 2D unsplit scheme.  `which`: 1 = stage 1, 2 = stage 2, 3 = both.
cudaError_t launch_2d_prepare_f64(double* U, const Geo2D& g, StepCtrl* ctrl, int p, cudaStream_t st);
cudaError_t launch_2d_step_f64(double* U, double* U1, const Geo2D& g, const LoopParams& lp,
                               StepCtrl* ctrl, double* partials, int p, int tx, int warps,
                               int which, cudaStream_t st, double* Uout = nullptr);
// The same FP64 stages as a row march fed by shared-memory rings (bit for bit
// the same results).
cudaError_t launch_2d_step_f64r(double* U, double* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl,
                                double* partials, int p, int tx, int warps, int which, cudaStream_t st,
                                double* Uout = nullptr);
cudaError_t launch_2d_prepare_f32(float* U, const Geo2D& g, StepCtrl* ctrl, int p, cudaStream_t st);
cudaError_t launch_2d_step_f32(float* U, float* U1, const Geo2D& g, const LoopParams& lp,
                               StepCtrl* ctrl, double* partials, int p, int tx, int warps,
                               bool repair, int which, cudaStream_t st);
// FP32 form with packed FP32x2 arithmetic, two columns per lane (60 output
// columns per warp).
cudaError_t launch_2d_step_f32x2(float* U, float* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl,
                                 double* partials, int p, int tx, int warps, bool repair, int which,
                                 cudaStream_t st, float* Uout = nullptr);

// nest's split 2D scheme (x-sweep = stage 1, y-sweep = stage 2), FP64.
cudaError_t launch_2d_compat_step(double* U, double* U1, const Geo2D& g, const LoopParams& lp, StepCtrl* ctrl, int p,
                                  int which, cudaStream_t st);

// Adjoint of one 2D stage: Lin = alpha * adj(U, Lout) + beta * Extra (periodic).
// dt is read on the device from *dtp (lx = dt/dx, ly = dt/dy).
cudaError_t launch_2d_adjoint_stage_f64(const double* U, const double* Lout, const double* Extra, double* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st);
cudaError_t launch_2d_adjoint_stage_f32(const float* U, const float* Lout, const float* Extra, float* Lin,
                                        const Geo2D& g, const double* dtp, double alpha, double beta,
                                        cudaStream_t st);
// Row-march form of the FP64 stage (one column per lane, any ny).
cudaError_t launch_2d_adjoint_stage_f64rm(const double* U, const double* Lout, const double* Extra, double* Lin,
                                          const Geo2D& g, const double* dtp, double alpha, double beta,
                                          cudaStream_t st);
// Packed FP32x2 row-march form of the same stage; cudaErrorNotSupported
// (nothing launched) for an odd ny.
cudaError_t launch_2d_adjoint_stage_f32x2(const float* U, const float* Lout, const float* Extra, float* Lin,
                                          const Geo2D& g, const double* dtp, double alpha, double beta,
                                          cudaStream_t st);

// Batched persistent stages (one launch per stage over the work list).
template <typename T> struct BatchArgs;
cudaError_t launch_batch_f64(const BatchArgs<double>& b, int which, int blocks, int warps, cudaStream_t st);
cudaError_t launch_batch_f32x2(const BatchArgs<float>& b, bool repair, int which, int blocks, int warps,
                               cudaStream_t st);
int batch_max_blocks_f64(int warps);
int batch_max_blocks_f32x2(int warps);
int strips_f32x2(int ny);
cudaError_t launch_sum_batch(const double* partials, const int* first, int count, double* out, cudaStream_t st);

// Records msg as the calling thread's last error (read by nest_last_error()).
nest_status record_error(nest_status st, const std::string& msg);
// Text of the error record of a control block whose err word is set:
// positivity violation or non-finite state, with the step and the first
// failing cell when one was recorded (`steps_now`: the solver's step count,
// used when no cell was).
std::string ctrl_error_text(const StepCtrl& c, int steps_now);

// Fixed-order sum of per-warp totals (deterministic).
cudaError_t launch_sum_partials(const double* partials, long long nrec, double* out4, cudaStream_t st);

}  // namespace nestb
