// Allocation-free entry point of the 1D solver.
//
// Some callers cannot allocate device memory: host codes that own every byte
// of the GPU through their own pool and forbid libraries from calling
// cudaMalloc, plugin hosts that sandbox device allocations, and real-time
// loops that must not pay allocation latency (or risk an allocation failure)
// after start-up.  nest_euler1d_run_noalloc serves them: the caller passes the
// state buffer, and the solver's scratch -- a second state buffer U1 and the
// step control block -- lives in a fixed file-scope device array below, so the
// call itself never allocates or frees memory.
//
// The array is part of the library image: every GPU that loads the library
// holds it (about 1.6 MB) until the process exits.  It reaches device memory
// when CUDA loads this file's code module into a context, which under the
// default lazy module loading happens at the first call; a caller that must
// not allocate after start-up makes its first call during start-up.  All calls share it, and it
// keeps the previous call's contents; each call clears the control block it
// needs, and calls that overlap on the GPU (two streams, or two threads at
// once) race on it.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/nest_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace {

// Largest extended length n_interior + 2*n_halo the scratch array holds.
constexpr int NOALLOC_MAX_TOTAL = NEST_NOALLOC_MAX_CELLS;

struct NoallocScratch {
    nestb::StepCtrl ctrl;
    double pad[(256 - sizeof(nestb::StepCtrl) % 256) / sizeof(double)];
    double U1[3 * NOALLOC_MAX_TOTAL];
};

static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

nest_status noalloc_fail(nest_status st, const std::string& msg) { return nestb::record_error(st, msg); }

// Device address of the scratch array in the current device's context.  In
// host code the array's name is only a host-side stand-in; the address comes
// from cudaGetSymbolAddress with the device current.  It is looked up on every
// call (a host-side table lookup once the module is loaded), so a device reset
// or another context, which can place the array elsewhere, never leaves a
// stale address behind.
nest_status scratch_for_current_device(NoallocScratch** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return noalloc_fail(NEST_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = static_cast<NoallocScratch*>(p);
    return NEST_OK;
}

}  // namespace

extern "C" nest_status nest_euler1d_run_noalloc(double* d_state, int n_interior, int n_halo, double dx,
                                                double gamma, int bc, double t_final, double cfl,
                                                int* steps_out, double* time_out, void* stream) {
    if (!d_state) return noalloc_fail(NEST_ERR_INVALID, "null state pointer");
    if (n_interior < 4 || n_halo < 2) return noalloc_fail(NEST_ERR_INVALID, "need n_interior >= 4 and n_halo >= 2");
    if ((long long)n_interior + 2ll * n_halo > NOALLOC_MAX_TOTAL)
        return noalloc_fail(NEST_ERR_INVALID, "n_interior + 2*n_halo exceeds NEST_NOALLOC_MAX_CELLS (" +
                                                  std::to_string(NOALLOC_MAX_TOTAL) + ")");
    if (!(dx > 0.0) || !(gamma > 1.0) || !(cfl > 0.0) || !(t_final > 0.0))
        return noalloc_fail(NEST_ERR_INVALID, "dx, cfl, t_final must be positive and gamma > 1");
    if (bc != NEST_BC_PERIODIC && bc != NEST_BC_OUTFLOW) return noalloc_fail(NEST_ERR_INVALID, "bad bc");

    NoallocScratch* sc = nullptr;
    nest_status r = scratch_for_current_device(&sc);
    if (r != NEST_OK) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    nestb::StepCtrl* ctrl = &sc->ctrl;
    double* U1 = sc->U1;

    // The control block starts from zero on every call (time, step count,
    // wave-speed slots and error word); U1 is fully written before it is read.
    cudaError_t e = cudaMemsetAsync(ctrl, 0, sizeof(nestb::StepCtrl), st);
    nestb::LoopParams lp{};
    lp.cfl = cfl;
    lp.t_final = t_final;
    int parity = 0;
    if (e == cudaSuccess) e = nestb::launch_1d_prepare(d_state, n_interior, n_halo, gamma, bc, ctrl, parity, st);
    nestb::StepCtrl host{};
    const int chunk = 32;
    int last_step = -1;
    while (e == cudaSuccess) {
        // one launch per step, out of place: d_state -> U1 -> d_state (the
        // chunk is even, so the state ends in the caller's buffer)
        for (int i = 0; i < chunk && e == cudaSuccess; i += 2) {
            e = nestb::launch_1d_fused(d_state, U1, nullptr, n_interior, n_halo, dx, gamma, bc, lp, ctrl, parity, st);
            if (e == cudaSuccess)
                e = nestb::launch_1d_fused(U1, d_state, nullptr, n_interior, n_halo, dx, gamma, bc, lp, ctrl,
                                           parity ^ 1, st);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&host, ctrl, sizeof host, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        if (host.err & nestb::ERRW_STOP)
            return noalloc_fail(NEST_ERR_NUMERIC, nestb::ctrl_error_text(host, host.step[parity]));
        if (!(host.time[parity] < t_final)) break;
        if (host.step[parity] == last_step) return noalloc_fail(NEST_ERR_NUMERIC, "time stopped advancing");
        last_step = host.step[parity];
    }
    if (e != cudaSuccess) return noalloc_fail(NEST_ERR_CUDA, std::string("1D run: ") + cudaGetErrorString(e));
    if (steps_out) *steps_out = host.step[parity];
    if (time_out) *time_out = host.time[parity];
    return NEST_OK;
}
