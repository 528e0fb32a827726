// Internal definitions shared by the host runtime files (capi.cpp, adjoint.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <string>
#include <tuple>

#include "../../include/nest_b200.h"
#include "common.cuh"
#include "euler2d_kernels.cuh"
#include "kernels.h"

namespace nestb {
namespace rt {

nest_status fail(nest_status st, const std::string& msg);
nest_status cuda_fail(cudaError_t e, const char* what);

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) return ::nestb::rt::cuda_fail(e__, #call); \
    } while (0)

double bits_to_double(unsigned long long b);

constexpr int GRAPH_STEPS = 16;  // steps per captured graph (even: parity-neutral)

struct GraphKey {
    int nsteps, parity;
    double cfl, t_final, fixed_dt;
    int max_steps;
    const double* dts_in;
    double* dts_out;
    int dts_cap, tx, warps;
    bool operator<(const GraphKey& o) const {
        return std::tie(nsteps, parity, cfl, t_final, fixed_dt, max_steps, dts_in, dts_out, dts_cap, tx, warps) <
               std::tie(o.nsteps, o.parity, o.cfl, o.t_final, o.fixed_dt, o.max_steps, o.dts_in, o.dts_out,
                        o.dts_cap, o.tx, o.warps);
    }
};

}  // namespace rt
}  // namespace nestb

struct nest_solver {
    nest_solver_desc d{};
    int h = 2;
    int n_total = 0;           // 1D: n + 2h
    int pitch = 0;             // 2D: elements per row
    long long vstride = 0;     // elements per variable plane
    int nvars = 3;
    size_t esize = 8;
    void* U = nullptr;
    void* U1 = nullptr;
    nestb::StepCtrl* ctrl = nullptr;
    nestb::StepCtrl* host_ctrl = nullptr;   // pinned mirror
    double* partials = nullptr;
    long long nrec = 0;
    double* totals_dev = nullptr;
    double* dts_in = nullptr;
    double* dts_out = nullptr;
    int dts_cap = 0;
    int dts_mode = 2;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int parity = 0;
    bool prepared = false;
    int tx = 64, warps = 4;
    int xlo_ex = 0, xhi_ex = 0;    // sharded domain: x sides filled by a halo exchange
    std::map<nestb::rt::GraphKey, cudaGraphExec_t> graphs;

    // 1D FP64 runs the resident solver when one CTA's shared memory holds the
    // domain or a thread-block cluster can split it (up to 16 x 255 cells)
    bool resident() const {
        return d.dim == 1 && d.precision == NEST_F64 && !(d.flags & NEST_FLAG_NO_RESIDENT) &&
               (nestb::resident_smem_bytes(d.nx, h) <= 220 * 1024 || nestb::cluster_1d_available(d.nx, h));
    }
    nestb::Geo2D geo() const {
        nestb::Geo2D g;
        g.nx = d.nx; g.ny = d.ny; g.pitch = pitch; g.vstride = vstride;
        g.bcx = d.bc_x; g.bcy = d.bc_y; g.dx = d.dx; g.dy = d.dy; g.gamma = d.gamma;
        g.xlo_ex = xlo_ex; g.xhi_ex = xhi_ex;
        return g;
    }
    size_t state_bytes() const { return esize * (size_t)nvars * (size_t)vstride; }
};

namespace nestb {
namespace rt {
// Ghost fill + wave-speed maxima of the solver's current state.
nest_status prepare(nest_solver* s);
// Enqueue one step (which: 1 = stage 1, 2 = stage 2, 3 = both) on the solver's buffers.
cudaError_t enqueue_step(nest_solver* s, const LoopParams& lp, int p, int which = 3);
nest_status read_ctrl(nest_solver* s);
// Releases the slab driver's captured step graphs of a solver (slab.cpp).
void slab_release(nest_solver* s);
}  // namespace rt
}  // namespace nestb
