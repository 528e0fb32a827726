// Host runtime and C ABI of the nest B200 hot path (C++20).
//
// One nest_solver owns its device state (U, the stage buffer U1, a StepCtrl
// control block and optional per-warp totals) and a stream.  Steps are
// enqueued without host synchronisation: dt is derived on the device from
// the wave-speed maximum that the previous stage 2 reduced, and runs of steps
// are captured once into CUDA graphs and replayed.
//
// The euler1d_gpu_* functions keep the names, signatures and semantics of
// nest's C ABI (src/backend_cuda/euler1d_solver.hpp:16-87,
// src/backend_cuda/euler1d_solver.cu:159-235) on top of a 1D FP64 solver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace {
thread_local std::string g_last_error;
}  // namespace

nest_status nestb::rt::fail(nest_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

nest_status nestb::rt::cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? NEST_ERR_OOM : NEST_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

double nestb::rt::bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof d);
    return d;
}

nest_status nestb::record_error(nest_status st, const std::string& msg) { return fail(st, msg); }

std::string nestb::ctrl_error_text(const StepCtrl& c, int steps_now) {
    char buf[256];
    if (c.bad_step > 0) {
        // the recorded cell names the failure: a NaN is a non-finite state
        const bool nan = !(c.bad_rho == c.bad_rho) || !(c.bad_p == c.bad_p);
        std::snprintf(buf, sizeof buf, "%s at step %d in cell (%d, %d): rho = %.17g, p = %.17g",
                      nan ? "non-finite state (NaN)" : "positivity violation (rho <= 0 or p <= 0)", c.bad_step,
                      c.bad_i, c.bad_j, c.bad_rho, c.bad_p);
    } else {
        std::snprintf(buf, sizeof buf, "non-finite state: infinite or NaN wave speed after step %d", steps_now);
    }
    return buf;
}

namespace {

nest_status drop_graphs(nest_solver* s) {
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    slab_release(s);
    return NEST_OK;
}

LoopParams base_params(const nest_solver* s) {
    LoopParams lp{};
    lp.lim = (s->d.flags & NEST_FLAG_LIMITER_MC) ? LIM_MC : (s->d.flags & NEST_FLAG_LIMITER_NONE) ? LIM_NONE : LIM_MINMOD;
    lp.dts_in = (s->dts_mode == 0) ? s->dts_in : nullptr;
    lp.dts_out = (s->dts_mode == 1) ? s->dts_out : nullptr;
    lp.dts_cap = s->dts_cap;
    return lp;
}

}  // namespace

// Ghost fill + wave-speed maxima of the current state into slot `parity`.
nest_status nestb::rt::prepare(nest_solver* s) {
    // both slots: the one-launch 1D step adds into maxs[1 - parity][1]
    CK(cudaMemsetAsync(&s->ctrl->maxs[0][0], 0, sizeof s->ctrl->maxs, s->st));
    cudaError_t e;
    if (s->d.dim == 1 && s->d.precision == NEST_F32) {
        e = launch_1d_prepare_f32((float*)s->U, s->d.nx, s->h, s->d.gamma, s->d.bc_x, s->ctrl, s->parity, s->st);
    } else if (s->d.dim == 1) {
        e = launch_1d_prepare((double*)s->U, s->d.nx, s->h, s->d.gamma, s->d.bc_x, s->ctrl, s->parity, s->st);
    } else if (s->d.precision == NEST_F64) {
        e = launch_2d_prepare_f64((double*)s->U, s->geo(), s->ctrl, s->parity, s->st);
    } else {
        e = launch_2d_prepare_f32((float*)s->U, s->geo(), s->ctrl, s->parity, s->st);
    }
    if (e != cudaSuccess) return cuda_fail(e, "prepare kernel");
    s->prepared = true;
    return NEST_OK;
}

// Enqueue one step (the two stage kernels, in place) with parity p; `which`
// selects the stages.
cudaError_t nestb::rt::enqueue_step(nest_solver* s, const LoopParams& lp, int p, int which) {
    if (s->d.dim == 1 && s->d.precision == NEST_F32)
        return launch_1d_step_f32((float*)s->U, (float*)s->U1, s->d.nx, s->h, s->d.dx, s->d.gamma, s->d.bc_x, lp,
                                  s->ctrl, p, which, s->st);
    if (s->d.dim == 1)
        return launch_1d_step((double*)s->U, (double*)s->U1, s->d.nx, s->h, s->d.dx, s->d.gamma, s->d.bc_x, lp,
                              s->ctrl, p, which, s->st);
    if (s->d.flags & NEST_FLAG_SPLIT_COMPAT)
        return launch_2d_compat_step((double*)s->U, (double*)s->U1, s->geo(), lp, s->ctrl, p, which, s->st);
    if (s->d.precision == NEST_F64)
        return launch_2d_step_f64((double*)s->U, (double*)s->U1, s->geo(), lp, s->ctrl, s->partials, p, s->tx,
                                  s->warps, which, s->st);
    if (s->d.flags & (NEST_FLAG_FP32_SCALAR | NEST_FLAG_LIMITER_MC | NEST_FLAG_LIMITER_NONE))
        return launch_2d_step_f32((float*)s->U, (float*)s->U1, s->geo(), lp, s->ctrl, s->partials, p, s->tx,
                                  s->warps, (s->d.flags & NEST_FLAG_REPAIR) != 0, which, s->st);
    return launch_2d_step_f32x2((float*)s->U, (float*)s->U1, s->geo(), lp, s->ctrl, s->partials, p, s->tx,
                                s->warps, (s->d.flags & NEST_FLAG_REPAIR) != 0, which, s->st);
}

namespace {

// Two 1D steps with parity p, one launch each, out of place: U -> U1 -> U
// (the stage buffer holds the state between them, so the state ends where it
// started).
cudaError_t enqueue_pair_1d(nest_solver* s, const LoopParams& lp, int p) {
    auto one = [&](void* from, void* to, int pp) {
        if (s->d.precision == NEST_F32)
            return launch_1d_fused_f32((const float*)from, (float*)to, nullptr, s->d.nx, s->h, s->d.dx, s->d.gamma,
                                       s->d.bc_x, lp, s->ctrl, pp, s->st);
        return launch_1d_fused((const double*)from, (double*)to, nullptr, s->d.nx, s->h, s->d.dx, s->d.gamma,
                               s->d.bc_x, lp, s->ctrl, pp, s->st);
    };
    cudaError_t e = one(s->U, s->U1, p);
    if (e == cudaSuccess) e = one(s->U1, s->U, p ^ 1);
    return e;
}

// Enqueue nsteps steps of the tiled path; whole chunks go through cached
// graphs.  1D steps go in pairs of one-launch steps; an odd last step runs
// the two stage launches in place.
nest_status enqueue_steps(nest_solver* s, int nsteps, const LoopParams& lp) {
    if (!s->prepared) {
        nest_status r = prepare(s);
        if (r != NEST_OK) return r;
    }
    bool use_graphs = s->st != nullptr;
    const bool pairs = s->d.dim == 1;
    while (nsteps > 0) {
        if (use_graphs && nsteps >= GRAPH_STEPS) {
            GraphKey k{GRAPH_STEPS, s->parity, lp.cfl, lp.t_final, lp.fixed_dt, lp.max_steps, lp.dts_in,
                       lp.dts_out, lp.dts_cap, s->tx, s->warps};
            auto it = s->graphs.find(k);
            if (it == s->graphs.end()) {
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
                int p = s->parity;
                cudaError_t e = cudaSuccess;
                if (pairs)
                    for (int i = 0; i < GRAPH_STEPS && e == cudaSuccess; i += 2) e = enqueue_pair_1d(s, lp, p);
                else
                    for (int i = 0; i < GRAPH_STEPS && e == cudaSuccess; ++i, p ^= 1) e = enqueue_step(s, lp, p);
                cudaError_t e2 = cudaStreamEndCapture(s->st, &g);
                if (e != cudaSuccess) {
                    if (e2 == cudaSuccess) cudaGraphDestroy(g);
                    return cuda_fail(e, "step capture");
                }
                if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
                cudaGraphExec_t ge;
                cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
                it = s->graphs.emplace(k, ge).first;
            }
            CK(cudaGraphLaunch(it->second, s->st));
            nsteps -= GRAPH_STEPS;  // parity unchanged (even chunk)
        } else if (pairs && nsteps >= 2) {
            cudaError_t e = enqueue_pair_1d(s, lp, s->parity);
            if (e != cudaSuccess) return cuda_fail(e, "step launch");
            nsteps -= 2;  // parity unchanged
        } else {
            cudaError_t e = enqueue_step(s, lp, s->parity);
            if (e != cudaSuccess) return cuda_fail(e, "step launch");
            s->parity ^= 1;
            --nsteps;
        }
    }
    return NEST_OK;
}

}  // namespace

nest_status nestb::rt::read_ctrl(nest_solver* s) {
    CK(cudaMemcpyAsync(s->host_ctrl, s->ctrl, sizeof(StepCtrl), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (s->host_ctrl->err & ERRW_STOP)
        return fail(NEST_ERR_NUMERIC, ctrl_error_text(*s->host_ctrl, s->host_ctrl->step[s->parity]));
    return NEST_OK;
}

namespace {

// Advance by at most `budget` steps (<= 0: unbounded) with the given loop
// parameters; on the resident 1D path this is a single launch.
nest_status advance(nest_solver* s, LoopParams lp, int budget) {
    if (s->resident()) {
        lp.step_budget = budget;
        cudaError_t e = launch_1d_resident((double*)s->U, s->d.nx, s->h, s->d.dx, s->d.gamma, s->d.bc_x, lp,
                                           s->ctrl, s->parity, s->st);
        if (e != cudaSuccess) return cuda_fail(e, "resident solver launch");
        s->prepared = false;  // the resident kernel does not leave maxs behind
        return NEST_OK;
    }
    return enqueue_steps(s, budget, lp);
}

nest_status check(const nest_solver* s) {
    if (!s) return fail(NEST_ERR_INVALID, "null solver handle");
    return NEST_OK;
}

nest_status copy_state(nest_solver* s, void* dst, const void* src, int layout, bool upload, cudaMemcpyKind kind) {
    if (layout != NEST_LAYOUT_EXTENDED && layout != NEST_LAYOUT_INTERIOR)
        return fail(NEST_ERR_INVALID, "unknown layout");
    size_t es = s->esize;
    if (s->d.dim == 1) {
        int n = s->d.nx, nt = s->n_total;
        if (layout == NEST_LAYOUT_EXTENDED) {
            if (upload) CK(cudaMemcpyAsync(s->U, src, es * 3 * nt, kind, s->st));
            else CK(cudaMemcpyAsync(dst, s->U, es * 3 * nt, kind, s->st));
        } else {
            // interior rows: 3 planes of n with the device plane stride nt
            if (upload)
                CK(cudaMemcpy2DAsync((char*)s->U + es * s->h, es * nt, src, es * n, es * n, 3, kind, s->st));
            else
                CK(cudaMemcpy2DAsync(dst, es * n, (char*)s->U + es * s->h, es * nt, es * n, 3, kind, s->st));
        }
        return NEST_OK;
    }
    int nx = s->d.nx, ny = s->d.ny;
    int rows = (layout == NEST_LAYOUT_EXTENDED) ? nx + 4 : nx;
    int cols = (layout == NEST_LAYOUT_EXTENDED) ? ny + 4 : ny;
    size_t off = (layout == NEST_LAYOUT_EXTENDED) ? 0 : (size_t)(2 * s->pitch + 2);
    for (int k = 0; k < 4; ++k) {
        char* dev = (char*)s->U + es * ((size_t)k * s->vstride + off);
        size_t hoff = es * (size_t)k * rows * cols;
        if (upload)
            CK(cudaMemcpy2DAsync(dev, es * s->pitch, (const char*)src + hoff, es * cols, es * cols, rows, kind, s->st));
        else
            CK(cudaMemcpy2DAsync((char*)dst + hoff, es * cols, dev, es * s->pitch, es * cols, rows, kind, s->st));
    }
    return NEST_OK;
}

}  // namespace

// ===========================================================================
// Solver API
// ===========================================================================

extern "C" {

const char* nest_last_error(void) { return g_last_error.c_str(); }

int nest_version(void) { return 10000; }

nest_status nest_solver_create(const nest_solver_desc* d, nest_solver** out) {
    if (!d || !out) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->dim != 1 && d->dim != 2) return fail(NEST_ERR_INVALID, "dim must be 1 or 2");
    if (d->nx < 4 || (d->dim == 2 && d->ny < 4)) return fail(NEST_ERR_INVALID, "need at least 4 interior cells per axis");
    if (!(d->dx > 0.0) || (d->dim == 2 && !(d->dy > 0.0))) return fail(NEST_ERR_INVALID, "cell sizes must be positive");
    if (!(d->gamma > 1.0)) return fail(NEST_ERR_INVALID, "gamma must exceed 1");
    if (d->bc_x != NEST_BC_PERIODIC && d->bc_x != NEST_BC_OUTFLOW) return fail(NEST_ERR_INVALID, "bad bc_x");
    if (d->dim == 2 && d->bc_y != NEST_BC_PERIODIC && d->bc_y != NEST_BC_OUTFLOW) return fail(NEST_ERR_INVALID, "bad bc_y");
    if (d->dim == 1 && d->halo < 2) return fail(NEST_ERR_INVALID, "PLM needs a halo of at least 2");
    if (d->dim == 2 && d->halo != 2) return fail(NEST_ERR_UNSUPPORTED, "2D solver uses a halo of exactly 2");
    if (d->dim == 1 && d->precision == NEST_F32 && (d->flags & (NEST_FLAG_TOTALS | NEST_FLAG_REPAIR)))
        return fail(NEST_ERR_UNSUPPORTED, "1D FP32 solver: totals and repair are 2D options");
    if (d->precision != NEST_F64 && d->precision != NEST_F32) return fail(NEST_ERR_INVALID, "bad precision");
    if (d->dim == 2 && (long long)d->nx * d->ny > (1ll << 31)) return fail(NEST_ERR_INVALID, "domain too large");
    if ((d->flags & NEST_FLAG_SPLIT_COMPAT) && (d->dim != 2 || d->precision != NEST_F64))
        return fail(NEST_ERR_UNSUPPORTED, "nest's split scheme runs in 2D FP64");
    if ((d->flags & NEST_FLAG_SPLIT_COMPAT) && (d->flags & NEST_FLAG_TOTALS))
        return fail(NEST_ERR_UNSUPPORTED, "totals are kept by the RK2 scheme only");
    if ((d->flags & NEST_FLAG_LIMITER_MC) && (d->flags & NEST_FLAG_LIMITER_NONE))
        return fail(NEST_ERR_INVALID, "choose one slope limiter");

    nest_solver* s = new (std::nothrow) nest_solver;
    if (!s) return fail(NEST_ERR_OOM, "host allocation failed");
    s->d = *d;
    s->h = d->halo;
    s->esize = d->precision == NEST_F64 ? 8 : 4;
    // default 2D launch shape: the autotuner's choice at 4096^2, one warp per
    // block, 16-row tiles in FP32 and 24-row tiles in FP64 (200 steps of the
    // 4096^2 Riemann problem 2.269 -> 2.233 ms per step, 1000 steps of the
    // 2048^2 KH state 585 -> 574 ms, against 16 rows; 32 rows took 627 ms on
    // KH).  At 2048^2
    // the earlier default of 64-row tiles and 4 warps per block left half the
    // warp slots empty: a 4000-step FP32 KH forward took 891 ms against 540 ms.
    if (d->dim == 2) {
        s->tx = d->precision == NEST_F64 ? 24 : 16;
        s->warps = 1;
    }
    if (d->dim == 1) {
        s->nvars = 3;
        s->n_total = d->nx + 2 * d->halo;
        s->vstride = s->n_total;
        s->pitch = s->n_total;
    } else {
        s->nvars = 4;
        int align = (int)(128 / s->esize);  // rows start on 128-byte boundaries
        s->pitch = ((d->ny + 4 + align - 1) / align) * align;
        s->vstride = (long long)s->pitch * (d->nx + 4);
        long long pad = 256 / (long long)s->esize;
        s->vstride = ((s->vstride + pad - 1) / pad) * pad;
    }
    auto cleanup = [&](nest_status st) { nest_solver_destroy(s); return st; };
    cudaError_t e;
    if (d->stream) {
        s->st = (cudaStream_t)d->stream;
    } else {
        e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaStreamCreate"));
        s->own_stream = true;
    }
    size_t bytes = s->state_bytes();
    if ((e = cudaMalloc(&s->U, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(U)"));
    if ((e = cudaMalloc(&s->U1, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(U1)"));
    if ((e = cudaMalloc(&s->ctrl, sizeof(StepCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(ctrl)"));
    if ((e = cudaMallocHost(&s->host_ctrl, sizeof(StepCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMallocHost"));
    if ((e = cudaMemsetAsync(s->U, 0, bytes, s->st)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMemsetAsync(s->U1, 0, bytes, s->st)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMemsetAsync(s->ctrl, 0, sizeof(StepCtrl), s->st)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if (d->dim == 2 && (d->flags & NEST_FLAG_TOTALS)) {
        long long nstrips = (d->ny + STRIP - 1) / STRIP;
        // sized for the smallest tile height the tiling hook accepts (8 rows)
        s->nrec = nstrips * ((d->nx + 7) / 8);
        if ((e = cudaMalloc(&s->partials, sizeof(double) * 4 * s->nrec)) != cudaSuccess)
            return cleanup(cuda_fail(e, "cudaMalloc(partials)"));
        if ((e = cudaMemsetAsync(s->partials, 0, sizeof(double) * 4 * s->nrec, s->st)) != cudaSuccess)
            return cleanup(cuda_fail(e, "memset"));
        if ((e = cudaMalloc(&s->totals_dev, sizeof(double) * 4)) != cudaSuccess)
            return cleanup(cuda_fail(e, "cudaMalloc(totals)"));
    }
    if ((e = cudaStreamSynchronize(s->st)) != cudaSuccess) return cleanup(cuda_fail(e, "sync"));
    *out = s;
    return NEST_OK;
}

nest_status nest_solver_destroy(nest_solver* s) {
    if (!s) return NEST_OK;
    if (s->st) cudaStreamSynchronize(s->st);
    drop_graphs(s);
    cudaFree(s->U); cudaFree(s->U1); cudaFree(s->ctrl); cudaFree(s->partials); cudaFree(s->totals_dev);
    cudaFree(s->dts_in); cudaFree(s->dts_out);
    if (s->host_ctrl) cudaFreeHost(s->host_ctrl);
    if (s->own_stream && s->st) cudaStreamDestroy(s->st);
    delete s;
    return NEST_OK;
}

static nest_status upload_impl(nest_solver* s, const void* src, int layout, cudaMemcpyKind kind) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!src) return fail(NEST_ERR_INVALID, "null source");
    r = copy_state(s, nullptr, src, layout, true, kind);
    if (r != NEST_OK) return r;
    // a new state starts without an error record
    CK(cudaMemsetAsync(&s->ctrl->err, 0, sizeof(StepCtrl) - offsetof(StepCtrl, err), s->st));
    r = prepare(s);
    if (r != NEST_OK) return r;
    CK(cudaStreamSynchronize(s->st));
    return NEST_OK;
}

static nest_status download_impl(nest_solver* s, void* dst, int layout, cudaMemcpyKind kind) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!dst) return fail(NEST_ERR_INVALID, "null destination");
    r = copy_state(s, dst, nullptr, layout, false, kind);
    if (r != NEST_OK) return r;
    CK(cudaStreamSynchronize(s->st));
    return NEST_OK;
}

nest_status nest_solver_upload(nest_solver* s, const void* host, int layout) {
    return upload_impl(s, host, layout, cudaMemcpyHostToDevice);
}
nest_status nest_solver_download(nest_solver* s, void* host, int layout) {
    return download_impl(s, host, layout, cudaMemcpyDeviceToHost);
}
nest_status nest_solver_upload_device(nest_solver* s, const void* dev, int layout) {
    return upload_impl(s, dev, layout, cudaMemcpyDeviceToDevice);
}
nest_status nest_solver_download_device(nest_solver* s, void* dev, int layout) {
    return download_impl(s, dev, layout, cudaMemcpyDeviceToDevice);
}

nest_status nest_solver_step(nest_solver* s, int nsteps, double cfl) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (nsteps < 0) return fail(NEST_ERR_INVALID, "negative step count");
    if (!(cfl > 0.0)) return fail(NEST_ERR_INVALID, "cfl must be positive");
    if (nsteps == 0) return NEST_OK;
    LoopParams lp = base_params(s);
    lp.cfl = cfl;
    return advance(s, lp, nsteps);
}

nest_status nest_solver_step_profiled(nest_solver* s, int nsteps, double cfl, float* stage_ms, float* total_ms) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (nsteps <= 0 || !(cfl > 0.0)) return fail(NEST_ERR_INVALID, "need nsteps > 0 and cfl > 0");
    if (s->resident()) return fail(NEST_ERR_UNSUPPORTED, "profiled steps use the tiled path (NEST_FLAG_NO_RESIDENT)");
    if (!s->prepared && (r = prepare(s)) != NEST_OK) return r;
    LoopParams lp = base_params(s);
    lp.cfl = cfl;
    int nev = 2 * nsteps + 1;
    cudaEvent_t* ev = new (std::nothrow) cudaEvent_t[nev];
    if (!ev) return fail(NEST_ERR_OOM, "host allocation failed");
    int made = 0;
    cudaError_t e = cudaSuccess;
    for (; made < nev && e == cudaSuccess; ++made) e = cudaEventCreate(&ev[made]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], s->st);
    for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
        e = enqueue_step(s, lp, s->parity, 1);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 1], s->st);
        if (e == cudaSuccess) e = enqueue_step(s, lp, s->parity, 2);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 2], s->st);
        s->parity ^= 1;
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[nev - 1]);
    for (int i = 0; i < 2 * nsteps && e == cudaSuccess; ++i) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        if (stage_ms) stage_ms[i] = ms;
    }
    if (e == cudaSuccess && total_ms) e = cudaEventElapsedTime(total_ms, ev[0], ev[nev - 1]);
    for (int i = 0; i < made; ++i) cudaEventDestroy(ev[i]);
    delete[] ev;
    if (e != cudaSuccess) return cuda_fail(e, "profiled steps");
    return read_ctrl(s);
}

nest_status nest_solver_step_dt(nest_solver* s, int nsteps, double dt) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (nsteps < 0) return fail(NEST_ERR_INVALID, "negative step count");
    if (!(dt > 0.0)) return fail(NEST_ERR_INVALID, "dt must be positive");
    if (nsteps == 0) return NEST_OK;
    LoopParams lp = base_params(s);
    lp.cfl = 1.0;
    lp.fixed_dt = dt;
    lp.dts_in = nullptr;
    return advance(s, lp, nsteps);
}

nest_status nest_solver_run_to(nest_solver* s, double t_final, double cfl, int max_steps, int* steps_out) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!(cfl > 0.0) || !(t_final > 0.0)) return fail(NEST_ERR_INVALID, "cfl and t_final must be positive");
    if ((r = read_ctrl(s)) != NEST_OK) return r;
    int start = s->host_ctrl->step[s->parity];
    LoopParams lp = base_params(s);
    lp.cfl = cfl;
    lp.t_final = t_final;
    lp.max_steps = max_steps > 0 ? start + max_steps : 0;
    if (s->resident()) {
        if ((r = advance(s, lp, 0)) != NEST_OK) return r;
        if ((r = read_ctrl(s)) != NEST_OK) return r;
    } else {
        const int chunk = 4 * GRAPH_STEPS;
        int last = -1;
        for (;;) {
            if ((r = enqueue_steps(s, chunk, lp)) != NEST_OK) return r;
            if ((r = read_ctrl(s)) != NEST_OK) return r;
            const StepCtrl* c = s->host_ctrl;
            int p = s->parity;
            if (!(c->time[p] < t_final)) break;
            if (lp.max_steps > 0 && c->step[p] >= lp.max_steps) break;
            if (s->dts_mode == 0 && c->step[p] >= s->dts_cap) break;
            if (c->step[p] == last) return fail(NEST_ERR_NUMERIC, "time stopped advancing");
            last = c->step[p];
        }
    }
    if (steps_out) *steps_out = s->host_ctrl->step[s->parity] - start;
    return NEST_OK;
}

nest_status nest_solver_compute_dt(nest_solver* s, double cfl, double* dt_out) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!dt_out) return fail(NEST_ERR_INVALID, "null output");
    if ((r = prepare(s)) != NEST_OK) return r;
    if ((r = read_ctrl(s)) != NEST_OK) return r;
    double sx = bits_to_double(s->host_ctrl->maxs[s->parity][0]);
    if (s->d.dim == 1) {
        *dt_out = cfl * s->d.dx / sx;  // benchmark_euler1d.cpp:179
    } else {
        double sy = bits_to_double(s->host_ctrl->maxs[s->parity][1]);
        double dtx = 1e10, dty = 1e10;  // euler2d.hpp:249-270
        if (sx > 0.0 && s->d.dx / sx < dtx) dtx = s->d.dx / sx;
        if (sy > 0.0 && s->d.dy / sy < dty) dty = s->d.dy / sy;
        *dt_out = cfl * (dty < dtx ? dty : dtx);
    }
    return NEST_OK;
}

nest_status nest_solver_time(nest_solver* s, double* time, int* steps) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if ((r = read_ctrl(s)) != NEST_OK) return r;
    if (time) *time = s->host_ctrl->time[s->parity];
    if (steps) *steps = s->host_ctrl->step[s->parity];
    return NEST_OK;
}

nest_status nest_solver_reset_time(nest_solver* s) { return nest_solver_set_time(s, 0.0, 0); }

nest_status nest_solver_set_time(nest_solver* s, double time, int steps) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!(time >= 0.0) || steps < 0) return fail(NEST_ERR_INVALID, "time and step count must be non-negative");
    CK(cudaStreamSynchronize(s->st));
    CK(cudaMemcpyAsync(s->host_ctrl, s->ctrl, sizeof(StepCtrl), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int p = 0; p < 2; ++p) { s->host_ctrl->time[p] = time; s->host_ctrl->step[p] = steps; }
    CK(cudaMemcpyAsync(s->ctrl, s->host_ctrl, sizeof(StepCtrl), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return NEST_OK;
}

nest_status nest_solver_totals(nest_solver* s, double out[4]) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!s->partials) return fail(NEST_ERR_UNSUPPORTED, "totals need a 2D solver created with NEST_FLAG_TOTALS");
    cudaError_t e = launch_sum_partials(s->partials, s->nrec, s->totals_dev, s->st);
    if (e != cudaSuccess) return cuda_fail(e, "totals kernel");
    CK(cudaMemcpyAsync(out, s->totals_dev, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int k = 0; k < 4; ++k) out[k] *= s->d.dx * s->d.dy;
    return NEST_OK;
}

nest_status nest_solver_repairs(nest_solver* s, unsigned* count) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if ((r = read_ctrl(s)) != NEST_OK) return r;
    if (count) *count = s->host_ctrl->repairs;
    return NEST_OK;
}

nest_status nest_solver_sync(nest_solver* s) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    return read_ctrl(s);
}

nest_status nest_solver_set_tiling(nest_solver* s, int rows_per_tile, int warps_per_block) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (rows_per_tile < 8 || rows_per_tile > 4096) return fail(NEST_ERR_INVALID, "rows per tile must be in [8, 4096]");
    if (warps_per_block < 1 || warps_per_block > 8) return fail(NEST_ERR_INVALID, "warps per block must be in [1, 8]");
    s->tx = rows_per_tile;
    s->warps = warps_per_block;
    if (s->partials) cudaMemsetAsync(s->partials, 0, sizeof(double) * 4 * s->nrec, s->st);
    return NEST_OK;
}

nest_status nest_solver_set_dt_sequence(nest_solver* s, const double* dts, int n, int mode) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    CK(cudaStreamSynchronize(s->st));
    drop_graphs(s);
    cudaFree(s->dts_in); s->dts_in = nullptr;
    cudaFree(s->dts_out); s->dts_out = nullptr;
    s->dts_cap = 0;
    s->dts_mode = 2;
    if (mode == 2) return NEST_OK;
    if (n <= 0) return fail(NEST_ERR_INVALID, "sequence length must be positive");
    if (mode == 0) {
        if (!dts) return fail(NEST_ERR_INVALID, "null dt sequence");
        CK(cudaMalloc(&s->dts_in, sizeof(double) * n));
        CK(cudaMemcpy(s->dts_in, dts, sizeof(double) * n, cudaMemcpyHostToDevice));
    } else if (mode == 1) {
        CK(cudaMalloc(&s->dts_out, sizeof(double) * n));
        CK(cudaMemset(s->dts_out, 0, sizeof(double) * n));
    } else {
        return fail(NEST_ERR_INVALID, "mode must be 0, 1 or 2");
    }
    s->dts_cap = n;
    s->dts_mode = mode;
    return NEST_OK;
}

nest_status nest_solver_get_dts(nest_solver* s, double* dts, int n) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (s->dts_mode != 1) return fail(NEST_ERR_INVALID, "no dt recording active");
    if (n > s->dts_cap) n = s->dts_cap;
    CK(cudaMemcpyAsync(dts, s->dts_out, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return NEST_OK;
}

nest_status nest_solver_set_exchange_sides(nest_solver* s, int xlo, int xhi) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (s->d.dim != 2) return fail(NEST_ERR_UNSUPPORTED, "halo-exchange sides apply to 2D solvers");
    if (s->d.flags & NEST_FLAG_SPLIT_COMPAT) return fail(NEST_ERR_UNSUPPORTED, "sharding runs the RK2 scheme");
    CK(cudaStreamSynchronize(s->st));
    s->xlo_ex = xlo ? 1 : 0;
    s->xhi_ex = xhi ? 1 : 0;
    s->prepared = false;
    drop_graphs(s);
    return NEST_OK;
}

nest_status nest_solver_stage(nest_solver* s, int which, double cfl, double t_final) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (which != 1 && which != 2) return fail(NEST_ERR_INVALID, "stage must be 1 or 2");
    if (!(cfl > 0.0)) return fail(NEST_ERR_INVALID, "cfl must be positive");
    if (s->resident()) return fail(NEST_ERR_UNSUPPORTED, "single stages use the tiled path (NEST_FLAG_NO_RESIDENT)");
    if (!s->prepared && (r = prepare(s)) != NEST_OK) return r;
    LoopParams lp = base_params(s);
    lp.cfl = cfl;
    lp.t_final = t_final > 0.0 ? t_final : 0.0;
    cudaError_t e = enqueue_step(s, lp, s->parity, which);
    if (e != cudaSuccess) return cuda_fail(e, "stage launch");
    if (which == 2) s->parity ^= 1;
    return NEST_OK;
}

nest_status nest_solver_speed_slot(nest_solver* s, void** dev) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!s->prepared && (r = prepare(s)) != NEST_OK) return r;
    if (dev) *dev = &s->ctrl->maxs[s->parity][0];
    return NEST_OK;
}

nest_status nest_solver_stage_ptr(nest_solver* s, void** dev) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (dev) *dev = s->U1;
    return NEST_OK;
}

nest_status nest_solver_stream(nest_solver* s, void** stream) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (stream) *stream = (void*)s->st;
    return NEST_OK;
}

nest_status nest_solver_state_ptr(nest_solver* s, void** dev, long long* pitch, long long* vstride) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (dev) *dev = s->U;
    if (pitch) *pitch = s->pitch;
    if (vstride) *vstride = s->vstride;
    return NEST_OK;
}

// ===========================================================================
// nest-compatible 1D ABI
// ===========================================================================

struct euler1d_gpu_t {
    nest_solver* s = nullptr;
    nest_status last = NEST_OK;
};

static nest_status note(euler1d_gpu_t* h, nest_status st) {
    if (h) h->last = st;
    return st;
}

euler1d_gpu_t* euler1d_gpu_create(int n_interior, int n_halo, double dx, double gamma) {
    nest_solver_desc d{};
    d.dim = 1; d.nx = n_interior; d.ny = 1; d.halo = n_halo;
    d.dx = dx; d.dy = dx; d.gamma = gamma;
    d.bc_x = NEST_BC_PERIODIC; d.bc_y = NEST_BC_PERIODIC;  // nest's solver is periodic (euler1d_cuda.cuh:337-360)
    d.precision = NEST_F64;
    auto* h = new (std::nothrow) euler1d_gpu_t;
    if (!h) { fail(NEST_ERR_OOM, "host allocation failed"); return nullptr; }
    if (nest_solver_create(&d, &h->s) != NEST_OK) { delete h; return nullptr; }
    return h;
}

void euler1d_gpu_destroy(euler1d_gpu_t* h) {
    if (!h) return;
    nest_solver_destroy(h->s);
    delete h;
}

void euler1d_gpu_upload(euler1d_gpu_t* h, const double* h_data) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return; }
    note(h, nest_solver_upload(h->s, h_data, NEST_LAYOUT_EXTENDED));
}

void euler1d_gpu_download(euler1d_gpu_t* h, double* h_data) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return; }
    note(h, nest_solver_download(h->s, h_data, NEST_LAYOUT_EXTENDED));
}

double euler1d_gpu_compute_dt(euler1d_gpu_t* h, double cfl) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return 0.0; }
    double dt = 0.0;
    note(h, nest_solver_compute_dt(h->s, cfl, &dt));
    return dt;
}

void euler1d_gpu_rk2_step(euler1d_gpu_t* h, double dt) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return; }
    nest_status r = nest_solver_step_dt(h->s, 1, dt);
    if (r == NEST_OK) r = nest_solver_sync(h->s);
    note(h, r);
}

int euler1d_gpu_run(euler1d_gpu_t* h, double t_final, double cfl) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return -1; }
    // nest's run() starts its own clock at 0 on every call (euler1d_solver.cu:159-174).
    nest_status r = nest_solver_reset_time(h->s);
    int steps = 0;
    if (r == NEST_OK) r = nest_solver_run_to(h->s, t_final, cfl, 0, &steps);
    note(h, r);
    return r == NEST_OK ? steps : -1;
}

double euler1d_gpu_run_timed(euler1d_gpu_t* h, double t_final, double cfl, int* steps) {
    if (!h) { fail(NEST_ERR_INVALID, "null solver handle"); return -1.0; }
    nest_solver_sync(h->s);
    auto t0 = std::chrono::high_resolution_clock::now();
    int n = euler1d_gpu_run(h, t_final, cfl);
    auto t1 = std::chrono::high_resolution_clock::now();
    if (steps) *steps = n;
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

nest_status euler1d_gpu_set_bc(euler1d_gpu_t* h, int bc) {
    if (!h) return fail(NEST_ERR_INVALID, "null solver handle");
    if (bc != NEST_BC_PERIODIC && bc != NEST_BC_OUTFLOW) return note(h, fail(NEST_ERR_INVALID, "bad bc"));
    h->s->d.bc_x = bc;
    h->s->prepared = false;
    drop_graphs(h->s);
    return note(h, NEST_OK);
}

nest_status euler1d_gpu_status(euler1d_gpu_t* h) {
    if (!h) return NEST_ERR_INVALID;
    return h->last;
}

}  // extern "C"

// ===========================================================================
// Batched independent 2D problems
// ===========================================================================

struct nest_batch {
    nest_batch_desc d{};
    int count = 0;
    std::vector<BatchProblem> probs;      // host copy
    std::vector<int> first;               // first item of each problem (+ total)
    std::vector<int4> items;
    size_t esize = 4;
    long long total_elems = 0;
    void* U = nullptr;
    void* U1 = nullptr;
    BatchProblem* dprobs = nullptr;
    int4* ditems = nullptr;
    int* dfirst = nullptr;
    StepCtrl* ctrls = nullptr;
    StepCtrl* host_ctrls = nullptr;
    double* partials = nullptr;
    double* totals_dev = nullptr;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int parity = 0;
    bool prepared = false;
    int tx = 32, warps = 2, blocks = 0;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    int strip_w() const { return d.precision == NEST_F64 ? STRIP : 60; }
};

namespace {

nest_status batch_build_items(nest_batch* b) {
    b->items.clear();
    b->first.assign(b->count + 1, 0);
    int sw = b->strip_w();
    for (int p = 0; p < b->count; ++p) {
        const Geo2D& g = b->probs[p].g;
        int nstrips = (g.ny + sw - 1) / sw, ntiles = (g.nx + b->tx - 1) / b->tx;
        b->first[p] = (int)b->items.size();
        b->probs[p].item0 = b->first[p];
        for (int t = 0; t < ntiles; ++t)
            for (int sidx = 0; sidx < nstrips; ++sidx) b->items.push_back(make_int4(p, sidx, t, 0));
    }
    b->first[b->count] = (int)b->items.size();
    cudaFree(b->ditems); b->ditems = nullptr;
    cudaFree(b->dfirst); b->dfirst = nullptr;
    cudaFree(b->partials); b->partials = nullptr;
    CK(cudaMalloc(&b->ditems, sizeof(int4) * b->items.size()));
    CK(cudaMalloc(&b->dfirst, sizeof(int) * (b->count + 1)));
    CK(cudaMemcpy(b->ditems, b->items.data(), sizeof(int4) * b->items.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->dfirst, b->first.data(), sizeof(int) * (b->count + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->dprobs, b->probs.data(), sizeof(BatchProblem) * b->count, cudaMemcpyHostToDevice));
    if (b->d.flags & NEST_FLAG_TOTALS) {
        CK(cudaMalloc(&b->partials, sizeof(double) * 4 * b->items.size()));
        CK(cudaMemset(b->partials, 0, sizeof(double) * 4 * b->items.size()));
    }
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    return NEST_OK;
}

template <typename T>
BatchArgs<T> batch_args(nest_batch* b, const LoopParams& lp, int p) {
    BatchArgs<T> a;
    a.U = (T*)b->U; a.U1 = (T*)b->U1; a.probs = b->dprobs; a.items = b->ditems; a.nitems = (int)b->items.size();
    a.ctrls = b->ctrls; a.partials = b->partials; a.lp = lp; a.p = p; a.tx = b->tx;
    a.nprobs = b->count;
    int ring = 0;
    for (const BatchProblem& q : b->probs) ring = std::max(ring, 4 * (q.g.nx + q.g.ny));
    a.ghost_blocks = std::min(32, (ring + 255) / 256);
    return a;
}

cudaError_t batch_enqueue_step(nest_batch* b, const LoopParams& lp, int p, int which = 3) {
    if (b->d.precision == NEST_F64)
        return launch_batch_f64(batch_args<double>(b, lp, p), which, b->blocks, b->warps, b->st);
    return launch_batch_f32x2(batch_args<float>(b, lp, p), (b->d.flags & NEST_FLAG_REPAIR) != 0, which,
                              b->blocks, b->warps, b->st);
}

nest_status batch_prepare(nest_batch* b) {
    for (int p = 0; p < b->count; ++p) {
        CK(cudaMemsetAsync(&b->ctrls[p].maxs[b->parity][0], 0, 2 * sizeof(unsigned long long), b->st));
        cudaError_t e;
        if (b->d.precision == NEST_F64)
            e = launch_2d_prepare_f64((double*)b->U + b->probs[p].off, b->probs[p].g, b->ctrls + p, b->parity, b->st);
        else
            e = launch_2d_prepare_f32((float*)b->U + b->probs[p].off, b->probs[p].g, b->ctrls + p, b->parity, b->st);
        if (e != cudaSuccess) return cuda_fail(e, "batch prepare");
    }
    b->prepared = true;
    return NEST_OK;
}

nest_status batch_check(const nest_batch* b) {
    if (!b) return fail(NEST_ERR_INVALID, "null batch handle");
    return NEST_OK;
}

}  // namespace

extern "C" {

nest_status nest_batch_create(const nest_batch_desc* d, nest_batch** out) {
    if (!d || !out || !d->nx || !d->ny) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->count <= 0) return fail(NEST_ERR_INVALID, "count must be positive");
    if (d->precision != NEST_F64 && d->precision != NEST_F32) return fail(NEST_ERR_INVALID, "bad precision");
    if (!(d->gamma > 1.0)) return fail(NEST_ERR_INVALID, "gamma must exceed 1");
    if (d->bc_x != NEST_BC_PERIODIC && d->bc_x != NEST_BC_OUTFLOW) return fail(NEST_ERR_INVALID, "bad bc_x");
    if (d->bc_y != NEST_BC_PERIODIC && d->bc_y != NEST_BC_OUTFLOW) return fail(NEST_ERR_INVALID, "bad bc_y");
    if (d->flags & (NEST_FLAG_LIMITER_MC | NEST_FLAG_LIMITER_NONE))
        return fail(NEST_ERR_UNSUPPORTED, "batched problems use the minmod limiter");
    for (int p = 0; p < d->count; ++p)
        if (d->nx[p] < 4 || d->ny[p] < 4) return fail(NEST_ERR_INVALID, "every problem needs >= 4 cells per axis");
    nest_batch* b = new (std::nothrow) nest_batch;
    if (!b) return fail(NEST_ERR_OOM, "host allocation failed");
    b->d = *d;
    b->count = d->count;
    b->esize = d->precision == NEST_F64 ? 8 : 4;
    auto cleanup = [&](nest_status st) { nest_batch_destroy(b); return st; };
    b->probs.resize(b->count);
    long long off = 0;
    int align = (int)(128 / b->esize);
    long long pad = 256 / (long long)b->esize;
    for (int p = 0; p < b->count; ++p) {
        Geo2D g;
        g.nx = d->nx[p]; g.ny = d->ny[p];
        g.pitch = ((g.ny + 4 + align - 1) / align) * align;
        g.vstride = (((long long)g.pitch * (g.nx + 4)) + pad - 1) / pad * pad;
        g.bcx = d->bc_x; g.bcy = d->bc_y;
        g.dx = d->dx ? d->dx[p] : 1.0 / g.nx;
        g.dy = d->dy ? d->dy[p] : 1.0 / g.ny;
        g.gamma = d->gamma;
        g.xlo_ex = 0; g.xhi_ex = 0;
        b->probs[p].g = g;
        b->probs[p].off = off;
        off += 4 * g.vstride;
    }
    b->total_elems = off;
    cudaError_t e;
    if (d->stream) {
        b->st = (cudaStream_t)d->stream;
    } else {
        if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess)
            return cleanup(cuda_fail(e, "cudaStreamCreate"));
        b->own_stream = true;
    }
    size_t bytes = b->esize * (size_t)off;
    if ((e = cudaMalloc(&b->U, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(U)"));
    if ((e = cudaMalloc(&b->U1, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(U1)"));
    if ((e = cudaMemset(b->U, 0, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMemset(b->U1, 0, bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMalloc(&b->dprobs, sizeof(BatchProblem) * b->count)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMalloc(probs)"));
    if ((e = cudaMalloc(&b->ctrls, sizeof(StepCtrl) * b->count)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMalloc(ctrls)"));
    if ((e = cudaMemset(b->ctrls, 0, sizeof(StepCtrl) * b->count)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMallocHost(&b->host_ctrls, sizeof(StepCtrl) * b->count)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMallocHost"));
    if ((e = cudaMalloc(&b->totals_dev, sizeof(double) * 4 * b->count)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMalloc(totals)"));
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = d->precision == NEST_F64 ? batch_max_blocks_f64(b->warps) : batch_max_blocks_f32x2(b->warps);
    b->blocks = sms * (per_sm > 0 ? per_sm : 1);
    nest_status r = batch_build_items(b);
    if (r != NEST_OK) return cleanup(r);
    *out = b;
    return NEST_OK;
}

nest_status nest_batch_destroy(nest_batch* b) {
    if (!b) return NEST_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(b->U); cudaFree(b->U1); cudaFree(b->dprobs); cudaFree(b->ditems); cudaFree(b->dfirst);
    cudaFree(b->ctrls); cudaFree(b->partials); cudaFree(b->totals_dev);
    if (b->host_ctrls) cudaFreeHost(b->host_ctrls);
    if (b->own_stream && b->st) cudaStreamDestroy(b->st);
    delete b;
    return NEST_OK;
}

static nest_status batch_copy(nest_batch* b, int p, void* dst, const void* src, int layout, bool up) {
    if (p < 0 || p >= b->count) return fail(NEST_ERR_INVALID, "problem index out of range");
    if (layout != NEST_LAYOUT_EXTENDED && layout != NEST_LAYOUT_INTERIOR) return fail(NEST_ERR_INVALID, "bad layout");
    const Geo2D& g = b->probs[p].g;
    size_t es = b->esize;
    int rows = layout == NEST_LAYOUT_EXTENDED ? g.nx + 4 : g.nx;
    int cols = layout == NEST_LAYOUT_EXTENDED ? g.ny + 4 : g.ny;
    size_t off = layout == NEST_LAYOUT_EXTENDED ? 0 : (size_t)(2 * g.pitch + 2);
    for (int k = 0; k < 4; ++k) {
        char* dev = (char*)b->U + es * (b->probs[p].off + (size_t)k * g.vstride + off);
        size_t hoff = es * (size_t)k * rows * cols;
        if (up)
            CK(cudaMemcpy2DAsync(dev, es * g.pitch, (const char*)src + hoff, es * cols, es * cols, rows,
                                 cudaMemcpyDefault, b->st));
        else
            CK(cudaMemcpy2DAsync((char*)dst + hoff, es * cols, dev, es * g.pitch, es * cols, rows,
                                 cudaMemcpyDefault, b->st));
    }
    CK(cudaStreamSynchronize(b->st));
    return NEST_OK;
}

nest_status nest_batch_upload(nest_batch* b, int problem, const void* host, int layout) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (!host) return fail(NEST_ERR_INVALID, "null source");
    if (problem < 0 || problem >= b->count) return fail(NEST_ERR_INVALID, "problem index out of range");
    b->prepared = false;
    // a new state starts without an error record
    CK(cudaMemsetAsync(&b->ctrls[problem].err, 0, sizeof(StepCtrl) - offsetof(StepCtrl, err), b->st));
    return batch_copy(b, problem, nullptr, host, layout, true);
}

nest_status nest_batch_download(nest_batch* b, int problem, void* host, int layout) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (!host) return fail(NEST_ERR_INVALID, "null destination");
    return batch_copy(b, problem, host, nullptr, layout, false);
}

nest_status nest_batch_set_tiling(nest_batch* b, int rows_per_tile, int warps_per_block, int blocks_per_sm) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (rows_per_tile < 8 || rows_per_tile > 4096) return fail(NEST_ERR_INVALID, "rows per tile must be in [8, 4096]");
    if (warps_per_block < 1 || warps_per_block > 8) return fail(NEST_ERR_INVALID, "warps per block must be in [1, 8]");
    CK(cudaStreamSynchronize(b->st));
    b->tx = rows_per_tile;
    b->warps = warps_per_block;
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = b->d.precision == NEST_F64 ? batch_max_blocks_f64(b->warps) : batch_max_blocks_f32x2(b->warps);
    if (per_sm < 1) per_sm = 1;
    if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
    b->blocks = sms * per_sm;
    return batch_build_items(b);
}

nest_status nest_batch_step(nest_batch* b, int nsteps, double cfl) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (nsteps < 0 || !(cfl > 0.0)) return fail(NEST_ERR_INVALID, "need nsteps >= 0 and cfl > 0");
    if (!b->prepared && (r = batch_prepare(b)) != NEST_OK) return r;
    LoopParams lp{};
    lp.cfl = cfl;
    while (nsteps > 0) {
        if (nsteps >= GRAPH_STEPS) {
            GraphKey k{GRAPH_STEPS, b->parity, cfl, 0.0, 0.0, 0, nullptr, nullptr, 0, b->tx, b->warps * 1000 + b->blocks};
            auto it = b->graphs.find(k);
            if (it == b->graphs.end()) {
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
                int p = b->parity;
                cudaError_t e = cudaSuccess;
                for (int i = 0; i < GRAPH_STEPS && e == cudaSuccess; ++i, p ^= 1) e = batch_enqueue_step(b, lp, p);
                cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
                if (e != cudaSuccess) {
                    if (e2 == cudaSuccess) cudaGraphDestroy(g);
                    return cuda_fail(e, "batch capture");
                }
                if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
                cudaGraphExec_t ge;
                cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
                it = b->graphs.emplace(k, ge).first;
            }
            CK(cudaGraphLaunch(it->second, b->st));
            nsteps -= GRAPH_STEPS;
        } else {
            cudaError_t e = batch_enqueue_step(b, lp, b->parity);
            if (e != cudaSuccess) return cuda_fail(e, "batch step");
            b->parity ^= 1;
            --nsteps;
        }
    }
    return NEST_OK;
}

nest_status nest_batch_step_profiled(nest_batch* b, int nsteps, double cfl, float* stage_ms, float* total_ms) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (nsteps <= 0 || !(cfl > 0.0)) return fail(NEST_ERR_INVALID, "need nsteps > 0 and cfl > 0");
    if (!b->prepared && (r = batch_prepare(b)) != NEST_OK) return r;
    LoopParams lp{};
    lp.cfl = cfl;
    std::vector<cudaEvent_t> ev(2 * nsteps + 1);
    int made = 0;
    cudaError_t e = cudaSuccess;
    for (; made < (int)ev.size() && e == cudaSuccess; ++made) e = cudaEventCreate(&ev[made]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], b->st);
    for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
        e = batch_enqueue_step(b, lp, b->parity, 1);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 1], b->st);
        if (e == cudaSuccess) e = batch_enqueue_step(b, lp, b->parity, 2);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * i + 2], b->st);
        b->parity ^= 1;
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(ev.back());
    for (int i = 0; i < 2 * nsteps && e == cudaSuccess; ++i) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        if (stage_ms) stage_ms[i] = ms;
    }
    if (e == cudaSuccess && total_ms) e = cudaEventElapsedTime(total_ms, ev[0], ev.back());
    for (int i = 0; i < made; ++i) cudaEventDestroy(ev[i]);
    if (e != cudaSuccess) return cuda_fail(e, "profiled batch steps");
    return NEST_OK;
}

nest_status nest_batch_times(nest_batch* b, double* times, int* steps) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    CK(cudaMemcpyAsync(b->host_ctrls, b->ctrls, sizeof(StepCtrl) * b->count, cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    for (int p = 0; p < b->count; ++p) {
        if (b->host_ctrls[p].err & ERRW_STOP)
            return fail(NEST_ERR_NUMERIC, "problem " + std::to_string(p) + ": " +
                                              ctrl_error_text(b->host_ctrls[p], b->host_ctrls[p].step[b->parity]));
        if (times) times[p] = b->host_ctrls[p].time[b->parity];
        if (steps) steps[p] = b->host_ctrls[p].step[b->parity];
    }
    return NEST_OK;
}

nest_status nest_batch_totals(nest_batch* b, double* out) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    if (!b->partials) return fail(NEST_ERR_UNSUPPORTED, "totals need a batch created with NEST_FLAG_TOTALS");
    cudaError_t e = launch_sum_batch(b->partials, b->dfirst, b->count, b->totals_dev, b->st);
    if (e != cudaSuccess) return cuda_fail(e, "batch totals kernel");
    CK(cudaMemcpyAsync(out, b->totals_dev, sizeof(double) * 4 * b->count, cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    for (int p = 0; p < b->count; ++p)
        for (int k = 0; k < 4; ++k) out[4 * p + k] *= b->probs[p].g.dx * b->probs[p].g.dy;
    return NEST_OK;
}

nest_status nest_batch_reset(nest_batch* b) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    CK(cudaMemsetAsync(b->ctrls, 0, sizeof(StepCtrl) * b->count, b->st));
    CK(cudaStreamSynchronize(b->st));
    b->parity = 0;
    b->prepared = false;
    return NEST_OK;
}

nest_status nest_batch_info(nest_batch* b, long long* cells, int* items, int* blocks) {
    nest_status r = batch_check(b);
    if (r != NEST_OK) return r;
    long long c = 0;
    for (auto& p : b->probs) c += (long long)p.g.nx * p.g.ny;
    if (cells) *cells = c;
    if (items) *items = (int)b->items.size();
    if (blocks) *blocks = b->blocks;
    return NEST_OK;
}

}  // extern "C"
