// Device pipeline executor over nest's per-patch storage.
//
// nest composes a time step from stages run over every patch in order
// (include/nest/pipeline.hpp:14-151): an Exchange stage fills the halos
// (fill_all_halos), a Compute stage maps each patch to a new patch
// (value(patch)), a Reduce stage folds a value over the patches and hands
// it back to each (init / reduce / finalize); execute() runs the stages of a
// pipeline in order.  nest's own examples drive the Euler solver this way
// from host loops over patches (examples/sod1d/sod1d.cpp:219-270).
//
// Here a pipeline is a list of stages, each one kernel launch over all
// patches of the storage an exchange plan describes (nest_exchange_*):
//   EXCHANGE   the plan's halo copies (the nest_exchange kernel),
//   EULER_RHS  compute: dst = src - (dt/dx) (F_{i+1/2} - F_{i-1/2}) on every
//              interior cell, nest's euler_rhs_t (examples/sod1d/
//              euler1d.hpp:279-397) including its one-sided reconstruction
//              at the first and last interior cell of each patch,
//   COPY       compute: dst = src on the interiors,
//   AVERAGE    compute: dst = 0.5 a + 0.5 b on the interiors (sod1d's SSPRK2
//              combine, sod1d.cpp:262-266),
//   CFL_DT     reduce: init 0, reduce the max |u| + c of each patch interior,
//              finalize dt = cfl dx / max, clipped to t_final - time
//              (compute_dt, sod1d.cpp:97-128 and :222-223),
//   CHECK      nest's positivity check every `k` steps (sod1d.cpp:279-301),
//   CLOCK      time += dt, step += 1.
// dt, time and the step count live in a device control block, so a step
// needs no host synchronisation and runs of steps are replayed from CUDA
// graphs.  A CFL_DT stage that finds time >= t_final marks the step
// inactive: the later stages of that execution do nothing.
//
// Compiled with -fmad=false: every formula keeps nest's operation order, so
// results equal nest's CPU code bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <new>
#include <vector>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace {

// One patch of the storage: element offset of its block, interior extents
// and extended extents (1D: n1 = ext1 = 1).
struct PatchInfo {
    long long off;
    int n0, n1, ext0, ext1;
};

// Device control block of a pipeline.
struct PipeCtrl {
    double time, dt, t_final;
    double maxs;          // CFL_DT: reduced max |u| + c (non-negative; bits compare like values)
    int step;
    int active;           // 0: the run is finished, stages after CFL_DT do nothing
    unsigned err;         // ERRW_* bits (CHECK)
    int bad_step, bad_cell, bad_patch;
    double bad_rho, bad_p;
};

__device__ __forceinline__ long long interior_at(const PatchInfo& P, int h, int dim, int v, int a, int b) {
    return P.off + (long long)v * P.ext0 * P.ext1 + (long long)(a + h) * P.ext1 + (dim == 2 ? b + h : 0);
}

// cons_to_prim, euler1d.hpp:69-84.
__device__ __forceinline__ void prim1d(const double* U, long long e, long long plane, double gm1, double& r, double& u,
                                       double& p) {
    r = U[e];
    const double m = U[plane + e];
    u = m / r;
    p = eos_pressure(gm1, r, m, U[2 * plane + e]);
}

// plm_reconstruct, euler1d.hpp:150-171: left and right face states of cell 0.
__device__ __forceinline__ void plm3(const double* Wm, const double* W0, const double* Wp, int lim, double* L,
                                     double* R) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double slope = limit(W0[k] - Wm[k], Wp[k] - W0[k], lim);
        L[k] = W0[k] - 0.5 * slope;
        R[k] = W0[k] + 0.5 * slope;
    }
}

// euler_rhs_t::operator() (euler1d.hpp:297-396) on every interior cell of
// every patch: grid.y = patch, one thread per cell.
__global__ void __launch_bounds__(128) k_pipe_rhs1d(const double* __restrict__ src, double* __restrict__ dst,
                                                     const PatchInfo* P, int h, double dx, double gamma, int lim,
                                                     const PipeCtrl* c) {
    if (!c->active) return;
    const PatchInfo pi = P[blockIdx.y];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pi.n0) return;
    const double gm1 = gamma - 1.0, dt = c->dt;
    const long long plane = pi.ext0, e = pi.off + h + i;
    double W[5][3];  // cells i-2 .. i+2
#pragma unroll
    for (int q = 1; q <= 3; ++q) prim1d(src, e + q - 2, plane, gm1, W[q][0], W[q][1], W[q][2]);
    // one-sided at the patch edges: i-2 -> i-1 on the first cell, i+2 -> i+1 on the last
    if (i >= 1) prim1d(src, e - 2, plane, gm1, W[0][0], W[0][1], W[0][2]);
    else for (int k = 0; k < 3; ++k) W[0][k] = W[1][k];
    if (i < pi.n0 - 1) prim1d(src, e + 2, plane, gm1, W[4][0], W[4][1], W[4][2]);
    else for (int k = 0; k < 3; ++k) W[4][k] = W[3][k];
    double aL[3], aR[3], bL[3], bR[3], cL[3], cR[3];
    plm3(W[0], W[1], W[2], lim, aL, aR);
    plm3(W[1], W[2], W[3], lim, bL, bR);
    plm3(W[2], W[3], W[4], lim, cL, cR);
    double fl[3], fr[3];
    hlle1d(gamma, gm1, aR[0], aR[1], aR[2], bL[0], bL[1], bL[2], fl[0], fl[1], fl[2]);
    hlle1d(gamma, gm1, bR[0], bR[1], bR[2], cL[0], cL[1], cL[2], fr[0], fr[1], fr[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[k * plane + e] = src[k * plane + e] - (dt / dx) * (fr[k] - fl[k]);
}

// dst = src (op 0) or dst = 0.5 a + 0.5 b (op 1) on every interior element.
__global__ void __launch_bounds__(256) k_pipe_interior(double* dst, const double* a, const double* b,
                                                        const PatchInfo* P, int h, int dim, int nvars, int op,
                                                        const PipeCtrl* c) {
    if (!c->active) return;
    const PatchInfo pi = P[blockIdx.y];
    const long long per = (long long)pi.n0 * pi.n1, total = per * nvars;
    for (long long t = blockIdx.x * 256ll + threadIdx.x; t < total; t += (long long)gridDim.x * 256) {
        const int v = (int)(t / per);
        const long long q = t - v * per;
        const int ia = (int)(q / pi.n1), ib = (int)(q - (long long)ia * pi.n1);
        const long long o = interior_at(pi, h, dim, v, ia, ib);
        dst[o] = op == 0 ? a[o] : 0.5 * a[o] + 0.5 * b[o];
    }
}

// CFL reduce: init (slot 0), reduce (one block per patch, atomic max on the
// bit pattern of the non-negative maximum), finalize (one thread).
__global__ void k_pipe_cfl_init(PipeCtrl* c) {
    if (c->t_final > 0.0) c->active = (c->time < c->t_final) && !(c->err & ERRW_STOP) ? 1 : 0;
    else c->active = (c->err & ERRW_STOP) ? 0 : 1;
    c->maxs = 0.0;
}

__global__ void __launch_bounds__(256) k_pipe_cfl_reduce(const double* U, const PatchInfo* P, int h, double gamma,
                                                          PipeCtrl* c) {
    if (!c->active) return;
    const PatchInfo pi = P[blockIdx.x];
    const double gm1 = gamma - 1.0;
    double ms = 0.0;
    for (int i = threadIdx.x; i < pi.n0; i += 256) {
        double r, u, p;
        prim1d(U, pi.off + h + i, pi.ext0, gm1, r, u, p);
        const double cs = sqrt(gamma * p / r);  // eos_t::sound_speed, euler1d.hpp:54-56
        ms = smax(ms, fabs(u) + cs);
    }
    ms = warp_max(ms);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ms;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < 8; ++w) m = smax(m, red[w]);
        atomicMax(reinterpret_cast<unsigned long long*>(&c->maxs), speed_bits(m));
    }
}

__global__ void k_pipe_cfl_finalize(PipeCtrl* c, double cfl, double dx) {
    if (!c->active) return;
    double dt = cfl * dx / c->maxs;
    if (c->t_final > 0.0) dt = smin(dt, c->t_final - c->time);
    c->dt = dt;
}

// nest's positivity check (sod1d.cpp:279-301) on the interiors, when the
// completed step count is a multiple of `every`.
__global__ void __launch_bounds__(256) k_pipe_check(const double* U, const PatchInfo* P, int h, double gamma,
                                                     int every, PipeCtrl* c) {
    if (!c->active || (c->step + 1) % every != 0) return;
    const PatchInfo pi = P[blockIdx.x];
    const double gm1 = gamma - 1.0;
    for (int i = threadIdx.x; i < pi.n0; i += 256) {
        double r, u, p;
        prim1d(U, pi.off + h + i, pi.ext0, gm1, r, u, p);
        if (!(r > 0.0) || !(p > 0.0)) {
            const unsigned bit = (r == r && p == p) ? ERRW_NONPOSITIVE : ERRW_NONFINITE;
            if (!(atomicOr(&c->err, bit) & ERRW_STOP)) {
                c->bad_step = c->step + 1; c->bad_cell = i; c->bad_patch = blockIdx.x;
                c->bad_rho = r; c->bad_p = p;
            }
        }
    }
}

__global__ void k_pipe_clock(PipeCtrl* c) {
    if (!c->active) return;
    c->time = c->time + c->dt;
    c->step = c->step + 1;
}

struct Stage {
    int kind, src, dst, aux;
    double param;
};

}  // namespace

struct nest_pipeline {
    nest_exchange* plan = nullptr;
    int dim = 1, nvars = 3, halo = 2, npatch = 0, nwork = 0, lim = LIM_MINMOD;
    double dx = 1.0, gamma = 1.4;
    long long total = 0;              // elements of one storage block (all patches)
    int max_n0 = 0;
    std::vector<PatchInfo> patches;
    PatchInfo* dpatches = nullptr;
    std::vector<double*> work;        // pipeline-owned buffers 1..nwork
    PipeCtrl* ctrl = nullptr;
    PipeCtrl* host_ctrl = nullptr;
    std::vector<Stage> stages;
    cudaStream_t own = nullptr;
    std::map<std::pair<void*, cudaStream_t>, cudaGraphExec_t> graphs;
};

namespace {

constexpr int PIPE_GRAPH_STEPS = 8;

void drop_pipe_graphs(nest_pipeline* p) {
    for (auto& kv : p->graphs) cudaGraphExecDestroy(kv.second);
    p->graphs.clear();
}

double* buffer(nest_pipeline* p, void* state, int b) { return b == 0 ? (double*)state : p->work[b - 1]; }

cudaError_t launch_stage(nest_pipeline* p, const Stage& s, void* state, cudaStream_t st) {
    double* src = buffer(p, state, s.src);
    const int h = p->halo;
    switch (s.kind) {
        case NEST_STAGE_EXCHANGE: {
            nest_status r = nest_exchange_execute(p->plan, src, NEST_F64, st);
            return r == NEST_OK ? cudaSuccess : cudaErrorLaunchFailure;
        }
        case NEST_STAGE_EULER_RHS: {
            dim3 gr((p->max_n0 + 127) / 128, p->npatch);
            k_pipe_rhs1d<<<gr, 128, 0, st>>>(src, buffer(p, state, s.dst), p->dpatches, h, p->dx, p->gamma, p->lim,
                                             p->ctrl);
            break;
        }
        case NEST_STAGE_COPY:
        case NEST_STAGE_AVERAGE: {
            long long per = 0;
            for (auto& q : p->patches) per = std::max(per, (long long)q.n0 * q.n1 * p->nvars);
            dim3 gr((unsigned)std::min<long long>((per + 255) / 256, 64), p->npatch);
            k_pipe_interior<<<gr, 256, 0, st>>>(buffer(p, state, s.dst), src,
                                                s.kind == NEST_STAGE_AVERAGE ? buffer(p, state, s.aux) : nullptr,
                                                p->dpatches, h, p->dim, p->nvars,
                                                s.kind == NEST_STAGE_AVERAGE ? 1 : 0, p->ctrl);
            break;
        }
        case NEST_STAGE_CFL_DT:
            k_pipe_cfl_init<<<1, 1, 0, st>>>(p->ctrl);
            k_pipe_cfl_reduce<<<p->npatch, 256, 0, st>>>(src, p->dpatches, h, p->gamma, p->ctrl);
            k_pipe_cfl_finalize<<<1, 1, 0, st>>>(p->ctrl, s.param, p->dx);
            break;
        case NEST_STAGE_CHECK:
            k_pipe_check<<<p->npatch, 256, 0, st>>>(src, p->dpatches, h, p->gamma, (int)s.param, p->ctrl);
            break;
        case NEST_STAGE_CLOCK:
            k_pipe_clock<<<1, 1, 0, st>>>(p->ctrl);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_all(nest_pipeline* p, void* state, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    for (const Stage& s : p->stages)
        if ((e = launch_stage(p, s, state, st)) != cudaSuccess) break;
    return e;
}

nest_status read_pipe_ctrl(nest_pipeline* p, cudaStream_t st) {
    CK(cudaMemcpyAsync(p->host_ctrl, p->ctrl, sizeof(PipeCtrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const PipeCtrl& c = *p->host_ctrl;
    if (c.err & ERRW_STOP) {
        char buf[256];
        const bool nan = !(c.bad_rho == c.bad_rho) || !(c.bad_p == c.bad_p);
        std::snprintf(buf, sizeof buf, "%s at step %d in patch %d, interior cell %d: rho = %.17g, p = %.17g",
                      nan ? "non-finite state (NaN)" : "positivity violation (rho <= 0 or p <= 0)", c.bad_step,
                      c.bad_patch, c.bad_cell, c.bad_rho, c.bad_p);
        return fail(NEST_ERR_NUMERIC, buf);
    }
    return NEST_OK;
}

nest_status pcheck(const nest_pipeline* p) {
    if (!p) return fail(NEST_ERR_INVALID, "null pipeline handle");
    return NEST_OK;
}

}  // namespace

extern "C" {

nest_status nest_pipeline_create(int dim, int nx, int ny, int npx, int npy, int halo, double dx, double gamma,
                                 int limiter, int nwork, nest_pipeline** out) {
    if (!out) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (dim != 1 && dim != 2) return fail(NEST_ERR_INVALID, "dim must be 1 or 2");
    if (!(dx > 0.0) || !(gamma > 1.0)) return fail(NEST_ERR_INVALID, "dx must be positive and gamma > 1");
    if (nwork < 0 || nwork > 16) return fail(NEST_ERR_INVALID, "work buffers must be 0..16");
    if (limiter != LIM_MINMOD && limiter != LIM_MC && limiter != LIM_NONE) return fail(NEST_ERR_INVALID, "bad limiter");
    auto* p = new (std::nothrow) nest_pipeline;
    if (!p) return fail(NEST_ERR_OOM, "host allocation failed");
    p->dim = dim; p->nvars = dim == 1 ? 3 : 4; p->halo = halo; p->dx = dx; p->gamma = gamma; p->lim = limiter;
    p->nwork = nwork;
    auto cleanup = [&](nest_status st) { nest_pipeline_destroy(p); return st; };
    nest_status r = nest_exchange_create_periodic(dim, nx, ny, npx, npy, p->nvars, halo, &p->plan);
    if (r != NEST_OK) return cleanup(r);
    p->npatch = dim == 2 ? npx * npy : npx;
    std::vector<long long> offs(p->npatch + 1);
    std::vector<int> boxes(4 * p->npatch);
    nest_exchange_layout(p->plan, offs.data(), boxes.data(), nullptr);
    p->total = offs[p->npatch];
    for (int q = 0; q < p->npatch; ++q) {
        PatchInfo pi;
        pi.off = offs[q];
        pi.n0 = boxes[4 * q + 2];
        pi.n1 = dim == 2 ? boxes[4 * q + 3] : 1;
        pi.ext0 = pi.n0 + 2 * halo;
        pi.ext1 = dim == 2 ? pi.n1 + 2 * halo : 1;
        p->patches.push_back(pi);
        p->max_n0 = std::max(p->max_n0, pi.n0);
    }
    cudaError_t e;
    if ((e = cudaMalloc(&p->dpatches, sizeof(PatchInfo) * p->npatch)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc"));
    if ((e = cudaMemcpy(p->dpatches, p->patches.data(), sizeof(PatchInfo) * p->npatch, cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMemcpy"));
    for (int w = 0; w < nwork; ++w) {
        double* b = nullptr;
        if ((e = cudaMalloc(&b, sizeof(double) * p->total)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(work)"));
        p->work.push_back(b);
        if ((e = cudaMemset(b, 0, sizeof(double) * p->total)) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    }
    if ((e = cudaMalloc(&p->ctrl, sizeof(PipeCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(ctrl)"));
    if ((e = cudaMemset(p->ctrl, 0, sizeof(PipeCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if ((e = cudaMallocHost(&p->host_ctrl, sizeof(PipeCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMallocHost"));
    if ((e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaStreamCreate"));
    // a step that starts active until a CFL stage says otherwise
    PipeCtrl c{};
    c.active = 1;
    if ((e = cudaMemcpy(p->ctrl, &c, sizeof c, cudaMemcpyHostToDevice)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMemcpy"));
    *out = p;
    return NEST_OK;
}

nest_status nest_pipeline_destroy(nest_pipeline* p) {
    if (!p) return NEST_OK;
    if (p->own) cudaStreamSynchronize(p->own);
    drop_pipe_graphs(p);
    for (double* b : p->work) cudaFree(b);
    cudaFree(p->dpatches);
    cudaFree(p->ctrl);
    if (p->host_ctrl) cudaFreeHost(p->host_ctrl);
    if (p->own) cudaStreamDestroy(p->own);
    nest_exchange_destroy(p->plan);
    delete p;
    return NEST_OK;
}

nest_status nest_pipeline_plan(nest_pipeline* p, nest_exchange** plan) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    if (plan) *plan = p->plan;
    return NEST_OK;
}

nest_status nest_pipeline_add(nest_pipeline* p, int kind, int src, int dst, int aux, double param) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    auto bad = [&](int b) { return b < 0 || b > p->nwork; };
    if (kind < NEST_STAGE_EXCHANGE || kind > NEST_STAGE_CLOCK) return fail(NEST_ERR_INVALID, "unknown stage kind");
    if (bad(src) || bad(dst) || bad(aux)) return fail(NEST_ERR_INVALID, "buffer index out of range");
    if ((kind == NEST_STAGE_EULER_RHS || kind == NEST_STAGE_CFL_DT || kind == NEST_STAGE_CHECK) && p->dim != 1)
        return fail(NEST_ERR_UNSUPPORTED, "Euler, CFL and positivity stages run nest's 1D patch scheme");
    if (kind == NEST_STAGE_EULER_RHS && src == dst) return fail(NEST_ERR_INVALID, "EULER_RHS needs dst != src");
    if (kind == NEST_STAGE_CFL_DT && !(param > 0.0)) return fail(NEST_ERR_INVALID, "CFL_DT needs cfl > 0");
    if (kind == NEST_STAGE_CHECK && !(param >= 1.0)) return fail(NEST_ERR_INVALID, "CHECK needs a period >= 1");
    p->stages.push_back(Stage{kind, src, dst, aux, param});
    drop_pipe_graphs(p);
    return NEST_OK;
}

nest_status nest_pipeline_execute(nest_pipeline* p, void* d_state, void* stream) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    if (!d_state) return fail(NEST_ERR_INVALID, "null state");
    cudaStream_t st = stream ? (cudaStream_t)stream : p->own;
    cudaError_t e = launch_all(p, d_state, st);
    if (e != cudaSuccess) return cuda_fail(e, "pipeline stage launch");
    return NEST_OK;
}

nest_status nest_pipeline_run(nest_pipeline* p, void* d_state, double t_final, int max_steps, int* steps_out,
                              void* stream) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    if (!d_state || !(t_final > 0.0)) return fail(NEST_ERR_INVALID, "need a state and t_final > 0");
    bool has_cfl = false;
    for (auto& s : p->stages) has_cfl |= s.kind == NEST_STAGE_CFL_DT;
    if (!has_cfl) return fail(NEST_ERR_INVALID, "run needs a CFL_DT stage (it decides when to stop)");
    cudaStream_t st = stream ? (cudaStream_t)stream : p->own;
    if ((r = read_pipe_ctrl(p, st)) != NEST_OK) return r;
    const int start = p->host_ctrl->step;
    // t_final into the control block (the CFL stages read it)
    CK(cudaMemcpyAsync(&p->ctrl->t_final, &t_final, sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    auto key = std::make_pair(d_state, st);
    auto it = p->graphs.find(key);
    if (it == p->graphs.end()) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < PIPE_GRAPH_STEPS && e == cudaSuccess; ++k) e = launch_all(p, d_state, st);
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) {
            if (e2 == cudaSuccess) cudaGraphDestroy(g);
            return cuda_fail(e, "pipeline capture");
        }
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
        cudaGraphExec_t ge;
        cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
        it = p->graphs.emplace(key, ge).first;
    }
    int last = -1;
    for (;;) {
        CK(cudaGraphLaunch(it->second, st));
        if ((r = read_pipe_ctrl(p, st)) != NEST_OK) break;
        const PipeCtrl& c = *p->host_ctrl;
        if (!(c.time < t_final) || !c.active) break;
        if (max_steps > 0 && c.step - start >= max_steps) break;
        if (c.step == last) { r = fail(NEST_ERR_NUMERIC, "time stopped advancing"); break; }
        last = c.step;
    }
    // later execute() calls run without a stopping time
    cudaStreamSynchronize(st);
    const double zero = 0.0;
    const int one = 1;
    cudaMemcpy(&p->ctrl->t_final, &zero, sizeof zero, cudaMemcpyHostToDevice);
    cudaMemcpy(&p->ctrl->active, &one, sizeof one, cudaMemcpyHostToDevice);
    if (steps_out) *steps_out = p->host_ctrl->step - start;
    return r;
}

nest_status nest_pipeline_clock(nest_pipeline* p, double* time, double* dt, int* step) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    if ((r = read_pipe_ctrl(p, p->own)) != NEST_OK) return r;
    if (time) *time = p->host_ctrl->time;
    if (dt) *dt = p->host_ctrl->dt;
    if (step) *step = p->host_ctrl->step;
    return NEST_OK;
}

nest_status nest_pipeline_set_clock(nest_pipeline* p, double time, double dt, int step) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    CK(cudaStreamSynchronize(p->own));
    PipeCtrl c{};
    c.time = time; c.dt = dt; c.step = step; c.active = 1;
    CK(cudaMemcpy(p->ctrl, &c, sizeof c, cudaMemcpyHostToDevice));
    return NEST_OK;
}

nest_status nest_pipeline_buffer(nest_pipeline* p, int index, void** dev) {
    nest_status r = pcheck(p);
    if (r != NEST_OK) return r;
    if (index < 1 || index > p->nwork) return fail(NEST_ERR_INVALID, "work buffer index out of range");
    if (dev) *dev = p->work[index - 1];
    return NEST_OK;
}

}  // extern "C"
