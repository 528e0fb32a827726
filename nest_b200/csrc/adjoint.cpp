// Checkpointed discrete adjoint of a solver's time loop (C++ host runtime).
//
// The forward sweep runs the solver's own step path with CFL dt and records
// the dt sequence; the adjoint then uses that frozen sequence.  Memory is
// bounded by checkpoint-and-recompute:
//   NEST_CKPT_UNIFORM  (param K): the forward sweep stores U every K steps;
//      each segment is recomputed once, storing its K states (and the stage
//      states U1), then reversed.  Cost: two forward sweeps.
//   NEST_CKPT_BINOMIAL (param s): s snapshot slots, schedule by the binomial
//      recursion of Griewank & Walther ("revolve", ACM TOMS 26(1), 2000):
//      with beta(s, r) = C(s + r, s), a range of t <= beta(s, r) steps is
//      split at d = beta(s, r - 1) from its start; the right part is reversed
//      first with s - 1 free slots, then the left part with s.  A slot cache
//      lets the recursion reuse the snapshots the forward sweep took along
//      the rightmost spine.
// Per reversed step: one stage-1 recompute of U1 from U^n, then
//   tmp      = 1/2 * S'(U1)^T lambda^{n+1}
//   lambda^n = S'(U^n)^T tmp + 1/2 lambda^{n+1}
// (Heun: U^{n+1} = 1/2 (U^n + S(S(U^n)))).
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <memory>
#include <new>
#include <vector>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace nestb {
// Both reverse stages of one Heun step in one launch (the intermediate adjoint
// stays in shared memory).
cudaError_t launch_1d_adjoint_step(const double* Un, const double* U1, const double* lam, double* lam_new, int n,
                                   int h, const double* dtp, double dx, double gamma, cudaStream_t st);
cudaError_t launch_1d_adjoint_step_f32(const float* Un, const float* U1, const float* lam, float* lam_new, int n,
                                       int h, const double* dtp, double dx, double gamma, cudaStream_t st);
}

namespace {

// Device operations the schedules need, for one solver form.  Stage
// launches take explicit loop parameters and parity (so a captured segment can
// read its dts from device memory); adjoint steps read dt through a device
// pointer.
struct Stepper {
    virtual ~Stepper() = default;
    // which = 1: U1 <- S(Un); which = 2: Uout <- (Un + S(U1)) / 2 after stage 1;
    // which = 3: both (Uout distinct from Un)
    virtual cudaError_t stage(int which, void* Un, void* U1, void* Uout, const LoopParams& lp, int p) = 0;
    virtual cudaError_t adjoint_step(void* Un, void* U1, const double* dtp, void* lam, void* lam_new, void* tmp) = 0;
};

LoopParams fixed(double dt) {
    LoopParams p{};
    p.cfl = 1.0;
    p.fixed_dt = dt;
    return p;
}

struct Stepper1D : Stepper {
    nest_solver* s;
    StepCtrl* ctrl;
    explicit Stepper1D(nest_solver* s_, StepCtrl* c) : s(s_), ctrl(c) {}
    cudaError_t stage(int which, void* Un, void* U1, void* Uout, const LoopParams& lp, int p) override {
        if (which == 3 && Uout && Uout != Un) {  // one launch, U1 of the step kept in U1
            if (s->d.precision == NEST_F32)
                return launch_1d_fused_f32((const float*)Un, (float*)Uout, (float*)U1, s->d.nx, s->h, s->d.dx,
                                           s->d.gamma, s->d.bc_x, lp, ctrl, p, s->st);
            return launch_1d_fused((const double*)Un, (double*)Uout, (double*)U1, s->d.nx, s->h, s->d.dx,
                                   s->d.gamma, s->d.bc_x, lp, ctrl, p, s->st);
        }
        if (s->d.precision == NEST_F32)
            return launch_1d_step_f32((float*)Un, (float*)U1, s->d.nx, s->h, s->d.dx, s->d.gamma, s->d.bc_x, lp, ctrl,
                                      p, which, s->st, (float*)Uout);
        return launch_1d_step((double*)Un, (double*)U1, s->d.nx, s->h, s->d.dx, s->d.gamma, s->d.bc_x, lp, ctrl, p,
                              which, s->st, (double*)Uout);
    }
    cudaError_t adjoint_step(void* Un, void* U1, const double* dtp, void* lam, void* lam_new, void*) override {
        const int n = s->d.nx, h = s->h;
        if (s->d.precision == NEST_F32)
            return launch_1d_adjoint_step_f32((const float*)Un, (const float*)U1, (const float*)lam, (float*)lam_new,
                                              n, h, dtp, s->d.dx, s->d.gamma, s->st);
        return launch_1d_adjoint_step((const double*)Un, (const double*)U1, (const double*)lam, (double*)lam_new, n,
                                      h, dtp, s->d.dx, s->d.gamma, s->st);
    }
};

// 2D solver (FP64 plain form or FP32 form): the stage kernels are the
// solver's own; the FP32 form's state is advanced by the packed kernel.
struct Stepper2D : Stepper {
    nest_solver* s;
    StepCtrl* ctrl;
    // NEST_ADJOINT2D_TILE=1 in the environment when the adjoint is created
    // selects the tile kernels instead of the row marches (a diagnostic: both
    // forms can then be compared on one trajectory)
    bool tile = false;
    Stepper2D(nest_solver* s_, StepCtrl* c) : s(s_), ctrl(c) {
        const char* e = std::getenv("NEST_ADJOINT2D_TILE");
        tile = e && e[0] == '1';
    }
    cudaError_t stage(int which, void* Un, void* U1, void* Uout, const LoopParams& lp, int p) override {
        if (s->d.precision == NEST_F64)
            return launch_2d_step_f64((double*)Un, (double*)U1, s->geo(), lp, ctrl, nullptr, p, s->tx, s->warps, which,
                                      s->st, (double*)Uout);
        return launch_2d_step_f32x2((float*)Un, (float*)U1, s->geo(), lp, ctrl, nullptr, p, s->tx, s->warps,
                                    (s->d.flags & NEST_FLAG_REPAIR) != 0, which, s->st, (float*)Uout);
    }
    cudaError_t adjoint_step(void* Un, void* U1, const double* dtp, void* lam, void* lam_new, void* tmp) override {
        cudaError_t e;
        if (s->d.precision == NEST_F64) {
            auto st64 = [&](const double* U, const double* Lo, const double* Ex, double* Li, double al, double be) {
                return tile ? launch_2d_adjoint_stage_f64(U, Lo, Ex, Li, s->geo(), dtp, al, be, s->st)
                            : launch_2d_adjoint_stage_f64rm(U, Lo, Ex, Li, s->geo(), dtp, al, be, s->st);
            };
            e = st64((const double*)U1, (const double*)lam, nullptr, (double*)tmp, 0.5, 0.0);
            if (e == cudaSuccess)
                e = st64((const double*)Un, (const double*)tmp, (const double*)lam, (double*)lam_new, 1.0, 0.5);
        } else {
            // packed row march; the tile kernel for an odd ny, which the packed
            // kernel does not take
            auto st32 = [&](const float* U, const float* Lo, const float* Ex, float* Li, double al, double be) {
                cudaError_t r = cudaErrorNotSupported;
                if (!tile) r = launch_2d_adjoint_stage_f32x2(U, Lo, Ex, Li, s->geo(), dtp, al, be, s->st);
                if (r == cudaErrorNotSupported)
                    r = launch_2d_adjoint_stage_f32(U, Lo, Ex, Li, s->geo(), dtp, al, be, s->st);
                return r;
            };
            e = st32((const float*)U1, (const float*)lam, nullptr, (float*)tmp, 0.5, 0.0);
            if (e == cudaSuccess)
                e = st32((const float*)Un, (const float*)tmp, (const float*)lam, (float*)lam_new, 1.0, 0.5);
        }
        return e;
    }
};

long long binom(int n, int k) {  // C(n, k), saturating
    if (k < 0 || k > n) return 0;
    long double r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r > 9.0e18L ? (long long)9.0e18 : (long long)(r + 0.5L);
}

}  // namespace

struct nest_adjoint {
    nest_solver* s = nullptr;
    int nsteps = 0, policy = 0, param = 0;
    std::unique_ptr<Stepper> stepper;
    StepCtrl* ctrl = nullptr;
    std::vector<double> dts;
    std::vector<void*> slots;      // snapshot slots (binomial) or checkpoints (uniform)
    std::vector<int> slot_pos;     // step index held by each slot (-1: none)
    std::vector<void*> seg_un, seg_u1;  // uniform: states of one segment
    void* work = nullptr;
    void* u1 = nullptr;
    void* lam[2] = {nullptr, nullptr};
    void* tmp = nullptr;
    double* d_dts = nullptr;       // all dts (device), for the adjoint kernels of the binomial schedule
    double* seg_dts = nullptr;     // dts of the current segment (device), uniform schedule
    double* h_seg_dts = nullptr;   // pinned staging for seg_dts
    std::map<int, cudaGraphExec_t> seg_graphs;  // uniform: one graph per segment length
    bool forward_done = false;
    double fwd_ms = 0.0, bwd_ms = 0.0;
    long long advanced = 0;        // forward steps run by the backward sweep (recompute)
    long long snap_bytes = 0;
};

namespace {

nest_status adj_alloc(nest_adjoint* a, void** p) {
    CK(cudaMalloc(p, a->s->state_bytes()));
    CK(cudaMemsetAsync(*p, 0, a->s->state_bytes(), a->s->st));
    a->snap_bytes += (long long)a->s->state_bytes();
    return NEST_OK;
}

nest_status copy_state_dev(nest_adjoint* a, void* dst, const void* src) {
    CK(cudaMemcpyAsync(dst, src, a->s->state_bytes(), cudaMemcpyDeviceToDevice, a->s->st));
    return NEST_OK;
}

// Advance the state of step j0 held in `src` by k >= 1 steps into `dst`
// without copying it first: the first step reads `src` (left unchanged), the
// steps between run in place in `work`, the last step writes `dst` (which may
// be `work`) out of place.
nest_status advance_from(nest_adjoint* a, void* src, void* dst, int j0, int k) {
    void* in = src;
    for (int s = 0; s < k; ++s) {
        const int j = j0 + s;
        void* out = (s == k - 1) ? dst : a->work;
        cudaError_t e = a->stepper->stage(1, in, a->u1, nullptr, fixed(a->dts[j]), 0);
        if (e == cudaSuccess) e = a->stepper->stage(2, in, a->u1, out == in ? nullptr : out, fixed(a->dts[j]), 0);
        if (e != cudaSuccess) return cuda_fail(e, "recompute step");
        ++a->advanced;
        in = out;
    }
    return NEST_OK;
}

// lambda <- adjoint of step j applied to lambda, given U^n of step j in `un`.
nest_status reverse_one(nest_adjoint* a, void* un, int j, int& cur) {
    cudaError_t e = a->stepper->stage(1, un, a->u1, nullptr, fixed(a->dts[j]), 0);
    if (e == cudaSuccess) e = a->stepper->adjoint_step(un, a->u1, a->d_dts + j, a->lam[cur], a->lam[cur ^ 1], a->tmp);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint step");
    cur ^= 1;
    return NEST_OK;
}

// Binomial reversal of steps [l, r); the state at l is in slot k; slots
// k+1 .. k+free are available.
nest_status reverse_binomial(nest_adjoint* a, int l, int r, int k, int free, int& cur) {
    nest_status st;
    int t = r - l;
    if (t == 1) return reverse_one(a, a->slots[k], l, cur);
    if (free == 0) {
        for (int j = r - 1; j > l; --j) {
            if ((st = advance_from(a, a->slots[k], a->work, l, j - l)) != NEST_OK) return st;
            if ((st = reverse_one(a, a->work, j, cur)) != NEST_OK) return st;
        }
        return reverse_one(a, a->slots[k], l, cur);
    }
    int rep = 1;
    while (binom(free + rep, free) < t) ++rep;
    long long d = binom(free + rep - 1, free);  // beta(free, rep - 1)
    d = std::max<long long>(1, std::min<long long>(d, t - 1));
    int m = l + (int)d;
    if (a->slot_pos[k + 1] != m) {
        if ((st = advance_from(a, a->slots[k], a->slots[k + 1], l, m - l)) != NEST_OK) return st;
        a->slot_pos[k + 1] = m;
    }
    if ((st = reverse_binomial(a, m, r, k + 1, free - 1, cur)) != NEST_OK) return st;
    a->slot_pos[k + 1] = -1;
    return reverse_binomial(a, l, m, k, free, cur);
}

// Uniform schedule, one segment of L steps starting from seg_un[0]:
// recompute (each step out of place into seg_un[r+1] with its U1 kept in
// seg_u1[r] -- one launch in 1D -- and U1 alone for the last step; dts read
// from seg_dts by step count) then reverse, lambda entering in lam[0] and
// leaving in lam[0].  Captured once per L and replayed.
nest_status segment_graph(nest_adjoint* a, int L, cudaGraphExec_t* out) {
    auto it = a->seg_graphs.find(L);
    if (it != a->seg_graphs.end()) { *out = it->second; return NEST_OK; }
    cudaStream_t st = a->s->st;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(a->ctrl, 0, sizeof(StepCtrl), st);
    LoopParams lp{};
    lp.cfl = 1.0;
    lp.dts_in = a->seg_dts;
    lp.dts_cap = L;
    for (int r = 0; r < L && e == cudaSuccess; ++r) {
        if (r + 1 < L) e = a->stepper->stage(3, a->seg_un[r], a->seg_u1[r], a->seg_un[r + 1], lp, r & 1);
        else e = a->stepper->stage(1, a->seg_un[r], a->seg_u1[r], nullptr, lp, r & 1);
    }
    int cur = 0;
    for (int r = L - 1; r >= 0 && e == cudaSuccess; --r, cur ^= 1)
        e = a->stepper->adjoint_step(a->seg_un[r], a->seg_u1[r], a->seg_dts + r, a->lam[cur], a->lam[cur ^ 1], a->tmp);
    if (e == cudaSuccess && cur == 1)
        e = cudaMemcpyAsync(a->lam[0], a->lam[1], a->s->state_bytes(), cudaMemcpyDeviceToDevice, st);
    cudaGraph_t g;
    cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) {
        if (e2 == cudaSuccess) cudaGraphDestroy(g);
        return cuda_fail(e, "segment capture");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
    cudaGraphExec_t ge;
    cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
    a->seg_graphs[L] = ge;
    *out = ge;
    return NEST_OK;
}

// Steps at which the forward sweep stores snapshots: uniform multiples of K,
// or the rightmost spine of the binomial recursion.
std::vector<std::pair<int, int>> forward_snapshots(const nest_adjoint* a) {
    std::vector<std::pair<int, int>> v;  // (step, slot)
    if (a->policy == NEST_CKPT_UNIFORM) {
        for (int j = 0, k = 0; j < a->nsteps; j += a->param, ++k) v.push_back({j, k});
        return v;
    }
    int l = 0, r = a->nsteps, k = 0, free = a->param - 1;
    v.push_back({0, 0});
    while (r - l > 1 && free > 0) {
        int t = r - l, rep = 1;
        while (binom(free + rep, free) < t) ++rep;
        long long d = std::max<long long>(1, std::min<long long>(binom(free + rep - 1, free), t - 1));
        l += (int)d;
        ++k;
        --free;
        v.push_back({l, k});
    }
    return v;
}

}  // namespace

extern "C" {

nest_status nest_adjoint_create(nest_solver* s, int nsteps, int policy, int param, nest_adjoint** out) {
    if (!s || !out) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (nsteps <= 0) return fail(NEST_ERR_INVALID, "nsteps must be positive");
    if (policy != NEST_CKPT_UNIFORM && policy != NEST_CKPT_BINOMIAL) return fail(NEST_ERR_INVALID, "bad policy");
    if (param < 1) return fail(NEST_ERR_INVALID, "checkpoint parameter must be >= 1");
    if (s->d.bc_x != NEST_BC_PERIODIC || (s->d.dim == 2 && s->d.bc_y != NEST_BC_PERIODIC))
        return fail(NEST_ERR_UNSUPPORTED, "adjoint: periodic boundaries");
    if (s->d.flags & (NEST_FLAG_SPLIT_COMPAT | NEST_FLAG_FP32_SCALAR))
        return fail(NEST_ERR_UNSUPPORTED, "adjoint: unsplit RK2 scheme only");
    if (s->d.flags & (NEST_FLAG_LIMITER_MC | NEST_FLAG_LIMITER_NONE))
        return fail(NEST_ERR_UNSUPPORTED, "adjoint: minmod limiter only");
    auto* a = new (std::nothrow) nest_adjoint;
    if (!a) return fail(NEST_ERR_OOM, "host allocation failed");
    a->s = s;
    a->nsteps = nsteps;
    a->policy = policy;
    a->param = policy == NEST_CKPT_UNIFORM ? std::min(param, nsteps) : std::min(param, nsteps);
    auto cleanup = [&](nest_status st) { nest_adjoint_destroy(a); return st; };
    cudaError_t e = cudaMalloc(&a->ctrl, sizeof(StepCtrl));
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(ctrl)"));
    if ((e = cudaMemset(a->ctrl, 0, sizeof(StepCtrl))) != cudaSuccess) return cleanup(cuda_fail(e, "memset"));
    if (s->d.dim == 1) a->stepper.reset(new Stepper1D(s, a->ctrl));
    else a->stepper.reset(new Stepper2D(s, a->ctrl));
    nest_status st;
    int nslots = policy == NEST_CKPT_UNIFORM ? (nsteps + a->param - 1) / a->param : a->param;
    a->slots.assign(nslots, nullptr);
    a->slot_pos.assign(nslots + 1, -1);
    for (auto& p : a->slots)
        if ((st = adj_alloc(a, &p)) != NEST_OK) return cleanup(st);
    if (policy == NEST_CKPT_UNIFORM) {
        a->seg_un.assign(a->param, nullptr);
        a->seg_u1.assign(a->param, nullptr);
        for (int i = 0; i < a->param; ++i) {
            if ((st = adj_alloc(a, &a->seg_un[i])) != NEST_OK) return cleanup(st);
            if ((st = adj_alloc(a, &a->seg_u1[i])) != NEST_OK) return cleanup(st);
        }
    }
    for (void** p : {&a->work, &a->u1, &a->lam[0], &a->lam[1], &a->tmp})
        if ((st = adj_alloc(a, p)) != NEST_OK) return cleanup(st);
    if ((e = cudaMalloc(&a->d_dts, sizeof(double) * nsteps)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(dts)"));
    if ((e = cudaMalloc(&a->seg_dts, sizeof(double) * a->param)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMalloc(seg dts)"));
    if ((e = cudaMallocHost(&a->h_seg_dts, sizeof(double) * a->param)) != cudaSuccess)
        return cleanup(cuda_fail(e, "cudaMallocHost"));
    *out = a;
    return NEST_OK;
}

nest_status nest_adjoint_destroy(nest_adjoint* a) {
    // Does not touch the solver (it may already be destroyed); cudaFree waits
    // for outstanding work on these buffers.
    if (!a) return NEST_OK;
    for (void* p : a->slots) cudaFree(p);
    for (void* p : a->seg_un) cudaFree(p);
    for (void* p : a->seg_u1) cudaFree(p);
    for (void* p : {a->work, a->u1, a->lam[0], a->lam[1], a->tmp}) cudaFree(p);
    for (auto& kv : a->seg_graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(a->d_dts);
    cudaFree(a->seg_dts);
    if (a->h_seg_dts) cudaFreeHost(a->h_seg_dts);
    cudaFree(a->ctrl);
    delete a;
    return NEST_OK;
}

nest_status nest_adjoint_forward(nest_adjoint* a, double cfl, const double* dts) {
    if (!a) return fail(NEST_ERR_INVALID, "null adjoint handle");
    nest_solver* s = a->s;
    nest_status st;
    if ((st = nest_solver_reset_time(s)) != NEST_OK) return st;
    if (dts) {
        a->dts.assign(dts, dts + a->nsteps);
        if ((st = nest_solver_set_dt_sequence(s, dts, a->nsteps, 0)) != NEST_OK) return st;
    } else {
        if ((st = nest_solver_set_dt_sequence(s, nullptr, a->nsteps, 1)) != NEST_OK) return st;
    }
    if (!s->prepared && (st = prepare(s)) != NEST_OK) return st;
    auto snaps = forward_snapshots(a);
    std::fill(a->slot_pos.begin(), a->slot_pos.end(), -1);
    CK(cudaStreamSynchronize(s->st));
    auto t0 = std::chrono::high_resolution_clock::now();
    int at = 0;
    for (auto [step, slot] : snaps) {
        if (step > at) {
            if ((st = nest_solver_step(s, step - at, cfl)) != NEST_OK) return st;
            at = step;
        }
        if ((st = copy_state_dev(a, a->slots[slot], s->U)) != NEST_OK) return st;
        a->slot_pos[slot] = step;
    }
    if (a->nsteps > at && (st = nest_solver_step(s, a->nsteps - at, cfl)) != NEST_OK) return st;
    if ((st = read_ctrl(s)) != NEST_OK) return st;
    auto t1 = std::chrono::high_resolution_clock::now();
    a->fwd_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (!dts) {
        a->dts.resize(a->nsteps);
        if ((st = nest_solver_get_dts(s, a->dts.data(), a->nsteps)) != NEST_OK) return st;
    }
    if ((st = nest_solver_set_dt_sequence(s, nullptr, 0, 2)) != NEST_OK) return st;
    CK(cudaMemcpy(a->d_dts, a->dts.data(), sizeof(double) * a->nsteps, cudaMemcpyHostToDevice));
    a->forward_done = true;
    return NEST_OK;
}

nest_status nest_adjoint_backward(nest_adjoint* a, const void* lam_final, void* lam_initial, int on_device) {
    if (!a) return fail(NEST_ERR_INVALID, "null adjoint handle");
    if (!a->forward_done) return fail(NEST_ERR_INVALID, "run nest_adjoint_forward first");
    if (!lam_final || !lam_initial) return fail(NEST_ERR_INVALID, "null adjoint buffer");
    nest_solver* s = a->s;
    size_t bytes = s->state_bytes();
    nest_status st;
    CK(cudaStreamSynchronize(s->st));
    auto t0 = std::chrono::high_resolution_clock::now();
    a->advanced = 0;
    int cur = 0;
    CK(cudaMemcpyAsync(a->lam[0], lam_final, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       s->st));
    if (a->policy == NEST_CKPT_UNIFORM) {
        int K = a->param;
        int nseg = (a->nsteps + K - 1) / K;
        for (int g = nseg - 1; g >= 0; --g) {
            int j0 = g * K, L = std::min(a->nsteps, j0 + K) - j0;
            cudaGraphExec_t ge;
            if ((st = segment_graph(a, L, &ge)) != NEST_OK) return st;
            for (int r = 0; r < L; ++r) a->h_seg_dts[r] = a->dts[j0 + r];
            CK(cudaMemcpyAsync(a->seg_dts, a->h_seg_dts, sizeof(double) * L, cudaMemcpyHostToDevice, s->st));
            if ((st = copy_state_dev(a, a->seg_un[0], a->slots[g])) != NEST_OK) return st;
            CK(cudaGraphLaunch(ge, s->st));
            // the staging buffer is reused by the next segment
            CK(cudaStreamSynchronize(s->st));
            a->advanced += L - 1;
        }
    } else {
        if ((st = reverse_binomial(a, 0, a->nsteps, 0, a->param - 1, cur)) != NEST_OK) return st;
    }
    CK(cudaMemcpyAsync(lam_initial, a->lam[cur], bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       s->st));
    CK(cudaStreamSynchronize(s->st));
    auto t1 = std::chrono::high_resolution_clock::now();
    a->bwd_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return NEST_OK;
}

nest_status nest_adjoint_get_dts(nest_adjoint* a, double* dts) {
    if (!a || !dts) return fail(NEST_ERR_INVALID, "null argument");
    if (!a->forward_done) return fail(NEST_ERR_INVALID, "run nest_adjoint_forward first");
    std::copy(a->dts.begin(), a->dts.end(), dts);
    return NEST_OK;
}

nest_status nest_adjoint_stats(nest_adjoint* a, double* fwd_ms, double* bwd_ms, long long* recomputed_steps,
                               long long* snapshot_bytes) {
    if (!a) return fail(NEST_ERR_INVALID, "null adjoint handle");
    if (fwd_ms) *fwd_ms = a->fwd_ms;
    if (bwd_ms) *bwd_ms = a->bwd_ms;
    if (recomputed_steps) *recomputed_steps = a->advanced;
    if (snapshot_bytes) *snapshot_bytes = a->snap_bytes;
    return NEST_OK;
}

}  // extern "C"
