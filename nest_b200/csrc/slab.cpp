// Multi-GPU x-slab driver in C++: the step loop of a sharded domain on the
// solver's stream, with NCCL for the two exchange steps, captured into CUDA
// graphs like the one-domain solver's steps.
//
// A domain cut into x-slabs (nest's subspace() split, include/nest/
// core.hpp:183-199), one per rank; per RK2 step (nest's exchange before each
// stage, examples/sod2d/sod2d.cpp:331-362):
//   1. max-all-reduce of the two wave-speed words of the step's speed slot
//      (bit patterns of non-negative doubles order like the doubles), so every
//      slab derives the same dt;
//   2. the two ghost rows of each cut side of the state from the neighbour
//      slab's edge rows (NCCL send / recv, one message per variable plane and
//      side: two rows of a plane are contiguous);
//   3. stage 1;  4. the same exchange on the stage buffer;  5. stage 2.
// All of it is enqueued on the solver's stream, so a step needs no host
// synchronisation, and runs of 16 steps are captured into a CUDA graph.
// Messages between one pair of ranks match in posting order: every rank
// posts its sends (hi side first, then lo side) before its receives (lo side
// first, then hi side), so with two ranks, whose lo and hi neighbour is the
// same rank, the hi rows of one land in the lo ghost rows of the other.
//
// NCCL is loaded at run time (dlopen of libnccl.so.2, the copy the process
// already has when torch loaded one), so the library has no link-time NCCL
// dependency.  No kernel here waits on another rank; only NCCL's own kernels
// do, bounded by the communicator's timeout.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace {

struct NcclApi {
    decltype(&ncclGetUniqueId) get_unique_id = nullptr;
    decltype(&ncclCommInitRank) comm_init_rank = nullptr;
    decltype(&ncclCommDestroy) comm_destroy = nullptr;
    decltype(&ncclAllReduce) all_reduce = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclGroupStart) group_start = nullptr;
    decltype(&ncclGroupEnd) group_end = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
    bool ok = false;
    std::string why;
};

const NcclApi& nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW);
        if (!h) { api.why = "libnccl.so.2 not found"; return; }
        auto sym = [&](const char* name) { return dlsym(h, name); };
        api.get_unique_id = (decltype(api.get_unique_id))sym("ncclGetUniqueId");
        api.comm_init_rank = (decltype(api.comm_init_rank))sym("ncclCommInitRank");
        api.comm_destroy = (decltype(api.comm_destroy))sym("ncclCommDestroy");
        api.all_reduce = (decltype(api.all_reduce))sym("ncclAllReduce");
        api.send = (decltype(api.send))sym("ncclSend");
        api.recv = (decltype(api.recv))sym("ncclRecv");
        api.group_start = (decltype(api.group_start))sym("ncclGroupStart");
        api.group_end = (decltype(api.group_end))sym("ncclGroupEnd");
        api.error_string = (decltype(api.error_string))sym("ncclGetErrorString");
        api.ok = api.get_unique_id && api.comm_init_rank && api.comm_destroy && api.all_reduce && api.send &&
                 api.recv && api.group_start && api.group_end && api.error_string;
        if (!api.ok) api.why = "libnccl.so.2 lacks a needed symbol";
    });
    return api;
}

nest_status nccl_fail(ncclResult_t r, const char* what) {
    return fail(NEST_ERR_CUDA, std::string(what) + ": " + nccl().error_string(r));
}

}  // namespace

struct nest_slab_comm {
    ncclComm_t comm = nullptr;
    int nranks = 0, rank = 0;
};

namespace {

// Key of a captured run of slab steps.
struct SlabGraphKey {
    nest_slab_comm* comm;
    int lo, hi, parity;
    double cfl, t_final;
    int tx, warps;
    bool operator<(const SlabGraphKey& o) const {
        return std::tie(comm, lo, hi, parity, cfl, t_final, tx, warps) <
               std::tie(o.comm, o.lo, o.hi, o.parity, o.cfl, o.t_final, o.tx, o.warps);
    }
};

std::mutex g_slab_graph_mutex;
std::map<nest_solver*, std::map<SlabGraphKey, cudaGraphExec_t>> g_slab_graphs;

// Ghost rows of the cut sides of buffer `base` from the neighbours (lo / hi =
// neighbour ranks, -1: that side is a domain boundary).
nest_status exchange_rows(nest_solver* s, nest_slab_comm* c, void* base, int lo, int hi) {
    const NcclApi& api = nccl();
    const ncclDataType_t dt = s->d.precision == NEST_F64 ? ncclFloat64 : ncclFloat32;
    const size_t es = s->esize, count = 2 * (size_t)s->pitch;
    const int n = s->d.nx;
    auto plane = [&](int v, int row) {  // element row `row` (-2 .. n+1) of plane v
        return (char*)base + es * ((size_t)v * s->vstride + (size_t)(row + 2) * s->pitch);
    };
    ncclResult_t r = api.group_start();
    if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
    for (int v = 0; v < 4 && r == ncclSuccess && hi >= 0; ++v) r = api.send(plane(v, n - 2), count, dt, hi, c->comm, s->st);
    for (int v = 0; v < 4 && r == ncclSuccess && lo >= 0; ++v) r = api.send(plane(v, 0), count, dt, lo, c->comm, s->st);
    for (int v = 0; v < 4 && r == ncclSuccess && lo >= 0; ++v) r = api.recv(plane(v, -2), count, dt, lo, c->comm, s->st);
    for (int v = 0; v < 4 && r == ncclSuccess && hi >= 0; ++v) r = api.recv(plane(v, n), count, dt, hi, c->comm, s->st);
    ncclResult_t r2 = api.group_end();
    if (r != ncclSuccess) return nccl_fail(r, "ncclSend/ncclRecv");
    if (r2 != ncclSuccess) return nccl_fail(r2, "ncclGroupEnd");
    return NEST_OK;
}

// One step with parity p: speed all-reduce, exchange, stage 1, exchange, stage 2.
nest_status enqueue_slab_step(nest_solver* s, nest_slab_comm* c, int lo, int hi, const LoopParams& lp, int p) {
    const NcclApi& api = nccl();
    unsigned long long* words = &s->ctrl->maxs[p][0];
    ncclResult_t r = api.all_reduce(words, words, 2, ncclUint64, ncclMax, c->comm, s->st);
    if (r != ncclSuccess) return nccl_fail(r, "ncclAllReduce(speeds)");
    nest_status st = exchange_rows(s, c, s->U, lo, hi);
    if (st != NEST_OK) return st;
    cudaError_t e = enqueue_step(s, lp, p, 1);
    if (e != cudaSuccess) return cuda_fail(e, "stage 1");
    if ((st = exchange_rows(s, c, s->U1, lo, hi)) != NEST_OK) return st;
    e = enqueue_step(s, lp, p, 2);
    if (e != cudaSuccess) return cuda_fail(e, "stage 2");
    return NEST_OK;
}

}  // namespace

// Called by the solver when it drops its graphs or is destroyed.
void nestb::rt::slab_release(nest_solver* s) {
    std::lock_guard<std::mutex> lock(g_slab_graph_mutex);
    auto it = g_slab_graphs.find(s);
    if (it == g_slab_graphs.end()) return;
    for (auto& kv : it->second) cudaGraphExecDestroy(kv.second);
    g_slab_graphs.erase(it);
}

extern "C" {

nest_status nest_slab_comm_id(unsigned char id[128]) {
    if (!id) return fail(NEST_ERR_INVALID, "null id buffer");
    const NcclApi& api = nccl();
    if (!api.ok) return fail(NEST_ERR_UNSUPPORTED, "NCCL unavailable: " + api.why);
    ncclUniqueId u;
    ncclResult_t r = api.get_unique_id(&u);
    if (r != ncclSuccess) return nccl_fail(r, "ncclGetUniqueId");
    std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
    return NEST_OK;
}

nest_status nest_slab_comm_create(const unsigned char id[128], int nranks, int rank, nest_slab_comm** out) {
    if (!id || !out) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (nranks < 1 || rank < 0 || rank >= nranks) return fail(NEST_ERR_INVALID, "bad rank / size");
    const NcclApi& api = nccl();
    if (!api.ok) return fail(NEST_ERR_UNSUPPORTED, "NCCL unavailable: " + api.why);
    auto* c = new (std::nothrow) nest_slab_comm;
    if (!c) return fail(NEST_ERR_OOM, "host allocation failed");
    ncclUniqueId u;
    std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
    ncclResult_t r = api.comm_init_rank(&c->comm, nranks, u, rank);
    if (r != ncclSuccess) {
        delete c;
        return nccl_fail(r, "ncclCommInitRank");
    }
    c->nranks = nranks;
    c->rank = rank;
    *out = c;
    return NEST_OK;
}

nest_status nest_slab_comm_destroy(nest_slab_comm* c) {
    if (!c) return NEST_OK;
    {
        // graphs that hold this communicator's calls go first
        std::lock_guard<std::mutex> lock(g_slab_graph_mutex);
        for (auto& per : g_slab_graphs)
            for (auto it = per.second.begin(); it != per.second.end();) {
                if (it->first.comm == c) {
                    cudaGraphExecDestroy(it->second);
                    it = per.second.erase(it);
                } else {
                    ++it;
                }
            }
    }
    if (c->comm) nccl().comm_destroy(c->comm);
    delete c;
    return NEST_OK;
}


nest_status nest_slab_step(nest_solver* s, nest_slab_comm* c, int lo, int hi, int nsteps, double cfl,
                           double t_final) {
    if (!s || !c) return fail(NEST_ERR_INVALID, "null argument");
    if (s->d.dim != 2 || (s->d.flags & NEST_FLAG_SPLIT_COMPAT))
        return fail(NEST_ERR_UNSUPPORTED, "slab steps run the 2D RK2 scheme");
    if (nsteps < 0 || !(cfl > 0.0)) return fail(NEST_ERR_INVALID, "need nsteps >= 0 and cfl > 0");
    if (lo >= c->nranks || hi >= c->nranks) return fail(NEST_ERR_INVALID, "neighbour rank out of range");
    if ((lo >= 0) != (s->xlo_ex != 0) || (hi >= 0) != (s->xhi_ex != 0))
        return fail(NEST_ERR_INVALID, "neighbours must match the solver's exchange sides");
    if (!s->prepared) {
        nest_status r = prepare(s);
        if (r != NEST_OK) return r;
    }
    LoopParams lp{};
    lp.lim = (s->d.flags & NEST_FLAG_LIMITER_MC) ? LIM_MC : (s->d.flags & NEST_FLAG_LIMITER_NONE) ? LIM_NONE
                                                                                                  : LIM_MINMOD;
    lp.cfl = cfl;
    lp.t_final = t_final > 0.0 ? t_final : 0.0;
    while (nsteps > 0) {
        if (nsteps >= GRAPH_STEPS) {
            SlabGraphKey k{c, lo, hi, s->parity, cfl, lp.t_final, s->tx, s->warps};
            cudaGraphExec_t ge = nullptr;
            {
                std::lock_guard<std::mutex> lock(g_slab_graph_mutex);
                auto& per = g_slab_graphs[s];
                auto it = per.find(k);
                if (it != per.end()) ge = it->second;
            }
            if (!ge) {
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
                nest_status r = NEST_OK;
                int p = s->parity;
                for (int i = 0; i < GRAPH_STEPS && r == NEST_OK; ++i, p ^= 1) r = enqueue_slab_step(s, c, lo, hi, lp, p);
                cudaError_t e2 = cudaStreamEndCapture(s->st, &g);
                if (r != NEST_OK) {
                    if (e2 == cudaSuccess) cudaGraphDestroy(g);
                    return r;
                }
                if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
                cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
                std::lock_guard<std::mutex> lock(g_slab_graph_mutex);
                g_slab_graphs[s][k] = ge;
            }
            CK(cudaGraphLaunch(ge, s->st));
            nsteps -= GRAPH_STEPS;
        } else {
            nest_status r = enqueue_slab_step(s, c, lo, hi, lp, s->parity);
            if (r != NEST_OK) return r;
            s->parity ^= 1;
            --nsteps;
        }
    }
    return NEST_OK;
}

}  // extern "C"
