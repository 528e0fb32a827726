// Patch halo exchange on nest's own per-patch storage, on the device.
//
// nest builds a plan of copy regions per patch (build_periodic_mesh_1d/2d,
// include/nest/patch.hpp:88-147, 207-326: for every face a region of width
// `halo` copied from the facing edge of the periodic neighbour; faces only,
// no corners) and executes it patch by patch on the host
// (execute_exchange / execute_all_exchanges, patch.hpp:153-190).  Here the
// plan is built the same way on the host, flattened into a table of regions,
// and executed by one kernel launch: every region reads only interior cells
// and writes only halo cells, so all copies are independent.
//
// Storage: patch p holds nvars SoA planes over its extended space
// (interior expanded by `halo`), row-major with idx[1] fastest
// (include/nest/core.hpp:206-215, 310-392); the patches' blocks are stored
// one after another in patch order.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace {

struct Region {
    long long dst, src;       // element offsets of the first element (variable 0)
    long long dvar, svar;     // plane strides (extended sizes) of the destination / source patch
    int ds0, ss0;             // row strides (extended extent along idx[1]; 1 for 1D)
    int n0, n1;               // region extents along idx[0], idx[1]
    long long first;          // index of the region's first element in the flattened launch
};

template <typename T>
__global__ void __launch_bounds__(256) k_exchange(T* data, const Region* regs, int nregs, int nvars, long long total) {
    for (long long e = blockIdx.x * 256ll + threadIdx.x; e < total; e += (long long)gridDim.x * 256) {
        int lo = 0, hi = nregs - 1;  // region containing element e
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (regs[mid].first <= e) lo = mid; else hi = mid - 1;
        }
        const Region& r = regs[lo];
        long long k = e - r.first;
        int per_var = r.n0 * r.n1;
        int v = (int)(k / per_var), q = (int)(k % per_var);
        int a = q / r.n1, b = q % r.n1;
        data[r.dst + v * r.dvar + (long long)a * r.ds0 + b] = data[r.src + v * r.svar + (long long)a * r.ss0 + b];
    }
}

struct Box { int s0, s1, n0, n1; };  // interior start and shape (idx[0], idx[1])

// subspace(), include/nest/core.hpp:183-199.
void split(int start, int total, int nparts, int part, int& off, int& len) {
    int base = total / nparts, extra = total % nparts;
    off = start + part * base + std::min(part, extra);
    len = base + (part < extra ? 1 : 0);
}

}  // namespace

struct nest_exchange {
    int dim = 1, nvars = 1, halo = 1, npatch = 0;
    std::vector<Box> boxes;
    std::vector<long long> offsets;  // element offset of each patch block (+ total)
    std::vector<Region> regs;
    std::vector<int> peers;          // per patch, per region: peer index (plan structure, patch.hpp:22-37)
    Region* dregs = nullptr;
    long long total = 0;
};

extern "C" {

nest_status nest_exchange_create_periodic(int dim, int nx, int ny, int npx, int npy, int nvars, int halo,
                                          nest_exchange** out) {
    if (!out) return fail(NEST_ERR_INVALID, "null argument");
    *out = nullptr;
    if (dim != 1 && dim != 2) return fail(NEST_ERR_INVALID, "dim must be 1 or 2");
    if (nvars < 1 || halo < 1 || npx < 1 || (dim == 2 && npy < 1)) return fail(NEST_ERR_INVALID, "bad plan sizes");
    if (nx < npx * halo || (dim == 2 && ny < npy * halo))
        return fail(NEST_ERR_INVALID, "every patch needs at least `halo` interior cells per axis");
    auto* x = new (std::nothrow) nest_exchange;
    if (!x) return fail(NEST_ERR_OOM, "host allocation failed");
    x->dim = dim; x->nvars = nvars; x->halo = halo;
    int nyp = dim == 2 ? npy : 1;
    x->npatch = npx * nyp;
    // patches in row-major order (py outer, px inner), patch.hpp:218-229
    for (int py = 0; py < nyp; ++py)
        for (int px = 0; px < npx; ++px) {
            Box b;
            split(0, nx, npx, px, b.s0, b.n0);
            if (dim == 2) split(0, ny, npy, py, b.s1, b.n1);
            else { b.s1 = 0; b.n1 = 1; }
            x->boxes.push_back(b);
        }
    auto ext1 = [&](const Box& b) { return dim == 2 ? b.n1 + 2 * halo : 1; };
    auto ext0 = [&](const Box& b) { return b.n0 + 2 * halo; };
    x->offsets.assign(x->npatch + 1, 0);
    for (int p = 0; p < x->npatch; ++p)
        x->offsets[p + 1] = x->offsets[p] + (long long)nvars * ext0(x->boxes[p]) * ext1(x->boxes[p]);
    // element offset of absolute index (i, j) inside patch p's plane 0
    auto at = [&](int p, int i, int j) {
        const Box& b = x->boxes[p];
        long long li = i - (b.s0 - halo), lj = dim == 2 ? j - (b.s1 - halo) : 0;
        return x->offsets[p] + li * ext1(b) + lj;
    };
    long long first = 0;
    auto add = [&](int p, int peer, int di, int dj, int si, int sj, int n0, int n1) {
        Region r;
        r.dst = at(p, di, dj);
        r.src = at(peer, si, sj);
        r.dvar = (long long)ext0(x->boxes[p]) * ext1(x->boxes[p]);
        r.svar = (long long)ext0(x->boxes[peer]) * ext1(x->boxes[peer]);
        r.ds0 = ext1(x->boxes[p]);
        r.ss0 = ext1(x->boxes[peer]);
        r.n0 = n0; r.n1 = n1;
        r.first = first;
        first += (long long)nvars * n0 * n1;
        x->regs.push_back(r);
        x->peers.push_back(peer);
    };
    for (int py = 0; py < nyp; ++py)
        for (int px = 0; px < npx; ++px) {
            int p = py * npx + px;
            const Box& b = x->boxes[p];
            int lp = py * npx + (px - 1 + npx) % npx, rp = py * npx + (px + 1) % npx;
            const Box& L = x->boxes[lp];
            const Box& R = x->boxes[rp];
            // x faces (patch.hpp:107-143, 237-278): receive the neighbours' edge columns
            add(p, lp, b.s0 - halo, dim == 2 ? b.s1 : 0, L.s0 + L.n0 - halo, dim == 2 ? L.s1 : 0, halo, b.n1);
            add(p, rp, b.s0 + b.n0, dim == 2 ? b.s1 : 0, R.s0, dim == 2 ? R.s1 : 0, halo, b.n1);
            if (dim == 2) {
                // y faces (patch.hpp:280-321)
                int bp = ((py - 1 + npy) % npy) * npx + px, tp = ((py + 1) % npy) * npx + px;
                const Box& B = x->boxes[bp];
                const Box& T = x->boxes[tp];
                add(p, bp, b.s0, b.s1 - halo, B.s0, B.s1 + B.n1 - halo, b.n0, halo);
                add(p, tp, b.s0, b.s1 + b.n1, T.s0, T.s1, b.n0, halo);
            }
        }
    x->total = first;
    cudaError_t e = cudaMalloc(&x->dregs, sizeof(Region) * x->regs.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(x->dregs, x->regs.data(), sizeof(Region) * x->regs.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        nest_exchange_destroy(x);
        return cuda_fail(e, "exchange plan upload");
    }
    *out = x;
    return NEST_OK;
}

nest_status nest_exchange_destroy(nest_exchange* x) {
    if (!x) return NEST_OK;
    cudaFree(x->dregs);
    delete x;
    return NEST_OK;
}

nest_status nest_exchange_layout(nest_exchange* x, long long* offsets, int* boxes, int* peers) {
    if (!x) return fail(NEST_ERR_INVALID, "null exchange handle");
    for (int p = 0; p <= x->npatch && offsets; ++p) offsets[p] = x->offsets[p];
    for (int p = 0; p < x->npatch && boxes; ++p) {
        boxes[4 * p] = x->boxes[p].s0; boxes[4 * p + 1] = x->boxes[p].s1;
        boxes[4 * p + 2] = x->boxes[p].n0; boxes[4 * p + 3] = x->boxes[p].n1;
    }
    for (size_t r = 0; r < x->peers.size() && peers; ++r) peers[r] = x->peers[r];
    return NEST_OK;
}

nest_status nest_exchange_execute(nest_exchange* x, void* d_data, int precision, void* stream) {
    if (!x || !d_data) return fail(NEST_ERR_INVALID, "null argument");
    if (precision != NEST_F64 && precision != NEST_F32) return fail(NEST_ERR_INVALID, "bad precision");
    if (x->total == 0) return NEST_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int blocks = (int)std::min<long long>((x->total + 255) / 256, 148ll * 16);
    if (precision == NEST_F64)
        k_exchange<double><<<blocks, 256, 0, st>>>((double*)d_data, x->dregs, (int)x->regs.size(), x->nvars, x->total);
    else
        k_exchange<float><<<blocks, 256, 0, st>>>((float*)d_data, x->dregs, (int)x->regs.size(), x->nvars, x->total);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "exchange kernel");
    return NEST_OK;
}

}  // extern "C"
