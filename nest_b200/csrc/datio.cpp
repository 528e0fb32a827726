// On-disk formats: nest's text snapshots and a restartable binary checkpoint.
//
// Text (.dat): the files nest's examples write for its plotting scripts.
//   1D, write_output (examples/sod1d/sod1d.cpp:50-91):
//     "# Sod shock tube at t = <t>" / "# x rho u p e" / one line per cell
//     "x rho u p e" with p from eos_t::pressure (clamped at 0) and
//     e = p / (rho (gamma - 1)) (examples/sod1d/euler1d.hpp:31-65).
//   2D, write_output_2d (examples/sod2d/sod2d.cpp:58-97):
//     "# 2D Sod shock tube at t = <t>" / "# x y rho u v p" / "x y rho u v p",
//     p = (gamma - 1)(E - 0.5 rho (u u + v v)) unclamped.
//   2D x-slice, write_xslice (sod2d.cpp:100-152): cells of row j = ny/2,
//     "# x-slice at y_mid, t = <t>" / "# x rho u p" / "x rho u p", sorted by x.
// Numbers use iostream's std::scientific with precision 10, i.e. "%.10e".
// Cells appear patch by patch in nest's patch order (build_periodic_mesh_1d /
// _2d, include/nest/patch.hpp:88-147, 207-229: py outer, px inner, pieces
// from subspace(), include/nest/core.hpp:183-199) and inside a patch in
// index_space order (last index fastest, core.hpp:103-121), so a state
// written here is byte for byte the file nest writes for the same state and
// patch grid.
//
// Checkpoint: header (magic "NESTCKP1", sizes, precision, boundary
// conditions, gamma, dx, dy, time, step), the interior planes in the
// solver's precision (row-major, y fastest) and an FNV-1a 64 checksum of
// the payload.  Loading restores state, time and step count, so a run
// continued from a checkpoint equals the uninterrupted run bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "solver_impl.h"

using namespace nestb;
using namespace nestb::rt;

namespace {

void piece(int total, int parts, int part, int& off, int& len) {
    int base = total / parts, extra = total % parts;
    off = part * base + std::min(part, extra);
    len = base + (part < extra ? 1 : 0);
}

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

// eos_t::pressure (euler1d.hpp:31-44), then cons_to_prim (euler1d.hpp:71-84).
void prim1d(double gamma, double rho, double mom, double erg, double& u, double& p) {
    u = mom / rho;
    double ke = 0.5 * rho * u * u;
    double pp = (gamma - 1.0) * (erg - ke);
    p = (pp < 0.0) ? 0.0 : pp;   // std::max(p, 0.0)
}

// Cell centre of index i on a grid starting at lo with spacing d.
inline double centre(double lo, double d, int i) { return lo + (i + 0.5) * d; }

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for (size_t i = 0; i < n; ++i) { h ^= p[i]; h *= 1099511628211ull; }
    return h;
}

nest_status check(const nest_solver* s) {
    return s ? NEST_OK : fail(NEST_ERR_INVALID, "null solver handle");
}

struct CkptHeader {
    char magic[8];
    int32_t version, dim, nx, ny, precision, bc_x, bc_y, halo;
    double gamma, dx, dy, time;
    int64_t step;
};

}  // namespace

extern "C" {

nest_status nest_write_dat_1d(const char* path, const double* U, int n, int halo, int npatch, double x_min,
                              double x_max, double gamma, double time) {
    if (!path || !U) return fail(NEST_ERR_INVALID, "null argument");
    if (n < 1 || halo < 0 || npatch < 1 || npatch > n) return fail(NEST_ERR_INVALID, "bad sizes");
    File out(path, "w");
    if (!out.f) return fail(NEST_ERR_INVALID, "cannot open output file");
    const long long nt = n + 2ll * halo;
    const double dx = (x_max - x_min) / n;
    std::fprintf(out.f, "# Sod shock tube at t = %.10e\n# x rho u p e\n", time);
    for (int k = 0; k < npatch; ++k) {
        int off, len;
        piece(n, npatch, k, off, len);
        for (int i = off; i < off + len; ++i) {
            double rho = U[halo + i], mom = U[nt + halo + i], erg = U[2 * nt + halo + i];
            double u, p;
            prim1d(gamma, rho, mom, erg, u, p);
            double e = p / (rho * (gamma - 1.0));
            std::fprintf(out.f, "%.10e %.10e %.10e %.10e %.10e\n", centre(x_min, dx, i), rho, u, p, e);
        }
    }
    if (std::ferror(out.f)) return fail(NEST_ERR_INVALID, "write failed");
    return NEST_OK;
}

nest_status nest_write_dat_2d(const char* path, const double* U, int nx, int ny, int npx, int npy, double x_min,
                              double x_max, double y_min, double y_max, double gamma, double time, int xslice) {
    if (!path || !U) return fail(NEST_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1 || npx < 1 || npy < 1 || npx > nx || npy > ny) return fail(NEST_ERR_INVALID, "bad sizes");
    File out(path, "w");
    if (!out.f) return fail(NEST_ERR_INVALID, "cannot open output file");
    const long long rowlen = ny + 4, plane = (long long)(nx + 4) * rowlen;
    const double dx = (x_max - x_min) / nx, dy = (y_max - y_min) / ny;
    auto at = [&](int i, int j) { return (long long)(i + 2) * rowlen + (j + 2); };
    auto prim = [&](int i, int j, double& rho, double& u, double& v, double& p) {
        long long o = at(i, j);
        rho = U[o];
        u = U[plane + o] / rho;
        v = U[2 * plane + o] / rho;
        double ke = 0.5 * rho * (u * u + v * v);
        p = (gamma - 1.0) * (U[3 * plane + o] - ke);
    };
    if (!xslice) {
        std::fprintf(out.f, "# 2D Sod shock tube at t = %.10e\n# x y rho u v p\n", time);
    } else {
        std::fprintf(out.f, "# x-slice at y_mid, t = %.10e\n# x rho u p\n", time);
    }
    const int jmid = ny / 2;
    struct Row { double x, rho, u, p; };
    std::vector<Row> slice;
    for (int py = 0; py < npy; ++py)
        for (int px = 0; px < npx; ++px) {
            int x0, lx, y0, ly;
            piece(nx, npx, px, x0, lx);
            piece(ny, npy, py, y0, ly);
            for (int i = x0; i < x0 + lx; ++i)
                for (int j = y0; j < y0 + ly; ++j) {
                    if (xslice && j != jmid) continue;
                    double rho, u, v, p;
                    prim(i, j, rho, u, v, p);
                    if (xslice) {
                        slice.push_back({centre(x_min, dx, i), rho, u, p});
                    } else {
                        std::fprintf(out.f, "%.10e %.10e %.10e %.10e %.10e %.10e\n", centre(x_min, dx, i),
                                     centre(y_min, dy, j), rho, u, v, p);
                    }
                }
        }
    if (xslice) {
        std::stable_sort(slice.begin(), slice.end(), [](const Row& a, const Row& b) { return a.x < b.x; });
        for (const Row& r : slice) std::fprintf(out.f, "%.10e %.10e %.10e %.10e\n", r.x, r.rho, r.u, r.p);
    }
    if (std::ferror(out.f)) return fail(NEST_ERR_INVALID, "write failed");
    return NEST_OK;
}

nest_status nest_solver_write_dat(nest_solver* s, const char* path, int npx, int npy, double x_min, double x_max,
                                  double y_min, double y_max, int xslice) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    const auto& d = s->d;
    size_t count = d.dim == 1 ? 3 * (size_t)(d.nx + 2 * s->h) : 4 * (size_t)(d.nx + 4) * (size_t)(d.ny + 4);
    std::vector<double> U(count);
    if (d.precision == NEST_F64) {
        if ((r = nest_solver_download(s, U.data(), NEST_LAYOUT_EXTENDED)) != NEST_OK) return r;
    } else {
        std::vector<float> F(count);
        if ((r = nest_solver_download(s, F.data(), NEST_LAYOUT_EXTENDED)) != NEST_OK) return r;
        for (size_t k = 0; k < count; ++k) U[k] = F[k];
    }
    double t = 0.0;
    if ((r = nest_solver_time(s, &t, nullptr)) != NEST_OK) return r;
    if (d.dim == 1) return nest_write_dat_1d(path, U.data(), d.nx, s->h, npx, x_min, x_max, d.gamma, t);
    return nest_write_dat_2d(path, U.data(), d.nx, d.ny, npx, npy, x_min, x_max, y_min, y_max, d.gamma, t, xslice);
}

nest_status nest_solver_save(nest_solver* s, const char* path) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!path) return fail(NEST_ERR_INVALID, "null path");
    const auto& d = s->d;
    const size_t es = d.precision == NEST_F64 ? 8 : 4;
    const size_t cells = d.dim == 1 ? (size_t)d.nx : (size_t)d.nx * (size_t)d.ny;
    std::vector<unsigned char> payload(s->nvars * cells * es);
    if ((r = nest_solver_download(s, payload.data(), NEST_LAYOUT_INTERIOR)) != NEST_OK) return r;
    CkptHeader h{};
    std::memcpy(h.magic, "NESTCKP1", 8);
    h.version = 1; h.dim = d.dim; h.nx = d.nx; h.ny = d.dim == 2 ? d.ny : 1; h.precision = d.precision;
    h.bc_x = d.bc_x; h.bc_y = d.bc_y; h.halo = s->h; h.gamma = d.gamma; h.dx = d.dx; h.dy = d.dy;
    int step = 0;
    if ((r = nest_solver_time(s, &h.time, &step)) != NEST_OK) return r;
    h.step = step;
    uint64_t sum = fnv1a(payload.data(), payload.size());
    File out(path, "wb");
    if (!out.f) return fail(NEST_ERR_INVALID, "cannot open checkpoint file");
    if (std::fwrite(&h, sizeof h, 1, out.f) != 1 || std::fwrite(payload.data(), 1, payload.size(), out.f) != payload.size() ||
        std::fwrite(&sum, sizeof sum, 1, out.f) != 1)
        return fail(NEST_ERR_INVALID, "checkpoint write failed");
    return NEST_OK;
}

nest_status nest_solver_load(nest_solver* s, const char* path) {
    nest_status r = check(s);
    if (r != NEST_OK) return r;
    if (!path) return fail(NEST_ERR_INVALID, "null path");
    File in(path, "rb");
    if (!in.f) return fail(NEST_ERR_INVALID, "cannot open checkpoint file");
    CkptHeader h{};
    if (std::fread(&h, sizeof h, 1, in.f) != 1 || std::memcmp(h.magic, "NESTCKP1", 8) != 0 || h.version != 1)
        return fail(NEST_ERR_INVALID, "not a nest_b200 checkpoint");
    const auto& d = s->d;
    if (h.dim != d.dim || h.nx != d.nx || (d.dim == 2 && h.ny != d.ny) || h.precision != d.precision ||
        h.bc_x != d.bc_x || h.bc_y != d.bc_y || h.gamma != d.gamma || h.dx != d.dx || h.dy != d.dy)
        return fail(NEST_ERR_INVALID, "checkpoint does not match this solver (sizes, precision, bc, gamma, dx, dy)");
    const size_t es = d.precision == NEST_F64 ? 8 : 4;
    const size_t cells = d.dim == 1 ? (size_t)d.nx : (size_t)d.nx * (size_t)d.ny;
    std::vector<unsigned char> payload(s->nvars * cells * es);
    uint64_t sum = 0;
    if (std::fread(payload.data(), 1, payload.size(), in.f) != payload.size() || std::fread(&sum, sizeof sum, 1, in.f) != 1)
        return fail(NEST_ERR_INVALID, "checkpoint truncated");
    if (sum != fnv1a(payload.data(), payload.size())) return fail(NEST_ERR_INVALID, "checkpoint checksum mismatch");
    if ((r = nest_solver_upload(s, payload.data(), NEST_LAYOUT_INTERIOR)) != NEST_OK) return r;
    return nest_solver_set_time(s, h.time, (int)h.step);
}

}  // extern "C"
