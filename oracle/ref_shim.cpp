// C entry points over nest's own CPU numerics -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile from the nest source tree (include/ and
// examples/ are put on the include path; nothing is copied into this
// repository) into oracle/_ref/libnest_ref.so.  Tests use it to pin the
// plain-C oracle (oracle/euler_oracle.c) to the reference's own functions.
#ifndef NDEBUG
#define NDEBUG 1  // release semantics: the debug asserts of euler1d.hpp:36-41 are off
#endif
#include "sod1d/euler1d.hpp"
#include "sod2d/euler2d.hpp"
#include "nest/patch.hpp"

#include <vector>

using namespace nest;
using namespace nest::euler1d;

extern "C" {

double ref_pressure(double gamma, double rho, double mom, double erg) {
    return eos_t{gamma}.pressure(rho, mom, erg);
}
double ref_total_energy(double gamma, double rho, double u, double p) {
    return eos_t{gamma}.total_energy(rho, u, p);
}
double ref_sound_speed(double gamma, double rho, double p) {
    return eos_t{gamma}.sound_speed(rho, p);
}
void ref_cons_to_prim(double gamma, const double* U, double* W) {
    cons_to_prim(U, W, eos_t{gamma});
}
void ref_prim_to_cons(double gamma, const double* W, double* U) {
    prim_to_cons(W, U, eos_t{gamma});
}
double ref_minmod(double a, double b) { return minmod(a, b); }
double ref_mc(double a, double b) { return mc_limiter(a, b); }
void ref_plm(const double* Wm, const double* W0, const double* Wp, int lim,
             double* WL, double* WR) {
    auto r = plm_reconstruct(Wm, W0, Wp, static_cast<limiter_t>(lim));
    for (int k = 0; k < 3; ++k) { WL[k] = r.W_L[k]; WR[k] = r.W_R[k]; }
}
void ref_hlle_flux(double gamma, const double* WL, const double* WR, double* F) {
    hlle_flux(WL, WR, F, eos_t{gamma});
}

// The reference's per-patch right-hand side (euler_rhs_t, euler1d.hpp:279-397)
// on one patch stored as SoA over its extended space [start-h, start+n+h).
void ref_patch_stage(const double* Uin, double* Uout, int n, int h, double dx,
                     double dt, double gamma) {
    auto interior = index_space(ivec(0), uvec(static_cast<unsigned>(n)));
    auto extended = expand(interior, h);
    std::size_t nt = size(extended);
    std::vector<double> in(Uin, Uin + 3 * nt), out(3 * nt, 0.0);
    field_t<double, 1> fin(in.data(), 3, extended);
    field_t<double, 1> fout(out.data(), 3, extended);
    eos_t eos{gamma};
    euler_rhs_t rhs(eos, dx, limiter_t::minmod);
    rhs(fin, fout, interior, dt);
    for (std::size_t i = 0; i < 3 * nt; ++i) Uout[i] = out[i];
}

// Periodic 1D/2D halo exchange through nest's own plan builder and executor
// (patch.hpp:88-190, 207-326).  Patches are given as one SoA block each over
// their extended space, concatenated in patch order; the data is updated in
// place.  Returns the number of patches built.
int ref_exchange_1d(double* data, int n_domain, int n_patches, int nvars, int halo) {
    auto domain = index_space(ivec(0), uvec(static_cast<unsigned>(n_domain)));
    auto patches = build_periodic_mesh_1d<double>(domain, n_patches, nvars, halo);
    std::size_t off = 0;
    for (auto& p : patches) {
        std::size_t sz = nvars * size(p.extended);
        for (std::size_t i = 0; i < sz; ++i) p.state.conserved._data[i] = data[off + i];
        off += sz;
    }
    execute_all_exchanges(patches);
    off = 0;
    for (auto& p : patches) {
        std::size_t sz = nvars * size(p.extended);
        for (std::size_t i = 0; i < sz; ++i) data[off + i] = p.state.conserved._data[i];
        off += sz;
    }
    return static_cast<int>(patches.size());
}

int ref_exchange_2d(double* data, int nx, int ny, int npx, int npy, int nvars, int halo) {
    auto domain = index_space(ivec(0, 0), uvec(static_cast<unsigned>(nx), static_cast<unsigned>(ny)));
    auto patches = build_periodic_mesh_2d<double>(domain, npx, npy, nvars, halo);
    std::size_t off = 0;
    for (auto& p : patches) {
        std::size_t sz = nvars * size(p.extended);
        for (std::size_t i = 0; i < sz; ++i) p.state.conserved._data[i] = data[off + i];
        off += sz;
    }
    execute_all_exchanges(patches);
    off = 0;
    for (auto& p : patches) {
        std::size_t sz = nvars * size(p.extended);
        for (std::size_t i = 0; i < sz; ++i) data[off + i] = p.state.conserved._data[i];
        off += sz;
    }
    return static_cast<int>(patches.size());
}

// Patch interior boxes as built by nest (start_x, start_y, shape_x, shape_y
// per patch), patch.hpp:207-229 with subspace() of core.hpp:183-199.
int ref_patch_boxes_2d(int nx, int ny, int npx, int npy, int* boxes) {
    auto domain = index_space(ivec(0, 0), uvec(static_cast<unsigned>(nx), static_cast<unsigned>(ny)));
    auto patches = build_periodic_mesh_2d<double>(domain, npx, npy, 1, 1);
    int k = 0;
    for (auto& p : patches) {
        boxes[4 * k + 0] = start(p.interior)[0];
        boxes[4 * k + 1] = start(p.interior)[1];
        boxes[4 * k + 2] = static_cast<int>(shape(p.interior)[0]);
        boxes[4 * k + 3] = static_cast<int>(shape(p.interior)[1]);
        ++k;
    }
    return k;
}

// limiter_t from an integer: 0 minmod, 1 MC, 2 none (euler1d.hpp:106-110).
static limiter_t ref_limiter(int lim) {
    return lim == 1 ? limiter_t::mc : (lim == 2 ? limiter_t::none : limiter_t::minmod);
}

// The reference's dimensionally split 2D sweeps (euler2d.hpp:67-239) and
// CFL (euler2d.hpp:242-271) on a single patch whose ghost ring is already
// filled.  Layout: SoA over the extended space, y fastest.
void ref_x_sweep(const double* Uin, double* Uout, int nx, int ny, int h, double dx,
                 double dt, double gamma, int lim) {
    auto interior = index_space(ivec(0, 0), uvec(static_cast<unsigned>(nx), static_cast<unsigned>(ny)));
    auto extended = expand(interior, h);
    std::size_t nt = size(extended);
    std::vector<double> in(Uin, Uin + 4 * nt), out(Uin, Uin + 4 * nt);
    field_t<double, 2> fin(in.data(), 4, extended), fout(out.data(), 4, extended);
    eos_t eos{gamma};
    euler2d::x_sweep_t sweep(eos, dx, ref_limiter(lim));
    sweep(fin, fout, interior, dt);
    for (std::size_t i = 0; i < 4 * nt; ++i) Uout[i] = out[i];
}

void ref_y_sweep(const double* Uin, double* Uout, int nx, int ny, int h, double dy,
                 double dt, double gamma, int lim) {
    auto interior = index_space(ivec(0, 0), uvec(static_cast<unsigned>(nx), static_cast<unsigned>(ny)));
    auto extended = expand(interior, h);
    std::size_t nt = size(extended);
    std::vector<double> in(Uin, Uin + 4 * nt), out(Uin, Uin + 4 * nt);
    field_t<double, 2> fin(in.data(), 4, extended), fout(out.data(), 4, extended);
    eos_t eos{gamma};
    euler2d::y_sweep_t sweep(eos, dy, ref_limiter(lim));
    sweep(fin, fout, interior, dt);
    for (std::size_t i = 0; i < 4 * nt; ++i) Uout[i] = out[i];
}

double ref_compute_dt_2d(const double* U, int nx, int ny, int h, double dx, double dy,
                         double cfl, double gamma) {
    auto interior = index_space(ivec(0, 0), uvec(static_cast<unsigned>(nx), static_cast<unsigned>(ny)));
    std::vector<patch_t<double, 2>> patches;
    patches.emplace_back(0, interior, 4, h);
    auto& p = patches[0];
    std::size_t nt = size(p.extended);
    for (std::size_t i = 0; i < 4 * nt; ++i) p.state.conserved._data[i] = U[i];
    return euler2d::compute_dt_2d(patches, dx, dy, cfl, eos_t{gamma});
}

}  // extern "C"
