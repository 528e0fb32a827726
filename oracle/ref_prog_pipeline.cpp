// nest's pipeline executor (include/nest/pipeline.hpp) driving nest's own 1D
// Euler right-hand side on nest's own patches -- TEST INFRASTRUCTURE ONLY.
// The three stages are written against nest's stage concepts
// (pipeline.hpp:14-56): a Reduce stage (init / reduce / finalize) giving
// dt = cfl dx / max |u| + c as sod1d's compute_dt does, an Exchange stage
// (no value / reduce members: fill_all_halos) and a Compute stage whose
// value(patch) applies euler_rhs_t (examples/sod1d/euler1d.hpp:279-397) and
// writes the result back into the patch interior.  nest::execute runs them in
// order; the caller repeats it.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#include <algorithm>
#include <cmath>
#include <vector>

#include "nest/patch.hpp"
#include "nest/pipeline.hpp"
#include "sod1d/euler1d.hpp"

namespace {

using namespace nest;
using namespace nest::euler1d;
using patch1 = patch_t<double, 1>;

struct dt_stage_t {
    using value_type = double;
    const eos_t* eos;
    double cfl, dx;
    double* dt;
    static value_type init() { return 0.0; }
    value_type reduce(value_type acc, const patch1& p) const {
        for (auto idx : p.interior) {
            double U[NCONS], W[NPRIM];
            for (std::size_t k = 0; k < NCONS; ++k) U[k] = p(k, idx);
            cons_to_prim(U, W, *eos);
            double speed = std::abs(W[I_VEL]) + eos->sound_speed(W[I_RHO], W[I_PRE]);
            acc = std::max(acc, speed);
        }
        return acc;
    }
    void finalize(value_type acc, patch1&) const { *dt = cfl * dx / acc; }
};

struct exchange_stage_t {};

struct rhs_stage_t {
    const euler_rhs_t* rhs;
    const double* dt;
    patch1 value(patch1 p) const {
        field_t<double, 1> out(NCONS, p.interior, field_init_t::uninitialized);
        (*rhs)(p.state.conserved, out, p.interior, *dt);
        for (std::size_t k = 0; k < NCONS; ++k)
            for (auto idx : p.interior) p(k, idx) = out(k, idx);
        return p;
    }
};

}  // namespace

// U: the global interior state [3][n]; npatch periodic patches with `halo`
// ghost cells; nexec executions of (dt, exchange, rhs).  U receives the final
// interior state and dts[nexec] the dt of each execution.
extern "C" void ref_pipeline_euler1d(double* U, int n, int npatch, int halo, double gamma, double cfl,
                                     int limiter, int nexec, double* dts) {
    const double dx = 1.0 / n;
    eos_t eos{gamma};
    const limiter_t lim = limiter == 1 ? limiter_t::mc : limiter == 2 ? limiter_t::none : limiter_t::minmod;
    auto domain = index_space(ivec(0), uvec(static_cast<unsigned int>(n)));
    auto patches = build_periodic_mesh_1d<double>(domain, npatch, NCONS, halo);
    for (auto& p : patches)
        for (auto idx : p.interior)
            for (std::size_t k = 0; k < NCONS; ++k) p(k, idx) = U[k * n + idx[0]];
    euler_rhs_t rhs(eos, dx, lim);
    double dt = 0.0;
    auto pipe = pipeline(dt_stage_t{&eos, cfl, dx, &dt}, exchange_stage_t{}, rhs_stage_t{&rhs, &dt});
    for (int e = 0; e < nexec; ++e) {
        execute(pipe, patches);
        dts[e] = dt;
    }
    for (auto& p : patches)
        for (auto idx : p.interior)
            for (std::size_t k = 0; k < NCONS; ++k) U[k * n + idx[0]] = p(k, idx);
}
