// nest's sod1d example as a callable function -- TEST INFRASTRUCTURE ONLY.
// examples/sod1d/sod1d.cpp is compiled where it lies; main() is renamed.
// Running it writes sod_*.dat into the current directory.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define main nest_ref_sod1d_main
#include "sod1d/sod1d.cpp"
#undef main

extern "C" int ref_sod1d_main(void) { return nest_ref_sod1d_main(); }

// nest's own 1D snapshot writer on a given state: fills nest patches (npatch
// pieces, halo 2) from U ([3][n + 2 halo], interior at halo..halo+n-1) and
// calls write_output, which writes sod_<step>.dat into the current directory.
extern "C" void ref_write_sod1d(const double* U, int n, int halo, int npatch, double x_min, double x_max,
                                double gamma, double time, int step) {
    auto cfg = config_t{};
    cfg.x_min = x_min;
    cfg.x_max = x_max;
    cfg.num_zones = n;
    cfg.num_patches = npatch;
    cfg.gamma = gamma;
    auto domain = index_space(ivec(0), uvec(static_cast<unsigned int>(n)));
    auto patches = build_periodic_mesh_1d<double>(domain, npatch, NCONS, 2);
    const long long nt = n + 2ll * halo;
    for (auto& patch : patches)
        for (auto idx : patch.interior)
            for (std::size_t k = 0; k < NCONS; ++k) patch(k, idx) = U[k * nt + halo + idx[0]];
    write_output(patches, cfg, time, step);
}
