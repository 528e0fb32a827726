// nest's sod2d example as a callable function -- TEST INFRASTRUCTURE ONLY.
// examples/sod2d/sod2d.cpp is compiled where it lies; main() is renamed.
// Running it writes sod2d_*.dat into the current directory.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define main nest_ref_sod2d_main
#include "sod2d/sod2d.cpp"
#undef main

extern "C" int ref_sod2d_main(void) { return nest_ref_sod2d_main(); }

// nest's own 2D snapshot writers on a given state: fills nest patches
// (npx x npy, halo 2) from U ([4][nx + 4][ny + 4]) and calls write_output_2d
// and write_xslice (sod2d_<step>.dat, sod2d_xslice_<step>.dat in the
// current directory).
extern "C" void ref_write_sod2d(const double* U, int nx, int ny, int npx, int npy, double x_min, double x_max,
                                double y_min, double y_max, double gamma, double time, int step) {
    auto cfg = config_t{};
    cfg.x_min = x_min;
    cfg.x_max = x_max;
    cfg.y_min = y_min;
    cfg.y_max = y_max;
    cfg.nx_zones = nx;
    cfg.ny_zones = ny;
    cfg.nx_patches = npx;
    cfg.ny_patches = npy;
    cfg.gamma = gamma;
    auto domain = index_space(ivec(0, 0), uvec(nx, ny));
    auto patches = build_periodic_mesh_2d<double>(domain, npx, npy, 4, 2);
    const long long row = ny + 4, plane = (long long)(nx + 4) * row;
    for (auto& patch : patches)
        for (auto idx : patch.interior)
            for (std::size_t k = 0; k < 4; ++k) patch(k, idx) = U[k * plane + (idx[0] + 2) * row + (idx[1] + 2)];
    write_output_2d(patches, cfg, time, step);
    write_xslice(patches, cfg, time, step);
}
