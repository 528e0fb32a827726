// nest's OpenMP Sod benchmark as a callable function -- TEST INFRASTRUCTURE ONLY.
// examples/benchmark/benchmark_euler1d.cpp is compiled where it lies in the
// nest source tree; its main() is renamed so ctypes can call benchmark_cpu().
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define main nest_ref_benchmark_main
#include "benchmark/benchmark_euler1d.cpp"
#undef main

extern "C" {
// benchmark_cpu() (benchmark_euler1d.cpp:90-221) with nest's own Sod set-up,
// loop and wall-clock timing.  Returns milliseconds.
double ref_benchmark_cpu(int n_zones, double t_final, int* steps, double* cells_per_sec) {
    bench_config_t cfg;
    cfg.n_zones = n_zones;
    cfg.t_final = t_final;
    auto r = benchmark_cpu(cfg);
    if (steps) *steps = r.steps;
    if (cells_per_sec) *cells_per_sec = r.cells_per_sec;
    return r.time_ms;
}
}
