// CPU half of nest's CPU-vs-GPU test as a callable function -- TEST
// INFRASTRUCTURE ONLY.  tests/test_euler_cuda.cpp is compiled where it lies;
// main() is renamed, and the nest C-ABI names its GPU half refers to are
// renamed to local stubs that are never called.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define euler1d_gpu_create ref_stub_gpu_create
#define euler1d_gpu_destroy ref_stub_gpu_destroy
#define euler1d_gpu_upload ref_stub_gpu_upload
#define euler1d_gpu_download ref_stub_gpu_download
#define euler1d_gpu_compute_dt ref_stub_gpu_compute_dt
#define euler1d_gpu_rk2_step ref_stub_gpu_rk2_step
#define euler1d_gpu_run ref_stub_gpu_run
#define euler1d_gpu_run_timed ref_stub_gpu_run_timed
#define main nest_ref_cudatest_main
#include "test_euler_cuda.cpp"
#undef main

extern "C" {
euler1d_gpu_t* ref_stub_gpu_create(int, int, double, double) { return nullptr; }
void ref_stub_gpu_destroy(euler1d_gpu_t*) {}
void ref_stub_gpu_upload(euler1d_gpu_t*, const double*) {}
void ref_stub_gpu_download(euler1d_gpu_t*, double*) {}
double ref_stub_gpu_compute_dt(euler1d_gpu_t*, double) { return 0.0; }
void ref_stub_gpu_rk2_step(euler1d_gpu_t*, double) {}
int ref_stub_gpu_run(euler1d_gpu_t*, double, double) { return 0; }
double ref_stub_gpu_run_timed(euler1d_gpu_t*, double, double, int* s) { if (s) *s = 0; return 0.0; }

// run_cpu_sod (tests/test_euler_cuda.cpp:49-185) with its periodic Sod
// set-up; U_out receives 3*(n+4) doubles (SoA with halos).
void ref_run_cpu_sod(int n_zones, double t_final, double cfl, double* U_out) {
    test_config_t cfg;
    cfg.n_zones = n_zones;
    cfg.t_final = t_final;
    cfg.cfl = cfl;
    std::vector<double> U;
    run_cpu_sod(cfg, U);
    for (std::size_t i = 0; i < U.size(); ++i) U_out[i] = U[i];
}
}
