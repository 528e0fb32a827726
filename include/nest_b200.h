/*
 * nest_b200 -- C ABI of the B200-native nest hot path.
 *
 * Plain C: pointers, sizes and status codes only.  Device memory is owned by
 * the library unless an entry point says otherwise; host buffers are owned
 * by the caller.  No entry point throws: failures return a status (or, for
 * the nest-compatible void/pointer functions, are recorded and readable
 * through nest_last_error() / euler1d_gpu_status()).
 *
 * Paths of the form file:line refer to the nest source tree.
 */
#ifndef NEST_B200_H
#define NEST_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status and errors                                                        */
/* ------------------------------------------------------------------------ */

/* nest's C ABI reports CUDA failures by throwing std::runtime_error through
 * extern "C" (src/backend_cuda/euler1d_solver.cu:24-29); here every failure
 * is a status code. */
typedef enum nest_status {
    NEST_OK = 0,
    NEST_ERR_INVALID = 1,     /* bad argument or handle */
    NEST_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    NEST_ERR_OOM = 3,         /* device allocation failed */
    NEST_ERR_NUMERIC = 4,     /* after a step: rho <= 0 or p <= 0 in an interior cell (nest's
                                 positivity check, examples/sod1d/sod1d.cpp:279-301, here after
                                 every step), or a NaN / Inf state; nest_last_error() names the
                                 step and the first failing cell.  The solver stops at that step
                                 (later steps are no-ops) until a new state is uploaded. */
    NEST_ERR_UNSUPPORTED = 6  /* valid request this build does not implement */
} nest_status;

/* Message of the last failing call on the calling thread ("" if none). */
const char* nest_last_error(void);
/* ABI version: major * 10000 + minor * 100 + patch. */
int nest_version(void);

enum { NEST_BC_PERIODIC = 0, NEST_BC_OUTFLOW = 1 };
enum { NEST_F64 = 0, NEST_F32 = 1 };
/* Host/device array layouts for upload/download.
 *   EXTENDED: SoA over the extended space, halos included.  1D: [var][n+2h]
 *             (euler1d_solver.hpp:38-40).  2D: [var][nx+4][ny+4] with the y
 *             index fastest (include/nest/core.hpp:206-215).
 *   INTERIOR: SoA over the interior only: 1D [var][n], 2D [var][nx][ny]. */
enum { NEST_LAYOUT_EXTENDED = 0, NEST_LAYOUT_INTERIOR = 1 };
enum {
    NEST_FLAG_TOTALS = 1,       /* keep FP64 conserved totals each step (2D) */
    NEST_FLAG_REPAIR = 2,       /* FP32 form: FP64 positivity repair near vacuum */
    NEST_FLAG_NO_RESIDENT = 4,  /* 1D: never use the single-CTA resident solver */
    NEST_FLAG_FP32_SCALAR = 8,  /* FP32 form: one column per lane instead of packed FP32x2 pairs */
    NEST_FLAG_SPLIT_COMPAT = 16, /* 2D FP64: nest's own dimensionally split forward-Euler sweeps
                                   (examples/sod2d/euler2d.hpp:67-271) instead of unsplit RK2 */
    NEST_FLAG_LIMITER_MC = 32,   /* slope limiter: monotonized central (mc_limiter, euler1d.hpp:117-125) */
    NEST_FLAG_LIMITER_NONE = 64  /* slope limiter: none, 0.5 (left + right) (apply_limiter, euler1d.hpp:127-137);
                                    default minmod.  The packed FP32 kernel is minmod-only: FP32 solvers
                                    with another limiter run the one-column-per-lane kernel. */
};

/* ------------------------------------------------------------------------ */
/* Drop-in: nest's 1D CUDA solver ABI                                       */
/* Same names, signatures, SoA-with-halo host layout and periodic boundary  */
/* as src/backend_cuda/euler1d_solver.hpp:16-87.                            */
/* ------------------------------------------------------------------------ */

typedef struct euler1d_gpu_t euler1d_gpu_t;

/* euler1d_solver.hpp:27.  NULL on failure (see nest_last_error()). */
euler1d_gpu_t* euler1d_gpu_create(int n_interior, int n_halo, double dx, double gamma);
/* euler1d_solver.hpp:32. */
void euler1d_gpu_destroy(euler1d_gpu_t* solver);
/* euler1d_solver.hpp:41: h_data is SoA [var * n_total + i], n_total = n_interior + 2 n_halo. */
void euler1d_gpu_upload(euler1d_gpu_t* solver, const double* h_data);
/* euler1d_solver.hpp:49. */
void euler1d_gpu_download(euler1d_gpu_t* solver, double* h_data);
/* euler1d_solver.hpp:58: cfl * dx / max(|u| + c) over the interior. */
double euler1d_gpu_compute_dt(euler1d_gpu_t* solver, double cfl);
/* euler1d_solver.hpp:66: one Heun step with the given dt. */
void euler1d_gpu_rk2_step(euler1d_gpu_t* solver, double dt);
/* euler1d_solver.hpp:76: run from time 0 until t_final; returns the step count (-1 on error). */
int euler1d_gpu_run(euler1d_gpu_t* solver, double t_final, double cfl);
/* euler1d_solver.hpp:87: as run, returns wall-clock milliseconds. */
double euler1d_gpu_run_timed(euler1d_gpu_t* solver, double t_final, double cfl, int* steps);

/* Extensions on the same handle (no counterpart in nest's ABI). */
nest_status euler1d_gpu_set_bc(euler1d_gpu_t* solver, int bc);
/* Status of the last call made on this handle. */
nest_status euler1d_gpu_status(euler1d_gpu_t* solver);

/* ------------------------------------------------------------------------ */
/* Solver API: 1D / 2D, FP64 plain or FP32 form, one domain per handle.     */
/* Replaces the time loops of examples/benchmark/benchmark_euler1d.cpp:     */
/* 185-209 and examples/sod2d/sod2d.cpp:318-366 on the device.  A step is   */
/* dt (CFL max-reduction on the device) -> ghost fill -> stage 1 -> ghost   */
/* fill -> stage 2 + Heun average, with no host synchronisation.            */
/* ------------------------------------------------------------------------ */

typedef struct nest_solver nest_solver;

typedef struct nest_solver_desc {
    int dim;          /* 1 or 2 */
    int nx, ny;       /* interior cells (ny unused for dim 1) */
    int halo;         /* ghost width: 2 (dim 1 accepts >= 2) */
    double dx, dy;    /* cell sizes (dy unused for dim 1) */
    double gamma;
    int bc_x, bc_y;   /* NEST_BC_* */
    int precision;    /* NEST_F64 or NEST_F32 (dim 2 only) */
    int flags;        /* NEST_FLAG_* */
    void* stream;     /* cudaStream_t to run on, or NULL for a private stream */
} nest_solver_desc;

nest_status nest_solver_create(const nest_solver_desc* desc, nest_solver** out);
nest_status nest_solver_destroy(nest_solver* s);
/* Host arrays are in the solver precision (double for F64, float for F32). */
nest_status nest_solver_upload(nest_solver* s, const void* host, int layout);
nest_status nest_solver_download(nest_solver* s, void* host, int layout);
/* Same with a device pointer (e.g. a torch tensor); no host staging. */
nest_status nest_solver_upload_device(nest_solver* s, const void* dev, int layout);
nest_status nest_solver_download_device(nest_solver* s, void* dev, int layout);
/* Enqueue nsteps steps with CFL dt; returns without waiting. */
nest_status nest_solver_step(nest_solver* s, int nsteps, double cfl);
/* nsteps CFL steps launched one kernel at a time with a CUDA event between
 * kernels on the solver stream (no graph); waits.  stage_ms (2*nsteps, may be
 * NULL) receives each kernel's duration in launch order, total_ms the span. */
nest_status nest_solver_step_profiled(nest_solver* s, int nsteps, double cfl, float* stage_ms, float* total_ms);
/* Enqueue nsteps steps with a fixed dt (nest's rk2_step(dt)). */
nest_status nest_solver_step_dt(nest_solver* s, int nsteps, double dt);
/* Advance until time >= t_final (dt clamped to hit it) or max_steps (> 0)
 * more steps; waits.  *steps_out = steps taken by this call. */
nest_status nest_solver_run_to(nest_solver* s, double t_final, double cfl, int max_steps, int* steps_out);
/* dt = CFL rule on the current state (waits). */
nest_status nest_solver_compute_dt(nest_solver* s, double cfl, double* dt_out);
/* Simulated time and completed steps since creation / last reset (waits). */
nest_status nest_solver_time(nest_solver* s, double* time, int* steps);
nest_status nest_solver_reset_time(nest_solver* s);
/* FP64 conserved totals of the state after the last step (2D, needs
 * NEST_FLAG_TOTALS): sum of rho, rho u, rho v, E over the interior times dx dy. */
nest_status nest_solver_totals(nest_solver* s, double out[4]);
/* Number of cells repaired by the FP32 form so far. */
nest_status nest_solver_repairs(nest_solver* s, unsigned* count);
nest_status nest_solver_sync(nest_solver* s);
/* 2D launch shape: rows per tile and warps per block (autotuner hook). */
nest_status nest_solver_set_tiling(nest_solver* s, int rows_per_tile, int warps_per_block);
/* dt sequence: mode 0 freezes the given n values (copied), mode 1 records the
 * next n dts (read back with nest_solver_get_dts), mode 2 clears. */
nest_status nest_solver_set_dt_sequence(nest_solver* s, const double* dts, int n, int mode);
nest_status nest_solver_get_dts(nest_solver* s, double* dts, int n);
/* Sharded domains (x-slabs on several GPUs).  xlo / xhi = 1 marks an x side
 * whose two ghost rows a halo exchange fills: the kernels then neither write
 * nor derive them.  Steps are driven stage by stage: before stage 1 the caller
 * max-reduces the two wave-speed words of nest_solver_speed_slot across ranks
 * (uint64 bit patterns of non-negative doubles, MAX) and fills the exchange
 * ghost rows of the state (nest_solver_state_ptr); before stage 2 those of
 * the stage buffer (nest_solver_stage_ptr, same pitch and plane stride).
 * Row i of plane v starts at element v * vstride + (i + 2) * pitch. */
nest_status nest_solver_set_exchange_sides(nest_solver* s, int xlo, int xhi);
/* Enqueue one stage (1 or 2) of the current step; stage 2 ends the step.
 * t_final > 0 clips dt to reach it; a step that would start at or past it is a no-op. */
nest_status nest_solver_stage(nest_solver* s, int which, double cfl, double t_final);
/* Device address of the current step's two wave-speed words. */
nest_status nest_solver_speed_slot(nest_solver* s, void** dev);
nest_status nest_solver_stage_ptr(nest_solver* s, void** dev);
nest_status nest_solver_stream(nest_solver* s, void** stream);
/* Device state: base pointer, row pitch (elements) and plane stride (elements). */
nest_status nest_solver_state_ptr(nest_solver* s, void** dev, long long* pitch, long long* vstride);

/* ------------------------------------------------------------------------ */
/* Several GPUs: the x-slab step loop in C++ with NCCL.                     */
/* One rank per GPU holds one x-slab solver (nest_solver_set_exchange_sides */
/* marks its cut sides).  nest_slab_step enqueues, per step and on the      */
/* solver's stream: a MAX all-reduce of the two wave-speed words, the two   */
/* ghost rows of each cut side from the neighbour ranks (NCCL send / recv,  */
/* one message per variable plane and side), stage 1, the same exchange of  */
/* the stage buffer, stage 2 (nest's exchange-before-each-stage, examples/  */
/* sod2d/sod2d.cpp:331-362); runs of 16 steps are replayed from captured    */
/* CUDA graphs; it returns without waiting.  lo / hi: neighbour ranks, -1   */
/* for a domain boundary (a rank can be its own neighbour).  NCCL is loaded */
/* at run time; NEST_ERR_UNSUPPORTED if it is absent.  Destroy solvers (or  */
/* the communicator) before tearing the process group down: their graphs   */
/* hold NCCL calls.                                                         */
/* ------------------------------------------------------------------------ */
typedef struct nest_slab_comm nest_slab_comm;
/* Rank 0 makes the communicator id (128 bytes) and sends it to the others. */
nest_status nest_slab_comm_id(unsigned char id[128]);
nest_status nest_slab_comm_create(const unsigned char id[128], int nranks, int rank, nest_slab_comm** out);
nest_status nest_slab_comm_destroy(nest_slab_comm* c);
nest_status nest_slab_step(nest_solver* s, nest_slab_comm* c, int lo, int hi, int nsteps, double cfl,
                           double t_final);

/* ------------------------------------------------------------------------ */
/* Batched independent 2D problems (uneven sizes).  One persistent launch   */
/* per stage walks a device work list of (problem, column strip, row tile); */
/* each problem keeps its own dt, time and FP64 totals; runs of steps are   */
/* captured into CUDA graphs.  No counterpart in nest (its patches are      */
/* advanced by serial host loops, examples/sod2d/sod2d.cpp:318-366).        */
/* ------------------------------------------------------------------------ */

typedef struct nest_batch nest_batch;

typedef struct nest_batch_desc {
    int count;            /* number of problems */
    const int* nx;        /* [count] interior cells along x */
    const int* ny;        /* [count] interior cells along y */
    const double* dx;     /* [count] or NULL: 1/nx */
    const double* dy;     /* [count] or NULL: 1/ny */
    double gamma;
    int bc_x, bc_y;       /* NEST_BC_*, shared by all problems */
    int precision;        /* NEST_F64 (bit-exact per problem) or NEST_F32 (packed FP32x2) */
    int flags;            /* NEST_FLAG_TOTALS, NEST_FLAG_REPAIR */
    void* stream;
} nest_batch_desc;

nest_status nest_batch_create(const nest_batch_desc* desc, nest_batch** out);
nest_status nest_batch_destroy(nest_batch* b);
/* One problem's state, in the batch precision and the solver layouts. */
nest_status nest_batch_upload(nest_batch* b, int problem, const void* host, int layout);
nest_status nest_batch_download(nest_batch* b, int problem, void* host, int layout);
/* Enqueue nsteps steps of every problem (CFL dt per problem); returns without waiting. */
nest_status nest_batch_step(nest_batch* b, int nsteps, double cfl);
/* As nest_batch_step with a CUDA event between kernels; waits (see nest_solver_step_profiled). */
nest_status nest_batch_step_profiled(nest_batch* b, int nsteps, double cfl, float* stage_ms, float* total_ms);
/* Per-problem simulated time and step count (waits). */
nest_status nest_batch_times(nest_batch* b, double* times, int* steps);
/* Per-problem FP64 totals [count][4] after the last step (needs NEST_FLAG_TOTALS). */
nest_status nest_batch_totals(nest_batch* b, double* out);
/* Launch shape: rows per work item, warps per block, blocks per SM (0 = occupancy limit). */
nest_status nest_batch_set_tiling(nest_batch* b, int rows_per_tile, int warps_per_block, int blocks_per_sm);
/* Zero every problem's time, step count and error word (states are kept;
 * ghost rings and wave speeds are rebuilt before the next step). */
nest_status nest_batch_reset(nest_batch* b);
/* Total interior cells, work items and persistent blocks. */
nest_status nest_batch_info(nest_batch* b, long long* cells, int* items, int* blocks);

/* ------------------------------------------------------------------------ */
/* Patch halo exchange on nest's per-patch storage (device).                */
/* Plan = build_periodic_mesh_1d / _2d (include/nest/patch.hpp:88-147,      */
/* 207-326); execute = execute_all_exchanges (patch.hpp:153-190) in one     */
/* kernel launch.  Patches are stored one after another in patch order,     */
/* each as nvars SoA planes over its extended space, idx[1] fastest.        */
/* ------------------------------------------------------------------------ */
typedef struct nest_exchange nest_exchange;
/* dim 1: nx cells in npx patches (ny, npy ignored); dim 2: nx x ny in npx x npy. */
nest_status nest_exchange_create_periodic(int dim, int nx, int ny, int npx, int npy, int nvars, int halo,
                                          nest_exchange** out);
nest_status nest_exchange_destroy(nest_exchange* x);
/* Element offset of each patch block (npatches + 1 values), interior boxes
 * (start0, start1, shape0, shape1 per patch) and the peer of every region
 * (2 per patch in 1D, 4 in 2D, in nest's order); any pointer may be NULL. */
nest_status nest_exchange_layout(nest_exchange* x, long long* offsets, int* boxes, int* peers);
/* Fill every patch's face halos from its periodic neighbours (device data). */
nest_status nest_exchange_execute(nest_exchange* x, void* d_data, int precision, void* stream);

/* ------------------------------------------------------------------------ */
/* Device pipeline executor over nest's per-patch storage (FP64).           */
/* Replaces nest's pipeline_t / execute (include/nest/pipeline.hpp:14-151)  */
/* and the host stage loops of examples/sod1d/sod1d.cpp:219-302: a pipeline */
/* is a list of stages, each one launch over every patch; execute() runs    */
/* them once in order, run() repeats them until time >= t_final with the   */
/* steps replayed from CUDA graphs.  The storage is the exchange plan's     */
/* (nest_pipeline_plan: patches one after another, nvars SoA planes over    */
/* each patch's extended space).  Buffers: 0 = the caller's device state,   */
/* 1..nwork = work arrays the pipeline owns, of the same layout.            */
/*   EXCHANGE   halos of buffer src (nest's fill_all_halos)                 */
/*   EULER_RHS  compute: dst = src - (dt/dx) (F_{i+1/2} - F_{i-1/2}) on the */
/*              interiors, nest's euler_rhs_t (examples/sod1d/euler1d.hpp:  */
/*              279-397) with its one-sided patch edges; 1D                 */
/*   COPY       compute: dst = src on the interiors                         */
/*   AVERAGE    compute: dst = 0.5 src + 0.5 aux on the interiors           */
/*   CFL_DT     reduce: init 0, max |u| + c over each interior of src,      */
/*              finalize dt = param * dx / max, clipped to t_final - time   */
/*              (compute_dt, sod1d.cpp:97-128); during run() a step that    */
/*              starts at or past t_final does nothing; 1D                  */
/*   CHECK      nest's positivity check (sod1d.cpp:279-301) of src when the */
/*              step in progress is a multiple of param; place it before    */
/*              CLOCK; failures surface as NEST_ERR_NUMERIC; 1D             */
/*   CLOCK      time += dt, step += 1                                       */
/* dt, time and the step count stay on the device (nest_pipeline_clock).   */
/* ------------------------------------------------------------------------ */
enum {
    NEST_STAGE_EXCHANGE = 1, NEST_STAGE_EULER_RHS = 2, NEST_STAGE_COPY = 3, NEST_STAGE_AVERAGE = 4,
    NEST_STAGE_CFL_DT = 5, NEST_STAGE_CHECK = 6, NEST_STAGE_CLOCK = 7
};
typedef struct nest_pipeline nest_pipeline;
/* Patch grid as nest_exchange_create_periodic; limiter 0 minmod, 1 MC, 2 none
 * (limiter_t, euler1d.hpp:106-137); nwork work buffers (0..16). */
nest_status nest_pipeline_create(int dim, int nx, int ny, int npx, int npy, int halo, double dx, double gamma,
                                 int limiter, int nwork, nest_pipeline** out);
nest_status nest_pipeline_destroy(nest_pipeline* p);
/* The pipeline's exchange plan (layout queries; owned by the pipeline). */
nest_status nest_pipeline_plan(nest_pipeline* p, nest_exchange** plan);
nest_status nest_pipeline_add(nest_pipeline* p, int kind, int src, int dst, int aux, double param);
/* All stages once, in order, enqueued on `stream` (NULL: the pipeline's own). */
nest_status nest_pipeline_execute(nest_pipeline* p, void* d_state, void* stream);
/* Execute until time >= t_final (needs a CFL_DT stage) or max_steps (> 0)
 * more steps; waits.  *steps_out = steps taken. */
nest_status nest_pipeline_run(nest_pipeline* p, void* d_state, double t_final, int max_steps, int* steps_out,
                              void* stream);
/* Clock (waits; NEST_ERR_NUMERIC after a failed CHECK). */
nest_status nest_pipeline_clock(nest_pipeline* p, double* time, double* dt, int* step);
nest_status nest_pipeline_set_clock(nest_pipeline* p, double time, double dt, int step);
/* Device address of work buffer `index` (1..nwork). */
nest_status nest_pipeline_buffer(nest_pipeline* p, int index, void** dev);

/* ------------------------------------------------------------------------ */
/* Discrete adjoint with checkpointing.  No counterpart in nest.            */
/* The forward sweep runs the solver from its current state for nsteps with */
/* CFL dt (recorded) or a given dt sequence; the backward sweep maps the    */
/* adjoint of the final state to the adjoint of the initial state with the  */
/* same frozen dts.  Memory is bounded by checkpoint-and-recompute:         */
/*   NEST_CKPT_UNIFORM  param = K: a checkpoint every K steps;              */
/*   NEST_CKPT_BINOMIAL param = s: s snapshot slots, binomial schedule.     */
/* Adjoint arrays use the solver's device layout (1D: [3][n + 2h]); on      */
/* device or host memory.  This build: 1D FP64, periodic.                   */
/* ------------------------------------------------------------------------ */
enum { NEST_CKPT_UNIFORM = 0, NEST_CKPT_BINOMIAL = 1 };
typedef struct nest_adjoint nest_adjoint;
/* The adjoint object refers to its solver: destroy it before the solver, or
 * after (destroy never touches the solver). */
nest_status nest_adjoint_create(nest_solver* s, int nsteps, int policy, int param, nest_adjoint** out);
nest_status nest_adjoint_destroy(nest_adjoint* a);
/* dts: NULL for CFL dt (recorded), else nsteps frozen values. */
nest_status nest_adjoint_forward(nest_adjoint* a, double cfl, const double* dts);
nest_status nest_adjoint_backward(nest_adjoint* a, const void* lam_final, void* lam_initial, int on_device);
nest_status nest_adjoint_get_dts(nest_adjoint* a, double* dts);
/* Wall-clock ms of the two sweeps, forward steps recomputed by the backward
 * sweep, and device bytes held for checkpoints and work buffers. */
nest_status nest_adjoint_stats(nest_adjoint* a, double* fwd_ms, double* bwd_ms, long long* recomputed_steps,
                               long long* snapshot_bytes);

/* ------------------------------------------------------------------------ */
/* Self-test of the FP64 stage kernels' checked division.  No counterpart   */
/* in nest.  For n pairs (device arrays), q[i] = the fast quotient of       */
/* a[i] / b[i] and ok[i] = 1 where the kernels accept it as the correctly   */
/* rounded IEEE quotient (0 where they fall back to the IEEE division).     */
/* Enqueued on the legacy stream; synchronises before returning.            */
/* ------------------------------------------------------------------------ */
nest_status nest_selftest_div_f64(const double* d_a, const double* d_b, double* d_q, int* d_ok, int n);

/* ------------------------------------------------------------------------ */
/* Allocation-free 1D run.  No counterpart in nest's ABI.                   */
/*                                                                          */
/* For callers that cannot allocate device memory (a host code that owns    */
/* the whole GPU through its own pool, a plugin host that forbids library   */
/* allocations, a real-time loop that must not allocate after start-up).    */
/* The caller passes the state; the solver's scratch (a second state buffer */
/* and the control block) is a fixed array inside the library, so this call */
/* makes no cudaMalloc / cudaFree.  The array holds n_interior + 2*n_halo   */
/* <= NEST_NOALLOC_MAX_CELLS cells (about 1.6 MB, held by every GPU that    */
/* loads the library until exit); larger sizes return NEST_ERR_INVALID.     */
/* Every call looks up the array's address in the current device's context  */
/* and waits for its stream (it reads the step count back every 32 steps).  */
/* All calls share the array: calls that overlap on the GPU race.           */
/* The array reaches device memory with the library's code module, which    */
/* CUDA loads into a context on first use (with the default lazy module     */
/* loading, at the first call of this function there): a caller that must   */
/* not allocate after start-up makes its first call during start-up.        */
/*                                                                          */
/* d_state: device SoA [var * n_total + i], n_total = n_interior + 2 n_halo */
/* (nest's layout), advanced in place from time 0 to t_final with CFL dt,   */
/* periodic or outflow boundaries, on `stream` (NULL: legacy stream); waits */
/* for the result.  Same arithmetic as euler1d_gpu_run (bit for bit).       */
/* ------------------------------------------------------------------------ */
#define NEST_NOALLOC_MAX_CELLS 65552
nest_status nest_euler1d_run_noalloc(double* d_state, int n_interior, int n_halo, double dx, double gamma,
                                     int bc, double t_final, double cfl, int* steps_out, double* time_out,
                                     void* stream);

/* ------------------------------------------------------------------------
 * On-disk formats.
 * nest's text snapshots, byte for byte the files its examples write for the
 * same state and patch grid (replace write_output, examples/sod1d/sod1d.cpp:
 * 50-91; write_output_2d and write_xslice, examples/sod2d/sod2d.cpp:58-152).
 * U is a host array in the extended layout: 1D [3][n + 2 halo], 2D
 * [4][nx + 4][ny + 4]; npatch / npx x npy is the patch grid that sets the
 * order of the lines.  xslice = 1 writes the row j = ny / 2 sorted by x.
 * ------------------------------------------------------------------------ */
nest_status nest_write_dat_1d(const char* path, const double* U, int n, int halo, int npatch, double x_min,
                              double x_max, double gamma, double time);
nest_status nest_write_dat_2d(const char* path, const double* U, int nx, int ny, int npx, int npy, double x_min,
                              double x_max, double y_min, double y_max, double gamma, double time, int xslice);
/* The solver's current state and time (downloads; FP32 states are widened). */
nest_status nest_solver_write_dat(nest_solver* s, const char* path, int npx, int npy, double x_min, double x_max,
                                  double y_min, double y_max, int xslice);
/* Restartable binary checkpoint (nest has none): state, time and step count,
 * checksummed; loading into a solver of the same sizes, precision, boundary
 * conditions, gamma and spacing continues the run bit for bit. */
nest_status nest_solver_save(nest_solver* s, const char* path);
nest_status nest_solver_load(nest_solver* s, const char* path);
/* Set the solver clock (time, completed steps). */
nest_status nest_solver_set_time(nest_solver* s, double time, int steps);


#ifdef __cplusplus
}
#endif

#endif /* NEST_B200_H */
