// Shared device definitions for the nest B200 kernels.
//
// Precision policy
//   double : the plain form.  Every translation unit that instantiates it is
//            compiled with -fmad=false and IEEE division / square root, and
//            the formulas below keep the operation order of nest's CPU code
//            (examples/sod1d/euler1d.hpp), so results match the CPU path bit
//            for bit.
//   float  : the FP32 form (reconstruction, Riemann solve and update in
//            FP32; totals, time and positivity repair in FP64).  Its
//            translation unit is compiled with FMA contraction and fast
//            reciprocal / square-root approximations.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace nestb {

// Programmatic dependent launch (sm_90 and later).  A kernel launched by
// launch_pdl may be scheduled while the kernel before it in the stream is
// still running: pdl_wait() returns once that kernel has completed and its
// memory is visible (immediately for an ordinary launch), so nothing is read
// before it; pdl_trigger() then lets the next such kernel be scheduled,
// which hides its launch and block start-up behind this kernel's run.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Boundary conditions on the domain edges.
enum { BC_PERIODIC = 0, BC_OUTFLOW = 1 };

// Device error word bits (read back by the host after a run).  A step that
// starts with either bit set does not run: the state stays as the failing
// step left it.
enum : unsigned {
    ERRW_NONFINITE = 1u,   // a wave speed, density or pressure was NaN / Inf
    ERRW_NONPOSITIVE = 2u, // rho <= 0 or p <= 0 in an interior cell after a step
};
constexpr unsigned ERRW_STOP = ERRW_NONFINITE | ERRW_NONPOSITIVE;

// Per-solver control block in device memory.  Fields indexed [p] belong to
// the step launched with parity p; a step with parity p reads slot p and
// prepares slot 1-p, so the two kernels of a step never race on a field.
struct StepCtrl {
    double time[2];                 // simulated time at the start of the step
    double dt[2];                   // dt chosen by stage 1 of the step
    unsigned long long maxs[2][2];  // [p][axis] max wave speed of U at the start of step p (bits of a non-negative double)
    int step[2];                    // completed steps at the start of the step
    int active[2];                  // stage 1 sets it: 1 = the step runs, 0 = finished
    unsigned repairs;               // FP32 form: number of repaired cells
    // error record (cleared by an upload; the fields from `err` on)
    unsigned err;                   // ERRW_* bits
    int bad_step;                   // first failing cell: steps completed when it was found (0: none recorded),
    int bad_i, bad_j;               // its interior index (1D: bad_j = 0)
    int pad_;
    double bad_rho, bad_p;          // and its density and pressure
    // one-launch 1D steps: blocks of the running step that have added their
    // wave speed to maxs[q][1] (the last one moves the maximum to maxs[q][0],
    // clears maxs[q][1] and resets this count)
    unsigned blocks_done;
    unsigned pad2_;
};

// Time-loop parameters shared by all launches of a solver.
struct LoopParams {
    double cfl;
    double t_final;        // > 0: stop when time >= t_final and clamp dt
    int max_steps;         // > 0: stop after this many steps
    const double* dts_in;  // frozen dt sequence (adjoint forward) or null
    double* dts_out;       // records the dt of every step, or null
    int dts_cap;           // capacity of dts_in / dts_out
    double fixed_dt;       // > 0: every step uses this dt (nest's rk2_step(dt))
    int step_budget;       // resident 1D kernel: > 0 = at most this many steps per launch
    int lim;               // slope limiter: LIM_MINMOD, LIM_MC or LIM_NONE
};

enum { LIM_MINMOD = 0, LIM_MC = 1, LIM_NONE = 2 };

// std::min / std::max semantics (first argument wins ties).
template <typename T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

__device__ __forceinline__ unsigned long long speed_bits(double s) {
    return (unsigned long long)__double_as_longlong(s);
}
__device__ __forceinline__ double bits_speed(unsigned long long b) {
    return __longlong_as_double((long long)b);
}

// Max over non-negative doubles: their IEEE bit patterns order like the values.
__device__ __forceinline__ void atomic_max_speed(unsigned long long* slot, double s) {
    atomicMax(slot, speed_bits(s));
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// nest's positivity check (examples/sod1d/sod1d.cpp:279-301: rho <= 0 or
// p <= 0 in an interior cell is an error) runs on every cell after every
// step (nest: every 10th step).  The kernels test !(rho > 0) || !(p > 0),
// which a NaN fails too, and call this on the rare failing path: the bit is
// ERRW_NONFINITE for a NaN, else ERRW_NONPOSITIVE, and the first failing
// cell records the step (`step_done` = steps completed, this one included),
// its interior index and its values.
__device__ __forceinline__ void flag_cell(StepCtrl* c, int step_done, double rho, double pr, int i, int j) {
    const unsigned bit = (rho == rho && pr == pr) ? ERRW_NONPOSITIVE : ERRW_NONFINITE;
    if (atomicOr(&c->err, bit) & ERRW_STOP) return;  // an earlier cell holds the record
    c->bad_step = step_done;
    c->bad_i = i;
    c->bad_j = j;
    c->bad_rho = rho;
    c->bad_p = pr;
}

// Decide the step: returns false when the run is finished.  Every block of
// stage 1 evaluates this on the same inputs, so all agree; block 0 publishes.
__device__ __forceinline__ bool step_is_done(const StepCtrl* c, int p, const LoopParams& lp) {
    if (c->err & ERRW_STOP) return true;
    double t = c->time[p];
    int s = c->step[p];
    if (lp.t_final > 0.0 && !(t < lp.t_final)) return true;
    if (lp.max_steps > 0 && s >= lp.max_steps) return true;
    if (lp.dts_in && s >= lp.dts_cap) return true;
    return false;
}

// dt of the step in slot p when it is not derived from the CFL condition:
// a frozen sequence or a caller-given constant.  Returns a negative value
// when the CFL rule applies.
__device__ __forceinline__ double prescribed_dt(const StepCtrl* c, int p, const LoopParams& lp) {
    if (lp.fixed_dt > 0.0) return lp.fixed_dt;
    if (lp.dts_in) return lp.dts_in[c->step[p]];
    return -1.0;
}

// Block 0 / thread 0 of stage 1: publish dt and prepare the next slot.
// clear_next = false in a one-launch 1D step, whose other blocks may already
// be adding to slot q (its last block writes maxs[q][0]).
__device__ __forceinline__ void publish_step(StepCtrl* c, int p, const LoopParams& lp, bool done, double dt,
                                             bool clear_next = true) {
    int q = p ^ 1;
    if (done) {
        c->active[p] = 0;
        c->time[q] = c->time[p];
        c->step[q] = c->step[p];
        c->maxs[q][0] = c->maxs[p][0];
        c->maxs[q][1] = c->maxs[p][1];
        c->active[q] = 0;
        return;
    }
    c->active[p] = 1;
    c->dt[p] = dt;
    c->time[q] = c->time[p] + dt;
    c->step[q] = c->step[p] + 1;
    if (clear_next) {
        c->maxs[q][0] = 0ull;
        c->maxs[q][1] = 0ull;
    }
    int s = c->step[p];
    if (lp.dts_out && s < lp.dts_cap) lp.dts_out[s] = dt;
}

// ---------------------------------------------------------------------------
// 1D numerics (3 variables), examples/sod1d/euler1d.hpp
// ---------------------------------------------------------------------------

// eos_t::pressure, euler1d.hpp:31-44.  T = double is the plain form (IEEE
// division, nest's operation order); T = float the FP32 form.
template <typename T>
__device__ __forceinline__ T eos_pressure(T gm1, T rho, T mom, T erg) {
    T u = mom / rho;
    T ke = T(0.5) * rho * u * u;
    T p = gm1 * (erg - ke);
    return smax(p, T(0));
}

// minmod, euler1d.hpp:112-115.
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {
    if (a * b <= T(0)) return T(0);
    return (fabs(a) < fabs(b)) ? a : b;
}

// apply_limiter, euler1d.hpp:127-137 (mc_limiter = minmod3(2a, (a+b)/2, 2b),
// euler1d.hpp:117-125).  `lim` is uniform across a launch.
template <typename T>
__device__ __forceinline__ T limit(T a, T b, int lim) {
    if (lim == LIM_MINMOD) return minmod(a, b);
    if (lim == LIM_MC) {
        T c = T(0.5) * (a + b);
        return minmod(T(2) * a, minmod(c, T(2) * b));
    }
    return T(0.5) * (a + b);
}

// hlle_flux, euler1d.hpp:178-242 (Davis speeds, three branches).
template <typename T>
__device__ __forceinline__ void hlle1d(T gamma, T gm1, T rL, T uL, T pL, T rR, T uR, T pR, T& f0, T& f1, T& f2) {
    T cL = sqrt(gamma * pL / rL);
    T EL = pL / gm1 + T(0.5) * rL * uL * uL;
    T cR = sqrt(gamma * pR / rR);
    T ER = pR / gm1 + T(0.5) * rR * uR * uR;
    T SL = smin(uL - cL, uR - cR);
    T SR = smax(uL + cL, uR + cR);
    T FL0 = rL * uL, FL1 = rL * uL * uL + pL, FL2 = (EL + pL) * uL;
    T FR0 = rR * uR, FR1 = rR * uR * uR + pR, FR2 = (ER + pR) * uR;
    if (SL >= T(0)) {
        f0 = FL0; f1 = FL1; f2 = FL2;
    } else if (SR <= T(0)) {
        f0 = FR0; f1 = FR1; f2 = FR2;
    } else {
        T SLR = SL * SR, dS = SR - SL;
        f0 = (SR * FL0 - SL * FR0 + SLR * (rR - rL)) / dS;
        f1 = (SR * FL1 - SL * FR1 + SLR * (rR * uR - rL * uL)) / dS;
        f2 = (SR * FL2 - SL * FR2 + SLR * (ER - EL)) / dS;
    }
}

}  // namespace nestb
