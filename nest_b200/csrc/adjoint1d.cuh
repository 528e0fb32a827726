// Discrete adjoint of the 1D fused stage, sm_100a, templated on the
// arithmetic type: double (adjoint1d.cu, IEEE arithmetic) and float
// (adjoint1d_f32.cu, fast reciprocal / square root) for the FP32 form.
//
// Forward stage (nest's OpenMP path, examples/benchmark/benchmark_euler1d.cpp:113-165):
//   W_c   = prim(U_c)                          (euler1d.hpp:69-84, p clamped at 0)
//   s_c   = minmod(W_c - W_{c-1}, W_{c+1} - W_c)
//   F_f   = HLLE(W_a + s_a/2, W_b - s_b/2)     (face f between cells a = b-1 and b)
//   U'_i  = U_i - lambda (F_{i+1/2} - F_{i-1/2}),  lambda = dt/dx (dt read from device memory)
// Adjoint (dt frozen), for a given adjoint Ubar' of the stage output:
//   Fbar_f   = lambda (Ubar'_b - Ubar'_a)
//   WLbar_f, WRbar_f = HLLE Jacobians^T Fbar_f   (branch of the forward: S_L >= 0,
//              S_R <= 0 or the HLLE average, with the active argument of each Davis min/max)
//   sbar_c   = WLbar_{c+1/2}/2 - WRbar_{c-1/2}/2
//   Wbar_i   = WRbar_{i-1/2} + WLbar_{i+1/2}
//              + sbar_i ([d1 active] - [d2 active]) + sbar_{i-1} [d2 active at i-1]
//              - sbar_{i+1} [d1 active at i+1]          (minmod subgradient; 0 if d1 d2 <= 0)
//   Ubar_i   = Ubar'_i + (dW/dU)_i^T Wbar_i
// Each thread gathers one cell (no atomics).  Periodic indices wrap modulo n,
// which is exactly the transpose of the periodic ghost fill
// (benchmark_euler1d.cpp:102-110): a ghost cell's adjoint lands on its source.
// A Heun step reverses both stages in one launch (k1d_adjoint_step): the
// stage-2 adjoint of the CTA's cells and a two-cell halo stays in shared
// memory and feeds the stage-1 reverse.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace nestb {
namespace {

constexpr int TA = 112;       // cells per CTA (586 CTAs at 65536 cells: at most 4 per SM, 448 cells)
constexpr int NTA = TA + 10;  // threads per CTA: one per cell of the widest phase (TA + 4 outputs + 6)

template <typename T>
struct St3 { T r, u, p; };

// Reverse of hlle1d (common.cuh) for one face: accumulates Wbar of the left
// and right face states for the flux adjoint fb.
template <typename T>
__device__ void hlle1d_adj(T gamma, T gm1, St3<T> L, St3<T> R, const T fb[3], T wl[3], T wr[3]) {
    const T igm1 = T(1) / gm1;
    T cL = sqrt(gamma * L.p / L.r), cR = sqrt(gamma * R.p / R.r);
    T EL = L.p * igm1 + T(0.5) * L.r * L.u * L.u, ER = R.p * igm1 + T(0.5) * R.r * R.u * R.u;
    T aL = L.u - cL, aR = R.u - cR;
    T bL = L.u + cL, bR = R.u + cR;
    T SL = smin(aL, aR), SR = smax(bL, bR);
    bool slR = aR < aL;   // std::min picks the right argument only when it is smaller
    bool srR = bL < bR;   // std::max picks the right argument when the left is smaller
    T FL[3] = { L.r * L.u, L.r * L.u * L.u + L.p, (EL + L.p) * L.u };
    T FR[3] = { R.r * R.u, R.r * R.u * R.u + R.p, (ER + R.p) * R.u };
    T UL[3] = { L.r, L.r * L.u, EL }, UR[3] = { R.r, R.r * R.u, ER };
    T fLb[3] = {0, 0, 0}, fRb[3] = {0, 0, 0}, uLb[3] = {0, 0, 0}, uRb[3] = {0, 0, 0};
    T SLb = T(0), SRb = T(0);
    if (SL >= T(0)) {
        for (int k = 0; k < 3; ++k) fLb[k] = fb[k];
    } else if (SR <= T(0)) {
        for (int k = 0; k < 3; ++k) fRb[k] = fb[k];
    } else {
        // one reciprocal per face: the adjoint needs the derivative, not the
        // forward's rounding
        const T iD = T(1) / (SR - SL);
        for (int k = 0; k < 3; ++k) {
            T dU = UR[k] - UL[k];
            T F = (SR * FL[k] - SL * FR[k] + SL * SR * dU) * iD;
            T g = fb[k] * iD;
            fLb[k] = g * SR;
            fRb[k] = -g * SL;
            uRb[k] = g * SL * SR;
            uLb[k] = -uRb[k];
            SLb += g * (-FR[k] + SR * dU + F);
            SRb += g * (FL[k] + SL * dU - F);
        }
    }
    // Davis speeds -> u and c of the active side
    T uLb_ = T(0), uRb_ = T(0), cLb = T(0), cRb = T(0);
    if (slR) { uRb_ += SLb; cRb -= SLb; } else { uLb_ += SLb; cLb -= SLb; }
    if (srR) { uRb_ += SRb; cRb += SRb; } else { uLb_ += SRb; cLb += SRb; }
    // one side: fluxes, conserved state, energy, sound speed -> (rho, u, p)
    auto side = [&](St3<T> S, T E, T c, const T* fb_, const T* ub_, T ubar, T cbar, T* wo) {
        T rb = T(0), ub = ubar, pb = T(0), Eb = T(0);
        // F0 = r u
        rb += fb_[0] * S.u; ub += fb_[0] * S.r;
        // F1 = (r u) u + p
        rb += fb_[1] * S.u * S.u; ub += fb_[1] * T(2) * S.r * S.u; pb += fb_[1];
        // F2 = (E + p) u
        Eb += fb_[2] * S.u; pb += fb_[2] * S.u; ub += fb_[2] * (E + S.p);
        // U = (r, r u, E)
        rb += ub_[0]; rb += ub_[1] * S.u; ub += ub_[1] * S.r; Eb += ub_[2];
        // E = p / (g-1) + 0.5 r u^2
        pb += Eb * igm1; rb += Eb * T(0.5) * S.u * S.u; ub += Eb * S.r * S.u;
        // c = sqrt(g p / r): dc/dp = g / (2 r c), dc/dr = -c / (2 r)
        if (c > T(0)) {  // 1 / (2 r c) once: dc/dr = -c^2 / (2 r c)
            const T q = T(0.5) / (S.r * c);
            pb += cbar * gamma * q;
            rb -= cbar * (c * c) * q;
        }
        wo[0] += rb; wo[1] += ub; wo[2] += pb;
    };
    side(L, EL, cL, fLb, uLb, uLb_, cLb, wl);
    side(R, ER, cR, fRb, uRb, uRb_, cRb, wr);
}

// Periodic index.  Tile halo cells past the domain (read by threads that
// return early) can lie more than one period away on small domains.
__device__ __forceinline__ int wrap(int c, int n) {
    int r = c % n;
    return r < 0 ? r + n : r;
}

// Shared-memory work arrays of one reverse stage over up to NOC output cells.
template <typename T, int NOC>
struct Rev1 {
    T W[3][NOC + 6];               // primitives of cells c0-3 ..
    T Lo[3][NOC + 4];              // output adjoint of cells c0-2 .. (alpha applied)
    T S[3][NOC + 4];               // slopes of cells c0-2 ..
    signed char B[3][NOC + 4];     // minmod branch: 0 none, 1 d1, 2 d2
    T WL[3][NOC + 3], WR[3][NOC + 3];  // face state adjoints, faces c0-2+1/2 ..
    T Sb[3][NOC + 2];              // slope adjoints, cells c0-1 ..
};

// One reverse stage over the NO output cells c0 .. c0+NO-1 (wrapped
// periodically), run by the CTA's NTA threads: Lo[t] = alpha * lo(k, t) for
// cell c0-2+t, W from U; calls put(q, rb, mb, Eb) with q < NO and the
// stage's Jacobian-transpose term of cell c0+q (the caller adds Lo[q + 2]
// and any Extra).  Ends with the CTA synchronised.
template <typename T, int NO, int NOC, class LoFn, class PutFn>
__device__ __forceinline__ void rev_stage(Rev1<T, NOC>& R, const T* __restrict__ U, int n, int h, int c0, T lambda,
                                          T gamma, T gm1, T alpha, LoFn lo, PutFn put) {
    static_assert(NO <= NOC, "work arrays too small");
    const int nt = n + 2 * h;
    for (int t = threadIdx.x; t < NO + 6; t += NTA) {
        int c = wrap(c0 - 3 + t, n) + h;
        T rho = U[c], mom = U[nt + c], erg = U[2 * nt + c];
        R.W[0][t] = rho; R.W[1][t] = mom / rho; R.W[2][t] = eos_pressure(gm1, rho, mom, erg);
    }
    for (int t = threadIdx.x; t < NO + 4; t += NTA)
        for (int k = 0; k < 3; ++k) R.Lo[k][t] = alpha * lo(k, t);
    __syncthreads();
    for (int t = threadIdx.x; t < NO + 4; t += NTA) {  // cell c0-2+t <-> W index t+1
        for (int k = 0; k < 3; ++k) {
            T d1 = R.W[k][t + 1] - R.W[k][t], d2 = R.W[k][t + 2] - R.W[k][t + 1];
            T s;
            signed char br;
            if (d1 * d2 <= T(0)) { s = T(0); br = 0; }
            else if (fabs(d1) < fabs(d2)) { s = d1; br = 1; }
            else { s = d2; br = 2; }
            R.S[k][t] = s; R.B[k][t] = br;
        }
    }
    __syncthreads();
    // faces: f = 0 .. NO+2 between cells a = c0-2+f and b = a+1 (S/Lo index f and f+1)
    for (int f = threadIdx.x; f < NO + 3; f += NTA) {
        St3<T> L = { R.W[0][f + 1] + T(0.5) * R.S[0][f], R.W[1][f + 1] + T(0.5) * R.S[1][f],
                     R.W[2][f + 1] + T(0.5) * R.S[2][f] };
        St3<T> Rs = { R.W[0][f + 2] - T(0.5) * R.S[0][f + 1], R.W[1][f + 2] - T(0.5) * R.S[1][f + 1],
                      R.W[2][f + 2] - T(0.5) * R.S[2][f + 1] };
        T fb[3], wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) fb[k] = lambda * (R.Lo[k][f + 1] - R.Lo[k][f]);
        hlle1d_adj(gamma, gm1, L, Rs, fb, wl, wr);
        for (int k = 0; k < 3; ++k) { R.WL[k][f] = wl[k]; R.WR[k][f] = wr[k]; }
    }
    __syncthreads();
    // slope adjoints of cells c0-1 .. c0+NO (index q): right face q+1, left face q
    for (int q = threadIdx.x; q < NO + 2; q += NTA)
        for (int k = 0; k < 3; ++k) R.Sb[k][q] = T(0.5) * R.WL[k][q + 1] - T(0.5) * R.WR[k][q];
    __syncthreads();
    for (int c = threadIdx.x; c < NO; c += NTA) {
        const int q = c + 1;  // Sb index of cell c0+c; S/B index q+1; faces q (left), q+1 (right)
        T wb[3];
        for (int k = 0; k < 3; ++k) {
            T v = R.WR[k][q] + R.WL[k][q + 1];
            int b0 = R.B[k][q + 1], bm = R.B[k][q], bp = R.B[k][q + 2];
            if (b0 == 1) v += R.Sb[k][q];
            else if (b0 == 2) v -= R.Sb[k][q];
            if (bm == 2) v += R.Sb[k][q - 1];
            if (bp == 1) v -= R.Sb[k][q + 1];
            wb[k] = v;
        }
        // (rho, u, p) = prim(rho, m, E): transpose of its Jacobian at the cell
        const int e = wrap(c0 + c, n) + h;
        T rho = U[e], mom = U[nt + e], erg = U[2 * nt + e];
        T u = mom / rho, ir = T(1) / rho;
        T praw = gm1 * (erg - T(0.5) * rho * u * u);
        T act = (praw < T(0)) ? T(0) : T(1);
        T rb = wb[0] - wb[1] * u * ir + act * wb[2] * gm1 * T(0.5) * u * u;
        T mb = wb[1] * ir - act * wb[2] * gm1 * u;
        T Eb = act * wb[2] * gm1;
        put(c, rb, mb, Eb);
    }
    __syncthreads();
}

// Output of a reverse stage into the solver layout, with the adjoint's ghost
// cells kept consistent with the periodic wrap.
template <typename T>
__device__ __forceinline__ void put_global(T* Lin, int n, int h, int i, const T v[3]) {
    const int nt = n + 2 * h, e = h + i;
    for (int k = 0; k < 3; ++k) {
        Lin[k * nt + e] = v[k];
        if (i < h) Lin[k * nt + h + n + i] = v[k];
        if (i >= n - h) Lin[k * nt + (i - (n - h))] = v[k];
    }
}

// One reverse Heun step in one launch: tmp = S'(U1)^T lam / 2 over the CTA's
// cells and a two-cell halo on each side (kept in shared memory), then
// lam_new = S'(Un)^T tmp + lam / 2 over its cells (the halo's tmp is
// recomputed by both neighbouring CTAs, bit for bit the same).
template <typename T>
__global__ void __launch_bounds__(NTA)
k1d_adjoint_step(const T* __restrict__ Un, const T* __restrict__ U1, const T* __restrict__ lam,
                 T* __restrict__ lam_new, int n, int h, const double* dtp, double dx, double gamma_d) {
    __shared__ Rev1<T, TA + 4> R;
    __shared__ T tmp[3][TA + 4];  // cells c0-2 .. c0+TA+1
    pdl_wait();
    pdl_trigger();
    const T lambda = (T)(*dtp / dx);
    const T gamma = (T)gamma_d, gm1 = (T)(gamma_d - 1.0);
    const int nt = n + 2 * h, c0 = blockIdx.x * TA;
    {
        auto lo = [&](int k, int t) { return lam[k * nt + wrap(c0 - 4 + t, n) + h]; };
        auto put = [&](int c, T rb, T mb, T Eb) {
            tmp[0][c] = R.Lo[0][c + 2] + rb;
            tmp[1][c] = R.Lo[1][c + 2] + mb;
            tmp[2][c] = R.Lo[2][c + 2] + Eb;
        };
        rev_stage<T, TA + 4>(R, U1, n, h, c0 - 2, lambda, gamma, gm1, T(0.5), lo, put);
    }
    {
        auto lo = [&](int k, int t) { return tmp[k][t]; };
        auto put = [&](int c, T rb, T mb, T Eb) {
            const int i = c0 + c;
            if (i >= n) return;
            const int e = h + i;
            T v[3] = { R.Lo[0][c + 2] + rb, R.Lo[1][c + 2] + mb, R.Lo[2][c + 2] + Eb };
            for (int k = 0; k < 3; ++k) v[k] += T(0.5) * lam[k * nt + e];
            put_global(lam_new, n, h, i, v);
        };
        rev_stage<T, TA>(R, Un, n, h, c0, lambda, gamma, gm1, T(1), lo, put);
    }
}

template <typename T>
cudaError_t launch_1d_adjoint_step_t(const T* Un, const T* U1, const T* lam, T* lam_new, int n, int h,
                                     const double* dtp, double dx, double gamma, cudaStream_t st) {
    int blocks = (n + TA - 1) / TA;
    return launch_pdl(k1d_adjoint_step<T>, dim3(blocks), dim3(NTA), 0, st, Un, U1, lam, lam_new, n, h, dtp, dx, gamma);
}

}  // namespace
}  // namespace nestb
