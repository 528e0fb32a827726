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
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace nestb {
namespace {

constexpr int TA = 128;  // cells per CTA

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

// Lin = alpha * adj(U, Lout) + beta * Extra (Extra may be null).  U, Lout,
// Extra, Lin: SoA [3][n + 2h], interior at offset h; periodic.
template <typename T>
__global__ void __launch_bounds__(TA)
k1d_adjoint_stage(const T* __restrict__ U, const T* __restrict__ Lout, const T* __restrict__ Extra,
                  T* __restrict__ Lin, int n, int h, const double* dtp, double dx, double gamma_d, double alpha_d,
                  double beta_d) {
    const T lambda = (T)(*dtp / dx);
    const T gamma = (T)gamma_d, alpha = (T)alpha_d, beta = (T)beta_d;
    __shared__ T W[3][TA + 6];     // cells c0-3 .. c0+TA+2
    __shared__ T Lo[3][TA + 4];    // cells c0-2 .. c0+TA+1 (alpha applied)
    __shared__ T S[3][TA + 4];     // slopes of cells c0-2 .. c0+TA+1
    __shared__ signed char B[3][TA + 4];  // minmod branch: 0 none, 1 d1, 2 d2
    __shared__ T WL[3][TA + 3], WR[3][TA + 3];  // face state adjoints, faces c0-2+1/2 .. c0+TA+1/2
    __shared__ T Sb[3][TA + 2];    // slope adjoints, cells c0-1 .. c0+TA
    const int nt = n + 2 * h;
    const int c0 = blockIdx.x * TA;
    const T gm1 = (T)(gamma_d - 1.0);
    for (int t = threadIdx.x; t < TA + 6; t += TA) {
        int c = wrap(c0 - 3 + t, n) + h;
        T rho = U[c], mom = U[nt + c], erg = U[2 * nt + c];
        W[0][t] = rho; W[1][t] = mom / rho; W[2][t] = eos_pressure(gm1, rho, mom, erg);
    }
    for (int t = threadIdx.x; t < TA + 4; t += TA) {
        int c = wrap(c0 - 2 + t, n) + h;
        for (int k = 0; k < 3; ++k) Lo[k][t] = alpha * Lout[k * nt + c];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < TA + 4; t += TA) {  // cell c0-2+t <-> W index t+1
        for (int k = 0; k < 3; ++k) {
            T d1 = W[k][t + 1] - W[k][t], d2 = W[k][t + 2] - W[k][t + 1];
            T s;
            signed char br;
            if (d1 * d2 <= T(0)) { s = T(0); br = 0; }
            else if (fabs(d1) < fabs(d2)) { s = d1; br = 1; }
            else { s = d2; br = 2; }
            S[k][t] = s; B[k][t] = br;
        }
    }
    __syncthreads();
    // faces: f = 0 .. TA+2 between cells a = c0-2+f and b = a+1 (S/Lo index f and f+1)
    for (int f = threadIdx.x; f < TA + 3; f += TA) {
        St3<T> L = { W[0][f + 1] + T(0.5) * S[0][f], W[1][f + 1] + T(0.5) * S[1][f], W[2][f + 1] + T(0.5) * S[2][f] };
        St3<T> R = { W[0][f + 2] - T(0.5) * S[0][f + 1], W[1][f + 2] - T(0.5) * S[1][f + 1], W[2][f + 2] - T(0.5) * S[2][f + 1] };
        T fb[3], wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) fb[k] = lambda * (Lo[k][f + 1] - Lo[k][f]);
        hlle1d_adj(gamma, gm1, L, R, fb, wl, wr);
        for (int k = 0; k < 3; ++k) { WL[k][f] = wl[k]; WR[k][f] = wr[k]; }
    }
    __syncthreads();
    // slope adjoints of cells c0-1 .. c0+TA (index q): right face q+1, left face q
    for (int q = threadIdx.x; q < TA + 2; q += TA)
        for (int k = 0; k < 3; ++k) Sb[k][q] = T(0.5) * WL[k][q + 1] - T(0.5) * WR[k][q];
    __syncthreads();
    int i = c0 + threadIdx.x;
    if (i >= n) return;
    const int q = threadIdx.x + 1;  // Sb index of cell i; S/B index q+1; faces q (left), q+1 (right)
    T wb[3];
    for (int k = 0; k < 3; ++k) {
        T v = WR[k][q] + WL[k][q + 1];
        int b0 = B[k][q + 1], bm = B[k][q], bp = B[k][q + 2];
        if (b0 == 1) v += Sb[k][q];
        else if (b0 == 2) v -= Sb[k][q];
        if (bm == 2) v += Sb[k][q - 1];
        if (bp == 1) v -= Sb[k][q + 1];
        wb[k] = v;
    }
    // (rho, u, p) = prim(rho, m, E): transpose of its Jacobian at cell i
    int e = h + i;
    T rho = U[e], mom = U[nt + e], erg = U[2 * nt + e];
    T u = mom / rho, ir = T(1) / rho;
    T praw = gm1 * (erg - T(0.5) * rho * u * u);
    T act = (praw < T(0)) ? T(0) : T(1);
    T rb = wb[0] - wb[1] * u * ir + act * wb[2] * gm1 * T(0.5) * u * u;
    T mb = wb[1] * ir - act * wb[2] * gm1 * u;
    T Eb = act * wb[2] * gm1;
    T out[3] = { Lo[0][q + 1] + rb, Lo[1][q + 1] + mb, Lo[2][q + 1] + Eb };
    for (int k = 0; k < 3; ++k) {
        T v = out[k];
        if (Extra) v += beta * Extra[k * nt + e];
        Lin[k * nt + e] = v;
    }
    // keep the adjoint's ghost cells consistent with the periodic wrap
    for (int k = 0; k < 3; ++k) {
        if (i < h) Lin[k * nt + h + n + i] = Lin[k * nt + e];
        if (i >= n - h) Lin[k * nt + (i - (n - h))] = Lin[k * nt + e];
    }
}

template <typename T>
cudaError_t launch_1d_adjoint_stage_t(const T* U, const T* Lout, const T* Extra, T* Lin, int n, int h, const double* dtp,
                                      double dx, double gamma, double alpha, double beta, cudaStream_t st) {
    int blocks = (n + TA - 1) / TA;
    k1d_adjoint_stage<T><<<blocks, TA, 0, st>>>(U, Lout, Extra, Lin, n, h, dtp, dx, gamma, alpha, beta);
    return cudaGetLastError();
}

}  // namespace
}  // namespace nestb
