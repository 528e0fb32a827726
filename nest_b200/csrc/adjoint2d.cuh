// Discrete adjoint of the unsplit 2D stage (template; instantiated for FP32
// and FP64 in adjoint2d.cu).  Periodic domains.
//
// Forward stage (euler2d_kernels.cuh):
//   W = prim(U) = (rho, u, v, p), p clamped at 0
//   sx, sy = minmod slopes along x and y
//   F_{i+1/2,j} = HLLE4(W_i + sx_i/2, W_{i+1} - sx_{i+1}/2)   normal u, transverse v
//   G_{i,j+1/2} = HLLE4(W_j + sy_j/2, W_{j+1} - sy_{j+1}/2)   normal v, transverse u
//   U' = U - (lx (F_{i+1/2} - F_{i-1/2}) + ly (G_{j+1/2} - G_{j-1/2}))
// Adjoint for a given Ubar':
//   Fbar = lx (Ubar'_{i+1} - Ubar'_i), Gbar = ly (Ubar'_{j+1} - Ubar'_j)
//   face-state adjoints from the HLLE4 reverse sweep (branch of the forward,
//   active argument of each Davis min / max), slope adjoints
//   sbar = WLbar/2 (face above) - WRbar/2 (face below) per axis, minmod
//   subgradients, Wbar gathered per cell, Ubar = Ubar' + (dW/dU)^T Wbar.
// A CTA of 256 threads owns a tile of ATX = 13 rows x ATY = 16 columns; every
// intermediate lives in shared memory.  The tile shape makes both face sets
// fit one pass of the CTA: (ATX + 3) x ATY = 256 x-faces and ATX x (ATY + 3)
// = 247 y-faces, so every thread runs one x-face and one y-face reverse HLLE.
#pragma once

#include "euler2d_kernels.cuh"

namespace nestb {

#ifndef NEST_ADJ_ATX
#define NEST_ADJ_ATX 13
#define NEST_ADJ_ATY 16
#define NEST_ADJ_NT 256
#endif
constexpr int ATX = NEST_ADJ_ATX, ATY = NEST_ADJ_ATY;  // tile rows, tile columns
constexpr int ANT = NEST_ADJ_NT;                       // threads per CTA

template <typename T>
struct Adj4 { T r, n, t, p; };

// Reverse sweep of hlle4 (normal n, transverse t) for one face.
template <typename T>
__device__ __forceinline__ void hlle4_adj(T gamma, T igm1, Adj4<T> L, Adj4<T> R, const T fb[4], T wl[4], T wr[4]) {
    T cL = sqrt(gamma * L.p / L.r), cR = sqrt(gamma * R.p / R.r);
    T EL = L.p * igm1 + T(0.5) * L.r * (L.n * L.n + L.t * L.t);
    T ER = R.p * igm1 + T(0.5) * R.r * (R.n * R.n + R.t * R.t);
    T aL = L.n - cL, aR = R.n - cR, bL = L.n + cL, bR = R.n + cR;
    T SL = smin(aL, aR), SR = smax(bL, bR);
    bool slR = aR < aL, srR = bL < bR;
    T FL[4] = { L.r * L.n, L.r * L.n * L.n + L.p, L.r * L.n * L.t, (EL + L.p) * L.n };
    T FR[4] = { R.r * R.n, R.r * R.n * R.n + R.p, R.r * R.n * R.t, (ER + R.p) * R.n };
    T UL[4] = { L.r, L.r * L.n, L.r * L.t, EL }, UR[4] = { R.r, R.r * R.n, R.r * R.t, ER };
    T fLb[4] = {0, 0, 0, 0}, fRb[4] = {0, 0, 0, 0}, uLb[4] = {0, 0, 0, 0}, uRb[4] = {0, 0, 0, 0};
    T SLb = 0, SRb = 0;
    if (SL >= T(0)) {
        for (int k = 0; k < 4; ++k) fLb[k] = fb[k];
    } else if (SR <= T(0)) {
        for (int k = 0; k < 4; ++k) fRb[k] = fb[k];
    } else {
        const T iD = T(1) / (SR - SL);
        for (int k = 0; k < 4; ++k) {
            T dU = UR[k] - UL[k];
            T F = (SR * FL[k] - SL * FR[k] + SL * SR * dU) * iD;
            T gk = fb[k] * iD;
            fLb[k] = gk * SR;
            fRb[k] = -gk * SL;
            uRb[k] = gk * SL * SR;
            uLb[k] = -uRb[k];
            SLb += gk * (-FR[k] + SR * dU + F);
            SRb += gk * (FL[k] + SL * dU - F);
        }
    }
    T nLb = 0, nRb = 0, cLb = 0, cRb = 0;
    if (slR) { nRb += SLb; cRb -= SLb; } else { nLb += SLb; cLb -= SLb; }
    if (srR) { nRb += SRb; cRb += SRb; } else { nLb += SRb; cLb += SRb; }
    auto side = [&](Adj4<T> S, T E, T c, const T* fb_, const T* ub_, T nb0, T cb, T* wo) {
        T rb = 0, nb = nb0, tb = 0, pb = 0, Eb = 0;
        rb += fb_[0] * S.n; nb += fb_[0] * S.r;                                   // rho n
        rb += fb_[1] * S.n * S.n; nb += fb_[1] * T(2) * S.r * S.n; pb += fb_[1]; // rho n n + p
        rb += fb_[2] * S.n * S.t; nb += fb_[2] * S.r * S.t; tb += fb_[2] * S.r * S.n;  // rho n t
        Eb += fb_[3] * S.n; pb += fb_[3] * S.n; nb += fb_[3] * (E + S.p);         // (E + p) n
        rb += ub_[0]; rb += ub_[1] * S.n; nb += ub_[1] * S.r;
        rb += ub_[2] * S.t; tb += ub_[2] * S.r; Eb += ub_[3];
        pb += Eb * igm1; rb += Eb * T(0.5) * (S.n * S.n + S.t * S.t); nb += Eb * S.r * S.n; tb += Eb * S.r * S.t;
        if (c > T(0)) {  // c = sqrt(g p / r): dc/dp = g / (2 r c), dc/dr = -c / (2 r) = -c^2 / (2 r c)
            const T q = T(0.5) / (S.r * c);
            pb += cb * gamma * q;
            rb -= cb * (c * c) * q;
        }
        wo[0] += rb; wo[1] += nb; wo[2] += tb; wo[3] += pb;
    };
    side(L, EL, cL, fLb, uLb, nLb, cLb, wl);
    side(R, ER, cR, fRb, uRb, nRb, cRb, wr);
}

// Minmod slope and its branch: 0 none, 1 first difference, 2 second; for
// FP32 states 3 = a near-tie (|d1| and |d2| within 2^-19 |w| of each other,
// w the cell's primitive), whose slope adjoint is split half and half between
// the two differences (the reasoning is at tie_mask in adjoint2d_f32x2.cu).
// FP64 keeps the exact branch.
template <typename T>
__device__ __forceinline__ T mmslope(T d1, T d2, signed char& br, T w) {
    if (d1 * d2 <= T(0)) { br = 0; return T(0); }
    const bool first = fabs(d1) < fabs(d2);
    if (sizeof(T) == 4 && fabs(fabs(d1) - fabs(d2)) <= T(1.9073486e-06) * fabs(w)) br = 3;
    else br = first ? 1 : 2;
    return first ? d1 : d2;
}

// Shared-memory image of one tile.
template <typename T>
struct AdjSmem {
    static constexpr int RX3 = ATX + 6, RY3 = ATY + 6, RX2 = ATX + 4, RY2 = ATY + 4;
    T W[4][RX3][RY3];                // primitives of cells (i0-3 .., j0-3 ..)
    T Lo[4][RX2][RY2];               // output adjoint of cells (i0-2 .., j0-2 ..), alpha applied
    T Sx[4][RX2][ATY];               // x slopes of rows i0-2 .. under the tile columns
    T Sy[4][ATX][RY2];               // y slopes of columns j0-2 .. in the tile rows
    T XL[4][ATX + 3][ATY], XR[4][ATX + 3][ATY];  // x-face state adjoints, faces between rows i0-2+f, i0-1+f
    T YL[4][ATX][ATY + 3], YR[4][ATX][ATY + 3];  // y-face state adjoints, faces between columns j0-2+f, j0-1+f
    T Uc[4][ATX][ATY];               // conserved values of the tile's own cells (kept from the load pass)
    T Ex[4][ATX][ATY];               // Extra of the tile's cells, fetched asynchronously at the start
    signed char Bx[4][RX2][ATY], By[4][ATX][RY2];  // minmod branch: 0 none, 1 first, 2 second difference
};

// Per-thread asynchronous global -> shared copy of one value (cp.async).
template <typename T>
__device__ __forceinline__ void adj_cp(T* smem_dst, const T* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}

// Lin = alpha * adj(U, Lout) + beta * Extra.  All arrays use the solver's
// 2D device layout (Geo2D); periodic wrap on both axes.  Needs
// sizeof(AdjSmem<T>) bytes of dynamic shared memory and AT*AT threads.
template <typename T>
__device__ void adjoint2d_tile(const T* __restrict__ U, const T* __restrict__ Lout, const T* __restrict__ Extra,
                               T* __restrict__ Lin, const Geo2D& g, T lx, T ly, T alpha, T beta) {
    constexpr int RX3 = ATX + 6, RY3 = ATY + 6, RX2 = ATX + 4, RY2 = ATY + 4;
    static_assert((ATX + 3) * ATY <= ANT && ATX * (ATY + 3) <= ANT, "one face of each kind per thread");
    extern __shared__ __align__(16) unsigned char adj_smem_raw[];
    AdjSmem<T>& S = *reinterpret_cast<AdjSmem<T>*>(adj_smem_raw);
    auto& W = S.W;
    auto& Lo = S.Lo;
    auto& Sx = S.Sx;
    auto& Sy = S.Sy;
    auto& Bx = S.Bx;
    auto& By = S.By;
    auto& XL = S.XL;
    auto& XR = S.XR;
    auto& YL = S.YL;
    auto& YR = S.YR;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.y * ATX, j0 = blockIdx.x * ATY;
    const long long vs = g.vstride;
    const T gamma = (T)g.gamma, gm1 = (T)(g.gamma - 1.0), igm1 = (T)(1.0 / (g.gamma - 1.0));
    // periodic wrap; tile cells beyond the domain (only read by threads that
    // return early) may lie more than one period away on small domains
    auto wrapi = [&](int i) {
        if ((unsigned)i < (unsigned)g.nx) return i;
        int r = i % g.nx;
        return r < 0 ? r + g.nx : r;
    };
    auto wrapj = [&](int j) {
        if ((unsigned)j < (unsigned)g.ny) return j;
        int r = j % g.ny;
        return r < 0 ? r + g.ny : r;
    };
    // Extra of this thread's output cell: requested now, read in the last pass
    // (the thread reads back only what it copied itself)
    const bool has_cell = tid < ATX * ATY && i0 + tid / ATY < g.nx && j0 + tid % ATY < g.ny;
    if (Extra && has_cell) {
        const int a = tid / ATY, b = tid % ATY;
        const long long o = g.at(i0 + a, j0 + b);
        for (int k = 0; k < 4; ++k) adj_cp(&S.Ex[k][a][b], Extra + k * vs + o);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int t = tid; t < RX3 * RY3; t += ANT) {
        int a = t / RY3, b = t % RY3;
        long long o = g.at(wrapi(i0 - 3 + a), wrapj(j0 - 3 + b));
        const T u0 = U[o], u1 = U[vs + o], u2 = U[2 * vs + o], u3 = U[3 * vs + o];
        Prim4<T> w = cons2prim<T, false>(u0, u1, u2, u3, gm1);
        W[0][a][b] = w.r; W[1][a][b] = w.u; W[2][a][b] = w.v; W[3][a][b] = w.p;
        if (a >= 3 && a < ATX + 3 && b >= 3 && b < ATY + 3) {
            S.Uc[0][a - 3][b - 3] = u0; S.Uc[1][a - 3][b - 3] = u1;
            S.Uc[2][a - 3][b - 3] = u2; S.Uc[3][a - 3][b - 3] = u3;
        }
    }
    for (int t = tid; t < RX2 * RY2; t += ANT) {
        int a = t / RY2, b = t % RY2;
        long long o = g.at(wrapi(i0 - 2 + a), wrapj(j0 - 2 + b));
        for (int k = 0; k < 4; ++k) Lo[k][a][b] = alpha * Lout[k * vs + o];
    }
    __syncthreads();
    // x slopes of rows i0-2 .. i0+ATX+1 (index a) under the tile columns
    for (int t = tid; t < RX2 * ATY; t += ANT) {
        int a = t / ATY, b = t % ATY;
        for (int k = 0; k < 4; ++k) {
            signed char br;
            Sx[k][a][b] = mmslope(W[k][a + 1][b + 3] - W[k][a][b + 3], W[k][a + 2][b + 3] - W[k][a + 1][b + 3], br,
                                  W[k][a + 1][b + 3]);
            Bx[k][a][b] = br;
        }
    }
    // y slopes of columns j0-2 .. j0+ATY+1 (index c) in the tile rows
    for (int t = tid; t < ATX * RY2; t += ANT) {
        int a = t / RY2, c = t % RY2;
        for (int k = 0; k < 4; ++k) {
            signed char br;
            Sy[k][a][c] = mmslope(W[k][a + 3][c + 1] - W[k][a + 3][c], W[k][a + 3][c + 2] - W[k][a + 3][c + 1], br,
                                  W[k][a + 3][c + 1]);
            By[k][a][c] = br;
        }
    }
    __syncthreads();
    if (tid < (ATX + 3) * ATY) {
        // x face f between rows i0-2+f and i0-1+f under tile column b (Sx index f, f+1; Lo row f, f+1)
        const int f = tid / ATY, b = tid % ATY;
        Adj4<T> L = { W[0][f + 1][b + 3] + T(0.5) * Sx[0][f][b], W[1][f + 1][b + 3] + T(0.5) * Sx[1][f][b],
                      W[2][f + 1][b + 3] + T(0.5) * Sx[2][f][b], W[3][f + 1][b + 3] + T(0.5) * Sx[3][f][b] };
        Adj4<T> R = { W[0][f + 2][b + 3] - T(0.5) * Sx[0][f + 1][b], W[1][f + 2][b + 3] - T(0.5) * Sx[1][f + 1][b],
                      W[2][f + 2][b + 3] - T(0.5) * Sx[2][f + 1][b], W[3][f + 2][b + 3] - T(0.5) * Sx[3][f + 1][b] };
        T fb[4], wl[4] = {0, 0, 0, 0}, wr[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k) fb[k] = lx * (Lo[k][f + 1][b + 2] - Lo[k][f][b + 2]);
        // components (rho, mu, mv, E) -> (rho, normal, transverse, E): x normal = u
        hlle4_adj(gamma, igm1, L, R, fb, wl, wr);
        for (int k = 0; k < 4; ++k) { XL[k][f][b] = wl[k]; XR[k][f][b] = wr[k]; }
    }
    if (tid < ATX * (ATY + 3)) {
        // y face f between columns j0-2+f and j0-1+f in tile row a
        const int a = tid / (ATY + 3), f = tid % (ATY + 3);
        Adj4<T> L = { W[0][a + 3][f + 1] + T(0.5) * Sy[0][a][f], W[2][a + 3][f + 1] + T(0.5) * Sy[2][a][f],
                      W[1][a + 3][f + 1] + T(0.5) * Sy[1][a][f], W[3][a + 3][f + 1] + T(0.5) * Sy[3][a][f] };
        Adj4<T> R = { W[0][a + 3][f + 2] - T(0.5) * Sy[0][a][f + 1], W[2][a + 3][f + 2] - T(0.5) * Sy[2][a][f + 1],
                      W[1][a + 3][f + 2] - T(0.5) * Sy[1][a][f + 1], W[3][a + 3][f + 2] - T(0.5) * Sy[3][a][f + 1] };
        // flux order (rho, normal = mv, transverse = mu, E)
        T fb[4] = { ly * (Lo[0][a + 2][f + 1] - Lo[0][a + 2][f]), ly * (Lo[2][a + 2][f + 1] - Lo[2][a + 2][f]),
                    ly * (Lo[1][a + 2][f + 1] - Lo[1][a + 2][f]), ly * (Lo[3][a + 2][f + 1] - Lo[3][a + 2][f]) };
        T wl[4] = {0, 0, 0, 0}, wr[4] = {0, 0, 0, 0};
        hlle4_adj(gamma, igm1, L, R, fb, wl, wr);
        // back to (rho, u, v, p)
        YL[0][a][f] = wl[0]; YL[1][a][f] = wl[2]; YL[2][a][f] = wl[1]; YL[3][a][f] = wl[3];
        YR[0][a][f] = wr[0]; YR[1][a][f] = wr[2]; YR[2][a][f] = wr[1]; YR[3][a][f] = wr[3];
    }
    __syncthreads();
    if (tid >= ATX * ATY) return;
    const int a = tid / ATY, b = tid % ATY;
    const int i = i0 + a, j = j0 + b;
    if (i >= g.nx || j >= g.ny) return;
    // Sx/Bx index of row i0-2+q is q; cell row i is q = a+2.  x face f lies between
    // rows i0-2+f and i0-1+f, so cell row i0-2+q has lower face q-1 and upper face q.
    // Columns likewise with r = b+2.
    auto sbx = [&](int k, int q) { return T(0.5) * XL[k][q][b] - T(0.5) * XR[k][q - 1][b]; };
    auto sby = [&](int k, int q) { return T(0.5) * YL[k][a][q] - T(0.5) * YR[k][a][q - 1]; };
    T wb[4];
    for (int k = 0; k < 4; ++k) {
        const int q = a + 2, r = b + 2;
        T v = XR[k][q - 1][b] + XL[k][q][b] + YR[k][a][r - 1] + YL[k][a][r];
        int bx0 = Bx[k][q][b], bxm = Bx[k][q - 1][b], bxp = Bx[k][q + 1][b];
        if (bx0 == 1) v += sbx(k, q); else if (bx0 == 2) v -= sbx(k, q);
        if (bxm == 2) v += sbx(k, q - 1); else if (bxm == 3) v += T(0.5) * sbx(k, q - 1);
        if (bxp == 1) v -= sbx(k, q + 1); else if (bxp == 3) v -= T(0.5) * sbx(k, q + 1);
        int by0 = By[k][a][r], bym = By[k][a][r - 1], byp = By[k][a][r + 1];
        if (by0 == 1) v += sby(k, r); else if (by0 == 2) v -= sby(k, r);
        if (bym == 2) v += sby(k, r - 1); else if (bym == 3) v += T(0.5) * sby(k, r - 1);
        if (byp == 1) v -= sby(k, r + 1); else if (byp == 3) v -= T(0.5) * sby(k, r + 1);
        wb[k] = v;
    }
    const long long o = g.at(i, j);
    T rho = S.Uc[0][a][b], mu = S.Uc[1][a][b], mv = S.Uc[2][a][b], E = S.Uc[3][a][b];
    const T ir = T(1) / rho;
    T u = mu / rho, v = mv / rho;
    T praw = gm1 * (E - (T(0.5) * rho * u * u + T(0.5) * rho * v * v));
    T act = (praw < T(0)) ? T(0) : T(1);
    T q2 = T(0.5) * (u * u + v * v);
    T rb = wb[0] - (wb[1] * u + wb[2] * v) * ir + act * wb[3] * gm1 * q2;
    T mub = wb[1] * ir - act * wb[3] * gm1 * u;
    T mvb = wb[2] * ir - act * wb[3] * gm1 * v;
    T Eb = act * wb[3] * gm1;
    T out[4] = { Lo[0][a + 2][b + 2] + rb, Lo[1][a + 2][b + 2] + mub, Lo[2][a + 2][b + 2] + mvb, Lo[3][a + 2][b + 2] + Eb };
    if (Extra) asm volatile("cp.async.wait_group 0;" ::: "memory");
    for (int k = 0; k < 4; ++k) {
        T val = out[k];
        if (Extra) val += beta * S.Ex[k][a][b];
        Lin[k * vs + o] = val;
    }
}

}  // namespace nestb
