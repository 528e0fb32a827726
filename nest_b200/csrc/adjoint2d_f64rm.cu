// FP64 discrete adjoint of the unsplit 2D stage as a row march (sm_100a).
//
// Same map and subgradients as the tile kernel of adjoint2d.cuh and the FP32
// row march of adjoint2d_f32x2.cu:
//   Lin = alpha * S'(U)^T Lout + beta * Extra, periodic on both axes.
// One column per lane: a warp owns a strip of 32 columns c0 .. c0+31 and
// writes the 26 columns c0+3 .. c0+28 (lanes 3..28), marching down a segment
// of rows with the step structure of the FP32 kernel (x-face a+1/2, the
// y-direction part of row a through shuffles, row a-1 written).
//
// The branch decisions of the reverse sweep (the minmod argument, the HLLE
// regime and the active Davis arguments) must be the ones the forward FP64
// stage took, so the quantities they compare are computed exactly as the
// forward computes them: this unit is compiled with -fmad=false, the
// primitives divide (u = m / rho), ke2 keeps its operation order and the sound
// speed is sqrt(gamma p / rho).  Terms that only enter derivatives use
// explicit fma().
#include "euler2d_kernels.cuh"
#include "kernels.h"

#include <algorithm>
#include <mutex>

namespace nestb {
namespace {

// Launch shape and register budget, measured on the 2048^2 FP64 KH adjoint
// (300 steps, backward ms): 2 warps per CTA at 168 registers (12 warps per
// SM, no spills) 570; unbounded (176 registers, 10 warps per SM) 611 with 1,
// 2 or 4 warps per CTA; 152 / 128 registers (spills) 591 / 592.
#ifndef NEST_ADJ64_WARPS
#define NEST_ADJ64_WARPS 2
#define NEST_ADJ64_REGS 168
#endif
constexpr int DSTRIP = 26;                // output columns per warp
constexpr int DWARPS = NEST_ADJ64_WARPS;  // warps per CTA
constexpr int DRU = 2, DRL = 4, DRE = 2;  // ring slots: conserved rows, Lout rows, Extra rows
constexpr int DRING = (DRU + DRL + DRE) * 4 * 32;  // doubles per warp
extern __shared__ __align__(16) double adj64_ring[];

struct D4 { double a, b, c, d; };

__device__ __forceinline__ void cp8d(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpd_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpd_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Primitives of one cell exactly as the forward FP64 stage (cons2prim, no
// contraction); `act` = 1 where the pressure clamp p = max(p_raw, 0) is not
// active (p_raw >= 0).
__device__ __forceinline__ D4 prim64(const D4& U, double gm1, int& act) {
    D4 w;
    w.a = U.a;
    w.b = U.b / U.a;
    w.c = U.c / U.a;
    const double praw = gm1 * (U.d - ke2(w.a, w.b, w.c));
    act = praw < 0.0 ? 0 : 1;
    w.d = smax(praw, 0.0);
    return w;
}

// nest's minmod and the code of its active argument: 0 none (product <= 0),
// 1 the first difference, 2 the second (ties: the second).
__device__ __forceinline__ double mmb(double d1, double d2, int& br) {
    if (d1 * d2 <= 0.0) { br = 0; return 0.0; }
    if (fabs(d1) < fabs(d2)) { br = 1; return d1; }
    br = 2;
    return d2;
}

// Reverse of hlle4 for one face in the relative-flux form of the FP32 row
// march (adjoint2d_f32x2.cu, hlle2_adj): states (r, n, t, p) per side, flux
// adjoint (f0..f3) in the order (mass, normal, transverse, energy); the
// face-state adjoints are added to Lb and Rb.  The regime and the active
// arguments come from the forward's own sound speeds and Davis speeds.
__device__ __forceinline__ void hlle_adj64(double gamma, double igm1, const D4& L, const D4& R, double f0,
                                           double f1, double f2, double f3, D4& Lb, D4& Rb) {
    const double rL = L.a, nL = L.b, tL = L.c, pL = L.d;
    const double rR = R.a, nR = R.b, tR = R.c, pR = R.d;
    const double cL = sqrt(gamma * pL / rL), cR = sqrt(gamma * pR / rR);
    // nsl = -min(S_L, 0), sr = max(S_R, 0) (cL - nL is exactly -(nL - cL))
    const double aL = cL - nL, aR = cR - nR, bL = nL + cL, bR = nR + cR;
    const double nsl = fmax(fmax(aL, aR), 0.0), sr = fmax(fmax(bL, bR), 0.0);
    const double den = sr + nsl;
    double wL = 1.0, wR = 0.0, i2 = 0.0;  // S_L = S_R = 0: the forward takes F_L
    if (den > 0.0) {
        const double inv = 1.0 / den;
        wL = sr * inv;
        wR = nsl * inv;
        i2 = inv * inv;
    }
    const double kL = 0.5 * fma(tL, tL, nL * nL), kR = 0.5 * fma(tR, tR, nR * nR);
    const double EL = fma(pL, igm1, rL * kL), ER = fma(pR, igm1, rR * kR);
    const double gL = wL * (nL + nsl), gR = wR * (nR - sr);
    const double XL = fma(f2, tL, fma(f1, nL, f0)), XR = fma(f2, tR, fma(f1, nR, f0));
    const double YL = fma(f3, nL, f1), YR = fma(f3, nR, f1);
    const double ZL = fma(rL, XL, f3 * EL), ZR = fma(rR, XR, f3 * ER);
    const double D = fma(pL, YL, -(pR * YR));
    const double s1 = fma(nL - sr, ZL, fma(sr - nR, ZR, D));
    const double s2 = fma(nR + nsl, ZR, fma(-(nL + nsl), ZL, -D));
    // speed adjoints, each only where its clamp is open (S_L < 0, S_R > 0)
    const double Slb = nsl > 0.0 ? sr * i2 * s1 : 0.0;
    const double Srb = sr > 0.0 ? -nsl * i2 * s2 : 0.0;
    // S_L = min(nL - cL, nR - cR): the right argument only where strictly smaller
    const bool lr = aR > aL, rr = bL < bR;
    const double slL = lr ? 0.0 : Slb, slR = Slb - slL;
    const double srL = rr ? 0.0 : Srb, srR = Srb - srL;
    auto side = [&](double w, double gs, double r, double n, double t, double p, double E, double k, double X,
                    double Y, double c, double nb0, double cb, D4& out) {
        double rb = gs * fma(f3, k, X);
        double nb = fma(w, fma(r, X, f3 * (E + p)), fma(gs * r, Y, nb0));
        double tb = gs * r * fma(f3, t, f2);
        double pb = fma(w, Y, gs * f3 * igm1);
        if (c > 0.0) {  // dc/dp = gamma / (2 r c), dc/dr = -c^2 / (2 r c)
            const double h = 0.5 / (r * c);
            pb = fma(cb * gamma, h, pb);
            rb = fma(-cb * (c * c), h, rb);
        }
        out.a += rb;
        out.b += nb;
        out.c += tb;
        out.d += pb;
    };
    side(wL, gL, rL, nL, tL, pL, EL, kL, XL, YL, cL, slL + srL, srL - slL, Lb);
    side(wR, gR, rR, nR, tR, pR, ER, kR, XR, YR, cR, slR + srR, srR - slR, Rb);
}

struct AdjD64Args {
    const double* U;
    const double* Lout;
    const double* Extra;
    double* Lin;
    Geo2D g;
    const double* dtp;
    double alpha, beta;
    int seg_rows;
};

#if NEST_ADJ64_REGS > 0
#define NEST_ADJ64_ATTR __maxnreg__(NEST_ADJ64_REGS)
#else
#define NEST_ADJ64_ATTR __launch_bounds__(32 * DWARPS)
#endif
__global__ void NEST_ADJ64_ATTR k2d_adjoint_rm64(AdjD64Args A) {
    const Geo2D& g = A.g;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = blockIdx.x * DWARPS + warp;
    const int nx = g.nx, ny = g.ny, pitch = g.pitch;
    const int j0 = strip * DSTRIP;
    if (j0 >= ny) return;
    const int r0 = blockIdx.y * A.seg_rows;
    if (r0 >= nx) return;
    const int rows = min(A.seg_rows, nx - r0);
    const long long vs = g.vstride;
    const double dt = *A.dtp;
    const double lx = dt / g.dx, ly = dt / g.dy;
    const double gamma = g.gamma, gm1 = g.gamma - 1.0, igm1 = 1.0 / (g.gamma - 1.0);

    const int col = j0 - 3 + lane;
    int cw = col % ny;
    if (cw < 0) cw += ny;
    const long long coff = cw + 2;
    const bool out = lane >= 3 && lane <= 28 && col < ny;
    auto wrapr = [&](int i) {
        int r = i % nx;
        return r < 0 ? r + nx : r;
    };
    auto rowoff = [&](int i) { return (long long)(wrapr(i) + 2) * pitch + coff; };
    // wrapped rows of the three streams issued at march step a (conserved
    // row a+3, Lout row a+2, Extra row a), advanced by one per step
    auto next_row = [&](int& r) { r = (r + 1 == nx) ? 0 : r + 1; };
    int ru = wrapr(r0 + 1), rl = wrapr(r0), re = wrapr(r0 - 2);

    double* const ring = adj64_ring + warp * DRING + lane;
    double* const ringU = ring;
    double* const ringL = ring + DRU * 128;
    double* const ringE = ring + (DRU + DRL) * 128;
    auto issue_row = [&](const double* base, int r, double* slot) {  // r: wrapped row
        const double* q = base + (long long)(r + 2) * pitch + coff;
        cp8d(slot, q);
        cp8d(slot + 32, q + vs);
        cp8d(slot + 64, q + 2 * vs);
        cp8d(slot + 96, q + 3 * vs);
    };
    auto rd = [&](const double* slot) { return D4{ slot[0], slot[32], slot[64], slot[96] }; };
    auto ld = [&](const double* base, int i) {
        const long long o = rowoff(i);
        return D4{ __ldg(base + o), __ldg(base + vs + o), __ldg(base + 2 * vs + o), __ldg(base + 3 * vs + o) };
    };
    const bool has_extra = A.Extra != nullptr;

    // act bits of rows a-1 .. a+2 (bit 3: row a-1), minmod codes of row a's
    // x-slope (2 bits per variable)
    unsigned actb = 0;
    int brm = 0;
    D4 Wm, W0, W1, P0;
    {
        int k0, k1, k2;
        Wm = prim64(ld(A.U, r0 - 3), gm1, k0);
        W0 = prim64(ld(A.U, r0 - 2), gm1, k1);
        W1 = prim64(ld(A.U, r0 - 1), gm1, k2);
        actb = ((unsigned)k0 << 2) | ((unsigned)k1 << 1) | (unsigned)k2;
        int b0, b1, b2, b3;
        D4 s{ mmb(W0.a - Wm.a, W1.a - W0.a, b0), mmb(W0.b - Wm.b, W1.b - W0.b, b1),
              mmb(W0.c - Wm.c, W1.c - W0.c, b2), mmb(W0.d - Wm.d, W1.d - W0.d, b3) };
        brm = b0 | (b1 << 2) | (b2 << 4) | (b3 << 6);
        P0 = { W0.a + 0.5 * s.a, W0.b + 0.5 * s.b, W0.c + 0.5 * s.c, W0.d + 0.5 * s.d };
        issue_row(A.U, wrapr(r0), ringU + (r0 & (DRU - 1)) * 128);
        issue_row(A.Lout, wrapr(r0 - 2), ringL + ((r0 - 2) & (DRL - 1)) * 128);
        issue_row(A.Lout, wrapr(r0 - 1), ringL + ((r0 - 1) & (DRL - 1)) * 128);
        cpd_commit();
    }
    D4 Bm{ 0, 0, 0, 0 }, B0{ 0, 0, 0, 0 }, Sp{ 0, 0, 0, 0 };

#pragma unroll 1
    for (int a = r0 - 2; a <= r0 + rows; ++a) {
        issue_row(A.U, ru, ringU + ((a + 3) & (DRU - 1)) * 128);
        issue_row(A.Lout, rl, ringL + ((a + 2) & (DRL - 1)) * 128);
        if (has_extra) issue_row(A.Extra, re, ringE + (a & (DRE - 1)) * 128);
        next_row(ru);
        next_row(rl);
        next_row(re);
        cpd_commit();
        cpd_wait1();

        // row a+2, x-slope of row a+1
        int k2;
        const D4 W2 = prim64(rd(ringU + ((a + 2) & (DRU - 1)) * 128), gm1, k2);
        actb = (actb << 1) | (unsigned)k2;
        int c0, c1, c2, c3;
        const D4 s1{ mmb(W1.a - W0.a, W2.a - W1.a, c0), mmb(W1.b - W0.b, W2.b - W1.b, c1),
                     mmb(W1.c - W0.c, W2.c - W1.c, c2), mmb(W1.d - W0.d, W2.d - W1.d, c3) };
        const int brn = c0 | (c1 << 2) | (c2 << 4) | (c3 << 6);

        // x-face a+1/2: left P0, right W1 - s1/2 (normal u, transverse v)
        const D4 L0 = rd(ringL + (a & (DRL - 1)) * 128);
        const D4 L1 = rd(ringL + ((a + 1) & (DRL - 1)) * 128);
        D4 B1{ 0, 0, 0, 0 };
        {
            const D4 M1{ W1.a - 0.5 * s1.a, W1.b - 0.5 * s1.b, W1.c - 0.5 * s1.c, W1.d - 0.5 * s1.d };
            D4 wl{ 0, 0, 0, 0 }, wr{ 0, 0, 0, 0 };
            hlle_adj64(gamma, igm1, P0, M1, lx * (L1.a - L0.a), lx * (L1.b - L0.b), lx * (L1.c - L0.c),
                       lx * (L1.d - L0.d), wl, wr);
            // slope adjoint of row a is complete: wl/2 + Sp, scattered by its code
            auto scat = [&](double wl_, double wr_, double sp, int br, double& bm, double& b0, double& b1) {
                const double s = fma(0.5, wl_, sp);
                const double t1 = br == 1 ? s : 0.0, t2 = br == 2 ? s : 0.0;
                bm -= t1;
                b0 += wl_ + (t1 - t2);
                b1 = wr_ + t2;
            };
            scat(wl.a, wr.a, Sp.a, brm & 3, Bm.a, B0.a, B1.a);
            scat(wl.b, wr.b, Sp.b, (brm >> 2) & 3, Bm.b, B0.b, B1.b);
            scat(wl.c, wr.c, Sp.c, (brm >> 4) & 3, Bm.c, B0.c, B1.c);
            scat(wl.d, wr.d, Sp.d, (brm >> 6) & 3, Bm.d, B0.d, B1.d);
            Sp = { -0.5 * wr.a, -0.5 * wr.b, -0.5 * wr.c, -0.5 * wr.d };
        }

        // y-direction part of row a
        if (a >= r0 && a < r0 + rows) {
            D4 P, R;
            int y0, y1, y2, y3;
            auto yvar = [&](double w, int& br, double& p, double& rr) {
                const double lw = __shfl_up_sync(0xffffffffu, w, 1);
                const double rw = __shfl_down_sync(0xffffffffu, w, 1);
                const double s = mmb(w - lw, rw - w, br);
                p = w + 0.5 * s;
                rr = __shfl_down_sync(0xffffffffu, w - 0.5 * s, 1);
            };
            yvar(W0.a, y0, P.a, R.a);
            yvar(W0.b, y1, P.b, R.b);
            yvar(W0.c, y2, P.c, R.c);
            yvar(W0.d, y3, P.d, R.d);
            const D4 Lr{ __shfl_down_sync(0xffffffffu, L0.a, 1), __shfl_down_sync(0xffffffffu, L0.b, 1),
                         __shfl_down_sync(0xffffffffu, L0.c, 1), __shfl_down_sync(0xffffffffu, L0.d, 1) };
            // face (c | c+1): normal v, transverse u; flux order (mass, mv, mu, E)
            const D4 PL{ P.a, P.c, P.b, P.d }, RR{ R.a, R.c, R.b, R.d };
            D4 wl{ 0, 0, 0, 0 }, wr{ 0, 0, 0, 0 };
            hlle_adj64(gamma, igm1, PL, RR, ly * (Lr.a - L0.a), ly * (Lr.c - L0.c), ly * (Lr.b - L0.b),
                       ly * (Lr.d - L0.d), wl, wr);
            auto ycell = [&](double l, double r, int br, double& b) {
                const double q = __shfl_up_sync(0xffffffffu, r, 1);  // right-state adjoint of the face on the left
                const double sb = 0.5 * (l - q);
                const double t1 = br == 1 ? sb : 0.0, t2 = br == 2 ? sb : 0.0;
                const double t1n = __shfl_down_sync(0xffffffffu, t1, 1);
                const double t2p = __shfl_up_sync(0xffffffffu, t2, 1);
                b += (l + q) + ((t1 - t2) + (t2p - t1n));
            };
            ycell(wl.a, wr.a, y0, B0.a);
            ycell(wl.c, wr.c, y1, B0.b);
            ycell(wl.b, wr.b, y2, B0.c);
            ycell(wl.d, wr.d, y3, B0.d);
        }

        // row a-1 is complete
        if (a - 1 >= r0 && out) {
            const D4 Lm = rd(ringL + ((a - 1) & (DRL - 1)) * 128);
            const double ir = 1.0 / Wm.a, u = Wm.b, v = Wm.c;
            const double g3 = ((actb >> 3) & 1u) ? gm1 * Bm.d : 0.0;
            const double q2 = 0.5 * fma(v, v, u * u);
            D4 o{ fma(g3, q2, Bm.a - fma(Bm.c, v, Bm.b * u) * ir), fma(-g3, u, Bm.b * ir), fma(-g3, v, Bm.c * ir),
                  g3 };
            o = { A.alpha * (Lm.a + o.a), A.alpha * (Lm.b + o.b), A.alpha * (Lm.c + o.c), A.alpha * (Lm.d + o.d) };
            if (has_extra) {
                const D4 E = rd(ringE + ((a - 1) & (DRE - 1)) * 128);
                o = { fma(A.beta, E.a, o.a), fma(A.beta, E.b, o.b), fma(A.beta, E.c, o.c), fma(A.beta, E.d, o.d) };
            }
            const long long off = (long long)(a - 1 + 2) * pitch + col + 2;
            A.Lin[off] = o.a;
            A.Lin[vs + off] = o.b;
            A.Lin[2 * vs + off] = o.c;
            A.Lin[3 * vs + off] = o.d;
        }

        Wm = W0; W0 = W1; W1 = W2;
        P0 = { W0.a + 0.5 * s1.a, W0.b + 0.5 * s1.b, W0.c + 0.5 * s1.c, W0.d + 0.5 * s1.d };
        brm = brn;
        Bm = B0; B0 = B1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

}  // namespace

// Row-march form of the FP64 2D adjoint stage (any ny).
cudaError_t launch_2d_adjoint_stage_f64rm(const double* U, const double* Lout, const double* Extra, double* Lin,
                                          const Geo2D& g, const double* dtp, double alpha, double beta,
                                          cudaStream_t st) {
    const size_t smem = sizeof(double) * DRING * DWARPS;
    constexpr int MAXDEV = 64;
    static std::mutex mu;
    static int dev_sms[MAXDEV] = {}, dev_per_sm[MAXDEV] = {};
    int dev = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    int sms = 0, per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < MAXDEV && dev_sms[dev] > 0) {
            sms = dev_sms[dev];
            per_sm = dev_per_sm[dev];
        } else {
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k2d_adjoint_rm64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
                return e;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2d_adjoint_rm64, 32 * DWARPS, smem)) !=
                cudaSuccess)
                return e;
            if (per_sm < 1) per_sm = 1;
            if (dev < MAXDEV) {
                dev_sms[dev] = sms;
                dev_per_sm[dev] = per_sm;
            }
        }
    }
    const int strips = (g.ny + DSTRIP - 1) / DSTRIP;
    const int cx = (strips + DWARPS - 1) / DWARPS;
    const long long slots = (long long)sms * per_sm * DWARPS;
    int segs = (int)std::max<long long>(1, slots / ((long long)cx * DWARPS));
    int seg_rows = (g.nx + segs - 1) / segs;
    if (seg_rows < 16) seg_rows = 16;
    segs = (g.nx + seg_rows - 1) / seg_rows;
    AdjD64Args a{ U, Lout, Extra, Lin, g, dtp, alpha, beta, seg_rows };
    k2d_adjoint_rm64<<<dim3(cx, segs), 32 * DWARPS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace nestb
