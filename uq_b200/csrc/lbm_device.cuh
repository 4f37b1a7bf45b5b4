// Device-side building blocks of the D2Q13 thermal LBM step (sm_100a).
//
// Every function restates a piece of the reference FP64 CPU solver
// CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp (cited per function) for the GPU's
// structure-of-arrays layout: per sample, 26 planes (f_0..f_12, h_0..h_12),
// each plane ny rows of `pitch` elements, x fastest.  Templates take the
// storage type S (double or float) and the compute type C; moment sums are
// always accumulated in double.
#pragma once

#include <cstdint>

namespace uqlbm {

constexpr int NQ = 13;
constexpr int NPL = 26;  // f and h planes

// node-flag byte: cell type in bits 0-1 (0 fluid, 1 permanent, 2 solid);
// bits 2-5 say whether the 5-point x / y stencil of the node meets a solid
// node or the domain edge (then the exact boundary-aware stencil runs).
constexpr uint8_t NF_TYPE = 3;
constexpr uint8_t NF_SOLX = 4;
constexpr uint8_t NF_SOLY = 8;
constexpr uint8_t NF_EDGX = 16;   // near a clamped/mirrored x edge
constexpr uint8_t NF_EDGY = 32;
constexpr uint8_t NF_WRPX = 64;   // x stencil wraps across a periodic edge
constexpr uint8_t NF_WRPY = 128;

// sample flag bits
constexpr int SF_PERX = 1, SF_PERY = 2, SF_MIRN = 4, SF_MIRS = 8, SF_MIRE = 16, SF_MIRW = 32;

struct SampleParams {
    int nx, ny, pitch, flags;
    int rk, fm;          // RKMETHOD, FMETHOD
    int ntile;           // tiles of this sample in the full tile list
    int first_tile;
    long long state_off; // element offset of plane 0 in every state buffer
    long long plane;     // elements per plane
    long long node_off;  // offset into per-node arrays
    int xoff, yoff;      // offsets into the per-column / per-row spacing tables
    double R, bR, K, Tc, inv_sRTc, RTc, mu, Pr, dt, c;
    // Reference rest state of the stored deviations (mixed path): the state
    // holds f - f_ref, h - h_ref with f_ref, h_ref the equilibria at
    // (rho0, 0, 0, T0); rho0 = shref = 0 (full storage) on the FP64 path.
    double rho0, T0n, shref;  // T0n = T0 / Tc
    double inv_mu, two_over_bR;
    int wide;  // FP32 WENO5 weights in the range-safe form (see weno5)
    // ghost columns of the stage buffers (0 or GHOST_X): x-periodic samples
    // keep, left and right of every row of buffers 2 and 3, the periodic
    // images of the gx columns at the other edge, so the staged halo boxes
    // of tiles at those edges load them as they load any interior node.
    // Rows stay aligned (pitch >= nx + 2 gx, a multiple of 32): the right
    // ghosts follow the row, the left ones are the last gx elements of the
    // row before (the sample's region starts GHOST_SLACK elements before
    // plane 0 for the first row's).  The per-node arrays have no ghosts.
    int gx;
    // viscosity law (codeCL.py:986-990): 0 constant mu, 1 VHS, 2 Sutherland;
    // mu(T) = mu (T/visc_T)^visc_exp [(visc_T + visc_S)/(T + visc_S)]
    int visc;
    double visc_exp, visc_S, visc_T;
};

constexpr int GHOST_X = 4;       // = the staged box's x halo
constexpr int GHOST_SLACK = 32;  // state elements before plane 0 of a sample with ghosts (keeps it aligned)

struct Tile {
    int sample;
    int x0, y0;
    int gid;  // index of the tile in the batch's full tile list; bit 30: simple
};

// A simple tile lies at least 3 nodes inside its domain and neither it nor
// its 3-node halo holds a solid/permanent node or a node whose stencil meets
// a solid or an edge: every flux it needs comes straight from the staged box.
// A wrap tile is a full tile that would be simple but for a periodic edge:
// its halo crosses it (along a periodic axis) and holds only plain fluid
// nodes, so once the periodic images are copied into the staged box every
// flux comes from the box as in a simple tile.
constexpr int TILE_SIMPLE = 1 << 30;
constexpr int TILE_WRAP = 1 << 29;
__host__ __device__ inline int tile_gid(const Tile &t) { return t.gid & (TILE_WRAP - 1); }
__host__ __device__ inline bool tile_simple(const Tile &t) { return (t.gid & TILE_SIMPLE) != 0; }
__host__ __device__ inline bool tile_wrap(const Tile &t) { return (t.gid & TILE_WRAP) != 0; }

// lattice (setupVars, cpuLBM.cpp:376-388) in units of c, its signs, and the
// reflection maps of mirIndex (cpuLBM.cpp:1147-1169)
__constant__ int c_EX[NQ] = {0, 1, 0, -1, 0, 1, -1, -1, 1, 2, 0, -2, 0};
__constant__ int c_EY[NQ] = {0, 0, 1, 0, -1, 1, 1, -1, -1, 0, 2, 0, -2};
__constant__ int c_MIR_NS[NQ] = {0, 1, 4, 3, 2, 8, 7, 6, 5, 9, 12, 11, 10};
__constant__ int c_MIR_EW[NQ] = {0, 3, 2, 1, 4, 6, 5, 8, 7, 11, 10, 9, 12};

// the same lattice as compile-time constants (for unrolled direction loops)
constexpr int kEX[NQ] = {0, 1, 0, -1, 0, 1, -1, -1, 1, 2, 0, -2, 0};
constexpr int kEY[NQ] = {0, 0, 1, 0, -1, 1, 1, -1, -1, 0, 2, 0, -2};

// the same as functions: compile-time values in unrolled loops, no table
__host__ __device__ constexpr int lat_ex(int i)
{
    return (i == 1 || i == 5 || i == 8) ? 1 : (i == 3 || i == 6 || i == 7) ? -1 : i == 9 ? 2 : i == 11 ? -2 : 0;
}
__host__ __device__ constexpr int lat_ey(int i)
{
    return (i == 2 || i == 5 || i == 6) ? 1 : (i == 4 || i == 7 || i == 8) ? -1 : i == 10 ? 2 : i == 12 ? -2 : 0;
}
constexpr bool lat_fn_match()
{
    for (int i = 0; i < NQ; ++i)
        if (lat_ex(i) != kEX[i] || lat_ey(i) != kEY[i]) return false;
    return true;
}
static_assert(lat_fn_match(), "lattice functions differ from the table");

__device__ __forceinline__ int isgn(int a) { return (a > 0) - (a < 0); }

// Round-to-nearest operations the compiler may neither fuse nor split:
// NND, WENO5, the flux divergence, the wall fluxes and, on the FP32 path,
// the equilibria and the RK3 stage updates are written with them so that
// every compiled instance (the
// simple-tile paths per scheme, the boundary-aware
// paths, the wall factors, the tile-shape instances) rounds a node the same
// way, and results do not depend on which path a node took (tile shape,
// batch packing).
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float xneg(float a) { return -a; }
__device__ __forceinline__ double xneg(double a) { return -a; }
__device__ __forceinline__ float xmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double xmin(double a, double b) { return fmin(a, b); }
// The same operations on a packed pair of FP32 values (the f and h planes
// of one face), one sm_100 f32x2 instruction each: every lane is rounded
// exactly as the scalar operation rounds it, so a face reconstructed in
// pairs equals the scalar reconstruction bit for bit.  a - b is formed as
// fma(b, -1, a), which is a - b correctly rounded.
__device__ __forceinline__ float2 xmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 xadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 xsub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 xfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 xneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 xmin(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }

// a constant in the arithmetic type (both lanes of a pair)
template <class C>
__device__ __forceinline__ C kc(double v) { return C(v); }
template <>
__device__ __forceinline__ float2 kc<float2>(double v) { return make_float2((float)v, (float)v); }
// FP32 arithmetic, scalar or packed
template <class C>
struct IsF32 { static constexpr bool value = false; };
template <>
struct IsF32<float> { static constexpr bool value = true; };
template <>
struct IsF32<float2> { static constexpr bool value = true; };

// ------------------------------------------------------------ equilibria
// equilibrium2D (cpuLBM.cpp:785-844) with the polynomials of
// inlineFunctions.cpp:10-61, evaluated per symmetry family.  Normalised
// u, v, T are u/sqrt(R Tc), v/sqrt(R Tc), T/Tc; with a = u^2, c = v^2:
//   f0      = 1 + 5/2 T^2 + 5/2 T (a + c - 1) + (a^2 + c^2)/4 + a c - 5/4 (a + c)
//   f1, f3  = E1(u, v) +- O1(u, v);   f2, f4 = E1(v, u) +- O1(v, u)
//   f5..f8  = (T + a +- u)(T + c +- v) / 4
//   f9, f11 = E9(u) +- O9(u);         f10, f12 = E9(v) +- O9(v)
// times rho, and the h families times rho R Tc.
template <class C>
struct EqState {
    C rho, u, v, T, K, rRTc;  // normalised velocity/temperature
};

template <class C>
__device__ __forceinline__ EqState<C> eq_state(double rho, double ux, double uy, double T, const SampleParams &sp)
{
    EqState<C> e;
    e.rho = (C)rho;
    e.u = (C)(ux * sp.inv_sRTc);
    e.v = (C)(uy * sp.inv_sRTc);
    e.T = (C)(T / sp.Tc);
    e.K = (C)sp.K;
    e.rRTc = (C)(rho * sp.RTc);
    return e;
}

// family 0: direction 0
template <class C>
__device__ __forceinline__ void eq_fam0(const EqState<C> &q, C &f0, C &h0)
{
    const C a = q.u * q.u, c = q.v * q.v, s2 = a + c, pc = a * c, T = q.T, T2 = T * T, T3 = T2 * T, K = q.K;
    f0 = q.rho * (C(1) + C(2.5) * T2 + C(2.5) * T * (s2 - C(1)) + C(0.25) * (a * a + c * c) + pc - C(1.25) * s2);
    h0 = q.rRTc * (T3 * (C(1.25) * K + C(20.0 / 3.0)) + T2 * ((C(1.25) * K + C(11.25)) * s2 - C(1.25) * K - C(5))
                   + T * (C(0.125) * K * (s2 * s2 + C(2) * pc) - C(0.625) * K * s2 + C(0.5) * K + C(2.5) * s2 * s2
                          + C(2.5) * pc - C(5) * s2 + C(1))
                   + s2 * s2 * s2 * C(0.125) + C(0.25) * pc * s2 - C(0.625) * s2 * s2 + C(0.5) * s2);
}

// family 1: directions 1..4 (out[0..3] = f1..f4, h1..h4)
template <class C>
__device__ __forceinline__ void eq_fam1(const EqState<C> &q, C *f, C *h)
{
    const C T = q.T, T2 = T * T, T3 = T2 * T, K = q.K;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const C U = k == 0 ? q.u : q.v;
        const C W = k == 0 ? q.v : q.u;
        const C A = U * U, Cc = W * W;
        C E = -T2 + T * (C(2.0 / 3.0) - C(1.5) * A - C(0.5) * Cc) + C(2.0 / 3.0) * A - A * A * C(1.0 / 6.0) - C(0.5) * A * Cc;
        C O = U * (C(2.0 / 3.0) - T - A * C(1.0 / 6.0) - C(0.5) * Cc);
        f[k] = q.rho * (E + O);
        f[k + 2] = q.rho * (E - O);
        E = T3 * (C(-0.5) * K - C(8.0 / 3.0))
            + T2 * (-(C(0.75) * K + C(6.5)) * A - (C(0.25) * K + C(2.5)) * Cc + K * C(1.0 / 3.0) + C(4.0 / 3.0))
            + T * (-(K * C(1.0 / 12.0) + C(19.0 / 12.0)) * A * A - (C(0.25) * K + C(3.5)) * A * Cc
                   + (K * C(1.0 / 3.0) + C(7.0 / 3.0)) * A - C(0.25) * Cc * Cc + Cc * C(1.0 / 3.0))
            - A * A * A * C(1.0 / 12.0) - A * A * Cc * C(1.0 / 3.0) + A * A * C(1.0 / 3.0) - C(0.25) * A * Cc * Cc
            + A * Cc * C(1.0 / 3.0);
        O = U * (T2 * (C(-0.5) * K - C(3))
                 + T * (-(K * C(1.0 / 12.0) + C(7.0 / 6.0)) * A - (C(0.25) * K + C(2.5)) * Cc + K * C(1.0 / 3.0) + C(4.0 / 3.0))
                 - A * A * C(1.0 / 12.0) - A * Cc * C(1.0 / 3.0) + A * C(1.0 / 3.0) - C(0.25) * Cc * Cc + Cc * C(1.0 / 3.0));
        h[k] = q.rRTc * (E + O);
        h[k + 2] = q.rRTc * (E - O);
    }
}

// family 5: directions 5..8
template <class C>
__device__ __forceinline__ void eq_fam5(const EqState<C> &q, C *f, C *h)
{
    const C u = q.u, v = q.v, a = u * u, c = v * v, s2 = a + c, pc = a * c, T = q.T, T2 = T * T, T3 = T2 * T, K = q.K;
    const C Ap = T + a + u, Am = T + a - u, Bp = T + c + v, Bm = T + c - v, r4 = C(0.25) * q.rho;
    f[0] = r4 * (Ap * Bp);
    f[1] = r4 * (Am * Bp);
    f[2] = r4 * (Am * Bm);
    f[3] = r4 * (Ap * Bm);
    const C k8 = C(0.125) * K;
    const C EE = T3 * (k8 + C(2.0 / 3.0)) + T2 * (k8 + C(1.125)) * s2 + T * ((k8 + C(1.5)) * pc + C(0.125) * (a * a + c * c))
                 + C(0.125) * pc * s2;
    const C OE = u * (T2 * (k8 + C(0.75)) + T * ((k8 + C(1.125)) * c + C(0.125) * a) + C(0.125) * c * s2);
    const C EO = v * (T2 * (k8 + C(0.75)) + T * ((k8 + C(1.125)) * a + C(0.125) * c) + C(0.125) * a * s2);
    const C OO = u * v * (T * (k8 + C(0.75)) + C(0.125) * s2);
    h[0] = q.rRTc * (EE + OE + EO + OO);
    h[1] = q.rRTc * (EE - OE + EO - OO);
    h[2] = q.rRTc * (EE - OE - EO + OO);
    h[3] = q.rRTc * (EE + OE - EO - OO);
}

// family 9: directions 9..12
template <class C>
__device__ __forceinline__ void eq_fam9(const EqState<C> &q, C *f, C *h)
{
    const C T = q.T, T2 = T * T, T3 = T2 * T, K = q.K;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const C U = k == 0 ? q.u : q.v;
        const C W = k == 0 ? q.v : q.u;
        const C A = U * U, Cc = W * W;
        C E = C(0.125) * T2 + T * (C(0.25) * A - C(1.0 / 24.0)) + (A * A - A) * C(1.0 / 24.0);
        C O = U * (C(0.25) * T + (A - C(1)) * C(1.0 / 12.0));
        f[k] = q.rho * (E + O);
        f[k + 2] = q.rho * (E - O);
        E = T3 * (K * C(1.0 / 16.0) + C(1.0 / 3.0))
            + T2 * ((C(0.125) * K + C(17.0 / 16.0)) * A + Cc * C(1.0 / 16.0) - K * C(1.0 / 48.0) - C(1.0 / 12.0))
            + T * ((K * C(1.0 / 48.0) + C(1.0 / 3.0)) * A * A - (K * C(1.0 / 48.0) + C(7.0 / 48.0)) * A + C(0.125) * A * Cc
                   - Cc * C(1.0 / 48.0))
            + (A * A * A + A * A * Cc - A * A - A * Cc) * C(1.0 / 48.0);
        O = U * (T2 * (C(0.125) * K + C(0.75)) + T * ((K * C(1.0 / 24.0) + C(11.0 / 24.0)) * A - K * C(1.0 / 24.0) - C(1.0 / 6.0) + C(0.125) * Cc)
                 + (A * A + A * Cc - A - Cc) * C(1.0 / 24.0));
        h[k] = q.rRTc * (E + O);
        h[k + 2] = q.rRTc * (E - O);
    }
}

// ------------------------------------------------ equilibria as deviations
// The same polynomials as deviations from the rest state (rho0, 0, 0, T0)
// of the sample, for the FP32 path: f_eq - f_ref = rho dP + (rho - rho0) P0
// where dP = P(u, v, T) - P(0, 0, T0) keeps only terms that vanish at rest:
// the T-only part g(T) - g(T0) is factored as (T - T0) G(T, T0), so no
// O(1) terms cancel in FP32.  Likewise for h with the factor R Tc.
template <class C>
struct EqDev {
    C rho, drho, u, v, T, tau, T0, K, RTc;
};

template <class C>
__device__ __forceinline__ EqDev<C> eq_dev(double rho, double ux, double uy, double T, const SampleParams &sp)
{
    EqDev<C> e;
    e.rho = (C)rho;
    e.drho = (C)(rho - sp.rho0);
    e.u = (C)(ux * sp.inv_sRTc);
    e.v = (C)(uy * sp.inv_sRTc);
    const double Tn = T / sp.Tc;
    e.T = (C)Tn;
    e.tau = (C)(Tn - sp.T0n);
    e.T0 = (C)sp.T0n;
    e.K = (C)sp.K;
    e.RTc = (C)sp.RTc;
    return e;
}

template <class C>
__device__ __forceinline__ void eqd_fam0(const EqDev<C> &q, C &f0, C &h0)
{
    const C a = q.u * q.u, c = q.v * q.v, s2 = a + c, pc = a * c, T = q.T, T2 = T * T, K = q.K, T0 = q.T0;
    const C S2 = T + T0, S3 = T2 + T * T0 + T0 * T0;
    const C dP = C(2.5) * T * s2 + C(0.25) * (a * a + c * c) + pc - C(1.25) * s2 + q.tau * (C(2.5) * S2 - C(2.5));
    const C P0 = C(1) + C(2.5) * T0 * T0 - C(2.5) * T0;
    f0 = q.rho * dP + q.drho * P0;
    const C dQ = T2 * (C(1.25) * K + C(11.25)) * s2
                 + T * (C(0.125) * K * (s2 * s2 + C(2) * pc) - C(0.625) * K * s2 + C(2.5) * s2 * s2 + C(2.5) * pc - C(5) * s2)
                 + s2 * s2 * s2 * C(0.125) + C(0.25) * pc * s2 - C(0.625) * s2 * s2 + C(0.5) * s2
                 + q.tau * ((C(1.25) * K + C(20.0 / 3.0)) * S3 + (C(-1.25) * K - C(5)) * S2 + C(0.5) * K + C(1));
    const C Q0 = T0 * T0 * T0 * (C(1.25) * K + C(20.0 / 3.0)) + T0 * T0 * (C(-1.25) * K - C(5)) + T0 * (C(0.5) * K + C(1));
    h0 = q.RTc * (q.rho * dQ + q.drho * Q0);
}

template <class C>
__device__ __forceinline__ void eqd_fam1(const EqDev<C> &q, C *f, C *h)
{
    const C T = q.T, T2 = T * T, K = q.K, T0 = q.T0;
    const C S2 = T + T0, S3 = T2 + T * T0 + T0 * T0;
    const C P0 = -T0 * T0 + C(2.0 / 3.0) * T0;
    const C Q0 = T0 * T0 * T0 * (C(-0.5) * K - C(8.0 / 3.0)) + T0 * T0 * (K * C(1.0 / 3.0) + C(4.0 / 3.0));
    const C Gf = -S2 + C(2.0 / 3.0);
    const C Gh = (C(-0.5) * K - C(8.0 / 3.0)) * S3 + (K * C(1.0 / 3.0) + C(4.0 / 3.0)) * S2;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const C U = k == 0 ? q.u : q.v;
        const C W = k == 0 ? q.v : q.u;
        const C A = U * U, Cc = W * W;
        C E = T * (C(-1.5) * A - C(0.5) * Cc) + C(2.0 / 3.0) * A - A * A * C(1.0 / 6.0) - C(0.5) * A * Cc + q.tau * Gf;
        C O = U * (C(2.0 / 3.0) - T - A * C(1.0 / 6.0) - C(0.5) * Cc);
        f[k] = q.rho * (E + O) + q.drho * P0;
        f[k + 2] = q.rho * (E - O) + q.drho * P0;
        E = T2 * (-(C(0.75) * K + C(6.5)) * A - (C(0.25) * K + C(2.5)) * Cc)
            + T * (-(K * C(1.0 / 12.0) + C(19.0 / 12.0)) * A * A - (C(0.25) * K + C(3.5)) * A * Cc
                   + (K * C(1.0 / 3.0) + C(7.0 / 3.0)) * A - C(0.25) * Cc * Cc + Cc * C(1.0 / 3.0))
            - A * A * A * C(1.0 / 12.0) - A * A * Cc * C(1.0 / 3.0) + A * A * C(1.0 / 3.0) - C(0.25) * A * Cc * Cc
            + A * Cc * C(1.0 / 3.0) + q.tau * Gh;
        O = U * (T2 * (C(-0.5) * K - C(3))
                 + T * (-(K * C(1.0 / 12.0) + C(7.0 / 6.0)) * A - (C(0.25) * K + C(2.5)) * Cc + K * C(1.0 / 3.0) + C(4.0 / 3.0))
                 - A * A * C(1.0 / 12.0) - A * Cc * C(1.0 / 3.0) + A * C(1.0 / 3.0) - C(0.25) * Cc * Cc + Cc * C(1.0 / 3.0));
        h[k] = q.RTc * (q.rho * (E + O) + q.drho * Q0);
        h[k + 2] = q.RTc * (q.rho * (E - O) + q.drho * Q0);
    }
}

template <class C>
__device__ __forceinline__ void eqd_fam5(const EqDev<C> &q, C *f, C *h)
{
    const C u = q.u, v = q.v, a = u * u, c = v * v, s2 = a + c, pc = a * c, T = q.T, T2 = T * T, K = q.K, T0 = q.T0;
    const C S2 = T + T0, S3 = T2 + T * T0 + T0 * T0;
    const C P0 = C(0.25) * T0 * T0;
    const C base = C(0.25) * q.tau * S2;
    const C Ap = a + u, Am = a - u, Bp = c + v, Bm = c - v;
    f[0] = q.rho * (base + C(0.25) * (T * (Ap + Bp) + Ap * Bp)) + q.drho * P0;
    f[1] = q.rho * (base + C(0.25) * (T * (Am + Bp) + Am * Bp)) + q.drho * P0;
    f[2] = q.rho * (base + C(0.25) * (T * (Am + Bm) + Am * Bm)) + q.drho * P0;
    f[3] = q.rho * (base + C(0.25) * (T * (Ap + Bm) + Ap * Bm)) + q.drho * P0;
    const C k8 = C(0.125) * K;
    const C Q0 = T0 * T0 * T0 * (k8 + C(2.0 / 3.0));
    const C EE = T2 * (k8 + C(1.125)) * s2 + T * ((k8 + C(1.5)) * pc + C(0.125) * (a * a + c * c)) + C(0.125) * pc * s2
                 + q.tau * (k8 + C(2.0 / 3.0)) * S3;
    const C OE = u * (T2 * (k8 + C(0.75)) + T * ((k8 + C(1.125)) * c + C(0.125) * a) + C(0.125) * c * s2);
    const C EO = v * (T2 * (k8 + C(0.75)) + T * ((k8 + C(1.125)) * a + C(0.125) * c) + C(0.125) * a * s2);
    const C OO = u * v * (T * (k8 + C(0.75)) + C(0.125) * s2);
    h[0] = q.RTc * (q.rho * (EE + OE + EO + OO) + q.drho * Q0);
    h[1] = q.RTc * (q.rho * (EE - OE + EO - OO) + q.drho * Q0);
    h[2] = q.RTc * (q.rho * (EE - OE - EO + OO) + q.drho * Q0);
    h[3] = q.RTc * (q.rho * (EE + OE - EO - OO) + q.drho * Q0);
}

template <class C>
__device__ __forceinline__ void eqd_fam9(const EqDev<C> &q, C *f, C *h)
{
    const C T = q.T, T2 = T * T, K = q.K, T0 = q.T0;
    const C S2 = T + T0, S3 = T2 + T * T0 + T0 * T0;
    const C P0 = C(0.125) * T0 * T0 - T0 * C(1.0 / 24.0);
    const C Q0 = T0 * T0 * T0 * (K * C(1.0 / 16.0) + C(1.0 / 3.0)) + T0 * T0 * (-K * C(1.0 / 48.0) - C(1.0 / 12.0));
    const C Gf = S2 * C(0.125) - C(1.0 / 24.0);
    const C Gh = (K * C(1.0 / 16.0) + C(1.0 / 3.0)) * S3 + (-K * C(1.0 / 48.0) - C(1.0 / 12.0)) * S2;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const C U = k == 0 ? q.u : q.v;
        const C W = k == 0 ? q.v : q.u;
        const C A = U * U, Cc = W * W;
        C E = T * A * C(0.25) + (A * A - A) * C(1.0 / 24.0) + q.tau * Gf;
        C O = U * (C(0.25) * T + (A - C(1)) * C(1.0 / 12.0));
        f[k] = q.rho * (E + O) + q.drho * P0;
        f[k + 2] = q.rho * (E - O) + q.drho * P0;
        E = T2 * ((C(0.125) * K + C(17.0 / 16.0)) * A + Cc * C(1.0 / 16.0))
            + T * ((K * C(1.0 / 48.0) + C(1.0 / 3.0)) * A * A - (K * C(1.0 / 48.0) + C(7.0 / 48.0)) * A + C(0.125) * A * Cc
                   - Cc * C(1.0 / 48.0))
            + (A * A * A + A * A * Cc - A * A - A * Cc) * C(1.0 / 48.0) + q.tau * Gh;
        O = U * (T2 * (C(0.125) * K + C(0.75)) + T * ((K * C(1.0 / 24.0) + C(11.0 / 24.0)) * A - K * C(1.0 / 24.0) - C(1.0 / 6.0) + C(0.125) * Cc)
                 + (A * A + A * Cc - A - Cc) * C(1.0 / 24.0));
        h[k] = q.RTc * (q.rho * (E + O) + q.drho * Q0);
        h[k + 2] = q.RTc * (q.rho * (E - O) + q.drho * Q0);
    }
}

// ------------------------- FP32 deviations: explicitly rounded, lanes paired
// The FP32 path evaluates the deviation polynomials above with every
// operation explicitly rounded (no compiler contraction), so every kernel
// that computes a node's equilibria gives it the same bits.  The terms are
// those of the generic form, regrouped (common factors, Horner form).  In
// families 1 and 9 the two axis pairs (k = 0: U = u, W = v; k = 1: U = v,
// W = u) are the two lanes of packed f32x2 operations; in family 5 the
// lanes are the sign of u in f (for v + and -) and (OE, EO) in h.
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }

__device__ __forceinline__ void eqd_fam0(const EqDev<float> &q, float &f0, float &h0)
{
    const float u = q.u, v = q.v, T = q.T, K = q.K, T0 = q.T0, tau = q.tau;
    const float a = xmul(u, u), c = xmul(v, v), s2 = xadd(a, c), pc = xmul(a, c), T2 = xmul(T, T);
    const float S2 = xadd(T, T0), S3 = xfma(T, S2, xmul(T0, T0));
    // dP = s2 (5/2 T - 5/4 + s2/4) + pc/2 + 5/2 tau (S2 - 1), P0 = 1 + 5/2 T0 (T0 - 1)
    const float dP = xfma(s2, xfma(0.25f, s2, xfma(2.5f, T, -1.25f)),
                          xfma(0.5f, pc, xmul(xmul(2.5f, tau), xadd(S2, -1.0f))));
    const float P0 = xfma(xmul(2.5f, T0), xadd(T0, -1.0f), 1.0f);
    f0 = xfma(q.rho, dP, xmul(q.drho, P0));
    // dQ = T2 (5/4 K + 45/4) s2 + T (s2 ((K/8 + 5/2) s2 - 5/8 K - 5) + (K/4 + 5/2) pc)
    //      + s2 (s2 (s2/8 - 5/8) + pc/4 + 1/2) + tau (k3 S3 + k2 S2 + k1),
    // Q0 = T0 (T0 (T0 k3 + k2) + k1)
    const float k3 = xfma(1.25f, K, 20.0f / 3.0f), k2 = xfma(-1.25f, K, -5.0f), k1 = xfma(0.5f, K, 1.0f);
    const float tT = xfma(s2, xfma(xfma(0.125f, K, 2.5f), s2, xfma(-0.625f, K, -5.0f)), xmul(xfma(0.25f, K, 2.5f), pc));
    const float rest = xmul(s2, xfma(s2, xfma(0.125f, s2, -0.625f), xfma(0.25f, pc, 0.5f)));
    const float tG = xmul(tau, xfma(k3, S3, xfma(k2, S2, k1)));
    const float dQ = xfma(T2, xmul(xfma(1.25f, K, 11.25f), s2), xfma(T, tT, xadd(rest, tG)));
    const float Q0 = xmul(T0, xfma(T0, xfma(T0, k3, k2), k1));
    h0 = xmul(q.RTc, xfma(q.rho, dQ, xmul(q.drho, Q0)));
}

__device__ __forceinline__ void eqd_fam1(const EqDev<float> &q, float *f, float *h)
{
    const float T = q.T, K = q.K, T0 = q.T0, tau = q.tau, T2 = xmul(T, T);
    const float S2 = xadd(T, T0), S3 = xfma(T, S2, xmul(T0, T0));
    const float kh3 = xfma(-0.5f, K, -8.0f / 3.0f), kh2 = xfma(K, 1.0f / 3.0f, 4.0f / 3.0f);
    const float P0 = xmul(T0, xsub(2.0f / 3.0f, T0));
    const float Q0 = xmul(xmul(T0, T0), xfma(T0, kh3, kh2));
    const float tGf = xmul(tau, xsub(2.0f / 3.0f, S2));
    const float tGh = xmul(tau, xfma(kh3, S3, xmul(kh2, S2)));
    const float2 U = make_float2(q.u, q.v), W = make_float2(q.v, q.u);
    const float2 A = xmul(U, U), Cc = xmul(W, W), vT = bc2(T), vT2 = bc2(T2), vr = bc2(q.rho);
    // f: E = T (-3/2 A - Cc/2) + A (m - A/6) + tau Gf, O = U (m - T - A/6), m = 2/3 - Cc/2
    const float2 m = xfma(kc<float2>(-0.5), Cc, kc<float2>(2.0 / 3.0));
    const float2 Ef = xfma(vT, xfma(kc<float2>(-1.5), A, xmul(kc<float2>(-0.5), Cc)),
                           xfma(A, xfma(kc<float2>(-1.0 / 6.0), A, m), bc2(tGf)));
    const float2 Of = xmul(U, xfma(kc<float2>(-1.0 / 6.0), A, xsub(m, vT)));
    const float2 dP0 = bc2(xmul(q.drho, P0));
    const float2 fp = xfma(vr, xadd(Ef, Of), dP0), fm = xfma(vr, xsub(Ef, Of), dP0);
    f[0] = fp.x; f[1] = fp.y; f[2] = fm.x; f[3] = fm.y;
    // h: with CB = Cc (1/3 - Cc/4) and R = A (1/3 - A/12 - Cc/3) + CB,
    // E = T2 (c1 A + c2 Cc) + T (A (c3 A + c4 Cc + c5) + CB) + A R + tau Gh,
    // O = U (T2 c8 + T (c6 A + c2 Cc + kh2) + R)
    const float c1 = xfma(-0.75f, K, -6.5f), c2 = xfma(-0.25f, K, -2.5f), c3 = xfma(K, -1.0f / 12.0f, -19.0f / 12.0f);
    const float c4 = xfma(-0.25f, K, -3.5f), c5 = xfma(K, 1.0f / 3.0f, 7.0f / 3.0f), c6 = xfma(K, -1.0f / 12.0f, -7.0f / 6.0f);
    const float c8 = xfma(-0.5f, K, -3.0f);
    const float2 CB = xmul(Cc, xfma(kc<float2>(-0.25), Cc, kc<float2>(1.0 / 3.0)));
    const float2 R = xfma(A, xfma(kc<float2>(-1.0 / 12.0), A, xfma(kc<float2>(-1.0 / 3.0), Cc, kc<float2>(1.0 / 3.0))), CB);
    const float2 Eh = xfma(vT2, xfma(bc2(c1), A, xmul(bc2(c2), Cc)),
                           xfma(vT, xfma(A, xfma(bc2(c3), A, xfma(bc2(c4), Cc, bc2(c5))), CB), xfma(A, R, bc2(tGh))));
    const float2 Oh = xmul(U, xfma(vT2, bc2(c8), xfma(vT, xfma(bc2(c6), A, xfma(bc2(c2), Cc, bc2(kh2))), R)));
    const float2 dQ0 = bc2(xmul(q.drho, Q0)), vR = bc2(q.RTc);
    const float2 hp = xmul(vR, xfma(vr, xadd(Eh, Oh), dQ0)), hm = xmul(vR, xfma(vr, xsub(Eh, Oh), dQ0));
    h[0] = hp.x; h[1] = hp.y; h[2] = hm.x; h[3] = hm.y;
}

__device__ __forceinline__ void eqd_fam5(const EqDev<float> &q, float *f, float *h)
{
    const float u = q.u, v = q.v, T = q.T, K = q.K, T0 = q.T0, tau = q.tau;
    const float a = xmul(u, u), c = xmul(v, v), s2 = xadd(a, c), pc = xmul(a, c), T2 = xmul(T, T);
    const float S2 = xadd(T, T0), S3 = xfma(T, S2, xmul(T0, T0));
    // f = rho (base + (T (X + Y) + X Y)/4) + drho P0, X = a +- u, Y = c +- v
    const float P0 = xmul(0.25f, xmul(T0, T0)), base = xmul(xmul(0.25f, tau), S2);
    const float2 X = make_float2(xadd(a, u), xsub(a, u));
    const float2 vT = bc2(T), vr = bc2(q.rho), vb = bc2(base), dP0 = bc2(xmul(q.drho, P0));
    const float2 Yp = bc2(xadd(c, v)), Ym = bc2(xsub(c, v));
    const float2 fp = xfma(vr, xfma(kc<float2>(0.25), xfma(X, Yp, xmul(vT, xadd(X, Yp))), vb), dP0);
    const float2 fm = xfma(vr, xfma(kc<float2>(0.25), xfma(X, Ym, xmul(vT, xadd(X, Ym))), vb), dP0);
    f[0] = fp.x; f[1] = fp.y; f[2] = fm.y; f[3] = fm.x;
    // h = RTc (rho (EE +- OE +- EO +- OO) + drho Q0) with
    // EE = T2 (k8 + 9/8) s2 + T ((k8 + 5/4) pc + s2^2/8) + pc s2/8 + tau (k8 + 2/3) S3,
    // (OE, EO) = (u, v) (T2 (k8 + 3/4) + T ((k8 + 9/8) (c, a) + (a, c)/8) + (c, a) s2/8),
    // OO = u v (T (k8 + 3/4) + s2/8)
    const float k8 = xmul(0.125f, K), e1 = xadd(k8, 0.75f), e2 = xadd(k8, 1.125f), e3 = xadd(k8, 2.0f / 3.0f);
    const float Q0 = xmul(xmul(xmul(T0, T0), T0), e3);
    const float EE = xfma(T2, xmul(e2, s2),
                          xfma(T, xfma(xadd(k8, 1.25f), pc, xmul(0.125f, xmul(s2, s2))),
                               xfma(xmul(0.125f, pc), s2, xmul(xmul(tau, e3), S3))));
    const float2 P = make_float2(a, c), Q = make_float2(c, a);
    const float2 OEO = xmul(make_float2(u, v),
                            xfma(bc2(T2), bc2(e1), xfma(vT, xfma(bc2(e2), Q, xmul(kc<float2>(0.125), P)),
                                                         xmul(kc<float2>(0.125), xmul(Q, bc2(s2))))));
    const float OO = xmul(xmul(u, v), xfma(T, e1, xmul(0.125f, s2)));
    const float p = xadd(EE, OO), mm = xsub(EE, OO), so = xadd(OEO.x, OEO.y), dd = xsub(OEO.x, OEO.y);
    const float2 vR = bc2(q.RTc), dQ0 = bc2(xmul(q.drho, Q0));
    const float2 h01 = xmul(vR, xfma(vr, make_float2(xadd(p, so), xsub(mm, dd)), dQ0));
    const float2 h23 = xmul(vR, xfma(vr, make_float2(xsub(p, so), xadd(mm, dd)), dQ0));
    h[0] = h01.x; h[1] = h01.y; h[2] = h23.x; h[3] = h23.y;
}

__device__ __forceinline__ void eqd_fam9(const EqDev<float> &q, float *f, float *h)
{
    const float T = q.T, K = q.K, T0 = q.T0, tau = q.tau, T2 = xmul(T, T);
    const float S2 = xadd(T, T0), S3 = xfma(T, S2, xmul(T0, T0));
    const float kh3 = xfma(K, 1.0f / 16.0f, 1.0f / 3.0f), kh2 = xfma(K, -1.0f / 48.0f, -1.0f / 12.0f);
    const float P0 = xmul(T0, xfma(0.125f, T0, -1.0f / 24.0f));
    const float Q0 = xmul(xmul(T0, T0), xfma(T0, kh3, kh2));
    const float tGf = xmul(tau, xfma(0.125f, S2, -1.0f / 24.0f));
    const float tGh = xmul(tau, xfma(kh3, S3, xmul(kh2, S2)));
    const float2 U = make_float2(q.u, q.v), W = make_float2(q.v, q.u);
    const float2 A = xmul(U, U), Cc = xmul(W, W), vT = bc2(T), vT2 = bc2(T2), vr = bc2(q.rho);
    const float2 qT = bc2(xmul(0.25f, T)), Am1 = xadd(A, kc<float2>(-1.0));
    // f: E = A (T/4 + (A - 1)/24) + tau Gf, O = U (T/4 + (A - 1)/12)
    const float2 Ef = xfma(A, xfma(kc<float2>(1.0 / 24.0), Am1, qT), bc2(tGf));
    const float2 Of = xmul(U, xfma(kc<float2>(1.0 / 12.0), Am1, qT));
    const float2 dP0 = bc2(xmul(q.drho, P0));
    const float2 fp = xfma(vr, xadd(Ef, Of), dP0), fm = xfma(vr, xsub(Ef, Of), dP0);
    f[0] = fp.x; f[1] = fp.y; f[2] = fm.x; f[3] = fm.y;
    // h: with M = (A + Cc)(A - 1),
    // E = T2 (d1 A + Cc/16) + T (A (d2 A + Cc/8 - d3) - Cc/48) + A M/48 + tau Gh,
    // O = U (T2 d4 + T (d5 A + Cc/8 + d6) + M/24)
    const float d1 = xfma(0.125f, K, 17.0f / 16.0f), d2 = xfma(K, 1.0f / 48.0f, 1.0f / 3.0f);
    const float d3 = xfma(K, 1.0f / 48.0f, 7.0f / 48.0f), d4 = xfma(0.125f, K, 0.75f);
    const float d5 = xfma(K, 1.0f / 24.0f, 11.0f / 24.0f), d6 = xfma(K, -1.0f / 24.0f, -1.0f / 6.0f);
    const float2 M = xmul(xadd(A, Cc), Am1);
    const float2 Eh = xfma(vT2, xfma(bc2(d1), A, xmul(kc<float2>(1.0 / 16.0), Cc)),
                           xfma(vT, xfma(A, xfma(bc2(d2), A, xfma(kc<float2>(0.125), Cc, bc2(xneg(d3)))),
                                         xmul(kc<float2>(-1.0 / 48.0), Cc)),
                                xfma(kc<float2>(1.0 / 48.0), xmul(A, M), bc2(tGh))));
    const float2 Oh = xmul(U, xfma(vT2, bc2(d4), xfma(vT, xfma(bc2(d5), A, xfma(kc<float2>(0.125), Cc, bc2(d6))),
                                                      xmul(kc<float2>(1.0 / 24.0), M))));
    const float2 dQ0 = bc2(xmul(q.drho, Q0)), vR = bc2(q.RTc);
    const float2 hp = xmul(vR, xfma(vr, xadd(Eh, Oh), dQ0)), hm = xmul(vR, xfma(vr, xsub(Eh, Oh), dQ0));
    h[0] = hp.x; h[1] = hp.y; h[2] = hm.x; h[3] = hm.y;
}

// Equilibria of one family in the stored representation: full values on the
// FP64 path, deviations from the rest state on the FP32 path.
template <class C, bool DEV>
struct EqArgs;
template <class C>
struct EqArgs<C, false> {
    EqState<C> q;
    __device__ __forceinline__ EqArgs(double rho, double ux, double uy, double T, const SampleParams &sp)
        : q(eq_state<C>(rho, ux, uy, T, sp)) {}
    __device__ __forceinline__ void fam(int f, C *fe, C *he) const
    {
        if (f == 0) eq_fam0(q, fe[0], he[0]);
        else if (f == 1) eq_fam1(q, fe, he);
        else if (f == 2) eq_fam5(q, fe, he);
        else eq_fam9(q, fe, he);
    }
};
template <class C>
struct EqArgs<C, true> {
    EqDev<C> q;
    __device__ __forceinline__ EqArgs(double rho, double ux, double uy, double T, const SampleParams &sp)
        : q(eq_dev<C>(rho, ux, uy, T, sp)) {}
    __device__ __forceinline__ void fam(int f, C *fe, C *he) const
    {
        if (f == 0) eqd_fam0(q, fe[0], he[0]);
        else if (f == 1) eqd_fam1(q, fe, he);
        else if (f == 2) eqd_fam5(q, fe, he);
        else eqd_fam9(q, fe, he);
    }
};

// all 26 values (init, pointwise stages)
template <class C>
__device__ __forceinline__ void eq_all(const EqState<C> &q, C *f, C *h)
{
    eq_fam0(q, f[0], h[0]);
    eq_fam1(q, f + 1, h + 1);
    eq_fam5(q, f + 5, h + 5);
    eq_fam9(q, f + 9, h + 9);
}

// ---------------------------------------------------------------- moments
// macroProp/macroPropShort (cpuLBM.cpp:877-970): FP64 sums over the node's
// 13 f and 13 h values.  The relaxation times tau_f = mu/p, tau_h =
// tau_f/Pr, tau_hf = tau_h tau_f / (tau_f - tau_h) (cpuLBM.cpp:952-955)
// enter every formula as their inverses, which are all linear in
// q = p / mu: 1/tau_f = q, 1/tau_h = Pr q, 1/tau_hf = (Pr - 1) q (so
// Pr = 1 gives 1/tau_hf = 0, the reference's x / inf).
struct Macro {
    double rho, ux, uy, T, p, q;
};

__device__ __forceinline__ Macro macro_from_sums(double r, double rux, double ruy, double sh, const SampleParams &sp)
{
    // stored deviations: add the rest state's rho0 and sum of h (0 when the
    // state is stored in full)
    r = sp.rho0 + r;
    sh = sp.shref + sh;
    Macro m;
    const double ir = 1.0 / r;
    m.rho = r;
    m.ux = rux * ir;
    m.uy = ruy * ir;
    const double usq = m.ux * m.ux + m.uy * m.uy;
    m.T = (sh * ir - 0.5 * usq) * sp.two_over_bR;
    m.p = r * sp.R * m.T;
    if (sp.visc == 0) {
        m.q = m.p * sp.inv_mu;  // 1/tau_f = p/mu
    } else {
        double mu = sp.mu * pow(m.T / sp.visc_T, sp.visc_exp);
        if (sp.visc == 2) mu *= (sp.visc_T + sp.visc_S) / (m.T + sp.visc_S);
        m.q = m.p / mu;
    }
    return m;
}

// ---------------------------------------------------------- index and BCs
// index (cpuLBM.cpp:1033-1113): periodic wrap, mirror (-i-1 / 2N-i-1 with a
// reflection flag) or zeroth-order extrapolation (clamp).
__device__ __forceinline__ int bc_index(const SampleParams &sp, int i, int pm, int axis, int &mir)
{
    i += pm;
    mir = 0;
    const int N = axis == 0 ? sp.nx : sp.ny;
    if (i < 0) {
        if (sp.flags & (axis == 0 ? SF_PERX : SF_PERY)) i = N + i;
        else if (sp.flags & (axis == 0 ? SF_MIRW : SF_MIRS)) { i = -i - 1; mir = 1; }
        else i = 0;
    } else if (i > N - 1) {
        if (sp.flags & (axis == 0 ? SF_PERX : SF_PERY)) i = i - N;
        else if (sp.flags & (axis == 0 ? SF_MIRE : SF_MIRN)) { i = 2 * N - i - 1; mir = 1; }
        else i = N - 1;
    }
    return i;
}

// -------------------------------------------------------------- NND, WENO5
// minmod with the reference's case order (cpuLBM.cpp:1130-1145): same
// signs -> the smaller magnitude (equal magnitudes mean a == b), else 0
template <class C>
__device__ __forceinline__ C minmod(C a, C b)
{
    return a * b > C(0) ? (fabs(a) < fabs(b) ? a : b) : C(0);
}
// lane-wise on the packed pair (f, h) of one face
template <>
__device__ __forceinline__ float2 minmod<float2>(float2 a, float2 b)
{
    return make_float2(minmod<float>(a.x, b.x), minmod<float>(a.y, b.y));
}

// NND (cpuLBM.cpp:1328-1356) on the 3 upwind-ordered values s0, s1, s2
template <class C>
__device__ __forceinline__ C nnd3(C ae, C s0, C s1, C s2)
{
    const C c = xmul(ae, s1);
    return xfma(kc<C>(0.5), minmod<C>(xfma(ae, s2, xneg(c)), xfma(xneg(ae), s0, c)), c);
}

// one division per face (the FP64 path keeps it correctly rounded)
__device__ __forceinline__ double face_div(double n, double d) { return n / d; }
// FP32: n times the approximate reciprocal of d (PTX rcp.approx, then one
// correctly rounded product).  Inline PTX, so that no compiled instance may
// lower the division another way: a face then rounds the same in every
// kernel that reconstructs it.  d here is a positive normal number (a sum
// of weights, or eps + b_k).
__device__ __forceinline__ float rcp_approx(float d)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    return r;
}
__device__ __forceinline__ float face_div(float n, float d) { return __fmul_rn(n, rcp_approx(d)); }
__device__ __forceinline__ float2 face_div(float2 n, float2 d)
{
    return __fmul2_rn(n, make_float2(rcp_approx(d.x), rcp_approx(d.y)));
}

// WENO5 (cpuLBM.cpp:1358-1403): Jiang-Shu indicators b_k, linear weights
// 1/10, 6/10, 3/10, epsilon 1e-6, on |e| times the upwind-ordered values.
// The nonlinear weights d_k/(eps+b_k)^2 normalised by their sum are formed
// as d_k prod_{j!=k} (eps+b_j)^2 over the same sum (one division per face).
// That fourth power (times the candidate values in the numerator) leaves
// the FP32 range on dimensional data; for samples whose scales allow that
// (SampleParams::wide, set on the host) the FP32 weights are formed as
// d_k (m/(eps+b_k))^2 instead, m the smallest eps+b_j, each ratio in (0, 1].
template <class C, bool WIDE = false>
__device__ __forceinline__ C weno5(C ae, C s0, C s1, C s2, C s3, C s4)
{
    const C q0 = xmul(ae, s0), q1 = xmul(ae, s1), q2 = xmul(ae, s2), q3 = xmul(ae, s3), q4 = xmul(ae, s4);
    // second differences d_k and one-sided slopes l_k of the three stencils
    const C d0 = xfma(kc<C>(-2), q1, xadd(q0, q2));
    const C d1 = xfma(kc<C>(-2), q2, xadd(q1, q3));
    const C d2 = xfma(kc<C>(-2), q3, xadd(q2, q4));
    const C l0 = xfma(kc<C>(3), q2, xfma(kc<C>(-4), q1, q0));
    const C l1 = xsub(q1, q3);
    const C l2 = xfma(kc<C>(-4), q3, xfma(kc<C>(3), q2, q4));
    // eps + b_k
    const C a0 = xfma(xmul(kc<C>(13.0 / 12.0), d0), d0, xfma(xmul(kc<C>(0.25), l0), l0, kc<C>(1e-6)));
    const C a1 = xfma(xmul(kc<C>(13.0 / 12.0), d1), d1, xfma(xmul(kc<C>(0.25), l1), l1, kc<C>(1e-6)));
    const C a2 = xfma(xmul(kc<C>(13.0 / 12.0), d2), d2, xfma(xmul(kc<C>(0.25), l2), l2, kc<C>(1e-6)));
    C w0, w1, w2;
    if (IsF32<C>::value && WIDE) {
        const C m = xmin(a0, xmin(a1, a2));
        const C s0 = face_div(m, a0), s1 = face_div(m, a1), s2 = face_div(m, a2);
        w0 = xmul(kc<C>(0.1), xmul(s0, s0));
        w1 = xmul(kc<C>(0.6), xmul(s1, s1));
        w2 = xmul(kc<C>(0.3), xmul(s2, s2));
    } else {
        const C p0 = xmul(a0, a0), p1 = xmul(a1, a1), p2 = xmul(a2, a2);
        w0 = xmul(kc<C>(0.1), xmul(p1, p2));
        w1 = xmul(kc<C>(0.6), xmul(p0, p2));
        w2 = xmul(kc<C>(0.3), xmul(p0, p1));
    }
    // candidate reconstructions (times 6)
    const C r0 = xfma(kc<C>(11), q2, xfma(kc<C>(-7), q1, xmul(kc<C>(2), q0)));
    const C r1 = xfma(kc<C>(2), q3, xfma(kc<C>(5), q2, xneg(q1)));
    const C r2 = xsub(xfma(kc<C>(5), q3, xmul(kc<C>(2), q2)), q4);
    return face_div(xfma(w2, r2, xfma(w1, r1, xmul(w0, r0))), xmul(kc<C>(6), xadd(xadd(w0, w1), w2)));
}

// the range-safe form out of line: the general paths that choose the form
// at run time keep one inlined WENO5 (their code stays compact)
template <class C>
__device__ __noinline__ C weno5_wide(C ae, C s0, C s1, C s2, C s3, C s4)
{
    return weno5<C, true>(ae, s0, s1, s2, s3, s4);
}

// WENO5 with the weight form of the sample
template <class C>
__device__ __forceinline__ C weno5_sp(const SampleParams &sp, C ae, C s0, C s1, C s2, C s3, C s4)
{
    if (sizeof(C) == 4 && sp.wide) return weno5_wide<C>(ae, s0, s1, s2, s3, s4);
    return weno5<C, false>(ae, s0, s1, s2, s3, s4);
}

// view of one sample's stage buffer and node flags
// One sample's stage buffer and node flags; offsets inside a sample fit in
// 32 bits (26 planes of up to 2^26 nodes).
template <class S>
struct StageView {
    const S *__restrict__ st;        // plane 0 of the sample in the stage buffer
    const uint8_t *__restrict__ nf;  // node flags of the sample
    int plane;
    int pitch;
};

template <class S>
__device__ __forceinline__ S ldv(const StageView<S> &v, int p, int x, int y)
{
    return __ldg(v.st + (p * v.plane + y * v.pitch + x));
}

// Exact stencil + reconstruction (stencil, cpuLBM.cpp:1171-1326, then NND/
// WENO5) for the flux of plane p along `axis` at (x, y): boundary-aware
// indices with reflections, and the linear extrapolation 2 f(m1) - f(m2)
// over the first solid/fluid edge met by the stencil.
template <class S, class C>
__device__ __noinline__ C flux_exact(const SampleParams &sp, const StageView<S> &v, int x, int y, int p, int axis)
{
    const int i = p < NQ ? p : p - NQ, pb = p - i;
    const int e = axis == 0 ? isgn(c_EX[i]) : isgn(c_EY[i]);
    if (e == 0) return C(0);
    const C ae = (C)(sp.c * (double)abs(axis == 0 ? c_EX[i] : c_EY[i]));
    const int L = sp.fm ? 5 : 3, low = (L - 1) / 2;
    const int pos = axis == 0 ? x : y;
    const int j1 = pos - e * low;
    C S5[5];
    int sld[5];
    int any = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        if (j < L) {
            int m;
            const int r = bc_index(sp, j1, e * j, axis, m);
            const int pp = m ? pb + (axis == 0 ? c_MIR_EW[i] : c_MIR_NS[i]) : p;
            const int xr = axis == 0 ? r : x, yr = axis == 0 ? y : r;
            S5[j] = (C)ldv(v, pp, xr, yr);
            sld[j] = (v.nf[yr * v.pitch + xr] & NF_TYPE) == 2;
            any |= sld[j];
        }
    }
    if (any) {
        int diff = 0, jj = 0, pe = 0, m;
        for (int j = 0; j < L - 1; ++j) {
            diff = sld[j] - sld[j + 1];
            if (diff > 0) { jj = j; pe = bc_index(sp, j1, e * j, axis, m); break; }
            if (diff < 0) { jj = j + 1; pe = bc_index(sp, j1, e * (j + 1), axis, m); break; }
        }
        const int r1 = bc_index(sp, pe, e * diff, axis, m);
        const int r2 = bc_index(sp, pe, e * 2 * diff, axis, m);
        const C v1 = axis == 0 ? (C)ldv(v, p, r1, y) : (C)ldv(v, p, x, r1);
        const C v2 = axis == 0 ? (C)ldv(v, p, r2, y) : (C)ldv(v, p, x, r2);
        const C ext = C(2) * v1 - v2;
        // S5[jj] = ext; S5[jj - diff] = ext when inside the stencil
#pragma unroll
        for (int j = 0; j < 5; ++j)
            if (j < L && (j == jj || (j == jj - diff))) S5[j] = ext;
    }
    if (sp.fm) return weno5_sp<C>(sp, ae, S5[0], S5[1], S5[2], S5[3], S5[4]);
    return nnd3<C>(ae, S5[0], S5[1], S5[2]);
}

// Stencil across a periodic edge with no solid in it: the five neighbours
// with single periodic wrap, read from global memory.
template <class S, class C>
__device__ __forceinline__ C flux_wrap(const SampleParams &sp, const StageView<S> &v, int x, int y, int p, int axis)
{
    const int i = p < NQ ? p : p - NQ;
    const int ev = axis == 0 ? c_EX[i] : c_EY[i];
    if (ev == 0) return C(0);
    const int e = ev > 0 ? 1 : -1;
    const C ae = (C)(sp.c * (double)abs(ev));
    const int N = axis == 0 ? sp.nx : sp.ny;
    const int pos = axis == 0 ? x : y;
    C q[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        int r = pos + e * (j - 2);
        r += r < 0 ? N : 0;
        r -= r >= N ? N : 0;
        q[j] = axis == 0 ? (C)ldv(v, p, r, y) : (C)ldv(v, p, x, r);
    }
    if (sp.fm) return weno5_sp<C>(sp, ae, q[0], q[1], q[2], q[3], q[4]);
    return nnd3<C>(ae, q[1], q[2], q[3]);
}

// Outgoing face flux of plane p along `axis` at a non-solid node; the fast
// path (no solid, no domain edge within the stencil) reads the five
// neighbours directly.
template <class S, class C>
__device__ __forceinline__ C flux_axis(const SampleParams &sp, const StageView<S> &v, int x, int y, int p, int axis,
                                       uint8_t nflag)
{
    const int i = p < NQ ? p : p - NQ;
    const int ev = axis == 0 ? c_EX[i] : c_EY[i];
    if (ev == 0) return C(0);
    const uint8_t slow = axis == 0 ? (NF_SOLX | NF_EDGX) : (NF_SOLY | NF_EDGY);
    if (nflag & slow) return flux_exact<S, C>(sp, v, x, y, p, axis);
    if (nflag & (axis == 0 ? NF_WRPX : NF_WRPY)) return flux_wrap<S, C>(sp, v, x, y, p, axis);
    const int e = ev > 0 ? 1 : -1;
    const C ae = (C)(sp.c * (double)abs(ev));
    const int stride = axis == 0 ? e : e * v.pitch;
    const S *c0 = v.st + (p * v.plane + y * v.pitch + x);
    if (sp.fm) {
        return weno5_sp<C>(sp, ae, (C)__ldg(c0 - 2 * stride), (C)__ldg(c0 - stride), (C)__ldg(c0), (C)__ldg(c0 + stride),
                        (C)__ldg(c0 + 2 * stride));
    }
    return nnd3<C>(ae, (C)__ldg(c0 - stride), (C)__ldg(c0), (C)__ldg(c0 + stride));
}

// wallFluxes (cpuLBM.cpp:1502-1590): for a solid node next to fluid,
// alpha = (f flux of the fluid 4-neighbours into it) / (|e| f out of it),
// weighted by the solid cell's 1/dx, 1/dy; one alpha for f and h.  Works on
// full values (stored values + fr, the rest state of stored deviations) and
// returns alpha - 1.
__constant__ int c_WXX[4] = {-1, 1, 0, 0};
__constant__ int c_WYY[4] = {0, 0, -1, 1};
__constant__ int c_WII[4][4] = {{1, 5, 8, 9}, {3, 6, 7, 11}, {2, 5, 6, 10}, {4, 7, 8, 12}};
__constant__ int c_WINV[4][4] = {{3, 6, 7, 11}, {1, 5, 8, 9}, {4, 8, 7, 12}, {2, 6, 5, 10}};

template <class S, class C>
__device__ double wall_alpha_m1(const SampleParams &sp, const StageView<S> &v, int x, int y, double dxm, double dym,
                                const double *fr)
{
    double fin = 0, fout = 0;
    for (int j = 0; j < 4; ++j) {
        int m;
        const int xm = bc_index(sp, x, c_WXX[j], 0, m);
        const int ym = bc_index(sp, y, c_WYY[j], 1, m);
        const uint8_t fl = v.nf[ym * v.pitch + xm];
        if ((fl & NF_TYPE) >= 2) continue;
        const int axis = j < 2 ? 0 : 1;
        const double dd = axis == 0 ? dxm : dym;
        for (int q = 0; q < 4; ++q) {
            const int i = c_WII[j][q], io = c_WINV[j][q];
            const double ai = sp.c * abs(axis == 0 ? c_EX[i] : c_EY[i]);
            const double F = (double)flux_axis<S, C>(sp, v, xm, ym, i, axis, fl) + ai * fr[i];
            fin += F / dd;
            const double fo = (double)ldv(v, io, x, y) + fr[io];
            fout += fo * (sp.c * abs(axis == 0 ? c_EX[io] : c_EY[io])) / dd;
        }
    }
    return fin / fout - 1.0;
}

}  // namespace uqlbm
