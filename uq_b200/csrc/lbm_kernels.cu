// CUDA kernels of the D2Q13 thermal LBM step for sm_100a.
//
// One time step of a batch is a short sequence of launches over a packed
// tile list of all samples (see lbm_engine.cu):
//   P0  pointwise stages      (RK3 stages 1+2 -> f2; RK1 stage 1 -> f1;
//                              EULER copies f) into stage buffer 2
//   W   wall fluxes           alpha for every solid node next to fluid
//   P1  stencil + stage       fluxes of buffer 2, divergence, then RK3 stage 3
//                              (-> buffer 3, and the update partial sum in
//                              place of f) or the RK1/EULER update of f
//   W   wall fluxes of buffer 3                        (RK3 only)
//   P2  stencil + update      fluxes of buffer 3, final RK3 combination
// The reference computes the same quantities in RK1/RK3/EULER/EULER_EQ
// (cpuLBM.cpp:1597-2283) with full-field temporaries.
#include "lbm_device.cuh"
#include "lbm_kernels.h"
#include "tma.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

namespace uqlbm {

template <class S>
__device__ __forceinline__ S *plane_ptr(S *base, const SampleParams &sp, int p)
{
    return base + sp.state_off + (long long)p * sp.plane;
}

// Ghost columns (SampleParams::gx): a node within gx of an x edge also
// stores its stage-buffer values at its periodic image beyond the other
// edge.  The offset of that image (0: none) for the node at x; RK3's stage
// 3 stores each buffer-3 value at o and, when this is nonzero, at
// o + offset too.  Buffer 2's ghosts are copied by k_fill_ghosts after the
// pointwise phase (the pointwise kernel runs at 64 registers, where the
// extra stores cost it spills).
__device__ __forceinline__ int ghost_offset(const SampleParams &sp, int x)
{
    return sp.gx ? (x < sp.gx ? sp.nx : (x >= sp.nx - sp.gx ? -sp.nx : 0)) : 0;
}

// ------------------------------------------------------------------- init
// initialiseFunctions (cpuLBM.cpp:846-875) for one node: f, h = equilibrium
// of (rho, ux, uy, T), stored as deviations from the rest state; solid and
// permanent nodes also seed stage buffers 2/3, whose contents never change
// for them.  Returns false when the equilibrium mass check fails.  One
// compiled body serves every initialising kernel, so a state set from
// fields is bit-for-bit the state built at creation.
template <class S>
__device__ __noinline__ bool init_node(double rho, double ux, double uy, double T, const SampleParams &sp,
                                       const double *fr, S *state, S *buf2, S *buf3, long long o, bool fixed)
{
    EqState<double> q = eq_state<double>(rho, ux, uy, T, sp);
    double f[NQ], h[NQ];
    eq_all(q, f, h);
    double sf = 0;
    for (int i = 0; i < NQ; ++i) sf += f[i];
    for (int i = 0; i < NQ; ++i) {
        const long long of = sp.state_off + (long long)i * sp.plane + o;
        const long long oh = sp.state_off + (long long)(NQ + i) * sp.plane + o;
        const S fv = (S)(f[i] - fr[i]), hv = (S)(h[i] - fr[NQ + i]);
        state[of] = fv;
        state[oh] = hv;
        if (fixed) {
            buf2[of] = fv; buf3[of] = fv;
            buf2[oh] = hv; buf3[oh] = hv;
        }
    }
    return !(fabs(sf - rho) > 1e-6);
}

template <class S>
__global__ void k_init(KArgs<S> a, const double *__restrict__ rho, const double *__restrict__ ux,
                       const double *__restrict__ uy, const double *__restrict__ T)
{
    const Tile t = a.tiles[blockIdx.x];
    const SampleParams sp = a.samples[t.sample];
    const int x = t.x0 + threadIdx.x % a.tx, y = t.y0 + threadIdx.x / a.tx;
    if (x >= sp.nx || y >= sp.ny) return;
    const long long node = sp.node_off + (long long)y * sp.pitch + x;
    const bool fixed = (a.nflags[node] & NF_TYPE) != 0;
    const long long o = (long long)y * sp.pitch + x;
    if (!init_node<S>(rho[node], ux[node], uy[node], T[node], sp, a.fref + NPL * t.sample, a.state, a.buf2, a.buf3, o,
                      fixed))
        atomicOr(&a.status[t.sample], STATUS_EQ);
}

// ------------------------------------------------------------------ moments
// macroPropShort of one node from its 26 stored values, read through
// rd(p) (p = i for f_i, NQ + i for h_i).
// The momentum sums are formed as sums of the values times the directions'
// integer components (0, +-1, +-2: exact, and no operation for 0 in the
// unrolled loops), scaled by c once.
__device__ __forceinline__ void mom_add(double &acc, int e, double v)
{
    if (e == 1) acc += v;
    else if (e == -1) acc -= v;
    else if (e != 0) acc = fma((double)e, v, acc);
}

// e_i . (cu, cv) for direction i, with cu = c u and cv = c v: the
// components are 0, +-1 or +-2, so each term is exact and only a diagonal
// direction adds (i a compile-time value in the unrolled loops)
template <class C>
__device__ __forceinline__ C e_dot(int i, C cu, C cv)
{
    const int ex = lat_ex(i), ey = lat_ey(i);
    const C x = ex == 1 ? cu : ex == -1 ? -cu : C(ex) * cu;
    const C y = ey == 1 ? cv : ey == -1 ? -cv : C(ey) * cv;
    return ex == 0 ? y : ey == 0 ? x : xadd(x, y);
}

template <class RD>
__device__ __forceinline__ Macro node_macro_rd(RD rd, const SampleParams &sp)
{
    double r = 0, rx = 0, ry = 0, sh = 0;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double fv = (double)rd(i);
        r += fv;
        mom_add(rx, lat_ex(i), fv);
        mom_add(ry, lat_ey(i), fv);
        sh += (double)rd(NQ + i);
    }
    return macro_from_sums(r, sp.c * rx, sp.c * ry, sh, sp);
}

// the same with stn the node's element in plane 0, the planes sp.plane
// elements apart (offsets in a sample fit in 32 bits)
template <class S>
__device__ __forceinline__ Macro node_macro(const S *__restrict__ stn, const SampleParams &sp)
{
    const int PL = (int)sp.plane;
    return node_macro_rd([&](int p) { return stn[p * PL]; }, sp);
}

// The same from the sample's plane 0 and the node's 64-bit offset o (the
// form the pointwise kernel keeps: it runs at 64 registers, where per-node
// pointers cost it more than they save).
template <class S>
__device__ __forceinline__ Macro node_macro_at(const S *__restrict__ st, const SampleParams &sp, long long o)
{
    double r = 0, rx = 0, ry = 0, sh = 0;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double fv = (double)st[(long long)i * sp.plane + o];
        r += fv;
        mom_add(rx, lat_ex(i), fv);
        mom_add(ry, lat_ey(i), fv);
        sh += (double)st[(long long)(NQ + i) * sp.plane + o];
    }
    return macro_from_sums(r, sp.c * rx, sp.c * ry, sh, sp);
}

// ------------------------------------------------------------------- P0
// RK: 1 (RK3 stages 1+2), 0 (RK1 stage 1), 2 (EULER / EULER_EQ: copy).
// Pointwise and memory-bound: the FP32 instances keep 64 registers so that
// four blocks (32 warps) per SM keep loads in flight.
template <class S>
struct Stage0Blocks {
    static constexpr int value = sizeof(S) == 4 ? 4 : 2;
};
template <class S, class C, int RK>
__global__ void __launch_bounds__(256, Stage0Blocks<S>::value) k_stage0(KArgs<S> a)
{
    const Tile t = a.tiles[blockIdx.x];
    const SampleParams sp = a.samples[t.sample];
    const int x = t.x0 + threadIdx.x % a.tx, y = t.y0 + threadIdx.x / a.tx;
    if (x >= sp.nx || y >= sp.ny) return;
    const long long o = (long long)y * sp.pitch + x;
    const long long node = sp.node_off + o;
    const int type = a.nflags[node] & NF_TYPE;
    const S *__restrict__ st = a.state + sp.state_off;
    S *__restrict__ b2 = a.buf2 + sp.state_off;
    if (RK >= 2) {  // EULER, EULER_EQ: fluxes of the state itself
        if (type == 0)
            for (int p = 0; p < NPL; ++p) b2[(long long)p * sp.plane + o] = st[(long long)p * sp.plane + o];
        if (a.want_residual && type == 0) a.told[node] = node_macro_at(st, sp, o).T;
        return;
    }
    if (type != 0) return;
    const Macro m = node_macro_at(st, sp, o);
    if (a.want_residual) a.told[node] = m.T;
    constexpr bool DEV = sizeof(S) == 4;
    const EqArgs<C, DEV> q(m.rho, m.ux, m.uy, m.T, sp);
    C fe[NQ], he[NQ];
    q.fam(0, fe, he);
    q.fam(1, fe + 1, he + 1);
    q.fam(2, fe + 5, he + 5);
    q.fam(3, fe + 9, he + 9);
    {
        // sum_i f_eq = rho (the stored values: sum = rho - rho0)
        double sf = 0;
#pragma unroll
        for (int i = 0; i < NQ; ++i) sf += (double)fe[i];
        if (fabs(sf - (m.rho - sp.rho0)) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(m.rho))))
            atomicOr(&a.status[t.sample], STATUS_EQ);
    }
    const C dt = (C)sp.dt, cu = (C)sp.c * (C)m.ux, cv = (C)sp.c * (C)m.uy;
    const C rq = (C)m.q, Pr = (C)sp.Pr;  // 1/tau_f
    if (RK == 1) {
        // RK3 stages 1 and 2 (cpuLBM.cpp:1819-1924); stage 2 reuses stage 1's
        // equilibrium, moments and relaxation times.  cf = dt/(2 tau_f),
        // ch = dt/(2 tau_h), g = 1/tau_hf.
        const C hdt = C(0.5) * dt;
        const C cf = hdt * rq, ch = hdt * Pr * rq, g = (Pr - C(1)) * rq;
        const C icf = C(1) / (C(1) + cf), ich = C(1) / (C(1) + ch), hg = hdt * g;
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            const C f = (C)st[(long long)i * sp.plane + o], h = (C)st[(long long)(NQ + i) * sp.plane + o];
            const C eu = e_dot<C>(i, cu, cv);
            C f2, h2;
            if constexpr (sizeof(S) == 4) {
                // FP32, explicitly rounded, with the stage-2 forms reduced:
                // -cf (fe - f1) + cf fe = cf f1, -ch (he - h1) + ch he = ch h1,
                // and the two coupling terms combine to hdt g eu (f1 - f2)
                const C hge = xmul(hg, eu);
                const C f1 = xmul(xfma(cf, fe[i], f), icf);
                const C h1 = xmul(xsub(xfma(ch, he[i], h), xmul(hge, xsub(fe[i], f1))), ich);
                f2 = xmul(xfma(cf, f1, f), icf);
                h2 = xmul(xfma(ch, h1, xsub(h, xmul(hge, xsub(f1, f2)))), ich);
            } else {
                const C f1 = (f + cf * fe[i]) * icf;
                const C h1 = (h - hdt * g * eu * (fe[i] - f1) + ch * he[i]) * ich;
                f2 = (f - cf * (fe[i] - f1) + cf * fe[i]) * icf;
                h2 = (h - hdt * (eu * g * (fe[i] - f2) - eu * g * (fe[i] - f1)) - ch * (he[i] - h1) + ch * he[i]) * ich;
            }
            b2[(long long)i * sp.plane + o] = (S)f2;
            b2[(long long)(NQ + i) * sp.plane + o] = (S)h2;
        }
    } else {
        // RK1 stage 1 (cpuLBM.cpp:1619-1663)
        const C cf = dt * rq, ch = dt * Pr * rq, g = (Pr - C(1)) * rq;
        const C icf = C(1) / (C(1) + cf), ich = C(1) / (C(1) + ch);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            const C f = (C)st[(long long)i * sp.plane + o], h = (C)st[(long long)(NQ + i) * sp.plane + o];
            const C eu = e_dot<C>(i, cu, cv);
            const C f1 = (f + cf * fe[i]) * icf;
            const C h1 = (h - dt * eu * ((fe[i] - f1) * g) + ch * he[i]) * ich;
            b2[(long long)i * sp.plane + o] = (S)f1;
            b2[(long long)(NQ + i) * sp.plane + o] = (S)h1;
        }
    }
}

// -------------------------------------------------------------------- W
template <class S, class C>
__global__ void k_wall(KArgs<S> a, const S *__restrict__ stage, const WallNode *__restrict__ walls, int nwalls)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nwalls) return;
    const WallNode w = walls[k];
    const SampleParams sp = a.samples[w.sample];
    const StageView<S> v{stage + sp.state_off, a.nflags + sp.node_off, (int)sp.plane, sp.pitch};
    const double am1 = wall_alpha_m1<S, C>(sp, v, w.x, w.y, a.dxv[sp.xoff + w.x], a.dyv[sp.yoff + w.y],
                                           a.fref + NPL * w.sample);
    a.template alpha_as<C>()[sp.node_off + (long long)w.y * sp.pitch + w.x] = (C)am1;
}

// ------------------------------------------------------------------ P1/P2
// Fast-path reconstruction along a line through c0 with element step `st`
// (upwind ordering already folded into the sign of st).
template <class S, class C>
__device__ __forceinline__ C line_flux(const SampleParams &sp, const S *__restrict__ c0, int st, C ae)
{
    if (sp.fm)
        return weno5_sp<C>(sp, ae, (C)__ldg(c0 - 2 * st), (C)__ldg(c0 - st), (C)__ldg(c0), (C)__ldg(c0 + st),
                        (C)__ldg(c0 + 2 * st));
    return nnd3<C>(ae, (C)__ldg(c0 - st), (C)__ldg(c0), (C)__ldg(c0 + st));
}

// Stage tiles in shared memory: per direction the f and h planes over the
// box [x0-4, x0+TX+4) x [y0-3, y0+TY+3) (x start kept on a 16-byte
// boundary), loaded by TMA ahead of use.  Directions are processed in
// groups of G, one barrier per group: G = 4 on the FP32 path (two +/-
// pairs per group: 3 barriers per phase, and the tile-edge items of four
// directions spread over more warps); G = 1 on the FP64 path, whose boxes
// are twice as large.
constexpr int HALO_X = 4, HALO_Y = 3;
constexpr uint32_t TMA_WAIT_POLLS = 1u << 16;

template <int G>
struct GroupCfg {
    static constexpr int NSTAGE = G >= 2 ? 2 : 3;  // groups in flight
    static constexpr int NGROUP = 12 / G;
};

// direction m of group g: G = 1 -> 1..12; G = 2 -> (1,3) (2,4) (5,7) (6,8)
// (9,11) (10,12); G = 4 -> (1,3,2,4) (5,7,6,8) (9,11,10,12)
template <int G>
__host__ __device__ constexpr int group_dir(int g, int m)
{
    if (G == 1) return g + 1;
    if (G == 4) return 4 * g + 1 + (m >> 1) + 2 * (m & 1);
    const int base = g < 2 ? g + 1 : (g < 4 ? g + 3 : g + 5);
    return base + 2 * m;
}

// Shared-memory layout of k_flux (bytes from a 128-byte aligned base).
struct FluxSmemLayout {
    size_t c_elems;      // C arrays: sf[2][G][4][NT], ring x[2][G][2][TY], ring y[2][G][2][TX], sD[26][NT]
    size_t stage_off;    // staged boxes
    size_t plane_bytes;  // one staged plane, padded to 128 bytes
    size_t pref_off;     // the h half of the prefetched state (the f half lands in a freed staging slot)
    size_t bar_off;      // NSTAGE mbarriers, then the prefetch's
    size_t total;        // including 128 bytes of base-alignment slack
};

// prefetch: the FP32 kernels load the update's state values of the tile
// into shared memory while the last direction group is computed
__host__ __device__ constexpr bool flux_prefetch(size_t es_s) { return es_s == 4; }

__host__ __device__ inline FluxSmemLayout flux_layout(size_t es_c, size_t es_s, int tx, int ty, int G, int nstage)
{
    FluxSmemLayout L;
    const size_t NT = (size_t)tx * ty;
    L.c_elems = 8 * (size_t)G * NT + 4 * (size_t)G * tx + 4 * (size_t)G * ty + (size_t)NPL * NT;
    L.stage_off = (L.c_elems * es_c + 127) / 128 * 128;
    L.plane_bytes = ((size_t)(tx + 2 * HALO_X) * (ty + 2 * HALO_Y) * es_s + 127) / 128 * 128;
    L.pref_off = L.stage_off + (size_t)nstage * 2 * G * L.plane_bytes;
    const size_t pref_bytes = flux_prefetch(es_s) ? ((size_t)PREFETCH_PLANES * NT * es_s + 127) / 128 * 128 : 0;
    L.bar_off = L.pref_off + pref_bytes;
    L.total = L.bar_off + (nstage + 1) * sizeof(uint64_t) + 128;
    return L;
}

template <class S, class C>
struct TileCtx {
    const SampleParams *sp;
    StageView<S> v;
    const C *alpha;  // alpha - 1 of this sample (node-indexed)
    const double *fref;  // this sample's 26 rest-state values
    C *sf;           // [2 buffers][G][4: fx_f, fx_h, fy_f, fy_h][NT]
    C *ringx;        // [2 buffers][G][2: f, h][TY]
    C *ringy;        // [2 buffers][G][2: f, h][TX]
    C *sD;           // [26][NT]
    const S *stg;    // [NSTAGE][G][2: f, h][BH][BW], planes `pstride` elements apart
    int pstride;
    uint64_t *bars;  // [NSTAGE], then the prefetch's
    const CUtensorMap *map;
    const CUtensorMap *smap;  // the state, box of the tile's own nodes over PREFETCH_PLANES planes
    S *pref_h;                // where the h half of the prefetch lands
    int gx;                   // the sample's ghost columns: TMA x coordinates are x + gx
    int *timed_out;  // shared flag
    bool wrap_fix;   // general tiles: the box crosses a periodic edge
    int *status;     // this sample's status word
    int NT, TX, TY, BW, BH, tid, tx, ty, x, y, x0, y0, x_end, y_end, o;
    uint8_t flag;
    bool active;
    C tdx, tdy;
};

template <int G, class S, class C>
__device__ __forceinline__ void issue_group_load(TileCtx<S, C> &k, int g, int slot)
{
    const uint32_t box = (uint32_t)(k.BW * k.BH * sizeof(S));
    S *dst = const_cast<S *>(k.stg) + (size_t)slot * 2 * G * k.pstride;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&k.bars[slot], 2 * G * box);
#pragma unroll
    for (int m = 0; m < G; ++m) {
        const int dir = group_dir<G>(g, m);
        tma_load_3d(dst + (size_t)(2 * m) * k.pstride, k.map, k.x0 - HALO_X + k.gx, k.y0 - HALO_Y, dir, &k.bars[slot]);
        tma_load_3d(dst + (size_t)(2 * m + 1) * k.pstride, k.map, k.x0 - HALO_X + k.gx, k.y0 - HALO_Y, NQ + dir,
                    &k.bars[slot]);
    }
}

// The update's state values of this tile (f planes into the freed staging
// slot, h planes into their own region), completing on bars[NSTAGE]; the
// slot's last readers passed the barrier before this is issued.
template <int G, class S, class C>
__device__ __forceinline__ void issue_state_prefetch(TileCtx<S, C> &k, int slot)
{
    const uint32_t bytes = (uint32_t)(k.NT * PREFETCH_PLANES * sizeof(S));
    constexpr int NST = GroupCfg<G>::NSTAGE;
    S *dst_f = const_cast<S *>(k.stg) + (size_t)slot * 2 * G * k.pstride;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&k.bars[NST], 2 * bytes);
    tma_load_3d(dst_f, k.smap, k.x0 + k.gx, k.y0, 0, &k.bars[NST]);
    tma_load_3d(k.pref_h, k.smap, k.x0 + k.gx, k.y0, NQ, &k.bars[NST]);
}

// reconstruction from the staged box (fast path; no solid, no domain edge
// within the stencil): element step `st` in the box, upwind sign folded in
// FM: 0 NND, 1 WENO5, 2 WENO5 with the range-safe weights, -1 the
// sample's FMETHOD and weight form (read at run time)
template <class S, class C, int FM = -1>
__device__ __forceinline__ C box_flux(const SampleParams &sp, const S *c0, int st, C ae)
{
    if (FM == 1) return weno5<C, false>(ae, (C)c0[-2 * st], (C)c0[-st], (C)c0[0], (C)c0[st], (C)c0[2 * st]);
    if (FM == 2) return weno5<C, true>(ae, (C)c0[-2 * st], (C)c0[-st], (C)c0[0], (C)c0[st], (C)c0[2 * st]);
    if (FM < 0 && sp.fm) return weno5_sp<C>(sp, ae, (C)c0[-2 * st], (C)c0[-st], (C)c0[0], (C)c0[st], (C)c0[2 * st]);
    return nnd3<C>(ae, (C)c0[-st], (C)c0[0], (C)c0[st]);
}

// Both planes of one face at once (FP32 simple tiles): cf and ch are the
// f and h values at the face's node, st the upwind element step.  Each lane
// takes the scalar reconstruction's operations, so the result is the pair
// box_flux would return for cf and ch.
template <class S, int FM>
__device__ __forceinline__ float2 box_flux2(const S *cf, const S *ch, int st, float ae)
{
    const float2 a = make_float2(ae, ae);
#define UQ_PAIR(j) make_float2((float)cf[(j) * st], (float)ch[(j) * st])
    if (FM == 1) return weno5<float2, false>(a, UQ_PAIR(-2), UQ_PAIR(-1), UQ_PAIR(0), UQ_PAIR(1), UQ_PAIR(2));
    if (FM == 2) return weno5<float2, true>(a, UQ_PAIR(-2), UQ_PAIR(-1), UQ_PAIR(0), UQ_PAIR(1), UQ_PAIR(2));
    return nnd3<float2>(a, UQ_PAIR(-1), UQ_PAIR(0), UQ_PAIR(1));
#undef UQ_PAIR
}

// Both planes of a face at a plain node from the staged box (f at cf, h at
// ch): one packed pair when the scheme is fixed at compile time in FP32,
// else two scalar reconstructions; the same values either way.
template <class S, class C, int FM>
__device__ __forceinline__ void box_flux_fh(const SampleParams &sp, const S *cf, const S *ch, int st, C ae, C &a, C &b)
{
    if constexpr (FM >= 0 && std::is_same<C, float>::value) {
        const float2 v = box_flux2<S, FM>(cf, ch, st, ae);
        a = v.x;
        b = v.y;
    } else {
        a = box_flux<S, C, FM>(sp, cf, st, ae);
        b = box_flux<S, C, FM>(sp, ch, st, ae);
    }
}

// simple FP32 tiles reconstruct the f and h planes of a face as one pair
template <class C, bool SIMPLE, int FM>
struct PairFaces {
    static constexpr bool value = SIMPLE && FM >= 0 && std::is_same<C, float>::value;
};

// flux_exact (the boundary-aware stencil with the linear extrapolation over
// a solid edge) for both planes of direction i at node (xn, yn), reading
// the values from the staged box (fb: the f plane; the h plane pstride
// further) instead of global memory.  (ux, uy) is the node's place in box
// coordinates before a periodic wrap.  Every point the stencil and the
// extrapolation touch lies within 3 nodes of the node along the axis,
// inside the box; positions come from bc_index as in flux_exact (clamped at
// a closed edge; along a periodic axis the box holds the images at the
// unwrapped places).  Not for an axis with a mirror edge (that reads the
// reflected direction's planes).
template <class S, class C>
__device__ __noinline__ void flux_exact_box(const SampleParams &sp, const StageView<S> &v, const S *fb, int pstride,
                                            int BW, int bx0, int by0, int xn, int yn, int ux, int uy, int i, int axis,
                                            C &outf, C &outh)
{
    const int ev = axis == 0 ? c_EX[i] : c_EY[i];
    const int e = isgn(ev);
    const C ae = (C)(sp.c * (double)abs(ev));
    const bool per = (sp.flags & (axis == 0 ? SF_PERX : SF_PERY)) != 0;
    const int L = sp.fm ? 5 : 3, low = (L - 1) / 2;
    const int pos = axis == 0 ? xn : yn, upos = axis == 0 ? ux : uy;
    const int j1 = pos - e * low, uj1 = upos - e * low;
    // box element of axis coordinate b (the other coordinate fixed)
    auto at = [&](int b) { return axis == 0 ? (uy - by0) * BW + (b - bx0) : (b - by0) * BW + (ux - bx0); };
    C Sf[5], Sh[5];
    int sld[5];
    int any = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        if (j < L) {
            int m;
            const int r = bc_index(sp, j1, e * j, axis, m);
            const int o = at(per ? uj1 + e * j : r);
            Sf[j] = (C)fb[o];
            Sh[j] = (C)fb[pstride + o];
            const int xr = axis == 0 ? r : xn, yr = axis == 0 ? yn : r;
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
        const int upe = uj1 + e * jj;
        const int o1 = at(per ? upe + e * diff : bc_index(sp, pe, e * diff, axis, m));
        const int o2 = at(per ? upe + 2 * e * diff : bc_index(sp, pe, e * 2 * diff, axis, m));
        const C extf = C(2) * (C)fb[o1] - (C)fb[o2];
        const C exth = C(2) * (C)fb[pstride + o1] - (C)fb[pstride + o2];
#pragma unroll
        for (int j = 0; j < 5; ++j)
            if (j < L && (j == jj || (j == jj - diff))) {
                Sf[j] = extf;
                Sh[j] = exth;
            }
    }
    if (sp.fm) {
        outf = weno5_sp<C>(sp, ae, Sf[0], Sf[1], Sf[2], Sf[3], Sf[4]);
        outh = weno5_sp<C>(sp, ae, Sh[0], Sh[1], Sh[2], Sh[3], Sh[4]);
    } else {
        outf = nnd3<C>(ae, Sf[0], Sf[1], Sf[2]);
        outh = nnd3<C>(ae, Sh[0], Sh[1], Sh[2]);
    }
}

// The axis has a mirror edge (its boundary-aware stencils read reflected
// planes from global memory).
__device__ __forceinline__ bool mirror_axis(const SampleParams &sp, int axis)
{
    return (sp.flags & (axis == 0 ? (SF_MIRW | SF_MIRE) : (SF_MIRN | SF_MIRS))) != 0;
}

// Flux of plane slot fh (0 f, 1 h) of direction i at node (xn, yn), along
// `axis`: solid nodes answer alpha |e| f; nodes whose stencil meets no
// solid or clamped/mirrored edge read the staged box at (ux, uy), the
// node's place before a periodic wrap (the box holds the periodic images);
// the rest run the exact boundary-aware stencil on global memory.
// `mirrored` selects the reflected plane (cFLUX at a mirror boundary).
template <class S, class C>
__device__ __forceinline__ C any_node_flux(TileCtx<S, C> &k, const S *box, int i, int xn, int yn, int ux, int uy,
                                          int fh, int axis, bool mirrored, bool in_box)
{
    const SampleParams &sp = *k.sp;
    const int ev = axis == 0 ? c_EX[i] : c_EY[i];
    const int pp = fh * NQ + (mirrored ? (axis == 0 ? c_MIR_EW[i] : c_MIR_NS[i]) : i);
    const int oo = yn * k.v.pitch + xn;
    const uint8_t fl = k.v.nf[oo];
    const C ae = (C)(sp.c * (double)abs(ev));
    if ((fl & NF_TYPE) == 2) {
        // wallFluxes' alpha |e| f on full values, written for stored ones:
        // |e| (f_s + (alpha - 1)(f_s + f_ref)) - |e| f_ref
        const C fs = (C)__ldg(k.v.st + (pp * k.v.plane + oo));
        return xmul(ae, xfma((C)k.alpha[oo], xadd(fs, (C)k.fref[pp]), fs));
    }
    const uint8_t edge = axis == 0 ? (NF_SOLX | NF_EDGX) : (NF_SOLY | NF_EDGY);
    if (in_box && !mirrored && !(fl & edge)) {
        const int lx = ux - (k.x0 - HALO_X), ly = uy - (k.y0 - HALO_Y);
        const S *c0 = box + (size_t)fh * k.pstride + ly * k.BW + lx;
        const int e = ev > 0 ? 1 : -1;
        return box_flux<S, C>(sp, c0, axis == 0 ? e : e * k.BW, ae);
    }
    return flux_axis<S, C>(sp, k.v, xn, yn, pp, axis, fl);
}

// Own-node face fluxes of direction i into sf_m (fx_f, fx_h, fy_f, fy_h)
// and the upwind fluxes across the tile edges into ringx_m / ringy_m
// (items numbered from ring0 over the block's threads).
// CEX, CEY: the direction's components when fixed at compile time (else
// DIR_RT and read from the table).
constexpr int DIR_RT = 99;

template <class S, class C, bool SIMPLE, int FM, int CEX = DIR_RT, int CEY = DIR_RT>
__device__ __forceinline__ void dir_fluxes(TileCtx<S, C> &k, const int i, const S *box, C *sf, C *ringx, C *ringy,
                                           int ring0)
{
    const int EX = CEX != DIR_RT ? CEX : c_EX[i], EY = CEY != DIR_RT ? CEY : c_EY[i];
    const int SX = isgn(EX), SY = isgn(EY);
    const int NT = k.NT;
    const SampleParams &sp = *k.sp;
    const C c = (C)sp.c;
    const C aex = C(abs(EX)) * c, aey = C(abs(EY)) * c;
    constexpr bool PAIR = PairFaces<C, SIMPLE, FM>::value;
    constexpr int PER = PAIR ? 1 : 2;  // ring items per edge node (f and h)
    const int nx_items = SX ? PER * k.TY : 0, ny_items = SY ? PER * k.TX : 0;
    // ring items of this direction start at thread ring0 (0 <= ring0 < NT)
    // and cover every item even when a group has more items than threads
    int r0 = k.tid - ring0;
    if (r0 < 0) r0 += NT;
    if (SIMPLE) {
        // every node fluid and fast-path, every upwind neighbour in the box
        const int lx = k.tx + HALO_X, ly = k.ty + HALO_Y;
        const S *cf = box + ly * k.BW + lx;
        const S *ch = cf + k.pstride;
        if constexpr (PAIR) {
            if (SX) {
                const float2 v = box_flux2<S, FM>(cf, ch, SX, aex);
                sf[k.tid] = v.x;
                sf[NT + k.tid] = v.y;
            }
            if (SY) {
                const float2 v = box_flux2<S, FM>(cf, ch, SY * k.BW, aey);
                sf[2 * NT + k.tid] = v.x;
                sf[3 * NT + k.tid] = v.y;
            }
            for (int r = r0; r < nx_items + ny_items; r += NT) {
                if (r < nx_items) {
                    const int row = r;
                    const int bx = (SX > 0 ? -1 : k.TX) + HALO_X, by = row + HALO_Y;
                    const S *e = box + by * k.BW + bx;
                    const float2 v = box_flux2<S, FM>(e, e + k.pstride, SX, aex);
                    ringx[row] = v.x;
                    ringx[k.TY + row] = v.y;
                } else {
                    const int col = r - nx_items;
                    const int bx = col + HALO_X, by = (SY > 0 ? -1 : k.TY) + HALO_Y;
                    const S *e = box + by * k.BW + bx;
                    const float2 v = box_flux2<S, FM>(e, e + k.pstride, SY * k.BW, aey);
                    ringy[col] = v.x;
                    ringy[k.TX + col] = v.y;
                }
            }
            return;
        }
        if (SX) {
            sf[k.tid] = box_flux<S, C, FM>(sp, cf, SX, aex);
            sf[NT + k.tid] = box_flux<S, C, FM>(sp, ch, SX, aex);
        }
        if (SY) {
            sf[2 * NT + k.tid] = box_flux<S, C, FM>(sp, cf, SY * k.BW, aey);
            sf[3 * NT + k.tid] = box_flux<S, C, FM>(sp, ch, SY * k.BW, aey);
        }
        for (int r = r0; r < nx_items + ny_items; r += NT) {
            if (r < nx_items) {
                const int fh = r / k.TY, row = r % k.TY;
                const int bx = (SX > 0 ? -1 : k.TX) + HALO_X, by = row + HALO_Y;
                ringx[fh * k.TY + row] = box_flux<S, C, FM>(sp, box + (size_t)fh * k.pstride + by * k.BW + bx, SX, aex);
            } else {
                const int q = r - nx_items, fh = q / k.TX, col = q % k.TX;
                const int bx = col + HALO_X, by = (SY > 0 ? -1 : k.TY) + HALO_Y;
                ringy[fh * k.TX + col] = box_flux<S, C, FM>(sp, box + (size_t)fh * k.pstride + by * k.BW + bx, SY * k.BW, aey);
            }
        }
        return;
    }
    if (k.active) {
        const int type = k.flag & NF_TYPE;
        const int lx = k.tx + HALO_X, ly = k.ty + HALO_Y;
        const S *cf = box + ly * k.BW + lx;
        const S *ch = cf + k.pstride;
        if (type == 2) {
            // alpha |e| f of wallFluxes on stored deviations (see any_node_flux)
            const C am1 = k.alpha[k.o];
            const C fv = (C)cf[0], hv = (C)ch[0];
            const C gf = xfma(am1, xadd(fv, (C)k.fref[i]), fv), gh = xfma(am1, xadd(hv, (C)k.fref[NQ + i]), hv);
            if (SX) { sf[k.tid] = xmul(aex, gf); sf[NT + k.tid] = xmul(aex, gh); }
            if (SY) { sf[2 * NT + k.tid] = xmul(aey, gf); sf[3 * NT + k.tid] = xmul(aey, gh); }
        } else {
            if (SX) {
                C a, b;
                if ((k.flag & (NF_SOLX | NF_EDGX)) && !mirror_axis(sp, 0)) {
                    flux_exact_box<S, C>(sp, k.v, box, k.pstride, k.BW, k.x0 - HALO_X, k.y0 - HALO_Y, k.x, k.y, k.x,
                                         k.y, i, 0, a, b);
                } else if (k.flag & (NF_SOLX | NF_EDGX)) {
                    a = flux_axis<S, C>(sp, k.v, k.x, k.y, i, 0, k.flag);
                    b = flux_axis<S, C>(sp, k.v, k.x, k.y, NQ + i, 0, k.flag);
                } else {
                    box_flux_fh<S, C, FM>(sp, cf, ch, SX, aex, a, b);
                }
                sf[k.tid] = a;
                sf[NT + k.tid] = b;
            }
            if (SY) {
                C a, b;
                if ((k.flag & (NF_SOLY | NF_EDGY)) && !mirror_axis(sp, 1)) {
                    flux_exact_box<S, C>(sp, k.v, box, k.pstride, k.BW, k.x0 - HALO_X, k.y0 - HALO_Y, k.x, k.y, k.x,
                                         k.y, i, 1, a, b);
                } else if (k.flag & (NF_SOLY | NF_EDGY)) {
                    a = flux_axis<S, C>(sp, k.v, k.x, k.y, i, 1, k.flag);
                    b = flux_axis<S, C>(sp, k.v, k.x, k.y, NQ + i, 1, k.flag);
                } else {
                    box_flux_fh<S, C, FM>(sp, cf, ch, SY * k.BW, aey, a, b);
                }
                sf[2 * NT + k.tid] = a;
                sf[3 * NT + k.tid] = b;
            }
        }
    }
    // upwind neighbours outside the tile: index(x, -e) with reflection
    for (int r = r0; r < nx_items + ny_items; r += NT) {
        if (r < nx_items) {
            const int fh = r / k.TY, row = r % k.TY, yy = k.y0 + row;
            C val = C(0);
            if (yy < k.y_end) {
                int m;
                const int xn = SX > 0 ? k.x0 : k.x_end - 1;
                const int xr = bc_index(sp, xn, -SX, 0, m);
                // in the box: the neighbour itself, or its periodic image
                const bool in_box = !m && (xr == xn - SX || (sp.flags & SF_PERX));
                val = any_node_flux<S, C>(k, box, i, xr, yy, xn - SX, yy, fh, 0, m != 0, in_box);
            }
            ringx[fh * k.TY + row] = val;
        } else {
            const int q = r - nx_items, fh = q / k.TX, col = q % k.TX, xx = k.x0 + col;
            C val = C(0);
            if (xx < k.x_end) {
                int m;
                const int yn = SY > 0 ? k.y0 : k.y_end - 1;
                const int yr = bc_index(sp, yn, -SY, 1, m);
                const bool in_box = !m && (yr == yn - SY || (sp.flags & SF_PERY));
                val = any_node_flux<S, C>(k, box, i, xx, yr, xx, yn - SY, fh, 1, m != 0, in_box);
            }
            ringy[fh * k.TX + col] = val;
        }
    }
}

// divergence D = (dt/dx, dt/dy).(F_out - F_in) of cFLUX
// (cpuLBM.cpp:1436-1470) for direction i at this node.  Every operation is
// an explicitly rounded one, so each kernel instance (simple, wrap and
// general tiles, any tile shape) gives a node the same bits.  FP64 keeps the
// reference's order (each flux scaled, out and in summed, then subtracted);
// FP32 takes the differences first (fewer operations).
template <class S, class C, int CEX = DIR_RT, int CEY = DIR_RT>
__device__ __forceinline__ void dir_divergence(TileCtx<S, C> &k, const int i, const C *sf, const C *ringx,
                                               const C *ringy)
{
    const int SX = isgn(CEX != DIR_RT ? CEX : c_EX[i]), SY = isgn(CEY != DIR_RT ? CEY : c_EY[i]);
    const int NT = k.NT;
    C fox = C(0), hox = C(0), fix = C(0), hix = C(0), foy = C(0), hoy = C(0), fiy = C(0), hiy = C(0);
    if (SX) {
        const int xu = k.x - SX;
        const bool inside = xu >= k.x0 && xu < k.x_end;
        fix = inside ? sf[k.tid - SX] : ringx[k.ty];
        hix = inside ? sf[NT + k.tid - SX] : ringx[k.TY + k.ty];
        fox = sf[k.tid];
        hox = sf[NT + k.tid];
    }
    if (SY) {
        const int yu = k.y - SY;
        const bool inside = yu >= k.y0 && yu < k.y_end;
        fiy = inside ? sf[2 * NT + k.tid - SY * k.TX] : ringy[k.tx];
        hiy = inside ? sf[3 * NT + k.tid - SY * k.TX] : ringy[k.TX + k.tx];
        foy = sf[2 * NT + k.tid];
        hoy = sf[3 * NT + k.tid];
    }
    C df, dh;
    if constexpr (IsF32<C>::value) {
        if (SX && SY) {
            df = xfma(k.tdy, xsub(foy, fiy), xmul(k.tdx, xsub(fox, fix)));
            dh = xfma(k.tdy, xsub(hoy, hiy), xmul(k.tdx, xsub(hox, hix)));
        } else if (SX) {
            df = xmul(k.tdx, xsub(fox, fix));
            dh = xmul(k.tdx, xsub(hox, hix));
        } else {
            df = xmul(k.tdy, xsub(foy, fiy));
            dh = xmul(k.tdy, xsub(hoy, hiy));
        }
    } else {
        if (SX && SY) {
            df = xsub(xadd(xmul(k.tdx, fox), xmul(k.tdy, foy)), xadd(xmul(k.tdx, fix), xmul(k.tdy, fiy)));
            dh = xsub(xadd(xmul(k.tdx, hox), xmul(k.tdy, hoy)), xadd(xmul(k.tdx, hix), xmul(k.tdy, hiy)));
        } else if (SX) {
            df = xsub(xmul(k.tdx, fox), xmul(k.tdx, fix));
            dh = xsub(xmul(k.tdx, hox), xmul(k.tdx, hix));
        } else {
            df = xsub(xmul(k.tdy, foy), xmul(k.tdy, fiy));
            dh = xsub(xmul(k.tdy, hoy), xmul(k.tdy, hiy));
        }
    }
    k.sD[i * NT + k.tid] = df;
    k.sD[(NQ + i) * NT + k.tid] = dh;
}

// General tiles whose box crosses a periodic edge: the box cells outside
// the domain along a periodic axis get the periodic images of the staged
// planes (TMA does not wrap), so wrapped stencils read the box like any
// other.  Along a non-periodic axis the cells outside stay as loaded; no box
// path reads them (nodes near such edges take the exact stencil).
template <int G, class S, class C>
__device__ void wrap_fixup(TileCtx<S, C> &k, int g, S *boxes)
{
    const SampleParams &sp = *k.sp;
    const bool px = (sp.flags & SF_PERX) != 0, py = (sp.flags & SF_PERY) != 0;
    const int nx = sp.nx, ny = sp.ny, BW = k.BW, BH = k.BH;
    const int gx0 = k.x0 - HALO_X, gy0 = k.y0 - HALO_Y;
    // box columns [0, cl) and [cr, BW) lie outside [0, nx); rows [0, rl), [rr, BH) outside [0, ny)
    const int cl = px ? max(0, min(BW, -gx0)) : 0, cr = px ? max(cl, min(BW, nx - gx0)) : BW;
    const int rl = py ? max(0, min(BH, -gy0)) : 0, rr = py ? max(rl, min(BH, ny - gy0)) : BH;
    const int ncol = cl + (BW - cr), nrow = rl + (BH - rr), inner = cr - cl;
    // the wrapped columns in every row, then the wrapped rows of the other columns
    const int n1 = ncol * BH, per = n1 + nrow * inner;
    for (int e = k.tid; e < 2 * G * per; e += k.NT) {
        const int pl = e / per, q = e - pl * per;
        int bx, by;
        if (q < n1) {
            const int c = q / BH;
            by = q - c * BH;
            bx = c < cl ? c : cr + (c - cl);
        } else {
            const int q2 = q - n1, r = q2 / inner;
            bx = cl + (q2 - r * inner);
            by = r < rl ? r : rr + (r - rl);
        }
        int gx = gx0 + bx, gy = gy0 + by;
        if (gx < 0 || gx >= nx) {
            if (!px) continue;
            gx = ((gx % nx) + nx) % nx;
        }
        if (gy < 0 || gy >= ny) {
            if (!py) continue;
            gy = ((gy % ny) + ny) % ny;
        }
        const int plane = (pl & 1) * NQ + group_dir<G>(g, pl >> 1);
        boxes[(size_t)pl * k.pstride + by * BW + bx] = ldv(k.v, plane, gx, gy);
    }
}

// Group g of G directions: wait for its staged boxes, the face fluxes
// (posFluxes/computeFlux, cpuLBM.cpp:1405-1500; solid nodes answer
// wallFluxes' alpha |e| f, cpuLBM.cpp:1576-1586) and edge fluxes of each,
// one barrier, refill the slot, then each direction's divergence.  WRAP:
// a wrap tile (simple code after the periodic images are copied in).
template <class S, class C, bool SIMPLE, int G, int FM, bool WRAP = false>
__device__ __forceinline__ void dir_group(TileCtx<S, C> &k, const int g)
{
    constexpr int NST = GroupCfg<G>::NSTAGE;
    const int buf = g & 1;
    const int slot = g % NST;
    const uint32_t parity = (g / NST) & 1;
    const int NT = k.NT;
    // every issued copy is waited for (boundedly), also after a timeout, so
    // no copy is still in flight when the block exits
    if (!mbar_wait_bounded(&k.bars[slot], parity, TMA_WAIT_POLLS)) {
        *k.timed_out = 1;
        atomicOr(k.status, STATUS_TIMEOUT);
    }
    const S *boxes = k.stg + (size_t)slot * 2 * G * k.pstride;
    if ((WRAP || !SIMPLE) && k.wrap_fix) {
        // k.wrap_fix is the same for the whole block
        wrap_fixup<G>(k, g, const_cast<S *>(boxes));
        __syncthreads();
    }
    int ring0 = 0;
#pragma unroll 1
    for (int m = 0; m < G; ++m) {
        const int i = group_dir<G>(g, m);
        C *sf = k.sf + (size_t)(buf * G + m) * 4 * NT;
        C *rx = k.ringx + (size_t)(buf * G + m) * 2 * k.TY;
        C *ry = k.ringy + (size_t)(buf * G + m) * 2 * k.TX;
        dir_fluxes<S, C, SIMPLE, FM>(k, i, boxes + (size_t)(2 * m) * k.pstride, sf, rx, ry, ring0);
        constexpr int PER = PairFaces<C, SIMPLE, FM>::value ? 1 : 2;
        ring0 += (c_EX[i] ? PER * k.TY : 0) + (c_EY[i] ? PER * k.TX : 0);
        while (ring0 >= NT) ring0 -= NT;
    }
    __syncthreads();
    // every thread is done with this slot: refill it NST groups ahead, or
    // (the first slot that no later group needs) take the state prefetch
    if (g + NST < GroupCfg<G>::NGROUP && k.tid == 0) issue_group_load<G>(k, g + NST, slot);
    else if (flux_prefetch(sizeof(S)) && g == GroupCfg<G>::NGROUP - NST && k.tid == 0)
        issue_state_prefetch<G>(k, slot);
    if (SIMPLE || (k.active && (k.flag & NF_TYPE) == 0)) {
#pragma unroll 1
        for (int m = 0; m < G; ++m) {
            const int i = group_dir<G>(g, m);
            dir_divergence<S, C>(k, i, k.sf + (size_t)(buf * G + m) * 4 * NT,
                                 k.ringx + (size_t)(buf * G + m) * 2 * k.TY, k.ringy + (size_t)(buf * G + m) * 2 * k.TX);
        }
    }
    // sf and the rings are double-buffered by group parity: buffer (g & 1)
    // is written again at group g + 2, after group g + 1's barrier, which
    // every reader of this group has passed.
}

// The D2Q13 velocity table as compile-time constants (c_EX, c_EY on the
// device); DirC<G, g, m>: direction m of group g (group_dir<G>) with its
// components.
struct DirTable {
    static constexpr int EX[NQ] = {0, 1, 0, -1, 0, 1, -1, -1, 1, 2, 0, -2, 0};
    static constexpr int EY[NQ] = {0, 0, 1, 0, -1, 1, 1, -1, -1, 0, 2, 0, -2};
};
template <int G, int g, int m>
struct DirC {
    static constexpr int i = group_dir<G>(g, m);
    static constexpr int EX = DirTable::EX[i], EY = DirTable::EY[i];
};

// Simple tiles with every direction fixed at compile time: the group loop
// and the loop over a group's directions unrolled, each direction's
// components constants (strides, signs, which faces and edge items exist).
template <class S, class C, int FM, int G, int g, int m>
__device__ __forceinline__ void group_fluxes_c(TileCtx<S, C> &k, const S *boxes, int &ring0)
{
    if constexpr (m < G) {
        using D = DirC<G, g, m>;
        const int NT = k.NT;
        constexpr int b = (g & 1) * G + m;
        dir_fluxes<S, C, true, FM, D::EX, D::EY>(k, D::i, boxes + (size_t)(2 * m) * k.pstride,
                                                 k.sf + (size_t)b * 4 * NT, k.ringx + (size_t)b * 2 * k.TY,
                                                 k.ringy + (size_t)b * 2 * k.TX, ring0);
        ring0 += (D::EX ? k.TY : 0) + (D::EY ? k.TX : 0);
        while (ring0 >= NT) ring0 -= NT;
        group_fluxes_c<S, C, FM, G, g, m + 1>(k, boxes, ring0);
    }
}

template <class S, class C, int G, int g, int m>
__device__ __forceinline__ void group_divergence_c(TileCtx<S, C> &k)
{
    if constexpr (m < G) {
        using D = DirC<G, g, m>;
        constexpr int b = (g & 1) * G + m;
        dir_divergence<S, C, D::EX, D::EY>(k, D::i, k.sf + (size_t)b * 4 * k.NT, k.ringx + (size_t)b * 2 * k.TY,
                                           k.ringy + (size_t)b * 2 * k.TX);
        group_divergence_c<S, C, G, g, m + 1>(k);
    }
}

// dir_group with the group fixed at compile time, then the next group
template <class S, class C, int FM, int G, int g, bool WRAP = false>
__device__ __forceinline__ void run_groups_c(TileCtx<S, C> &k)
{
    if constexpr (g < GroupCfg<G>::NGROUP) {
        constexpr int NST = GroupCfg<G>::NSTAGE;
        constexpr int slot = g % NST;
        constexpr uint32_t parity = (g / NST) & 1;
        if (!mbar_wait_bounded(&k.bars[slot], parity, TMA_WAIT_POLLS)) {
            *k.timed_out = 1;
            atomicOr(k.status, STATUS_TIMEOUT);
        }
        const S *boxes = k.stg + (size_t)slot * 2 * G * k.pstride;
        if constexpr (WRAP) {
            wrap_fixup<G>(k, g, const_cast<S *>(boxes));
            __syncthreads();
        }
        int ring0 = 0;
        group_fluxes_c<S, C, FM, G, g, 0>(k, boxes, ring0);
        __syncthreads();
        if (g + NST < GroupCfg<G>::NGROUP && k.tid == 0) issue_group_load<G>(k, g + NST, slot);
        else if (flux_prefetch(sizeof(S)) && g == GroupCfg<G>::NGROUP - NST && k.tid == 0)
            issue_state_prefetch<G>(k, slot);
        group_divergence_c<S, C, G, g, 0>(k);
        run_groups_c<S, C, FM, G, g + 1, WRAP>(k);
    }
}

template <class S>
struct FluxGroup {
    static constexpr int value = sizeof(S) == 4 ? 4 : 1;
};

size_t flux_smem_bytes_t(size_t es, int tx, int ty)
{
    const int G = es == 4 ? 4 : 1;
    return flux_layout(es, es, tx, ty, G, G == 4 ? GroupCfg<4>::NSTAGE : GroupCfg<1>::NSTAGE).total;
}

// MODE: 1 = RK3 stage 3 (fluxes of buffer 2), 2 = RK3 final (buffer 3),
// 3 = RK1 update, 4 = EULER update, 5 = EULER_EQ update (buffer 2)
// PATH (FluxPath): FLUX_SIMPLE / FLUX_GENERAL compile only the code of that
// kind of tile (the two together are far smaller per kernel than one kernel
// holding both, which the register allocation of the simple path needs);
// FLUX_WRAP is the simple code with the periodic images copied into each
// staged box before use.  A block given a tile of another kind returns at
// once.
// TC: the tile shape is the default TILE_CX x TILE_CY, compiled in (box
// widths, strides and the thread-to-node map become constants); otherwise
// read from the arguments.
template <class S, class C, int MODE, int PATH, bool TC>
__global__ void __launch_bounds__(256, 2) k_flux(KArgs<S> a)
{
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const int TX = TC ? TILE_CX : a.tx, TY = TC ? TILE_CY : a.ty, NT = TX * TY;
    const int BW = TX + 2 * HALO_X, BH = TY + 2 * HALO_Y;
    constexpr int G = FluxGroup<S>::value;
    constexpr int NST = GroupCfg<G>::NSTAGE;
    const FluxSmemLayout Ls = flux_layout(sizeof(C), sizeof(S), TX, TY, G, NST);
    unsigned char *smem_raw = smem_dyn + ((128 - (smem_u32(smem_dyn) & 127)) & 127);
    C *sf = reinterpret_cast<C *>(smem_raw);  // [2][G][4][NT]
    C *ringx = sf + 8 * G * NT;                // [2][G][2][TY]
    C *ringy = ringx + 4 * G * TY;             // [2][G][2][TX]
    C *sD = ringy + 4 * G * TX;                // [26][NT]
    S *stg = reinterpret_cast<S *>(smem_raw + Ls.stage_off);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + Ls.bar_off);
    __shared__ double red[32];
    __shared__ SampleParams s_sp;  // kept out of registers: read as needed
    __shared__ int s_timeout;

    const Tile t = a.tiles[blockIdx.x];
    if ((tile_simple(t) ? FLUX_SIMPLE : tile_wrap(t) ? FLUX_WRAP : FLUX_GENERAL) != PATH) return;
    constexpr bool WRAPT = PATH == FLUX_WRAP;
    const int tid = threadIdx.x;
    constexpr int PH = MODE == 2 ? 2 : 1;
    const CUtensorMap *map = a.tmaps + MAPS_PER_SAMPLE * t.sample + (PH == 1 ? 0 : 1);
    constexpr bool PREF = flux_prefetch(sizeof(S));

    TileCtx<S, C> k;
    k.NT = NT; k.TX = TX; k.TY = TY; k.BW = BW; k.BH = BH; k.tid = tid;
    k.x0 = t.x0; k.y0 = t.y0;
    k.stg = stg; k.pstride = (int)(Ls.plane_bytes / sizeof(S)); k.bars = bars; k.map = map; k.timed_out = &s_timeout;
    k.smap = a.tmaps + MAPS_PER_SAMPLE * t.sample + 2;
    k.pref_h = reinterpret_cast<S *>(smem_raw + Ls.pref_off);
    if (tid == 0) {
        s_sp = a.samples[t.sample];
        s_timeout = 0;
        k.gx = s_sp.gx;
        for (int b = 0; b < NST + (PREF ? 1 : 0); ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
        for (int g = 0; g < NST; ++g) issue_group_load<G>(k, g, g);
    }
    __syncthreads();
    const SampleParams &sp = s_sp;
    const int tx = tid % TX, ty = tid / TX;
    const int x = t.x0 + tx, y = t.y0 + ty;
    const int x_end = min(t.x0 + TX, sp.nx), y_end = min(t.y0 + TY, sp.ny);
    const bool active = x < sp.nx && y < sp.ny;
    const S *stage = PH == 1 ? a.buf2 : a.buf3;
    const StageView<S> v{stage + sp.state_off, a.nflags + sp.node_off, (int)sp.plane, sp.pitch};
    const int o = y * sp.pitch + x;
    const C *alpha = a.template alpha_as<C>() + sp.node_off;

    k.sp = &sp;
    k.gx = sp.gx;
    k.v = v;
    k.alpha = alpha;
    k.fref = a.fref + NPL * t.sample;
    k.sf = sf;
    k.ringx = ringx;
    k.ringy = ringy;
    k.sD = sD;
    k.status = &a.status[t.sample];
    k.tx = tx; k.ty = ty; k.x = x; k.y = y;
    k.x_end = x_end; k.y_end = y_end; k.o = o;
    k.active = active;
    k.wrap_fix = PATH != FLUX_SIMPLE &&
                 (((sp.flags & SF_PERX) && (t.x0 < HALO_X || t.x0 + TX + HALO_X > sp.nx)) ||
                  ((sp.flags & SF_PERY) && (t.y0 < HALO_Y || t.y0 + TY + HALO_Y > sp.ny)));
    k.flag = active ? v.nf[o] : 0;
    k.tdx = active ? (C)a.tdx[sp.xoff + x] : C(0);
    k.tdy = active ? (C)a.tdy[sp.yoff + y] : C(0);
    const int type = k.flag & NF_TYPE;
    sD[tid] = C(0);          // direction 0 streams nothing
    sD[NQ * NT + tid] = C(0);
    if (PATH != FLUX_GENERAL) {
        // simple tiles: the flux scheme fixed at compile time (smaller hot
        // code); for narrow-range WENO5, the common case, in FP32 and in the
        // FP64 final phase also every direction (the other instances lose
        // more to their larger code than they gain)
        if (sp.fm && sizeof(S) == 4 && sp.wide) {
#pragma unroll 1
            for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, true, G, 2, WRAPT>(k, g);
        } else if (sp.fm) {
            if constexpr (G == 4 || MODE == 2) {
                run_groups_c<S, C, 1, G, 0, WRAPT>(k);
            } else {
#pragma unroll 1
                for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, true, G, 1, WRAPT>(k, g);
            }
        } else {
#pragma unroll 1
            for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, true, G, 0, WRAPT>(k, g);
        }
    } else {
        // general tiles: the scheme fixed at compile time for their plain
        // nodes' faces (the boundary stencils read it at run time)
        if (sp.fm && sizeof(S) == 4 && sp.wide) {
#pragma unroll 1
            for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, false, G, 2>(k, g);
        } else if (sp.fm) {
#pragma unroll 1
            for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, false, G, 1>(k, g);
        } else {
#pragma unroll 1
            for (int g = 0; g < GroupCfg<G>::NGROUP; ++g) dir_group<S, C, false, G, 0>(k, g);
        }
    }

    // the prefetched state values: every thread waits (boundedly) for the
    // copies, so that none is in flight when the block exits
    const S *pref_f = nullptr;
    if constexpr (PREF) {
        if (!mbar_wait_bounded(&bars[NST], 0, TMA_WAIT_POLLS)) {
            s_timeout = 1;
            atomicOr(&a.status[t.sample], STATUS_TIMEOUT);
        }
        pref_f = stg + (size_t)((GroupCfg<G>::NGROUP - NST) % NST) * 2 * G * k.pstride;
    }
    double res_part = 0;
    if (active && type == 0) {
        // this node in plane 0 of each buffer; planes PL elements apart
        S *__restrict__ st = a.state + sp.state_off + o;
        const S *__restrict__ b2 = a.buf2 + sp.state_off + o;
        S *__restrict__ b3 = a.buf3 + sp.state_off + o;
        const int PL = (int)sp.plane;
        // the node's state value of plane p at the start of the update: from
        // the prefetch (FP32) or from memory
        const S *pref_h = k.pref_h;
        auto rd = [&](int p) -> S {
            if constexpr (PREF) return p < NQ ? pref_f[p * NT + tid] : pref_h[(p - NQ) * NT + tid];
            else return st[p * PL];
        };
        const C dt = (C)sp.dt;
        bool final_phase = true;
        double fin_r = 0, fin_sh = 0;  // FP64 sums of the new state (MODE 2)
        if (MODE == 1) {
            // RK3 stage 3 (cpuLBM.cpp:1928-1993) and the part of the update
            // (cpuLBM.cpp:1999-2042) that does not need the stage-3 fluxes
            final_phase = false;
            const int gd = ghost_offset(sp, x);
            // stage-1 moments (= stage 2's) and the moments of f - div F(f2)
            // (macroProp3, cpuLBM.cpp:973-1032), both summed in FP64
            constexpr bool DEV = sizeof(S) == 4;
            Macro m1, m3;
            C rq1, rq3, ux1, uy1, ux3, uy3;
            double rho3;
            {
                // one pass over the values for both
                double r1 = 0, x1 = 0, y1 = 0, s1 = 0, r3 = 0, x3 = 0, y3 = 0, s3 = 0;
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const double fv = (double)rd(i), hv = (double)rd(NQ + i);
                    const double d = fv - (double)sD[i * NT + tid];
                    r1 += fv;
                    mom_add(x1, lat_ex(i), fv);
                    mom_add(y1, lat_ey(i), fv);
                    s1 += hv;
                    r3 += d;
                    mom_add(x3, lat_ex(i), d);
                    mom_add(y3, lat_ey(i), d);
                    s3 += hv - (double)sD[(NQ + i) * NT + tid];
                }
                m1 = macro_from_sums(r1, sp.c * x1, sp.c * y1, s1, sp);
                m3 = macro_from_sums(r3, sp.c * x3, sp.c * y3, s3, sp);
                rq1 = (C)m1.q; ux1 = (C)m1.ux; uy1 = (C)m1.uy;
                rq3 = (C)m3.q; ux3 = (C)m3.ux; uy3 = (C)m3.uy;
                rho3 = m3.rho;
            }
            const EqArgs<C, DEV> q1(m1.rho, m1.ux, m1.uy, m1.T, sp);
            const EqArgs<C, DEV> q3(m3.rho, m3.ux, m3.uy, m3.T, sp);
            const C hdt = dt * C(0.5);
            const C cu1 = (C)sp.c * ux1, cv1 = (C)sp.c * uy1, cu3 = (C)sp.c * ux3, cv3 = (C)sp.c * uy3;
            // dt/(2 tau) and 1/tau of stages 2 (= 1) and 3, all from q = p/mu
            const C Pr = (C)sp.Pr;
            const C itf2 = rq1, itf3 = rq3, ith2 = Pr * rq1, ith3 = Pr * rq3;
            const C g2 = (Pr - C(1)) * rq1, g3 = (Pr - C(1)) * rq3;
            const C a2 = hdt * itf2, a3 = hdt * itf3, b2c = hdt * ith2, b3c = hdt * ith3;
            const C ia3 = C(1) / (C(1) + a3), ib3 = C(1) / (C(1) + b3c);
            double sf3 = 0;
            auto family = [&](const int fam) {
                C e1f[4], e1h[4], e3f[4], e3h[4];
                q1.fam(fam, e1f, e1h);
                q3.fam(fam, e3f, e3h);
                const int i0 = fam == 0 ? 0 : 4 * fam - 3, n = fam == 0 ? 1 : 4;
                C vf[4], vh[4], vf2[4], vh2[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= n) break;
                    const int of = (i0 + k) * PL, oh = (NQ + i0 + k) * PL;
                    vf[k] = (C)rd(i0 + k); vh[k] = (C)rd(NQ + i0 + k); vf2[k] = (C)b2[of]; vh2[k] = (C)b2[oh];
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= n) break;
                    const int i = i0 + k;
                    sf3 += (double)e3f[k];
                    const int of = i * PL, oh = (NQ + i) * PL;
                    const C f = vf[k], h = vh[k], f2 = vf2[k], h2 = vh2[k];
                    const C Df = sD[i * NT + tid], Dh = sD[(NQ + i) * NT + tid];
                    C eu2, eu3;
                    if constexpr (sizeof(S) == 4) {
                        eu2 = e_dot<C>(i, cu1, cv1);
                        eu3 = e_dot<C>(i, cu3, cv3);
                    } else {
                        const C exi = (C)(sp.c * c_EX[i]), eyi = (C)(sp.c * c_EY[i]);
                        eu2 = exi * ux1 + eyi * uy1;
                        eu3 = exi * ux3 + eyi * uy3;
                    }
                    // stage 3 (cpuLBM.cpp:1970, 1986) and the update without
                    // the stage-3 fluxes (cpuLBM.cpp:2022, 2039)
                    C f3, h3, accf, acch;
                    if constexpr (sizeof(S) == 4) {
                        // FP32: the f and h lanes as packed pairs, every
                        // operation explicitly rounded
                        // (a2, b2c) = hdt (1/tau_f, 1/tau_h) of stage 2, (a3, b3c) of stage 3
                        const float2 A2 = make_float2(a2, b2c), A3 = make_float2(a3, b3c);
                        const float2 D = make_float2(Df, Dh), E3 = make_float2(e3f[k], e3h[k]);
                        const float2 D1 = xsub(make_float2(e1f[k], e1h[k]), make_float2(f2, h2));
                        const float2 V = make_float2(f, h);
                        const float2 X = xfma(A2, D1, xfma(A3, E3, xsub(V, D)));
                        f3 = xmul(X.x, ia3);
                        // hdt times the coupling term cpl
                        const float hc = xmul(hdt, xfma(xmul(eu2, g2), D1.x, xmul(xmul(eu3, g3), xsub(E3.x, f3))));
                        h3 = xmul(xsub(X.y, hc), ib3);
                        const float2 acc = xfma(A3, xsub(E3, make_float2(f3, h3)), xfma(A2, D1, xfma(kc<float2>(-0.5), D, V)));
                        accf = acc.x;
                        acch = xsub(acc.y, hc);
                    } else {
                        f3 = (f - Df + a2 * (e1f[k] - f2) + a3 * e3f[k]) * ia3;
                        const C cpl = eu2 * g2 * (e1f[k] - f2) + eu3 * g3 * (e3f[k] - f3);
                        h3 = (h - Dh - hdt * cpl + b2c * (e1h[k] - h2) + b3c * e3h[k]) * ib3;
                        accf = f - C(0.5) * Df + hdt * ((e1f[k] - f2) * itf2 + (e3f[k] - f3) * itf3);
                        acch = h - C(0.5) * Dh + hdt * ((e1h[k] - h2) * ith2 + (e3h[k] - h3) * ith3) - hdt * cpl;
                    }
                    b3[of] = (S)f3;
                    b3[oh] = (S)h3;
                    if (gd) {
                        b3[of + gd] = (S)f3;
                        b3[oh + gd] = (S)h3;
                    }
                    st[of] = (S)accf;
                    st[oh] = (S)acch;
                }
            };
            if constexpr (sizeof(S) == 4) {
#pragma unroll
                for (int fam = 0; fam < 4; ++fam) family(fam);
            } else {
#pragma unroll 1
                for (int fam = 0; fam < 4; ++fam) family(fam);
            }
            if (fabs(sf3 - (rho3 - sp.rho0)) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(rho3))))
                atomicOr(&a.status[t.sample], STATUS_EQ);
        } else if (MODE == 2) {
            // final RK3 combination (cpuLBM.cpp:1999-2042): f = acc - D3/2,
            // f planes then h planes (loads of a half before its stores),
            // summing the new values in FP64 for the finiteness check
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                S acc[NQ];
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] = rd(half * NQ + i);
                // NaN / Inf propagate through an FP32 sum as through an FP64 one
                typename std::conditional<sizeof(S) == 4, float, double>::type sum = 0;
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const S v = (S)((C)acc[i] - C(0.5) * sD[(half * NQ + i) * NT + tid]);
                    st[(half * NQ + i) * PL] = v;
                    sum += v;
                }
                if (half == 0) fin_r = sum;
                else fin_sh = sum;
            }
        } else {
            // RK1 update (cpuLBM.cpp:1674-1710), EULER (:2130-2168), EULER_EQ (:2220-2258)
            const Macro m = node_macro_rd(rd, sp);
            constexpr bool DEV = sizeof(S) == 4;
            const EqArgs<C, DEV> q(m.rho, m.ux, m.uy, m.T, sp);
            const C ux = (C)m.ux, uy = (C)m.uy, Pr = (C)sp.Pr;
            const C cu = (C)sp.c * ux, cv = (C)sp.c * uy;
            const C rtf = dt * (C)m.q, rth = dt * Pr * (C)m.q, rg = (Pr - C(1)) * (C)m.q;  // dt/tau_f, dt/tau_h, 1/tau_hf
            double sf = 0;
            auto family = [&](const int fam) {
                C fe[4], he[4];
                q.fam(fam, fe, he);
                const int i0 = fam == 0 ? 0 : 4 * fam - 3, n = fam == 0 ? 1 : 4;
                C vf[4], vh[4], v1f[4], v1h[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= n) break;
                    const int of = (i0 + k) * PL, oh = (NQ + i0 + k) * PL;
                    vf[k] = (C)rd(i0 + k); vh[k] = (C)rd(NQ + i0 + k);
                    if (MODE == 3) { v1f[k] = (C)b2[of]; v1h[k] = (C)b2[oh]; }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= n) break;
                    const int i = i0 + k;
                    sf += (double)fe[k];
                    const int of = i * PL, oh = (NQ + i) * PL;
                    const C f = vf[k], h = vh[k];
                    const C Df = sD[i * NT + tid], Dh = sD[(NQ + i) * NT + tid];
                    C eu;
                    if constexpr (sizeof(S) == 4) eu = e_dot<C>(i, cu, cv);
                    else eu = (C)(sp.c * c_EX[i]) * ux + (C)(sp.c * c_EY[i]) * uy;
                    C fn, hn;
                    if (MODE == 3) {
                        const C f1 = v1f[k], h1 = v1h[k];
                        fn = f - Df + rtf * (fe[k] - f1);
                        hn = h - Dh + rth * (he[k] - h1) - (dt * eu * rg) * (fe[k] - f1);
                    } else if (MODE == 4) {
                        fn = f - Df + rtf * (fe[k] - f);
                        hn = h - Dh + rth * (he[k] - h) - (dt * eu * rg) * (fe[k] - f);
                    } else {
                        fn = fe[k] - Df;
                        hn = he[k] - Dh;
                    }
                    st[of] = (S)fn;
                    st[oh] = (S)hn;
                }
            };
            if constexpr (sizeof(S) == 4) {
#pragma unroll
                for (int fam = 0; fam < 4; ++fam) family(fam);
            } else {
#pragma unroll 1
                for (int fam = 0; fam < 4; ++fam) family(fam);
            }
            if (MODE >= 4 && fabs(sf - (m.rho - sp.rho0)) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(m.rho))))
                atomicOr(&a.status[t.sample], STATUS_EQ);
        }
        if (final_phase) {
            if (a.want_residual) {
                // macroPropShort of the new state: the residual's T, and the
                // finiteness / positive-density check
                const Macro mn = node_macro(st, sp);
                if (!(mn.rho > 0.0) || !isfinite(mn.rho) || !isfinite(mn.T) || !isfinite(mn.ux) || !isfinite(mn.uy))
                    atomicOr(&a.status[t.sample], STATUS_NONFINITE);
                const double d = mn.T - a.told[sp.node_off + o];
                res_part = d * d;
            } else {
                // finiteness / positive density from the FP64 sums alone
                double r = fin_r, sh = fin_sh;
                if (MODE != 2) {
#pragma unroll
                    for (int i = 0; i < NQ; ++i) {
                        r += (double)st[i * PL];
                        sh += (double)st[(NQ + i) * PL];
                    }
                }
                r += sp.rho0;
                if (!(r > 0.0) || !isfinite(r) || !isfinite(sh)) atomicOr(&a.status[t.sample], STATUS_NONFINITE);
            }
        }
    }
    if (a.want_residual && MODE != 1) {
        // per-tile partial sum, fixed order (deterministic)
        for (int off = 16; off > 0; off >>= 1) res_part += __shfl_down_sync(0xffffffffu, res_part, off);
        if ((tid & 31) == 0) red[tid >> 5] = res_part;
        __syncthreads();
        if (tid == 0) {
            double s = 0;
            for (int w = 0; w < (NT + 31) / 32; ++w) s += red[w];
            a.partial[tile_gid(t)] = s;
        }
    }
}

// Ghost columns (SampleParams::gx): block (s, p) copies, in every row of
// plane p of sample s0 + s, the gx columns at each x edge of the domain to
// the ghost columns beyond the other edge: x in [-gx, 0) gets x + nx, x in
// [nx, nx + gx) gets x - nx.  The stepping kernels keep the ghosts of the
// values they write; this refreshes them after the state is set from
// outside (the fixed nodes' stage values change there).
template <class S>
__global__ void k_fill_ghosts(const SampleParams *samples, int s0, S *buf)
{
    const SampleParams sp = samples[s0 + blockIdx.x];
    if (!sp.gx) return;  // else GHOST_X
    constexpr int gx = GHOST_X, w = 2 * GHOST_X, U = 4;
    const int nx = sp.nx, n = sp.ny * w, pitch = sp.pitch;
    S *pl = buf + sp.state_off + (long long)blockIdx.y * sp.plane;
    // element e: row e / w, ghost e % w (consecutive threads share a row);
    // each thread loads U elements before it stores them
    for (int base = threadIdx.x; base < n; base += U * blockDim.x) {
        S v[U];
        S *dst[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = base + u * blockDim.x;
            dst[u] = nullptr;
            if (e < n) {
                const int y = e / w, c = e % w;
                const int xg = c < gx ? c - gx : nx + (c - gx);  // the ghost
                const int xs = c < gx ? xg + nx : c - gx;        // its image in the domain
                S *row = pl + (long long)y * pitch;
                v[u] = row[xs];
                dst[u] = row + xg;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (dst[u]) *dst[u] = v[u];
    }
}

template <class S>
cudaError_t launch_fill_ghosts(const SampleParams *samples, int s0, int ns, S *buf2, S *buf3, cudaStream_t st)
{
    if (ns > 0) {
        if (buf2) k_fill_ghosts<S><<<dim3(ns, NPL), 256, 0, st>>>(samples, s0, buf2);
        if (buf3) k_fill_ghosts<S><<<dim3(ns, NPL), 256, 0, st>>>(samples, s0, buf3);
    }
    return cudaGetLastError();
}
template cudaError_t launch_fill_ghosts<double>(const SampleParams *, int, int, double *, double *, cudaStream_t);
template cudaError_t launch_fill_ghosts<float>(const SampleParams *, int, int, float *, float *, cudaStream_t);

// per-sample residual = sqrt(sum / (Nx Ny)) (runOne, cpuLBM.cpp:2322-2331)
__global__ void k_residual(const SampleParams *samples, int nsamples, const double *partial, const int *tile_first,
                           const int *tile_count, double *residual)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsamples) return;
    double sum = 0;
    for (int k = 0; k < tile_count[s]; ++k) sum += partial[tile_first[s] + k];
    residual[s] = sqrt(sum / ((double)samples[s].nx * samples[s].ny));
}

// ------------------------------------------------------------ boundary I/O
// macroPropShort for every node of one sample, written in the reference's
// [x*Ny + y] order: rho, ux, uy, T, p, each `stride` values apart.
template <class S>
__global__ void k_macro_out(const SampleParams *samples, int s, const S *state, double *out, long long stride)
{
    const SampleParams sp = samples[s];
    const long long n = (long long)sp.nx * sp.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k % sp.ny), x = (int)(k / sp.ny);
        const Macro m = node_macro_at(state + sp.state_off, sp, (long long)y * sp.pitch + x);
        out[k] = m.rho;
        out[stride + k] = m.ux;
        out[2 * stride + k] = m.uy;
        out[3 * stride + k] = m.T;
        out[4 * stride + k] = m.p;
    }
}

// planes <-> reference AoS [(x*Ny + y)*13 + i] in FP64
template <class S>
__global__ void k_dist_io(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, double *aos, int to_aos,
                          const uint8_t *nflags, const double *fref)
{
    const double *fr = fref + NPL * s;
    const SampleParams sp = samples[s];
    const long long n = (long long)sp.nx * sp.ny * NQ;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % NQ);
        const long long xy = k / NQ;
        const int y = (int)(xy % sp.ny), x = (int)(xy / sp.ny);
        const long long o = (long long)y * sp.pitch + x;
        S *f = state + sp.state_off + (long long)i * sp.plane + o;
        S *h = state + sp.state_off + (long long)(NQ + i) * sp.plane + o;
        if (to_aos) {
            aos[k] = (double)*f + fr[i];
            aos[n + k] = (double)*h + fr[NQ + i];
        } else {
            *f = (S)(aos[k] - fr[i]);
            *h = (S)(aos[n + k] - fr[NQ + i]);
            if (nflags[sp.node_off + o] & NF_TYPE) {  // fixed nodes seed the stage buffers
                const long long of = sp.state_off + (long long)i * sp.plane + o;
                const long long oh = sp.state_off + (long long)(NQ + i) * sp.plane + o;
                buf2[of] = *f; buf3[of] = *f;
                buf2[oh] = *h; buf3[oh] = *h;
            }
        }
    }
}

// f, h = equilibria of per-node fields given in [x*Ny + y] order (FP64):
// rho, ux, uy, T, each `stride` values apart
template <class S>
__global__ void k_set_macro(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, const double *fields,
                            long long stride, const uint8_t *nflags, const double *fref)
{
    const double *fr = fref + NPL * s;
    const SampleParams sp = samples[s];
    const long long n = (long long)sp.nx * sp.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k % sp.ny), x = (int)(k / sp.ny);
        const long long o = (long long)y * sp.pitch + x;
        const bool fixed = (nflags[sp.node_off + o] & NF_TYPE) != 0;
        init_node<S>(fields[k], fields[stride + k], fields[2 * stride + k], fields[3 * stride + k], sp, fr, state, buf2,
                     buf3, o, fixed);
    }
}

template <class S>
cudaError_t launch_set_macro_strided(const SampleParams *samples, int s, S *state, S *buf2, S *buf3,
                                     const double *fields, long long stride, const uint8_t *nflags, const double *fref,
                                     long long nodes, cudaStream_t st)
{
    const int blocks = (int)std::min<long long>((nodes + 255) / 256, 4096);
    k_set_macro<S><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(samples, s, state, buf2, buf3, fields, stride, nflags, fref);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_set_macro(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, const double *fields,
                             const uint8_t *nflags, const double *fref, long long nodes, cudaStream_t st)
{
    return launch_set_macro_strided<S>(samples, s, state, buf2, buf3, fields, nodes, nflags, fref, nodes, st);
}
template cudaError_t launch_set_macro_strided<double>(const SampleParams *, int, double *, double *, double *,
                                                      const double *, long long, const uint8_t *, const double *,
                                                      long long, cudaStream_t);
template cudaError_t launch_set_macro_strided<float>(const SampleParams *, int, float *, float *, float *,
                                                     const double *, long long, const uint8_t *, const double *,
                                                     long long, cudaStream_t);
template cudaError_t launch_set_macro<double>(const SampleParams *, int, double *, double *, double *, const double *,
                                              const uint8_t *, const double *, long long, cudaStream_t);
template cudaError_t launch_set_macro<float>(const SampleParams *, int, float *, float *, float *, const double *,
                                             const uint8_t *, const double *, long long, cudaStream_t);

// ----------------------------------------------------------------- launchers
// phase: 0 pointwise stages, 1 stencil phase over buffer 2, 2 RK3 final
// stencil phase over buffer 3, 3/4 wall fluxes of buffer 2/3.  rk selects
// the method of the tiles passed (one method per launch).
template <class S, class C, int PATH, bool TC>
void launch_flux_t(int mode, const KArgs<S> &k, int ntiles, int NT, size_t sm, cudaStream_t st)
{
    switch (mode) {
    case 1: k_flux<S, C, 1, PATH, TC><<<ntiles, NT, sm, st>>>(k); break;
    case 2: k_flux<S, C, 2, PATH, TC><<<ntiles, NT, sm, st>>>(k); break;
    case 3: k_flux<S, C, 3, PATH, TC><<<ntiles, NT, sm, st>>>(k); break;
    case 4: k_flux<S, C, 4, PATH, TC><<<ntiles, NT, sm, st>>>(k); break;
    default: k_flux<S, C, 5, PATH, TC><<<ntiles, NT, sm, st>>>(k); break;
    }
}

template <class S, class C, int PATH>
void launch_flux(int mode, const KArgs<S> &k, int ntiles, int NT, size_t sm, cudaStream_t st)
{
    if (k.tx == TILE_CX && k.ty == TILE_CY) launch_flux_t<S, C, PATH, true>(mode, k, ntiles, NT, sm, st);
    else launch_flux_t<S, C, PATH, false>(mode, k, ntiles, NT, sm, st);
}

template <class S, class C>
cudaError_t launch_phase(const KArgs<S> &a, int phase, int rk, const Tile *tiles, int ntiles, const WallNode *walls,
                         int nwalls, cudaStream_t st, int path)
{
    KArgs<S> k = a;
    k.tiles = tiles;
    k.ntiles = ntiles;
    const int NT = a.tx * a.ty;
    if (phase == 0) {
        if (!ntiles) return cudaSuccess;
        if (rk == 1) k_stage0<S, C, 1><<<ntiles, NT, 0, st>>>(k);
        else if (rk == 0) k_stage0<S, C, 0><<<ntiles, NT, 0, st>>>(k);
        else k_stage0<S, C, 2><<<ntiles, NT, 0, st>>>(k);
    } else if (phase == 1 || phase == 2) {
        if (!ntiles) return cudaSuccess;
        const size_t sm = flux_smem_bytes_t(sizeof(S), a.tx, a.ty);
        const int mode = phase == 2 ? 2 : (rk == 1 ? 1 : (rk == 0 ? 3 : (rk == 2 ? 4 : 5)));
        if (path == FLUX_BOTH || path == FLUX_SIMPLE) launch_flux<S, C, FLUX_SIMPLE>(mode, k, ntiles, NT, sm, st);
        if (path == FLUX_WRAP) launch_flux<S, C, FLUX_WRAP>(mode, k, ntiles, NT, sm, st);
        if (path == FLUX_BOTH || path == FLUX_GENERAL) launch_flux<S, C, FLUX_GENERAL>(mode, k, ntiles, NT, sm, st);
    } else if (phase == 3 || phase == 4) {
        if (nwalls) k_wall<S, C><<<(nwalls + 127) / 128, 128, 0, st>>>(k, phase == 3 ? a.buf2 : a.buf3, walls, nwalls);
    }
    return cudaGetLastError();
}

template <class S, class C>
cudaError_t prepare_kernels()
{
    const int maxsm = 200 * 1024;
    cudaError_t e = cudaSuccess;
#define UQ_FLUX_SMEM1(M, P, T)                                                                              \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_flux<S, C, M, P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
#define UQ_FLUX_SMEM(M, P) UQ_FLUX_SMEM1(M, P, true) UQ_FLUX_SMEM1(M, P, false)
    UQ_FLUX_SMEM(1, FLUX_SIMPLE) UQ_FLUX_SMEM(2, FLUX_SIMPLE) UQ_FLUX_SMEM(3, FLUX_SIMPLE)
    UQ_FLUX_SMEM(4, FLUX_SIMPLE) UQ_FLUX_SMEM(5, FLUX_SIMPLE)
    UQ_FLUX_SMEM(1, FLUX_GENERAL) UQ_FLUX_SMEM(2, FLUX_GENERAL) UQ_FLUX_SMEM(3, FLUX_GENERAL)
    UQ_FLUX_SMEM(4, FLUX_GENERAL) UQ_FLUX_SMEM(5, FLUX_GENERAL)
    UQ_FLUX_SMEM(1, FLUX_WRAP) UQ_FLUX_SMEM(2, FLUX_WRAP) UQ_FLUX_SMEM(3, FLUX_WRAP)
    UQ_FLUX_SMEM(4, FLUX_WRAP) UQ_FLUX_SMEM(5, FLUX_WRAP)
#undef UQ_FLUX_SMEM
#undef UQ_FLUX_SMEM1
    return e;
}

size_t flux_smem_bytes(int prec, int tx, int ty) { return flux_smem_bytes_t(prec == 0 ? 8 : 4, tx, ty); }

template <class S>
cudaError_t launch_init(const KArgs<S> &a, const double *rho, const double *ux, const double *uy, const double *T,
                        cudaStream_t st)
{
    if (a.ntiles) k_init<S><<<a.ntiles, a.tx * a.ty, 0, st>>>(a, rho, ux, uy, T);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_macro_out_strided(const SampleParams *samples, int s, const S *state, double *out,
                                     long long stride, long long nodes, cudaStream_t st)
{
    const int blocks = (int)std::min<long long>((nodes + 255) / 256, 4096);
    k_macro_out<S><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(samples, s, state, out, stride);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_macro_out(const SampleParams *samples, int s, const S *state, double *out, long long nodes,
                             cudaStream_t st)
{
    return launch_macro_out_strided<S>(samples, s, state, out, nodes, nodes, st);
}

template <class S>
cudaError_t launch_dist_io(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, double *aos, int to_aos,
                           const uint8_t *nflags, const double *fref, long long nodes, cudaStream_t st)
{
    const int blocks = (int)std::min<long long>((nodes * NQ + 255) / 256, 8192);
    k_dist_io<S><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(samples, s, state, buf2, buf3, aos, to_aos, nflags, fref);
    return cudaGetLastError();
}

// Self-test of the bounded mbarrier wait the stencil kernels use: one block
// initialises a barrier that expects one arrival and waits on it with the
// same poll limit.  With arrive = 0 nothing arrives, the wait runs out and
// the block records STATUS_TIMEOUT and returns; with arrive = 1 thread 0
// arrives first and the wait succeeds.  No copy is ever in flight.
__global__ void k_wait_selftest(int *status, int arrive, uint32_t polls)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && arrive) mbar_arrive_expect_tx(&bar, 0);
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, polls);
    if (!ok && threadIdx.x == 0) atomicOr(status, STATUS_TIMEOUT);
}

cudaError_t launch_wait_selftest(int *status, int arrive, cudaStream_t st)
{
    k_wait_selftest<<<1, 32, 0, st>>>(status, arrive, TMA_WAIT_POLLS);
    return cudaGetLastError();
}

cudaError_t launch_residual(const SampleParams *samples, int nsamples, const double *partial, const int *tile_first,
                            const int *tile_count, double *residual, cudaStream_t st)
{
    k_residual<<<(nsamples + 127) / 128, 128, 0, st>>>(samples, nsamples, partial, tile_first, tile_count, residual);
    return cudaGetLastError();
}

template cudaError_t launch_phase<double, double>(const KArgs<double> &, int, int, const Tile *, int, const WallNode *,
                                                  int, cudaStream_t, int);
template cudaError_t launch_phase<float, float>(const KArgs<float> &, int, int, const Tile *, int, const WallNode *, int,
                                                cudaStream_t, int);
template cudaError_t prepare_kernels<double, double>();
template cudaError_t prepare_kernels<float, float>();
template cudaError_t launch_init<double>(const KArgs<double> &, const double *, const double *, const double *,
                                         const double *, cudaStream_t);
template cudaError_t launch_init<float>(const KArgs<float> &, const double *, const double *, const double *,
                                        const double *, cudaStream_t);
template cudaError_t launch_macro_out_strided<double>(const SampleParams *, int, const double *, double *, long long,
                                                      long long, cudaStream_t);
template cudaError_t launch_macro_out_strided<float>(const SampleParams *, int, const float *, double *, long long,
                                                     long long, cudaStream_t);
template cudaError_t launch_macro_out<double>(const SampleParams *, int, const double *, double *, long long, cudaStream_t);
template cudaError_t launch_macro_out<float>(const SampleParams *, int, const float *, double *, long long, cudaStream_t);
template cudaError_t launch_dist_io<double>(const SampleParams *, int, double *, double *, double *, double *, int,
                                            const uint8_t *, const double *, long long, cudaStream_t);
template cudaError_t launch_dist_io<float>(const SampleParams *, int, float *, float *, float *, double *, int,
                                           const uint8_t *, const double *, long long, cudaStream_t);

}  // namespace uqlbm
