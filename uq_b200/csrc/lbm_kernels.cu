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

#include <cuda_runtime.h>

#include <algorithm>

namespace uqlbm {

template <class S>
__device__ __forceinline__ S *plane_ptr(S *base, const SampleParams &sp, int p)
{
    return base + sp.state_off + (long long)p * sp.plane;
}

// ------------------------------------------------------------------- init
// initialiseFunctions (cpuLBM.cpp:846-875): f, h = equilibrium of each
// node's property; solid and permanent nodes also seed stage buffers 2/3,
// whose contents never change for them.
template <class S>
__global__ void k_init(KArgs<S> a, const double *__restrict__ rho, const double *__restrict__ ux,
                       const double *__restrict__ uy, const double *__restrict__ T)
{
    const Tile t = a.tiles[blockIdx.x];
    const SampleParams sp = a.samples[t.sample];
    const int x = t.x0 + threadIdx.x % a.tx, y = t.y0 + threadIdx.x / a.tx;
    if (x >= sp.nx || y >= sp.ny) return;
    const long long node = sp.node_off + (long long)y * sp.pitch + x;
    EqState<double> q = eq_state<double>(rho[node], ux[node], uy[node], T[node], sp);
    double f[NQ], h[NQ];
    eq_all(q, f, h);
    double sf = 0;
    for (int i = 0; i < NQ; ++i) sf += f[i];
    if (fabs(sf - rho[node]) > 1e-6) atomicOr(&a.status[t.sample], STATUS_EQ);
    const bool fixed = (a.nflags[node] & NF_TYPE) != 0;
    const long long o = (long long)y * sp.pitch + x;
    for (int i = 0; i < NQ; ++i) {
        plane_ptr(a.state, sp, i)[o] = (S)f[i];
        plane_ptr(a.state, sp, NQ + i)[o] = (S)h[i];
        if (fixed) {
            plane_ptr(a.buf2, sp, i)[o] = (S)f[i];
            plane_ptr(a.buf2, sp, NQ + i)[o] = (S)h[i];
            plane_ptr(a.buf3, sp, i)[o] = (S)f[i];
            plane_ptr(a.buf3, sp, NQ + i)[o] = (S)h[i];
        }
    }
}

// ------------------------------------------------------------------ moments
template <class S>
__device__ __forceinline__ Macro node_macro(const S *__restrict__ st, const SampleParams &sp, long long o)
{
    double r = 0, rux = 0, ruy = 0, sh = 0;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double fv = (double)st[(long long)i * sp.plane + o];
        r += fv;
        rux += fv * (sp.c * c_EX[i]);
        ruy += fv * (sp.c * c_EY[i]);
        sh += (double)st[(long long)(NQ + i) * sp.plane + o];
    }
    return macro_from_sums(r, rux, ruy, sh, sp);
}

// ------------------------------------------------------------------- P0
template <class S, class C>
__global__ void __launch_bounds__(256) k_stage0(KArgs<S> a)
{
    const Tile t = a.tiles[blockIdx.x];
    const SampleParams sp = a.samples[t.sample];
    const int x = t.x0 + threadIdx.x % a.tx, y = t.y0 + threadIdx.x / a.tx;
    if (x >= sp.nx || y >= sp.ny) return;
    const long long o = (long long)y * sp.pitch + x;
    const long long node = sp.node_off + o;
    const int type = a.nflags[node] & NF_TYPE;
    const S *st = a.state + sp.state_off;
    S *b2 = a.buf2 + sp.state_off;
    if (sp.rk >= 2) {  // EULER, EULER_EQ: fluxes of the state itself
        if (type == 0)
            for (int p = 0; p < NPL; ++p) b2[(long long)p * sp.plane + o] = st[(long long)p * sp.plane + o];
        if (a.want_residual && type == 0) a.told[node] = node_macro(st, sp, o).T;
        return;
    }
    if (type != 0) return;
    const Macro m = node_macro(st, sp, o);
    if (a.want_residual) a.told[node] = m.T;
    const EqState<C> q = eq_state<C>(m.rho, m.ux, m.uy, m.T, sp);
    C fe[NQ], he[NQ];
    eq_all(q, fe, he);
    {
        double sf = 0;
#pragma unroll
        for (int i = 0; i < NQ; ++i) sf += (double)fe[i];
        if (fabs(sf - m.rho) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(m.rho))))
            atomicOr(&a.status[t.sample], STATUS_EQ);
    }
    const C dt = (C)sp.dt, ux = (C)m.ux, uy = (C)m.uy;
    const C tf = (C)m.tf, th = (C)m.th, thf = (C)m.thf;
    if (sp.rk == 1) {
        // RK3 stages 1 and 2 (cpuLBM.cpp:1819-1924); stage 2 reuses stage 1's
        // equilibrium, moments and relaxation times.
        const C cf = dt / (C(2) * tf), ch = dt / (C(2) * th), chf = dt / (C(2) * thf);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            const C f = (C)st[(long long)i * sp.plane + o], h = (C)st[(long long)(NQ + i) * sp.plane + o];
            const C eu = (C)(sp.c * c_EX[i]) * ux + (C)(sp.c * c_EY[i]) * uy;
            const C f1 = (f + cf * fe[i]) / (C(1) + cf);
            const C h1 = (h - chf * eu * (fe[i] - f1) + ch * he[i]) / (C(1) + ch);
            const C f2 = (f - cf * (fe[i] - f1) + cf * fe[i]) / (C(1) + cf);
            const C h2 = (h - (dt / C(2)) * ((eu / thf) * (fe[i] - f2) - (eu / thf) * (fe[i] - f1)) - ch * (he[i] - h1) + ch * he[i])
                         / (C(1) + ch);
            b2[(long long)i * sp.plane + o] = (S)f2;
            b2[(long long)(NQ + i) * sp.plane + o] = (S)h2;
        }
    } else {
        // RK1 stage 1 (cpuLBM.cpp:1619-1663)
        const C cf = dt / tf, ch = dt / th;
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            const C f = (C)st[(long long)i * sp.plane + o], h = (C)st[(long long)(NQ + i) * sp.plane + o];
            const C eu = (C)(sp.c * c_EX[i]) * ux + (C)(sp.c * c_EY[i]) * uy;
            const C f1 = (f + cf * fe[i]) / (C(1) + cf);
            const C h1 = (h - dt * eu * ((fe[i] - f1) / thf) + ch * he[i]) / (C(1) + ch);
            b2[(long long)i * sp.plane + o] = (S)f1;
            b2[(long long)(NQ + i) * sp.plane + o] = (S)h1;
        }
    }
}

// -------------------------------------------------------------------- W
// wallFluxes (cpuLBM.cpp:1502-1590): for a solid node next to fluid,
// alpha = (f flux of the fluid 4-neighbours into it) / (|e| f out of it),
// weighted by the solid cell's 1/dx, 1/dy.
__constant__ int c_WXX[4] = {-1, 1, 0, 0};
__constant__ int c_WYY[4] = {0, 0, -1, 1};
__constant__ int c_WII[4][4] = {{1, 5, 8, 9}, {3, 6, 7, 11}, {2, 5, 6, 10}, {4, 7, 8, 12}};
__constant__ int c_WINV[4][4] = {{3, 6, 7, 11}, {1, 5, 8, 9}, {4, 8, 7, 12}, {2, 6, 5, 10}};

template <class S, class C>
__global__ void k_wall(KArgs<S> a, const S *__restrict__ stage, const WallNode *__restrict__ walls, int nwalls)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nwalls) return;
    const WallNode w = walls[k];
    const SampleParams sp = a.samples[w.sample];
    const StageView<S> v{stage + sp.state_off, a.nflags + sp.node_off, sp.plane, sp.pitch};
    const double dxm = a.dxv[sp.xoff + w.x], dym = a.dyv[sp.yoff + w.y];
    double fin = 0, fout = 0;
    for (int j = 0; j < 4; ++j) {
        int m;
        const int xm = bc_index(sp, w.x, c_WXX[j], 0, m);
        const int ym = bc_index(sp, w.y, c_WYY[j], 1, m);
        const uint8_t fl = v.nf[(long long)ym * sp.pitch + xm];
        if ((fl & NF_TYPE) >= 2) continue;
        const int axis = j < 2 ? 0 : 1;
        const double dd = axis == 0 ? dxm : dym;
        for (int q = 0; q < 4; ++q) {
            const int i = c_WII[j][q], io = c_WINV[j][q];
            const double F = (double)flux_axis<S, C>(sp, v, xm, ym, i, axis, fl);
            fin += F / dd;
            const double fo = (double)ldv(v, io, w.x, w.y);
            fout += fo * (sp.c * abs(axis == 0 ? c_EX[io] : c_EY[io])) / dd;
        }
    }
    a.template alpha_as<C>()[sp.node_off + (long long)w.y * sp.pitch + w.x] = (C)(fin / fout);
}

// ------------------------------------------------------------------ P1/P2
// flux of plane p at a node, solid nodes answering alpha |e| f_stage
// (wallFluxes' outgoing flux, cpuLBM.cpp:1576-1586)
template <class S, class C>
__device__ __forceinline__ C node_flux(const KArgs<S> &a, const SampleParams &sp, const StageView<S> &v, int x, int y,
                                       int p, int axis)
{
    const long long o = (long long)y * sp.pitch + x;
    const uint8_t fl = v.nf[o];
    if ((fl & NF_TYPE) == 2) {
        const int i = p < NQ ? p : p - NQ;
        const C al = a.template alpha_as<C>()[sp.node_off + o];
        return al * (C)(sp.c * abs(axis == 0 ? c_EX[i] : c_EY[i])) * (C)ldv(v, p, x, y);
    }
    return flux_axis<S, C>(sp, v, x, y, p, axis, fl);
}

template <class S, class C, int PH>
__global__ void __launch_bounds__(256) k_flux(KArgs<S> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TX = a.tx, TY = a.ty, NT = TX * TY;
    C *sfx = reinterpret_cast<C *>(smem_raw);  // [2][NT]
    C *sfy = sfx + 2 * NT;                      // [2][NT]
    C *ringx = sfy + 2 * NT;                    // [26][TY]
    C *ringy = ringx + NPL * TY;                // [26][TX]
    C *sD = ringy + NPL * TX;                   // [26][NT]
    __shared__ double red[32];

    const Tile t = a.tiles[blockIdx.x];
    const SampleParams sp = a.samples[t.sample];
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x = t.x0 + tx, y = t.y0 + ty;
    const int x_end = min(t.x0 + TX, sp.nx), y_end = min(t.y0 + TY, sp.ny);
    const bool active = x < sp.nx && y < sp.ny;
    const S *stage = PH == 1 ? a.buf2 : a.buf3;
    const StageView<S> v{stage + sp.state_off, a.nflags + sp.node_off, sp.plane, sp.pitch};
    const long long o = (long long)y * sp.pitch + x;
    const uint8_t myflag = active ? v.nf[o] : 0;
    const int type = myflag & NF_TYPE;

    // upwind fluxes across the tile edges, for all planes (cFLUX's
    // index(x, -e) neighbour with its reflected direction, cpuLBM.cpp:1436-1470)
    for (int r = tid; r < NPL * (TX + TY); r += NT) {
        const int p = r / (TX + TY), k = r % (TX + TY);
        const int i = p < NQ ? p : p - NQ, pb = p - i;
        C val = C(0);
        if (k < TY) {
            const int yy = t.y0 + k, e = isgn(c_EX[i]);
            if (yy < y_end && e != 0) {
                int m;
                const int xn = e > 0 ? t.x0 : x_end - 1;
                const int xr = bc_index(sp, xn, -e, 0, m);
                val = node_flux<S, C>(a, sp, v, xr, yy, m ? pb + c_MIR_EW[i] : p, 0);
            }
            ringx[p * TY + k] = val;
        } else {
            const int xx = t.x0 + (k - TY), e = isgn(c_EY[i]);
            if (xx < x_end && e != 0) {
                int m;
                const int yn = e > 0 ? t.y0 : y_end - 1;
                const int yr = bc_index(sp, yn, -e, 1, m);
                val = node_flux<S, C>(a, sp, v, xx, yr, m ? pb + c_MIR_NS[i] : p, 1);
            }
            ringy[p * TX + (k - TY)] = val;
        }
    }

    const C tdx = active ? (C)a.tdx[sp.xoff + x] : C(0);
    const C tdy = active ? (C)a.tdy[sp.yoff + y] : C(0);
    for (int p = 0; p < NPL; ++p) {
        const int buf = p & 1;
        const int i = p < NQ ? p : p - NQ;
        if (active) {
            C Fx, Fy;
            if (type == 2) {
                const C al = a.template alpha_as<C>()[sp.node_off + o];
                const C sv = (C)ldv(v, p, x, y);
                Fx = al * (C)(sp.c * abs(c_EX[i])) * sv;
                Fy = al * (C)(sp.c * abs(c_EY[i])) * sv;
            } else {
                Fx = flux_axis<S, C>(sp, v, x, y, p, 0, myflag);
                Fy = flux_axis<S, C>(sp, v, x, y, p, 1, myflag);
            }
            sfx[buf * NT + tid] = Fx;
            sfy[buf * NT + tid] = Fy;
        }
        __syncthreads();
        if (active && type == 0) {
            const int ex = isgn(c_EX[i]), ey = isgn(c_EY[i]);
            const int xu = x - ex, yu = y - ey;
            const C Fx_in = (xu >= t.x0 && xu < x_end) ? sfx[buf * NT + ty * TX + (xu - t.x0)] : ringx[p * TY + ty];
            const C Fy_in = (yu >= t.y0 && yu < y_end) ? sfy[buf * NT + (yu - t.y0) * TX + tx] : ringy[p * TX + tx];
            const C out = tdx * sfx[buf * NT + tid] + tdy * sfy[buf * NT + tid];
            const C in = tdx * Fx_in + tdy * Fy_in;
            sD[p * NT + tid] = out - in;
        }
    }

    double res_part = 0;
    if (active && type == 0) {
        S *st = a.state + sp.state_off;
        const S *b2 = a.buf2 + sp.state_off;
        S *b3 = a.buf3 + sp.state_off;
        const C dt = (C)sp.dt;
        bool final_phase = true;
        if (PH == 1 && sp.rk == 1) {
            // RK3 stage 3 (cpuLBM.cpp:1928-1993) and the part of the update
            // (cpuLBM.cpp:1999-2042) that does not need the stage-3 fluxes
            final_phase = false;
            const Macro m1 = node_macro(st, sp, o);
            double r = 0, rux = 0, ruy = 0, sh = 0;
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const double fv = (double)st[(long long)i * sp.plane + o];
                const double Df = (double)sD[i * NT + tid];
                r += fv - Df;
                rux += fv * (sp.c * c_EX[i]) - Df * (sp.c * c_EX[i]);
                ruy += fv * (sp.c * c_EY[i]) - Df * (sp.c * c_EY[i]);
                sh += (double)st[(long long)(NQ + i) * sp.plane + o] - (double)sD[(NQ + i) * NT + tid];
            }
            const Macro m3 = macro_from_sums(r, rux, ruy, sh, sp);
            const EqState<C> q1 = eq_state<C>(m1.rho, m1.ux, m1.uy, m1.T, sp);
            const EqState<C> q3 = eq_state<C>(m3.rho, m3.ux, m3.uy, m3.T, sp);
            const C tf2 = (C)m1.tf, th2 = (C)m1.th, thf2 = (C)m1.thf;
            const C tf3 = (C)m3.tf, th3 = (C)m3.th, thf3 = (C)m3.thf;
            const C a2 = dt / (C(2) * tf2), a3 = dt / (C(2) * tf3), b2c = dt / (C(2) * th2), b3c = dt / (C(2) * th3);
            const C ux1 = (C)m1.ux, uy1 = (C)m1.uy, ux3 = (C)m3.ux, uy3 = (C)m3.uy;
            double sf3 = 0;
            for (int fam = 0; fam < 4; ++fam) {
                C e1f[4], e1h[4], e3f[4], e3h[4];
                int i0, n;
                if (fam == 0) { eq_fam0(q1, e1f[0], e1h[0]); eq_fam0(q3, e3f[0], e3h[0]); i0 = 0; n = 1; }
                else if (fam == 1) { eq_fam1(q1, e1f, e1h); eq_fam1(q3, e3f, e3h); i0 = 1; n = 4; }
                else if (fam == 2) { eq_fam5(q1, e1f, e1h); eq_fam5(q3, e3f, e3h); i0 = 5; n = 4; }
                else { eq_fam9(q1, e1f, e1h); eq_fam9(q3, e3f, e3h); i0 = 9; n = 4; }
                for (int k = 0; k < n; ++k) {
                    const int i = i0 + k;
                    sf3 += (double)e3f[k];
                    const long long of = (long long)i * sp.plane + o, oh = (long long)(NQ + i) * sp.plane + o;
                    const C f = (C)st[of], h = (C)st[oh], f2 = (C)b2[of], h2 = (C)b2[oh];
                    const C Df = sD[i * NT + tid], Dh = sD[(NQ + i) * NT + tid];
                    const C exi = (C)(sp.c * c_EX[i]), eyi = (C)(sp.c * c_EY[i]);
                    const C eu2 = exi * ux1 + eyi * uy1, eu3 = exi * ux3 + eyi * uy3;
                    const C f3 = (f - Df + a2 * (e1f[k] - f2) + a3 * e3f[k]) / (C(1) + a3);
                    const C h3 = (h - Dh - (dt / C(2)) * ((eu2 / thf2) * (e1f[k] - f2) + (eu3 / thf3) * (e3f[k] - f3))
                                  + b2c * (e1h[k] - h2) + b3c * e3h[k]) / (C(1) + b3c);
                    const C accf = f - C(0.5) * Df + (dt / C(2)) * ((e1f[k] - f2) / tf2 + (e3f[k] - f3) / tf3);
                    const C acch = h - C(0.5) * Dh + (dt / C(2)) * ((e1h[k] - h2) / th2 + (e3h[k] - h3) / th3)
                                   - (dt / C(2)) * ((eu2 / thf2) * (e1f[k] - f2) + (eu3 / thf3) * (e3f[k] - f3));
                    b3[of] = (S)f3;
                    b3[oh] = (S)h3;
                    st[of] = (S)accf;
                    st[oh] = (S)acch;
                }
            }
            if (fabs(sf3 - m3.rho) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(m3.rho))))
                atomicOr(&a.status[t.sample], STATUS_EQ);
        } else if (PH == 2) {
            // final RK3 combination (cpuLBM.cpp:1999-2042): f = acc - D3/2
            for (int p = 0; p < NPL; ++p) {
                const long long op = (long long)p * sp.plane + o;
                st[op] = (S)((C)st[op] - C(0.5) * sD[p * NT + tid]);
            }
        } else {
            // RK1 update (cpuLBM.cpp:1674-1710), EULER (:2130-2168), EULER_EQ (:2220-2258)
            const Macro m = node_macro(st, sp, o);
            const EqState<C> q = eq_state<C>(m.rho, m.ux, m.uy, m.T, sp);
            C fe[NQ], he[NQ];
            eq_all(q, fe, he);
            if (sp.rk >= 2) {
                double sf = 0;
#pragma unroll
                for (int i = 0; i < NQ; ++i) sf += (double)fe[i];
                if (fabs(sf - m.rho) > a.eq_tol * (sizeof(C) == 8 ? 1.0 : fmax(1.0, fabs(m.rho))))
                    atomicOr(&a.status[t.sample], STATUS_EQ);
            }
            const C tf = (C)m.tf, th = (C)m.th, thf = (C)m.thf, ux = (C)m.ux, uy = (C)m.uy;
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const long long of = (long long)i * sp.plane + o, oh = (long long)(NQ + i) * sp.plane + o;
                const C f = (C)st[of], h = (C)st[oh];
                const C Df = sD[i * NT + tid], Dh = sD[(NQ + i) * NT + tid];
                const C eu = (C)(sp.c * c_EX[i]) * ux + (C)(sp.c * c_EY[i]) * uy;
                C fn, hn;
                if (sp.rk == 0) {
                    const C f1 = (C)b2[of], h1 = (C)b2[oh];
                    fn = f - Df + (dt / tf) * (fe[i] - f1);
                    hn = h - Dh + (dt / th) * (he[i] - h1) - ((dt * eu) / thf) * (fe[i] - f1);
                } else if (sp.rk == 2) {
                    fn = f - Df + (dt / tf) * (fe[i] - f);
                    hn = h - Dh + (dt / th) * (he[i] - h) - ((dt * eu) / thf) * (fe[i] - f);
                } else {
                    fn = fe[i] - Df;
                    hn = he[i] - Dh;
                }
                st[of] = (S)fn;
                st[oh] = (S)hn;
            }
        }
        if (final_phase) {
            // macroPropShort of the new state: the residual's T and a
            // finiteness / positive-density check
            const Macro mn = node_macro(st, sp, o);
            if (!(mn.rho > 0.0) || !isfinite(mn.rho) || !isfinite(mn.T) || !isfinite(mn.ux) || !isfinite(mn.uy))
                atomicOr(&a.status[t.sample], STATUS_NONFINITE);
            if (a.want_residual) {
                const double d = mn.T - a.told[sp.node_off + o];
                res_part = d * d;
            }
        }
    }
    if (a.want_residual && ((PH == 2) || (PH == 1 && sp.rk != 1))) {
        // per-tile partial sum, fixed order (deterministic)
        for (int off = 16; off > 0; off >>= 1) res_part += __shfl_down_sync(0xffffffffu, res_part, off);
        if ((tid & 31) == 0) red[tid >> 5] = res_part;
        __syncthreads();
        if (tid == 0) {
            double s = 0;
            for (int w = 0; w < (NT + 31) / 32; ++w) s += red[w];
            a.partial[t.gid] = s;
        }
    }
}

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
// [x*Ny + y] order.
template <class S>
__global__ void k_macro_out(const SampleParams *samples, int s, const S *state, double *out)
{
    const SampleParams sp = samples[s];
    const long long n = (long long)sp.nx * sp.ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k % sp.ny), x = (int)(k / sp.ny);
        const Macro m = node_macro(state + sp.state_off, sp, (long long)y * sp.pitch + x);
        out[k] = m.rho;
        out[n + k] = m.ux;
        out[2 * n + k] = m.uy;
        out[3 * n + k] = m.T;
        out[4 * n + k] = m.p;
    }
}

// planes <-> reference AoS [(x*Ny + y)*13 + i] in FP64
template <class S>
__global__ void k_dist_io(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, double *aos, int to_aos,
                          const uint8_t *nflags)
{
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
            aos[k] = (double)*f;
            aos[n + k] = (double)*h;
        } else {
            *f = (S)aos[k];
            *h = (S)aos[n + k];
            if (nflags[sp.node_off + o] & NF_TYPE) {  // fixed nodes seed the stage buffers
                const long long of = sp.state_off + (long long)i * sp.plane + o;
                const long long oh = sp.state_off + (long long)(NQ + i) * sp.plane + o;
                buf2[of] = *f; buf3[of] = *f;
                buf2[oh] = *h; buf3[oh] = *h;
            }
        }
    }
}

// ----------------------------------------------------------------- launchers
template <class S, class C>
cudaError_t launch_phase(const KArgs<S> &a, int phase, const Tile *tiles, int ntiles, const WallNode *walls,
                         int nwalls, cudaStream_t st)
{
    KArgs<S> k = a;
    k.tiles = tiles;
    k.ntiles = ntiles;
    const int NT = a.tx * a.ty;
    if (phase == 0) {
        if (ntiles) k_stage0<S, C><<<ntiles, NT, 0, st>>>(k);
    } else if (phase == 1 || phase == 2) {
        const size_t sm = sizeof(C) * ((size_t)4 * NT + (size_t)NPL * (a.tx + a.ty) + (size_t)NPL * NT);
        if (ntiles) {
            if (phase == 1) k_flux<S, C, 1><<<ntiles, NT, sm, st>>>(k);
            else k_flux<S, C, 2><<<ntiles, NT, sm, st>>>(k);
        }
    } else if (phase == 3 || phase == 4) {  // walls of buffer 2 / buffer 3
        if (nwalls) k_wall<S, C><<<(nwalls + 127) / 128, 128, 0, st>>>(k, phase == 3 ? a.buf2 : a.buf3, walls, nwalls);
    }
    return cudaGetLastError();
}

template <class S, class C>
cudaError_t prepare_kernels()
{
    const int maxsm = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_flux<S, C, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_flux<S, C, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
}

size_t flux_smem_bytes(int prec, int tx, int ty)
{
    const size_t NT = (size_t)tx * ty;
    return (prec == 0 ? 8 : 4) * (4 * NT + (size_t)NPL * (tx + ty) + (size_t)NPL * NT);
}

template <class S>
cudaError_t launch_init(const KArgs<S> &a, const double *rho, const double *ux, const double *uy, const double *T,
                        cudaStream_t st)
{
    if (a.ntiles) k_init<S><<<a.ntiles, a.tx * a.ty, 0, st>>>(a, rho, ux, uy, T);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_macro_out(const SampleParams *samples, int s, const S *state, double *out, long long nodes,
                             cudaStream_t st)
{
    const int blocks = (int)std::min<long long>((nodes + 255) / 256, 4096);
    k_macro_out<S><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(samples, s, state, out);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_dist_io(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, double *aos, int to_aos,
                           const uint8_t *nflags, long long nodes, cudaStream_t st)
{
    const int blocks = (int)std::min<long long>((nodes * NQ + 255) / 256, 8192);
    k_dist_io<S><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(samples, s, state, buf2, buf3, aos, to_aos, nflags);
    return cudaGetLastError();
}

cudaError_t launch_residual(const SampleParams *samples, int nsamples, const double *partial, const int *tile_first,
                            const int *tile_count, double *residual, cudaStream_t st)
{
    k_residual<<<(nsamples + 127) / 128, 128, 0, st>>>(samples, nsamples, partial, tile_first, tile_count, residual);
    return cudaGetLastError();
}

template cudaError_t launch_phase<double, double>(const KArgs<double> &, int, const Tile *, int, const WallNode *, int,
                                                  cudaStream_t);
template cudaError_t launch_phase<float, float>(const KArgs<float> &, int, const Tile *, int, const WallNode *, int,
                                                cudaStream_t);
template cudaError_t prepare_kernels<double, double>();
template cudaError_t prepare_kernels<float, float>();
template cudaError_t launch_init<double>(const KArgs<double> &, const double *, const double *, const double *,
                                         const double *, cudaStream_t);
template cudaError_t launch_init<float>(const KArgs<float> &, const double *, const double *, const double *,
                                        const double *, cudaStream_t);
template cudaError_t launch_macro_out<double>(const SampleParams *, int, const double *, double *, long long, cudaStream_t);
template cudaError_t launch_macro_out<float>(const SampleParams *, int, const float *, double *, long long, cudaStream_t);
template cudaError_t launch_dist_io<double>(const SampleParams *, int, double *, double *, double *, double *, int,
                                            const uint8_t *, long long, cudaStream_t);
template cudaError_t launch_dist_io<float>(const SampleParams *, int, float *, float *, float *, double *, int,
                                           const uint8_t *, long long, cudaStream_t);

}  // namespace uqlbm
