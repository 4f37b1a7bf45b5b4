/* FP64 CPU restatement of the reference D2Q13 thermal LBM solver.
 *
 * TEST INFRASTRUCTURE ONLY (the parity oracle); see lbm_oracle.h.
 * Every function cites the reference function it restates; paths are
 * relative to CODE/C++/VS2010/simLB/simLB/ unless they name CODE/Python.
 * Arithmetic is FP64 with no FMA contraction (-ffp-contract=off), the same
 * evaluation model as the reference's x86-64 build.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NQ 13

struct orc {
    int Nx, Ny;
    int rk, fm;
    int perX, perY, mirN, mirS, mirE, mirW;
    double R, b, K, Tc, mu, Pr, dt, tol;
    int mu_model;            /* 0 constant, 1 VHS, 2 Sutherland */
    double visc_exp, S_v, T_ref;
    double ex[NQ], ey[NQ];
    double *dx, *dy;           /* per column / per row cell widths */
    unsigned char *type;       /* [x*Ny+y] cell type */
    double *f, *h;             /* [(x*Ny+y)*13+i] */
    double *rho, *ux, *uy, *T, *p;
    int nsteps, step;
    double residual, resNorm, initRes[100];
    int hasFailed;
    /* stage scratch, allocated once */
    double *w[16];
    struct macro_s *Ma, *Mc;
};

/* lattice directions in units of c (setupVars, cpuLBM.cpp:376-388) */
static const int EX[NQ] = {0, 1, 0, -1, 0, 1, -1, -1, 1, 2, 0, -2, 0};
static const int EY[NQ] = {0, 0, 1, 0, -1, 1, 1, -1, -1, 0, 2, 0, -2};
/* direction maps for reflections (mirIndex, cpuLBM.cpp:1147-1169):
 * MIR_NS flips the y component, MIR_EW flips the x component. */
static const int MIR_NS[NQ] = {0, 1, 4, 3, 2, 8, 7, 6, 5, 9, 12, 11, 10};
static const int MIR_EW[NQ] = {0, 3, 2, 1, 4, 6, 5, 8, 7, 11, 10, 9, 12};

#define AT(x, y) ((size_t)(x) * s->Ny + (y))
#define AT3(x, y, i) (((size_t)(x) * s->Ny + (y)) * NQ + (i))

/* ---------------------------------------------------------------- equilibria
 * equilibrium2D (cpuLBM.cpp:785-844) with the polynomials of
 * inlineFunctions.cpp:10-61, written here as even/odd parts in the
 * normalised velocity so that the four symmetry-mapped calls per family
 * share one evaluation.  In normalised units (u, v, T) = (u/sqrt(R Tc),
 * v/sqrt(R Tc), T/Tc) with a = u^2, c = v^2 the families are:
 *   f0     = 1 + 5/2 T^2 + 5/2 T (a + c - 1) + (a^2 + c^2)/4 + a c - 5/4 (a + c)
 *   f1,f3  = E1(u,v) +- O1(u,v),  f2,f4 = E1(v,u) +- O1(v,u)
 *   f5..f8 = (T + a +- u)(T + c +- v)/4
 *   f9,f11 = E9(u) +- O9(u),      f10,f12 = E9(v) +- O9(v)
 * times rho; the h family likewise times rho R Tc.  The identities
 * sum f_i = rho and sum h_i = rho (|u|^2 + b R T)/2 hold exactly. */
static void eq_normalised(double rho, double u, double v, double T, double K,
                          double *eqf, double *eqh, double rRTc)
{
    const double a = u * u, c = v * v, s2 = a + c, pc = a * c, T2 = T * T, T3 = T2 * T;

    eqf[0] = rho * (1.0 + 2.5 * T2 + 2.5 * T * (s2 - 1.0) + 0.25 * (a * a + c * c) + pc - 1.25 * s2);
    {
        double E = -T2 + T * (2.0 / 3.0 - 1.5 * a - 0.5 * c) + (2.0 / 3.0) * a - a * a / 6.0 - 0.5 * pc;
        double O = u * (2.0 / 3.0 - T - a / 6.0 - 0.5 * c);
        eqf[1] = rho * (E + O);
        eqf[3] = rho * (E - O);
        E = -T2 + T * (2.0 / 3.0 - 1.5 * c - 0.5 * a) + (2.0 / 3.0) * c - c * c / 6.0 - 0.5 * pc;
        O = v * (2.0 / 3.0 - T - c / 6.0 - 0.5 * a);
        eqf[2] = rho * (E + O);
        eqf[4] = rho * (E - O);
    }
    {
        double Ap = T + a + u, Am = T + a - u, Bp = T + c + v, Bm = T + c - v, r4 = 0.25 * rho;
        eqf[5] = r4 * (Ap * Bp);
        eqf[6] = r4 * (Am * Bp);
        eqf[7] = r4 * (Am * Bm);
        eqf[8] = r4 * (Ap * Bm);
    }
    {
        double E = 0.125 * T2 + T * (0.25 * a - 1.0 / 24.0) + (a * a - a) / 24.0;
        double O = u * (0.25 * T + (a - 1.0) / 12.0);
        eqf[9] = rho * (E + O);
        eqf[11] = rho * (E - O);
        E = 0.125 * T2 + T * (0.25 * c - 1.0 / 24.0) + (c * c - c) / 24.0;
        O = v * (0.25 * T + (c - 1.0) / 12.0);
        eqf[10] = rho * (E + O);
        eqf[12] = rho * (E - O);
    }

    /* h0 */
    eqh[0] = rRTc * (T3 * (1.25 * K + 20.0 / 3.0)
                     + T2 * ((1.25 * K + 11.25) * s2 - 1.25 * K - 5.0)
                     + T * (0.125 * K * (s2 * s2 + 2.0 * pc) - 0.625 * K * s2 + 0.5 * K
                            + 2.5 * s2 * s2 + 2.5 * pc - 5.0 * s2 + 1.0)
                     + s2 * s2 * s2 / 8.0 + 0.25 * pc * s2 - 0.625 * s2 * s2 + 0.5 * s2);
    /* h1..h4: even/odd parts of the x-type family, then swapped for y */
    {
        double A = a, C = c, U = u;
        for (int k = 0; k < 2; ++k) {
            double E = T3 * (-0.5 * K - 8.0 / 3.0)
                       + T2 * (-(0.75 * K + 6.5) * A - (0.25 * K + 2.5) * C + K / 3.0 + 4.0 / 3.0)
                       + T * (-(K / 12.0 + 19.0 / 12.0) * A * A - (0.25 * K + 3.5) * A * C
                              + (K / 3.0 + 7.0 / 3.0) * A - 0.25 * C * C + C / 3.0)
                       - A * A * A / 12.0 - A * A * C / 3.0 + A * A / 3.0 - 0.25 * A * C * C + A * C / 3.0;
            double O = U * (T2 * (-0.5 * K - 3.0)
                            + T * (-(K / 12.0 + 7.0 / 6.0) * A - (0.25 * K + 2.5) * C + K / 3.0 + 4.0 / 3.0)
                            - A * A / 12.0 - A * C / 3.0 + A / 3.0 - 0.25 * C * C + C / 3.0);
            eqh[1 + k] = rRTc * (E + O);
            eqh[3 + k] = rRTc * (E - O);
            A = c; C = a; U = v;
        }
    }
    /* h5..h8: parts even/odd in u and in v */
    {
        double EE = T3 * (0.125 * K + 2.0 / 3.0) + T2 * (0.125 * K + 1.125) * s2
                    + T * ((0.125 * K + 1.5) * pc + 0.125 * (a * a + c * c)) + 0.125 * pc * s2;
        double OE = u * (T2 * (0.125 * K + 0.75) + T * ((0.125 * K + 1.125) * c + 0.125 * a) + 0.125 * c * s2);
        double EO = v * (T2 * (0.125 * K + 0.75) + T * ((0.125 * K + 1.125) * a + 0.125 * c) + 0.125 * a * s2);
        double OO = u * v * (T * (0.125 * K + 0.75) + 0.125 * s2);
        eqh[5] = rRTc * (EE + OE + EO + OO);
        eqh[6] = rRTc * (EE - OE + EO - OO);
        eqh[7] = rRTc * (EE - OE - EO + OO);
        eqh[8] = rRTc * (EE + OE - EO - OO);
    }
    /* h9..h12 */
    {
        double A = a, C = c, U = u;
        for (int k = 0; k < 2; ++k) {
            double E = T3 * (K / 16.0 + 1.0 / 3.0)
                       + T2 * ((0.125 * K + 17.0 / 16.0) * A + C / 16.0 - K / 48.0 - 1.0 / 12.0)
                       + T * ((K / 48.0 + 1.0 / 3.0) * A * A - (K / 48.0 + 7.0 / 48.0) * A + 0.125 * A * C - C / 48.0)
                       + (A * A * A + A * A * C - A * A - A * C) / 48.0;
            double O = U * (T2 * (0.125 * K + 0.75) + T * ((K / 24.0 + 11.0 / 24.0) * A - K / 24.0 - 1.0 / 6.0 + 0.125 * C)
                            + (A * A + A * C - A - C) / 24.0);
            eqh[9 + k] = rRTc * (E + O);
            eqh[11 + k] = rRTc * (E - O);
            A = c; C = a; U = v;
        }
    }
}

void orc_equilibrium(double rho, double ux, double uy, double T, double R, double Tc, double K,
                     double *eqf, double *eqh)
{
    double sRTc = sqrt(R * Tc);
    eq_normalised(rho, ux / sRTc, uy / sRTc, T / Tc, K, eqf, eqh, rho * R * Tc);
}

/* equilibrium2D including its mass check (cpuLBM.cpp:825-843) */
static void equilibrium(orc *s, double rho, double ux, double uy, double T, double *eqf, double *eqh)
{
    orc_equilibrium(rho, ux, uy, T, s->R, s->Tc, s->K, eqf, eqh);
    double sum_f = 0;
    for (int i = 0; i < NQ; ++i) sum_f += eqf[i];
    if (fabs(sum_f - rho) > 1e-6) s->hasFailed = 1;
}

/* ------------------------------------------------------------------ moments
 * macroPropShort / macroProp / macroProp3 (cpuLBM.cpp:877-1032): rho, u, T, p
 * of a node from 13 f and 13 h values; optionally tau_f = mu/p,
 * tau_h = tau_f/Pr, tau_hf = tau_h tau_f/(tau_f - tau_h). */
typedef struct macro_s { double rho, ux, uy, T, p, tf, th, thf; } macro_t;

/* dynamic viscosity at temperature T: constant (cpuLBM.cpp:952), VHS or
 * Sutherland (CODE/Python/simLB/codeCL.py:986-990) */
static double viscosity(const orc *s, double T)
{
    if (s->mu_model == 0) return s->mu;
    double mu = s->mu * pow(T / s->T_ref, s->visc_exp);
    if (s->mu_model == 2) mu *= (s->T_ref + s->S_v) / (T + s->S_v);
    return mu;
}

static macro_t moments(const orc *s, const double *fv, const double *hv)
{
    macro_t m;
    double r = 0, rux = 0, ruy = 0, sh = 0;
    for (int i = 0; i < NQ; ++i) {
        r += fv[i];
        rux += fv[i] * s->ex[i];
        ruy += fv[i] * s->ey[i];
        sh += hv[i];
    }
    m.rho = r;
    m.ux = rux / r;
    m.uy = ruy / r;
    double ax = fabs(m.ux), ay = fabs(m.uy);
    double usq = ax * ax + ay * ay;
    m.T = 2.0 * (sh / r - usq / 2.0) / (s->b * s->R);
    m.p = r * s->R * m.T;
    m.tf = viscosity(s, m.T) / m.p;
    m.th = m.tf / s->Pr;
    m.thf = (m.th * m.tf) / (m.tf - m.th);
    return m;
}

static void store_macro(orc *s, int x, int y, const macro_t *m)
{
    size_t k = AT(x, y);
    s->rho[k] = m->rho;
    s->ux[k] = m->ux;
    s->uy[k] = m->uy;
    s->T[k] = m->T;
    s->p[k] = m->p;
}

static void macro_short(orc *s, int x, int y)
{
    macro_t m = moments(s, &s->f[AT3(x, y, 0)], &s->h[AT3(x, y, 0)]);
    store_macro(s, x, y, &m);
}

/* ------------------------------------------------------ boundary index maps
 * index (cpuLBM.cpp:1033-1113): periodic wrap, mirror (i -> -i-1 / 2N-i-1,
 * flagging a reflection) or zeroth-order extrapolation (clamp). */
static int bc_index(const orc *s, int i, int pm, int d, int *mir)
{
    i += pm;
    *mir = 0;
    int N = d == 0 ? s->Nx : s->Ny;
    int per = d == 0 ? s->perX : s->perY;
    int mlo = d == 0 ? s->mirW : s->mirS;
    int mhi = d == 0 ? s->mirE : s->mirN;
    if (i < 0) {
        if (per > 0) i = N + i;
        else if (mlo > 0) { i = -i - 1; *mir = 1; }
        else i = 0;
    } else if (i > N - 1) {
        if (per > 0) i = i - N;
        else if (mhi > 0) { i = 2 * N - i - 1; *mir = 1; }
        else i = N - 1;
    }
    return i;
}

static int sgn(double a) { return a > 0 ? 1 : (a < 0 ? -1 : 0); }

/* minmod (cpuLBM.cpp:1130-1145), including its case order */
static double minmod(double a, double b)
{
    double out = 0;
    if (fabs(a) < fabs(b) && a * b > 0) out = a;
    else if (fabs(b) < fabs(a) && a * b > 0) out = b;
    else if (a == b) out = a;
    else if (a * b <= 0) out = 0;
    return out;
}

/* stencil (cpuLBM.cpp:1171-1326): L points along x and along y through
 * (x, y), ordered upwind for direction i; a stencil that meets solid nodes
 * has its first solid/fluid edge point replaced by the linear extrapolation
 * 2 f(m1) - f(m2) from the two nearest fluid nodes, and the point beyond it
 * (if inside the stencil) by the same value. */
static void stencil(const orc *s, const double *f, int x, int y, int i, int L, double *Sx, double *Sy)
{
    if (i == 0) return;
    int ex = EX[i] > 0 ? 1 : (EX[i] < 0 ? -1 : 0);
    int ey = EY[i] > 0 ? 1 : (EY[i] < 0 ? -1 : 0);
    int low = (L - 1) / 2;
    int jx1 = x - ex * low, jy1 = y - ey * low;
    int sx[5], sy[5], any_x = 0, any_y = 0;
    for (int j = 0; j < L; ++j) {
        int m_ew, m_ns;
        int jx = bc_index(s, jx1, ex * j, 0, &m_ew);
        int jy = bc_index(s, jy1, ey * j, 1, &m_ns);
        int i_ns = m_ns ? MIR_NS[i] : i;
        int i_ew = m_ew ? MIR_EW[i] : i;
        Sx[j] = f[AT3(jx, y, i_ew)];
        sx[j] = s->type[AT(jx, y)] == 2;
        any_x |= sx[j];
        Sy[j] = f[AT3(x, jy, i_ns)];
        sy[j] = s->type[AT(x, jy)] == 2;
        any_y |= sy[j];
    }
    if (any_x) {
        int diff = 0, jj = 0, xe = 0, m;
        for (int j = 0; j < L - 1; ++j) {
            diff = sx[j] - sx[j + 1];
            if (diff > 0) { jj = j; xe = bc_index(s, jx1, ex * j, 0, &m); break; }
            if (diff < 0) { jj = j + 1; xe = bc_index(s, jx1, ex * (j + 1), 0, &m); break; }
        }
        int x1 = bc_index(s, xe, ex * diff, 0, &m);
        int x2 = bc_index(s, xe, ex * 2 * diff, 0, &m);
        Sx[jj] = 2 * f[AT3(x1, y, i)] - f[AT3(x2, y, i)];
        int jn = jj - diff;
        if (jn >= 0 && jn < L) Sx[jn] = Sx[jj];
    }
    if (any_y) {
        int diff = 0, jj = 0, ye = 0, m;
        for (int j = 0; j < L - 1; ++j) {
            diff = sy[j] - sy[j + 1];
            if (diff > 0) { jj = j; ye = bc_index(s, jy1, ey * j, 1, &m); break; }
            if (diff < 0) { jj = j + 1; ye = bc_index(s, jy1, ey * (j + 1), 1, &m); break; }
        }
        int y1 = bc_index(s, ye, ey * diff, 1, &m);
        int y2 = bc_index(s, ye, ey * 2 * diff, 1, &m);
        Sy[jj] = 2 * f[AT3(x, y1, i)] - f[AT3(x, y2, i)];
        int jn = jj - diff;
        if (jn >= 0 && jn < L) Sy[jn] = Sy[jj];
    }
}

/* NND (cpuLBM.cpp:1328-1356): |e| S1 + minmod(forward, backward)/2 */
static double nnd(double e, const double *S)
{
    double a = fabs(e);
    if (a == 0) return 0;
    double c = a * S[1], dp = a * S[2] - c, dm = c - a * S[0];
    return c + 0.5 * minmod(dp, dm);
}

/* WENO5 (cpuLBM.cpp:1358-1403): Jiang-Shu smoothness indicators, linear
 * weights 1/10, 6/10, 3/10, epsilon 1e-6, on the upwind-ordered stencil
 * scaled by |e|. */
static double weno5(double e, const double *S)
{
    double a = fabs(e);
    if (a == 0) return 0;
    double q0 = a * S[0], q1 = a * S[1], q2 = a * S[2], q3 = a * S[3], q4 = a * S[4];
    double d0 = q0 - 2 * q1 + q2, d1 = q1 - 2 * q2 + q3, d2 = q2 - 2 * q3 + q4;
    double l0 = q0 - 4 * q1 + 3 * q2, l1 = q1 - q3, l2 = 3 * q2 - 4 * q3 + q4;
    double b0 = (13.0 / 12.0) * d0 * d0 + 0.25 * l0 * l0;
    double b1 = (13.0 / 12.0) * d1 * d1 + 0.25 * l1 * l1;
    double b2 = (13.0 / 12.0) * d2 * d2 + 0.25 * l2 * l2;
    const double eps = 1e-6;
    double g0 = 1.0 / (eps + b0), g1 = 1.0 / (eps + b1), g2 = 1.0 / (eps + b2);
    double w0 = 0.1 * g0 * g0, w1 = 0.6 * g1 * g1, w2 = 0.3 * g2 * g2;
    double ws = w0 + w1 + w2;
    double r0 = (2.0 * q0 - 7.0 * q1 + 11.0 * q2) / 6.0;
    double r1 = (-q1 + 5.0 * q2 + 2.0 * q3) / 6.0;
    double r2 = (2.0 * q2 + 5.0 * q3 - q4) / 6.0;
    return (w0 / ws) * r0 + (w1 / ws) * r1 + (w2 / ws) * r2;
}

/* computeFlux (cpuLBM.cpp:1405-1434): outgoing face fluxes (x, y) of
 * direction i at a non-solid node */
static void compute_flux(const orc *s, const double *f, int x, int y, int i, double *Fx, double *Fy)
{
    double Sx[5], Sy[5];
    if (s->fm == 0) {
        stencil(s, f, x, y, i, 3, Sx, Sy);
        *Fx = nnd(s->ex[i], Sx);
        *Fy = nnd(s->ey[i], Sy);
    } else {
        stencil(s, f, x, y, i, 5, Sx, Sy);
        *Fx = weno5(s->ex[i], Sx);
        *Fy = weno5(s->ey[i], Sy);
    }
}

/* posFluxes + wallFluxes (cpuLBM.cpp:1471-1596).  Fluxes of non-solid nodes
 * from their stencils; each solid node gets alpha |e_i| f_solid with
 * alpha = (flux of the fluid 4-neighbours into it) / (|e| f_solid out of it),
 * one alpha from f applied to both f and h.  The in/out weights use the
 * solid cell's own dx, dy (the uniform case is the reference's /dx, /dy;
 * the non-uniform case is codeCL.py:715-742's area weighting divided by the
 * cell volume). */
static void boundary_fluxes(orc *s, const double *f, const double *h, double *Ff, double *Hf)
{
    /* Ff/Hf layout: [(x*Ny+y)*13+i][2] (x then y component) */
    for (int x = 0; x < s->Nx; ++x)
        for (int y = 0; y < s->Ny; ++y)
            for (int i = 0; i < NQ; ++i) {
                if (s->type[AT(x, y)] == 2) continue;
                size_t k = AT3(x, y, i) * 2;
                compute_flux(s, f, x, y, i, &Ff[k], &Ff[k + 1]);
                compute_flux(s, h, x, y, i, &Hf[k], &Hf[k + 1]);
            }
    static const int xx[4] = {-1, 1, 0, 0}, yy[4] = {0, 0, -1, 1};
    static const int ii[4][4] = {{1, 5, 8, 9}, {3, 6, 7, 11}, {2, 5, 6, 10}, {4, 7, 8, 12}};
    static const int inv[4][4] = {{3, 6, 7, 11}, {1, 5, 8, 9}, {4, 8, 7, 12}, {2, 6, 5, 10}};
    for (int x = 0; x < s->Nx; ++x)
        for (int y = 0; y < s->Ny; ++y) {
            if (s->type[AT(x, y)] != 2) continue;
            double fin = 0, fout = 0, m_dx = s->dx[x], m_dy = s->dy[y];
            for (int j = 0; j < 4; ++j) {
                int m;
                int xm = bc_index(s, x, xx[j], 0, &m);
                int ym = bc_index(s, y, yy[j], 1, &m);
                if (s->type[AT(xm, ym)] >= 2) continue;
                int inx = abs(xx[j]), iny = abs(yy[j]);
                for (int k = 0; k < 4; ++k) {
                    int i = ii[j][k], io = inv[j][k];
                    size_t kn = AT3(xm, ym, i) * 2;
                    fin += inx * Ff[kn] / m_dx + iny * Ff[kn + 1] / m_dy;
                    double fo = f[AT3(x, y, io)];
                    fout += inx * fo * fabs(s->ex[io]) / m_dx + iny * fo * fabs(s->ey[io]) / m_dy;
                }
            }
            double alpha = fin / fout;
            for (int i = 0; i < NQ; ++i) {
                size_t k = AT3(x, y, i) * 2;
                double ax = fabs(s->ex[i]), ay = fabs(s->ey[i]);
                Ff[k] = alpha * ax * f[AT3(x, y, i)];
                Ff[k + 1] = alpha * ay * f[AT3(x, y, i)];
                Hf[k] = alpha * ax * h[AT3(x, y, i)];
                Hf[k + 1] = alpha * ay * h[AT3(x, y, i)];
            }
        }
}

/* cFLUX (cpuLBM.cpp:1436-1470) with the node's own dt/dx, dt/dy
 * (codeCL.py:590-620 for non-uniform cells) */
static double div_flux(const orc *s, const double *Fl, int x, int y, int i)
{
    if (i == 0) return 0;
    int ex = sgn(s->ex[i]), ey = sgn(s->ey[i]);
    int m_ew, m_ns;
    int xu = bc_index(s, x, -ex, 0, &m_ew);
    int yu = bc_index(s, y, -ey, 1, &m_ns);
    int i_ns = m_ns ? MIR_NS[i] : i, i_ew = m_ew ? MIR_EW[i] : i;
    double tx = s->dt / s->dx[x], ty = s->dt / s->dy[y];
    double out = tx * Fl[AT3(x, y, i) * 2] + ty * Fl[AT3(x, y, i) * 2 + 1];
    double in = tx * Fl[AT3(xu, y, i_ew) * 2] + ty * Fl[AT3(x, yu, i_ns) * 2 + 1];
    return out - in;
}

static double edot(const orc *s, int i, double ux, double uy) { return s->ex[i] * ux + s->ey[i] * uy; }

/* ------------------------------------------------------------------ steppers */
enum { W_F1, W_H1, W_F2, W_H2, W_F3, W_H3, W_FF2, W_HF2, W_FF3, W_HF3, W_D2F, W_D2H, W_EQF1, W_EQH1, W_EQF3, W_EQH3 };

/* RK1 (cpuLBM.cpp:1597-1737): implicit BGK half of IMEX Euler */
static void rk1(orc *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    double *f1 = s->w[W_F1], *h1 = s->w[W_H1], *feq = s->w[W_EQF1], *heq = s->w[W_EQH1];
    double *Ff = s->w[W_FF2], *Hf = s->w[W_HF2];
    macro_t *M = s->Ma;
    const double dt = s->dt;
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            size_t b = AT3(x, y, 0);
            if (s->type[AT(x, y)] > 0) {
                memcpy(&f1[b], &s->f[b], NQ * sizeof(double));
                memcpy(&h1[b], &s->h[b], NQ * sizeof(double));
                continue;
            }
            macro_t m = moments(s, &s->f[b], &s->h[b]);
            store_macro(s, x, y, &m);
            M[AT(x, y)] = m;
            equilibrium(s, m.rho, m.ux, m.uy, m.T, &feq[b], &heq[b]);
            for (int i = 0; i < NQ; ++i) {
                f1[b + i] = (s->f[b + i] + (dt / m.tf) * feq[b + i]) / (1.0 + dt / m.tf);
                double eu = edot(s, i, m.ux, m.uy);
                h1[b + i] = (s->h[b + i] - dt * eu * ((feq[b + i] - f1[b + i]) / m.thf) + (dt / m.th) * heq[b + i])
                            / (1 + dt / m.th);
            }
        }
    boundary_fluxes(s, f1, h1, Ff, Hf);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            if (s->type[AT(x, y)] > 0) continue;
            size_t b = AT3(x, y, 0);
            macro_t m = M[AT(x, y)];
            for (int i = 0; i < NQ; ++i) {
                double fo = s->f[b + i];
                s->f[b + i] = fo - div_flux(s, Ff, x, y, i) + (dt / m.tf) * (feq[b + i] - f1[b + i]);
                double eu = edot(s, i, m.ux, m.uy);
                s->h[b + i] = s->h[b + i] - div_flux(s, Hf, x, y, i) + (dt / m.th) * (heq[b + i] - h1[b + i])
                              - ((dt * eu) / m.thf) * (feq[b + i] - f1[b + i]);
            }
        }
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y)
            if (s->type[AT(x, y)] != 2) macro_short(s, x, y);
}

/* RK3 (cpuLBM.cpp:1738-2103): three-stage IMEX scheme, implicit BGK with
 * weights 1/2, explicit flux from stage 2 and 3 states. */
static void rk3(orc *s)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const double dt = s->dt;
    double *f1 = s->w[W_F1], *h1 = s->w[W_H1], *f2 = s->w[W_F2], *h2 = s->w[W_H2];
    double *f3 = s->w[W_F3], *h3 = s->w[W_H3];
    double *feq1 = s->w[W_EQF1], *heq1 = s->w[W_EQH1], *feq3 = s->w[W_EQF3], *heq3 = s->w[W_EQH3];
    double *Ff2 = s->w[W_FF2], *Hf2 = s->w[W_HF2], *Ff3 = s->w[W_FF3], *Hf3 = s->w[W_HF3];
    double *D2f = s->w[W_D2F], *D2h = s->w[W_D2H];
    macro_t *Ma = s->Ma, *Mc = s->Mc;

    /* stage 1 (cpuLBM.cpp:1819-1865) */
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            size_t b = AT3(x, y, 0);
            if (s->type[AT(x, y)] > 0) {
                memcpy(&f1[b], &s->f[b], NQ * sizeof(double));
                memcpy(&h1[b], &s->h[b], NQ * sizeof(double));
                continue;
            }
            macro_t m = moments(s, &s->f[b], &s->h[b]);
            Ma[AT(x, y)] = m;
            equilibrium(s, m.rho, m.ux, m.uy, m.T, &feq1[b], &heq1[b]);
            for (int i = 0; i < NQ; ++i) {
                double c = dt / (2 * m.tf);
                f1[b + i] = (s->f[b + i] + c * feq1[b + i]) / (1 + c);
                double eu = edot(s, i, m.ux, m.uy);
                h1[b + i] = (s->h[b + i] - (dt / (2 * m.thf)) * eu * (feq1[b + i] - f1[b + i])
                             + (dt / (2 * m.th)) * heq1[b + i]) / (1 + dt / (2 * m.th));
            }
        }
    /* stage 2 (cpuLBM.cpp:1869-1924): the stage-2 equilibrium, moments and
     * relaxation times alias stage 1's */
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            size_t b = AT3(x, y, 0);
            if (s->type[AT(x, y)] > 0) {
                memcpy(&f2[b], &f1[b], NQ * sizeof(double));
                memcpy(&h2[b], &h1[b], NQ * sizeof(double));
                continue;
            }
            macro_t m = Ma[AT(x, y)];
            for (int i = 0; i < NQ; ++i) {
                f2[b + i] = (s->f[b + i] - (dt / (2 * m.tf)) * (feq1[b + i] - f1[b + i]) + (dt / (2 * m.tf)) * feq1[b + i])
                            / (1 + dt / (2 * m.tf));
                double eu = edot(s, i, m.ux, m.uy);
                h2[b + i] = (s->h[b + i]
                             - (dt / 2) * ((eu / m.thf) * (feq1[b + i] - f2[b + i]) - (eu / m.thf) * (feq1[b + i] - f1[b + i]))
                             - (dt / (2 * m.th)) * (heq1[b + i] - h1[b + i]) + (dt / (2 * m.th)) * heq1[b + i])
                            / (1 + dt / (2 * m.th));
            }
        }
    /* stage 3 (cpuLBM.cpp:1928-1993) */
    boundary_fluxes(s, f2, h2, Ff2, Hf2);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            size_t b = AT3(x, y, 0);
            if (s->type[AT(x, y)] > 0) {
                memcpy(&f3[b], &f2[b], NQ * sizeof(double));
                memcpy(&h3[b], &h2[b], NQ * sizeof(double));
                continue;
            }
            for (int i = 0; i < NQ; ++i) {
                D2f[b + i] = div_flux(s, Ff2, x, y, i);
                D2h[b + i] = div_flux(s, Hf2, x, y, i);
            }
            /* macroProp3 (cpuLBM.cpp:973-1032): moments of f - div F(f2) */
            double r = 0, rux = 0, ruy = 0, sh = 0;
            for (int i = 0; i < NQ; ++i) {
                r += s->f[b + i] - D2f[b + i];
                rux += s->f[b + i] * s->ex[i] - D2f[b + i] * s->ex[i];
                ruy += s->f[b + i] * s->ey[i] - D2f[b + i] * s->ey[i];
                sh += s->h[b + i] - D2h[b + i];
            }
            macro_t m;
            m.rho = r;
            m.ux = rux / r;
            m.uy = ruy / r;
            double ax = fabs(m.ux), ay = fabs(m.uy);
            m.T = 2.0 * (sh / r - (ax * ax + ay * ay) / 2.0) / (s->b * s->R);
            m.p = r * s->R * m.T;
            m.tf = viscosity(s, m.T) / m.p;
            m.th = m.tf / s->Pr;
            m.thf = (m.th * m.tf) / (m.tf - m.th);
            Mc[AT(x, y)] = m;
            macro_t m2 = Ma[AT(x, y)];
            equilibrium(s, m.rho, m.ux, m.uy, m.T, &feq3[b], &heq3[b]);
            for (int i = 0; i < NQ; ++i) {
                f3[b + i] = (s->f[b + i] - D2f[b + i] + (dt / (2 * m2.tf)) * (feq1[b + i] - f2[b + i])
                             + (dt / (2 * m.tf)) * feq3[b + i]) / (1 + dt / (2 * m.tf));
                double eu2 = edot(s, i, m2.ux, m2.uy), eu3 = edot(s, i, m.ux, m.uy);
                h3[b + i] = (s->h[b + i] - D2h[b + i]
                             - (dt / 2) * ((eu2 / m2.thf) * (feq1[b + i] - f2[b + i]) + (eu3 / m.thf) * (feq3[b + i] - f3[b + i]))
                             + (dt / (2 * m2.th)) * (heq1[b + i] - h2[b + i]) + (dt / (2 * m.th)) * heq3[b + i])
                            / (1 + dt / (2 * m.th));
            }
        }
    /* update (cpuLBM.cpp:1997-2042) */
    boundary_fluxes(s, f3, h3, Ff3, Hf3);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            if (s->type[AT(x, y)] > 0) continue;
            size_t b = AT3(x, y, 0);
            macro_t m2 = Ma[AT(x, y)], m3 = Mc[AT(x, y)];
            for (int i = 0; i < NQ; ++i) {
                double D3f = div_flux(s, Ff3, x, y, i), D3h = div_flux(s, Hf3, x, y, i);
                double eu2 = edot(s, i, m2.ux, m2.uy), eu3 = edot(s, i, m3.ux, m3.uy);
                s->f[b + i] = s->f[b + i] - 0.5 * (D2f[b + i] + D3f)
                              + (dt / 2.0) * ((feq1[b + i] - f2[b + i]) / m2.tf + (feq3[b + i] - f3[b + i]) / m3.tf);
                s->h[b + i] = s->h[b + i] - 0.5 * (D2h[b + i] + D3h)
                              + (dt / 2.0) * ((heq1[b + i] - h2[b + i]) / m2.th + (heq3[b + i] - h3[b + i]) / m3.th)
                              - (dt / 2.0) * ((eu2 / m2.thf) * (feq1[b + i] - f2[b + i]) + (eu3 / m3.thf) * (feq3[b + i] - f3[b + i]));
            }
        }
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y)
            if (s->type[AT(x, y)] != 2) macro_short(s, x, y);
}

/* EULER (cpuLBM.cpp:2104-2193) and EULER_EQ (cpuLBM.cpp:2194-2283) */
static void euler(orc *s, int to_eq)
{
    const int Nx = s->Nx, Ny = s->Ny;
    const double dt = s->dt;
    double *Ff = s->w[W_FF2], *Hf = s->w[W_HF2];
    /* fluxes come from the state at the start of the step */
    boundary_fluxes(s, s->f, s->h, Ff, Hf);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            if (s->type[AT(x, y)] > 0) continue;
            size_t b = AT3(x, y, 0);
            macro_t m = moments(s, &s->f[b], &s->h[b]);
            store_macro(s, x, y, &m);
            double feq[NQ], heq[NQ];
            equilibrium(s, m.rho, m.ux, m.uy, m.T, feq, heq);
            for (int i = 0; i < NQ; ++i) {
                double fo = s->f[b + i], ho = s->h[b + i];
                double Df = div_flux(s, Ff, x, y, i), Dh = div_flux(s, Hf, x, y, i);
                if (to_eq) {
                    s->f[b + i] = feq[i] - Df;
                    s->h[b + i] = heq[i] - Dh;
                } else {
                    double eu = edot(s, i, m.ux, m.uy);
                    s->f[b + i] = fo - Df + (dt / m.tf) * (feq[i] - fo);
                    s->h[b + i] = ho - Dh + (dt / m.th) * (heq[i] - ho) - ((dt * eu) / m.thf) * (feq[i] - fo);
                }
            }
        }
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y)
            if (s->type[AT(x, y)] != 2) macro_short(s, x, y);
}

/* runOne (cpuLBM.cpp:2284-2335) */
static int run_one(orc *s, int res)
{
    s->hasFailed = 0;
    size_t N = (size_t)s->Nx * s->Ny;
    double *Told = NULL;
    if (res > 0) {
        Told = (double *)malloc(N * sizeof(double));
        memcpy(Told, s->T, N * sizeof(double));
    }
    switch (s->rk) {
    case 0: rk1(s); break;
    case 1: rk3(s); break;
    case 2: euler(s, 0); break;
    case 3: euler(s, 1); break;
    default: break;
    }
    if (res > 0) {
        double sum = 0;
        for (size_t k = 0; k < N; ++k) sum += (s->T[k] - Told[k]) * (s->T[k] - Told[k]);
        s->residual = sqrt(sum / (double)N);
        free(Told);
    }
    return s->hasFailed;
}

int orc_step(orc *s, int n, int res, double *residual)
{
    int failed = 0;
    for (int k = 0; k < n; ++k) {
        s->step += 1; /* updateStepCount (cpuLBM.cpp:771-775) */
        failed |= run_one(s, res);
    }
    if (residual) *residual = s->residual;
    return failed;
}

/* the driver loop of main.cpp:32-112 (runSimStep), without file output */
int orc_run(orc *s, int max_steps, double *trace)
{
    const int numRes = 20;
    int stop = 0, k = 0;
    while (stop == 0 && (max_steps < 0 || k < max_steps)) {
        s->step += 1;
        if (s->tol != 0) {
            stop = run_one(s, 1);
            if (s->step >= 2 && s->step <= numRes) {
                s->initRes[s->step - 2] = s->residual;
                s->residual = 1;
            } else if (s->step == numRes + 1) {
                for (int i = 0; i < numRes - 1; ++i) s->resNorm = fmax(s->initRes[i], s->resNorm);
                s->residual = s->residual / s->resNorm;
            } else if (s->step >= numRes + 1) {
                s->residual = s->residual / s->resNorm;
            }
        } else {
            stop = run_one(s, 0);
        }
        if (trace) trace[k] = s->residual;
        if (s->step >= s->nsteps && s->nsteps != 0) stop = 2;
        if (s->tol != 0 && s->residual <= s->tol && s->step >= numRes + 1) stop = 2;
        ++k;
    }
    return stop;
}

/* --------------------------------------------------------------------- setup
 * refineInput (cpuLBM.cpp:283-358), setupVars (:360-450),
 * initialiseFunctions (:846-875). */
orc *orc_create(const orc_config *c, const orc_init *in)
{
    if (!c || !in || in->Nx < 1 || in->Ny < 1) return NULL;
    orc *s = (orc *)calloc(1, sizeof(orc));
    const int Nx = in->Nx, Ny = in->Ny;
    const size_t N = (size_t)Nx * Ny;
    s->Nx = Nx;
    s->Ny = Ny;
    s->rk = c->RKMETHOD;
    s->fm = c->FMETHOD;
    s->perX = c->periodicX;
    s->perY = c->periodicY;
    s->mirN = c->mirrorNorth;
    s->mirS = c->mirrorSouth;
    s->mirE = c->mirrorEast;
    s->mirW = c->mirrorWest;
    s->R = c->R;
    s->mu = c->mu;
    s->mu_model = c->mu_model;
    s->visc_exp = c->mu_model == 1 ? 0.5 + c->upsilon : 1.5;
    s->S_v = c->S_v;
    s->Pr = c->Pr;
    s->tol = c->tol;

    double dx = c->dx, dy = c->dy, Lx = c->Lx, Ly = c->Ly;
    if (dx == 0) dx = Lx / ((double)Nx - 1); else Lx = dx * (Nx - 1);
    if (dy == 0 && Ly != 0) dy = Ly / ((double)Ny - 1);
    else if (dy == 0 && Ly == 0) { dy = dx; Ly = dy * (Ny - 1); }
    else Ly = dy * (Ny - 1);
    double rho_ref = c->rho_ref, p_ref = c->p_ref, T_ref = c->T_ref;
    if (rho_ref == 0) rho_ref = p_ref / (c->R * T_ref);
    else if (p_ref == 0) p_ref = rho_ref * c->R * T_ref;
    else if (T_ref == 0) T_ref = p_ref / (rho_ref * c->R);
    s->T_ref = T_ref;

    s->dx = (double *)malloc(Nx * sizeof(double));
    s->dy = (double *)malloc(Ny * sizeof(double));
    double mind = dx < dy ? dx : dy;
    if (c->dx_array || c->dy_array) mind = INFINITY;
    for (int x = 0; x < Nx; ++x) {
        s->dx[x] = c->dx_array ? c->dx_array[x] : dx;
        if ((c->dx_array || c->dy_array) && s->dx[x] < mind) mind = s->dx[x];
    }
    for (int y = 0; y < Ny; ++y) {
        s->dy[y] = c->dy_array ? c->dy_array[y] : dy;
        if ((c->dx_array || c->dy_array) && s->dy[y] < mind) mind = s->dy[y];
    }

    s->b = 2 / (c->gamma - 1);
    s->K = s->b - 2;
    s->Tc = c->Tc_Tref * T_ref;
    double tau_ref = c->mu / p_ref;
    double u_ref = sqrt(c->R * T_ref);
    double t_ref = (Lx > Ly ? Lx : Ly) / u_ref;
    double cc = sqrt(c->R * s->Tc);
    for (int i = 0; i < NQ; ++i) {
        s->ex[i] = EX[i] * cc;
        s->ey[i] = EY[i] * cc;
    }
    s->dt = c->dtau == 0 ? (c->CFL * mind) / s->ex[9] : c->dtau * tau_ref;
    double ttotal = 0;
    int need = 0;
    if (c->tt_tref > 0) { ttotal = c->tt_tref * t_ref; need = 1; }
    else if (c->tt_time > 0) { ttotal = c->tt_time; need = 1; }
    else if (c->steps > 0) s->nsteps = c->steps;
    else if (c->tol > 0) s->nsteps = 0;
    if (need) s->nsteps = (int)ceil(ttotal / s->dt);

    s->type = (unsigned char *)malloc(N);
    s->f = (double *)malloc(N * NQ * sizeof(double));
    s->h = (double *)malloc(N * NQ * sizeof(double));
    s->rho = (double *)calloc(N, sizeof(double));
    s->ux = (double *)calloc(N, sizeof(double));
    s->uy = (double *)calloc(N, sizeof(double));
    s->T = (double *)calloc(N, sizeof(double));
    s->p = (double *)calloc(N, sizeof(double));
    for (int k = 0; k < 16; ++k) s->w[k] = (double *)calloc(N * NQ * 2, sizeof(double));
    s->Ma = (macro_t *)calloc(N, sizeof(macro_t));
    s->Mc = (macro_t *)calloc(N, sizeof(macro_t));

    /* property tables completed as refineInput does */
    int np = in->numProps;
    double *prho = (double *)malloc(np * sizeof(double)), *pT = (double *)malloc(np * sizeof(double));
    for (int r = 0; r < np; ++r) {
        double rho = in->density[r], p = in->pressure[r], T = in->temp[r];
        if (rho == 0) rho = p / (c->R * T);
        else if (p == 0) p = rho * c->R * T;
        else if (T == 0) T = p / (rho * c->R);
        prho[r] = rho;
        pT[r] = T;
    }
    for (int y = 0; y < Ny; ++y)
        for (int x = 0; x < Nx; ++x) {
            int id = in->bnd[(size_t)x * Ny + y];
            s->type[AT(x, y)] = (unsigned char)in->cellType[id];
            equilibrium(s, prho[id], in->velocityX[id], in->velocityY[id], pT[id], &s->f[AT3(x, y, 0)],
                        &s->h[AT3(x, y, 0)]);
            macro_short(s, x, y);
        }
    free(prho);
    free(pT);
    s->step = 0;
    s->residual = 1;
    return s;
}

void orc_destroy(orc *s)
{
    if (!s) return;
    free(s->dx); free(s->dy); free(s->type); free(s->f); free(s->h);
    free(s->rho); free(s->ux); free(s->uy); free(s->T); free(s->p);
    for (int k = 0; k < 16; ++k) free(s->w[k]);
    free(s->Ma); free(s->Mc);
    free(s);
}

void orc_get_macro(const orc *s, double *rho, double *ux, double *uy, double *T, double *p)
{
    size_t N = (size_t)s->Nx * s->Ny;
    if (rho) memcpy(rho, s->rho, N * sizeof(double));
    if (ux) memcpy(ux, s->ux, N * sizeof(double));
    if (uy) memcpy(uy, s->uy, N * sizeof(double));
    if (T) memcpy(T, s->T, N * sizeof(double));
    if (p) memcpy(p, s->p, N * sizeof(double));
}

void orc_get_dist(const orc *s, double *f, double *h)
{
    size_t N3 = (size_t)s->Nx * s->Ny * NQ;
    if (f) memcpy(f, s->f, N3 * sizeof(double));
    if (h) memcpy(h, s->h, N3 * sizeof(double));
}

void orc_set_dist(orc *s, const double *f, const double *h)
{
    size_t N3 = (size_t)s->Nx * s->Ny * NQ;
    memcpy(s->f, f, N3 * sizeof(double));
    memcpy(s->h, h, N3 * sizeof(double));
    for (int x = 0; x < s->Nx; ++x)
        for (int y = 0; y < s->Ny; ++y) macro_short(s, x, y);
}

/* the viscosity law alone at temperature T, with the parameters set as
 * orc_create sets them (for pinning against the reference's OpenCL
 * generator, codeCL.py:60-69, 986-990) */
double orc_viscosity(int mu_model, double mu_ref, double T_ref, double upsilon, double S_v, double T)
{
    orc s;
    memset(&s, 0, sizeof s);
    s.mu_model = mu_model;
    s.mu = mu_ref;
    s.T_ref = T_ref;
    s.S_v = S_v;
    s.visc_exp = mu_model == 1 ? 0.5 + upsilon : 1.5;
    return viscosity(&s, T);
}

double orc_dt(const orc *s) { return s->dt; }
int orc_nsteps(const orc *s) { return s->nsteps; }
int orc_step_count(const orc *s) { return s->step; }
double orc_residual(const orc *s) { return s->residual; }
