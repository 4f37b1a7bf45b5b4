/* FP64 CPU restatement of the reference D2Q13 thermal lattice-Boltzmann step.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle that the CUDA path is checked
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product never does.
 *
 * It restates CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp (the reference's FP64
 * CPU solver) function by function in plain C, in the reference's own AoS
 * layout f[(x*Ny + y)*13 + i], and adds the non-uniform cell widths of the
 * OpenCL generator (CODE/Python/simLB/codeCL.py:100-114, 590-620), which the
 * C++ solver cannot express.  On uniform grids it is pinned against the
 * reference binary built from the read-only sources (oracle/_ref).
 */
#ifndef LBM_ORACLE_H_
#define LBM_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_config {
    int RKMETHOD;  /* 0 RK1 (IMEX Euler), 1 RK3, 2 EULER, 3 EULER_EQ */
    int FMETHOD;   /* 0 NND, 1 WENO5 */
    double CFL, dtau, tt_tref, tt_time;
    int steps;
    double tol;
    int periodicX, periodicY, mirrorNorth, mirrorSouth, mirrorEast, mirrorWest;
    double gamma, R, mu, Pr, dx, dy, Lx, Ly, rho_ref, p_ref, T_ref, Tc_Tref;
    const double *dx_array; /* [Nx] cell widths, or NULL for uniform dx */
    const double *dy_array; /* [Ny] cell heights, or NULL for uniform dy */
    /* viscosity law of the OpenCL generator (codeCL.py:986-990): 0 constant
     * mu (the C++ solver), 1 VHS, 2 Sutherland; mu is the value at T_ref */
    int mu_model;
    double upsilon, S_v;
} orc_config;

typedef struct orc_init {
    int Nx, Ny, numProps;
    const int *bnd;       /* [Nx*Ny] property id, bnd[x*Ny + y] */
    const int *cellType;  /* [numProps] 0 fluid, 1 permanent, 2 solid */
    const double *density, *pressure, *temp, *velocityX, *velocityY; /* [numProps] */
} orc_init;

typedef struct orc orc;

orc *orc_create(const orc_config *cfg, const orc_init *init);
void orc_destroy(orc *s);

/* n x (updateStepCount + runOne(res)); returns 1 if any equilibrium check
 * failed (the reference's hasFailed), else 0. */
int orc_step(orc *s, int n, int res, double *residual);

/* The reference driver loop (main.cpp:32-112) until stop or max_steps steps
 * (max_steps < 0: no limit).  Returns the stop code (2 end, 1 failure). */
int orc_run(orc *s, int max_steps, double *residual_trace);

void orc_get_macro(const orc *s, double *rho, double *ux, double *uy, double *T, double *p);
void orc_get_dist(const orc *s, double *f, double *h);
void orc_set_dist(orc *s, const double *f, const double *h);
double orc_viscosity(int mu_model, double mu_ref, double T_ref, double upsilon, double S_v, double T);
double orc_dt(const orc *s);
int orc_nsteps(const orc *s);
int orc_step_count(const orc *s);
double orc_residual(const orc *s);

/* Equilibria of one node in physical units (equilibrium2D, cpuLBM.cpp:785-844). */
void orc_equilibrium(double rho, double ux, double uy, double T, double R, double Tc, double K,
                     double *eqf, double *eqh);

#ifdef __cplusplus
}
#endif
#endif
