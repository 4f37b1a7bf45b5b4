/* uq_lbm.h - C ABI of the B200 D2Q13 thermal lattice-Boltzmann step.
 *
 * Drop-in boundary for the reference solver's step API, the C++ class
 * cpuLBM (CODE/C++/VS2010/simLB/simLB/cpuLBM.h:16-175) and the PyOpenCL
 * ClassLBM.runSimStep (CODE/Python/simLB/LBM.py:571-594).  Plain C types
 * only; every entry point returns an lbm_status and never throws.
 *
 * Layout at the boundary is the reference's: per-node arrays are indexed
 * [x*Ny + y] (macros.h:8-14) and distributions [(x*Ny + y)*13 + i]
 * (macros.h:9-10).  Inside the library the state is structure-of-arrays on
 * the GPU; the conversion happens in lbm_get_* / lbm_set_*.
 *
 * Threading: a handle is not thread-safe; each handle owns one CUDA stream.
 * There is no CPU fallback: without a usable CUDA device lbm_create fails
 * with LBM_ERR_CUDA.
 */
#ifndef UQ_LBM_H_
#define UQ_LBM_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

typedef enum lbm_status {
    LBM_OK = 0,
    /* an equilibrium mass check failed: the reference's hasFailed
     * (cpuLBM.cpp:839-843) returned by runOne (cpuLBM.cpp:2334) */
    LBM_ERR_EQUILIBRIUM = 1,
    LBM_ERR_INVALID = 2,     /* bad argument or configuration */
    LBM_ERR_CUDA = 3,        /* CUDA runtime error / no device */
    LBM_ERR_NOMEM = 4,       /* device allocation failed */
    LBM_ERR_NONFINITE = 5,   /* the state became NaN/Inf or rho <= 0 */
    LBM_ERR_BUSY = 6,        /* serving: queue full / no capacity */
    LBM_ERR_NOT_FOUND = 7,   /* serving: unknown request id */
    LBM_ERR_TIMEOUT = 8,     /* a bounded wait ran out */
    LBM_ERR_CANCELLED = 9    /* serving: the request was cancelled */
} lbm_status;

/* Storage/compute precision of a handle or batch. */
enum {
    LBM_PREC_F64 = 0, /* plain path: FP64 state and arithmetic */
    LBM_PREC_F32 = 1  /* mixed path: FP32 state and stencil/collision math,
                         FP64 moment sums and reductions */
};

/* Configuration: the MAT variables read by cpuLBM::loadInput
 * (cpuLBM.cpp:113-199), same names and meaning; derived values follow
 * refineInput/setupVars (cpuLBM.cpp:283-450).  dx_array/dy_array (optional)
 * give per-column/per-row cell widths as in the OpenCL generator
 * (CODE/Python/simLB/codeCL.py:100-114); NULL selects uniform dx, dy. */
typedef struct lbm_config {
    int RKMETHOD; /* 0 RK1 (IMEX Euler), 1 RK3 (3-stage IMEX), 2 EULER, 3 EULER_EQ */
    int FMETHOD;  /* 0 NND, 1 WENO5 */
    double CFL, dtau, tt_tref, tt_time;
    int steps;
    double tol;
    int periodicX, periodicY, mirrorNorth, mirrorSouth, mirrorEast, mirrorWest;
    double gamma, R, mu, Pr;
    double dx, dy, Lx, Ly;
    double rho_ref, p_ref, T_ref, Tc_Tref;
    const double *dx_array; /* [Nx] or NULL */
    const double *dy_array; /* [Ny] or NULL */
    /* Viscosity law of the OpenCL generator (CODE/Python/simLB/codeCL.py:
     * 986-990; the C++ solver has the constant law only): 0 constant mu
     * (cpuLBM), 1 VHS mu (T/T_ref)^(0.5 + upsilon), 2 Sutherland
     * mu (T/T_ref)^(3/2) (T_ref + S_v)/(T + S_v); mu is the viscosity at
     * T_ref.  A zero-initialised config keeps the constant law. */
    int mu_model;
    double upsilon, S_v;
} lbm_config;

/* Domain: the property-id map and property tables of loadInput
 * (cpuLBM.cpp:202-266).  bndArray is in the solver's internal order
 * BNDARRAY(x,y) = bndArray[x*Ny + y] (i.e. after loadInput's y flip). */
typedef struct lbm_init {
    int Nx, Ny, numProps;
    const int *bndArray;  /* [Nx*Ny] */
    const int *cellType;  /* [numProps] 0 fluid, 1 permanent, 2 solid */
    const double *density, *pressure, *temp, *velocityX, *velocityY; /* [numProps] */
} lbm_init;

typedef struct lbm_info {
    int Nx, Ny;
    int step;       /* steps taken (cpuLBM::step) */
    int nsteps;     /* derived step count (cpuLBM::nsteps) */
    double dt;      /* cpuLBM::dt */
    double tstep;   /* step * dt (cpuLBM::tstep) */
    double residual;/* cpuLBM::residual */
    int precision;
    int rkmethod, fmethod;
    size_t device_bytes; /* device memory held by this handle */
} lbm_info;

typedef struct lbm_handle lbm_handle;

/* cpuLBM::cpuLBM (cpuLBM.cpp:7-20) + initSim (cpuLBM.cpp:452-462):
 * derive the run parameters, set f, h to the equilibria of each node's
 * property and upload.  precision: LBM_PREC_F64 or LBM_PREC_F32. */
LBM_API lbm_status lbm_create(const lbm_config *cfg, const lbm_init *init, int precision, lbm_handle **out);

/* n_steps x (cpuLBM::updateStepCount + cpuLBM::runOne(want_residual))
 * (cpuLBM.cpp:771-775, 2284-2335).  Returns LBM_ERR_EQUILIBRIUM where runOne
 * returns hasFailed = 1 (the failing step still completes, as in the
 * reference), LBM_ERR_NONFINITE if the state left the finite range.
 * residual_out (may be NULL) receives cpuLBM::residual after the last step. */
LBM_API lbm_status lbm_step(lbm_handle *h, int n_steps, int want_residual, double *residual_out);

/* The reference driver loop (main.cpp:32-112, runSimStep without file
 * output): steps until nsteps is reached, the normalised residual falls to
 * tol, an equilibrium check fails, or max_steps (<0: unlimited) steps ran.
 * stop_out: 0 still running, 1 failure, 2 finished.  residual_trace (may be
 * NULL) receives the per-step residual as main.cpp leaves it. */
LBM_API lbm_status lbm_run(lbm_handle *h, int max_steps, int *stop_out, double *residual_trace, int trace_len);

/* Public arrays rho_G, u_G, T_G, p_G (cpuLBM.h:93-96) in [x*Ny + y] order,
 * computed from the current f, h (macroPropShort, cpuLBM.cpp:877-914).
 * Any pointer may be NULL. */
LBM_API lbm_status lbm_get_macro(lbm_handle *h, double *rho, double *ux, double *uy, double *T, double *p);

/* f_G, h_G (cpuLBM.h:90-91) in [(x*Ny + y)*13 + i] order; may be NULL. */
LBM_API lbm_status lbm_get_dist(lbm_handle *h, double *f, double *hh);

/* Replace f, h (same layout); the checkpoint/resume entry point. */
LBM_API lbm_status lbm_set_dist(lbm_handle *h, const double *f, const double *hh);

LBM_API lbm_status lbm_get_info(lbm_handle *h, lbm_info *info);

/* The CUDA stream (cudaStream_t) the handle's kernels run on. */
LBM_API void *lbm_stream(lbm_handle *h);

LBM_API void lbm_destroy(lbm_handle *h);

/* Human-readable message of the last failure on the calling thread. */
LBM_API const char *lbm_last_error(void);

/* ------------------------------------------------------------- MAT files
 * The reference's MATLAB Level-5 files at the boundary.  Input: the
 * variables cpuLBM::loadInput reads (cpuLBM.cpp:46-281), same names, any
 * numeric class (converted to double as loadInput's mxGetPr reads it),
 * compressed or not; bndArray's y axis is flipped as loadInput does.
 * Output: the variables cpuLBM::createMAT writes (cpuLBM.cpp:467-745). */
typedef struct lbm_mat_case lbm_mat_case;

/* Read an input MAT file into a case (no GPU needed). */
LBM_API lbm_status lbm_mat_read_case(const char *path, lbm_mat_case **out);
/* The case as the lbm_create arguments; init's arrays stay owned by the
 * case (valid until lbm_mat_case_free).  Either pointer may be NULL. */
LBM_API lbm_status lbm_mat_case_get(const lbm_mat_case *c, lbm_config *cfg, lbm_init *init);
LBM_API void lbm_mat_case_free(lbm_mat_case *c);
/* new cpuLBM(files) on an input MAT file: read it and create a handle. */
LBM_API lbm_status lbm_create_from_mat(const char *path, int precision, lbm_handle **out);
/* createMAT: rho, ux, uy, p, T as {Ny, Nx} arrays over [x*Ny + y], t, dx,
 * dy and, when f, h, ex, ey are all given, f and h as {13, Ny, Nx} over
 * [(x*Ny + y)*13 + i] with the lattice vectors ex, ey (no GPU needed). */
LBM_API lbm_status lbm_mat_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux,
                                        const double *uy, const double *p, const double *T, double t, double dx,
                                        double dy, const double *f, const double *h, const double *ex,
                                        const double *ey);
/* createMAT(name, DF) of a handle's current state (t = step * dt). */
LBM_API lbm_status lbm_write_mat(lbm_handle *h, const char *path, int with_dist);
/* Checkpoint/resume, which the reference cannot do (it only dumps): f, h
 * and t of a file lbm_write_mat wrote with with_dist = 1 (no GPU needed;
 * f, h [(x*Ny + y)*13 + i], any pointer may be NULL) ... */
LBM_API lbm_status lbm_mat_read_dist(const char *path, int Nx, int Ny, double *f, double *h, double *t);
/* ... and into a handle of the same case: its f, h and step count
 * (round(t / dt)) become the checkpoint's. */
LBM_API lbm_status lbm_restore_mat(lbm_handle *h, const char *path);
/* The Python reference's result files, ClassLBM.saveHDF5
 * (CODE/Python/simLB/LBM.py:516-567): an HDF5 file with the datasets rho,
 * T, ux, uy ({Nx, Ny} over [x*Ny + y]), t, gamma, R, T_ref, rho_ref, dx, dy
 * (ndx / ndy values; scalars when 1), Nx, Ny (int64) and, when f and h are
 * both given, f and h ({Nx, Ny, 13} over [(x*Ny + y)*13 + i]).  Doubles are
 * little-endian IEEE.  No GPU needed. */
LBM_API lbm_status lbm_hdf5_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux,
                                         const double *uy, const double *T, double t, double gamma, double R,
                                         double T_ref, double rho_ref, const double *dx, int ndx, const double *dy,
                                         int ndy, const double *f, const double *h);
/* saveHDF5(all) of a handle's current state (t = step * dt). */
LBM_API lbm_status lbm_write_hdf5(lbm_handle *h, const char *path, int with_dist);

/* -------------------------------------------------------------- batches
 * Many independent samples (uneven grids, own parameters) advanced
 * together: every phase is one launch over a packed tile list of all
 * samples; runs of steps are captured in a CUDA graph.  Samples must share
 * RKMETHOD where they are stepped together; everything else may differ. */
typedef struct lbm_batch lbm_batch;

typedef struct lbm_batch_options {
    int precision;      /* LBM_PREC_F64 / LBM_PREC_F32 */
    int tile_x, tile_y; /* 0: chosen by the autotuner's table (32 x 8, the
                           shape the stencil kernels are also compiled for;
                           other shapes run the same kernels with the shape
                           read at run time, bit-identical and slower) */
    int use_graph;      /* capture step sequences in CUDA graphs */
} lbm_batch_options;

LBM_API lbm_status lbm_batch_create(int n, const lbm_config *cfgs, const lbm_init *inits,
                            const lbm_batch_options *opt, lbm_batch **out);
/* n_steps steps of every sample; want_residual as runOne(res). */
LBM_API lbm_status lbm_batch_step(lbm_batch *b, int n_steps, int want_residual);
/* Per-sample status (lbm_status values) of the steps since the last call. */
LBM_API lbm_status lbm_batch_status(lbm_batch *b, int *status);
/* Per-sample residual after the last step with want_residual. */
LBM_API lbm_status lbm_batch_residuals(lbm_batch *b, double *residual);
LBM_API lbm_status lbm_batch_get_macro(lbm_batch *b, int sample, double *rho, double *ux, double *uy,
                               double *T, double *p);
LBM_API lbm_status lbm_batch_get_dist(lbm_batch *b, int sample, double *f, double *hh);
LBM_API lbm_status lbm_batch_set_dist(lbm_batch *b, int sample, const double *f, const double *hh);
/* Set a sample's f, h to the equilibria of the given macroscopic fields
 * (each [x*Ny + y]), as initialiseFunctions does for property tables
 * (cpuLBM.cpp:846-875): the restart-from-fields / new-solve entry point. */
LBM_API lbm_status lbm_batch_set_macro(lbm_batch *b, int sample, const double *rho, const double *ux,
                                       const double *uy, const double *T);
/* Every sample's fields at once, for callers that move the whole ensemble
 * (no counterpart in the reference, which runs one solve per process): the
 * arrays hold the samples one after another in sample order, each in the
 * [x*Ny + y] order of its own grid (sum over samples of Nx*Ny values per
 * field).  One host<->device copy per field and one synchronisation, in
 * place of one of each per sample.  Results are those of the per-sample
 * calls. */
LBM_API lbm_status lbm_batch_set_macro_all(lbm_batch *b, const double *rho, const double *ux, const double *uy,
                                           const double *T);
LBM_API lbm_status lbm_batch_get_macro_all(lbm_batch *b, double *rho, double *ux, double *uy, double *T,
                                           double *p);
/* Run n_steps steps outside any graph with CUDA events around every phase
 * and return the mean device milliseconds per step of each phase in
 * phase_ms[0..5]: pointwise stages, walls of buffer 2, stencil phase 1,
 * walls of buffer 3, stencil phase 2, residual reduction. */
LBM_API lbm_status lbm_batch_profile(lbm_batch *b, int n_steps, double *phase_ms, int n_phases);
/* Autotuner: time n-step runs (CUDA events) of the batch for each
 * candidate tile shape (pairs tile_x, tile_y; NULL / 0 candidates: a
 * built-in list), switch the batch to the fastest and restore the state it
 * had, so tuning leaves results unchanged.  chosen (2 ints) and
 * ms_per_step (one per candidate) may be NULL. */
LBM_API lbm_status lbm_batch_autotune(lbm_batch *b, const int *candidates, int n_candidates, int steps, int *chosen,
                                      double *ms_per_step);
/* Kernel launches one step of the batch issues. */
LBM_API int lbm_batch_launches_per_step(lbm_batch *b, int want_residual);
/* Lattice updates (nodes) one step of the whole batch performs. */
LBM_API long long lbm_batch_nodes(lbm_batch *b);
LBM_API void *lbm_batch_stream(lbm_batch *b);
LBM_API void lbm_batch_destroy(lbm_batch *b);

/* ------------------------------------------------------------- serving
 * No single counterpart in the reference, whose driver runs one solve per
 * process (main.cpp:32-112).  A server owns a device arena carved from the
 * free HBM when it is created and a thread that runs solves submitted at
 * any time, as a continuous batch (the smallest resident solves take
 * several steps per server step, so that large ones do not pace them):
 *   - a submitted solve waits in a FIFO queue until a region of the arena
 *     large enough for its f, h and stage buffers is free, then joins the
 *     resident set at the next step boundary;
 *   - every step advances all resident solves with one launch per phase
 *     over their packed tile lists (the launches of lbm_batch_step);
 *   - at each step boundary finished, failed and cancelled solves leave,
 *     queued ones join, and the tile lists are repacked; when the arena is
 *     fragmented the resident regions are moved together first;
 *   - a finished solve's rho, ux, uy, T, p are copied to host memory by a
 *     second thread and its region is freed for the queue.
 * Each solve runs the same per-node arithmetic as alone in a batch of one
 * with the same precision and tile shape, so its result does not depend on
 * what else was resident.  The step count of a solve is its derived
 * nsteps (steps, tt_tref or tt_time of lbm_config); a residual tolerance
 * alone is not accepted.  A solve whose state fails a device check
 * (equilibrium mass, non-finite values) is removed within status_poll_steps
 * steps and completes with that status; the others are not affected. */
typedef struct lbm_server lbm_server;

typedef struct lbm_server_options {
    int precision;        /* LBM_PREC_F64 / LBM_PREC_F32, all solves */
    int tile_x, tile_y;   /* 0: 32 x 8 */
    size_t arena_bytes;   /* device memory for resident solves; 0: hbm_fraction of the free memory */
    double hbm_fraction;  /* used when arena_bytes is 0; 0: 0.6 */
    int max_resident;     /* most solves resident at once; 0: 1024 */
    int max_queued;       /* most solves waiting; 0: no limit */
    int use_graph;        /* replay steps from a CUDA graph while the resident set is unchanged */
    int status_poll_steps;/* steps between reads of the device status words; 0: 32 */
    int fast_lane_steps;  /* steps per server step of the smallest solves
                             (each at most 1/16 of the resident nodes, together
                             at most 1/4); 0: 4; 1: every solve takes one */
} lbm_server_options;

enum { LBM_REQ_QUEUED = 0, LBM_REQ_RESIDENT = 1, LBM_REQ_DONE = 2 };

typedef struct lbm_request_info {
    long long id;
    int Nx, Ny;
    int steps_total, steps_done;
    int state;           /* LBM_REQ_* */
    lbm_status status;   /* of the finished solve */
    double t_submit, t_admit, t_done;    /* seconds since the server was created */
    long long step_admit, step_done;     /* server step count at admission / retirement */
} lbm_request_info;

typedef struct lbm_server_stats {
    long long submitted, admitted, completed, failed, cancelled;
    long long steps;            /* server steps (each advances every resident solve) */
    long long lattice_updates;  /* sum over steps of the resident nodes */
    long long repacks, compactions, graph_captures;
    int resident, queued;
    long long arena_nodes, arena_nodes_used;
    size_t arena_bytes;
    double busy_seconds;        /* wall time with at least one resident solve */
    double uptime_seconds;
    /* host time of the loop thread by part: step boundaries (retire, admit,
     * repack, initialise), graph captures, and steps enqueued launch by
     * launch (no graph yet) or replayed from a graph */
    double boundary_seconds, capture_seconds;
    long long steps_eager, steps_graph;
} lbm_server_stats;

LBM_API lbm_status lbm_server_create(const lbm_server_options *opt, lbm_server **out);
/* Queue one solve (the arguments of lbm_create).  The host-side set-up
 * (derived parameters, node flags, tiles) runs on the calling thread.
 * LBM_ERR_NOMEM: it can never fit the arena; LBM_ERR_BUSY: the queue is full. */
LBM_API lbm_status lbm_server_submit(lbm_server *s, const lbm_config *cfg, const lbm_init *init, long long *id);
/* Wait until the solve is done (timeout_s < 0: no limit); LBM_ERR_TIMEOUT
 * when the time ran out first. */
LBM_API lbm_status lbm_server_wait(lbm_server *s, long long id, double timeout_s);
/* Wait for the next solve to finish that no earlier call returned. */
LBM_API lbm_status lbm_server_wait_any(lbm_server *s, double timeout_s, long long *id);
LBM_API lbm_status lbm_server_info(lbm_server *s, long long id, lbm_request_info *info);
/* Copy a finished solve's fields ([x*Ny + y], any pointer may be NULL) and
 * return its status; LBM_ERR_BUSY while it is not done. */
LBM_API lbm_status lbm_server_result(lbm_server *s, long long id, double *rho, double *ux, double *uy, double *T,
                                     double *p);
/* Cancel a queued or resident solve; it completes with LBM_ERR_CANCELLED. */
LBM_API lbm_status lbm_server_cancel(lbm_server *s, long long id);
/* Forget a solve and its result (cancelling it when not done). */
LBM_API lbm_status lbm_server_release(lbm_server *s, long long id);
LBM_API lbm_status lbm_server_get_stats(lbm_server *s, lbm_server_stats *st);
/* Stop the threads; solves not done are dropped. */
LBM_API void lbm_server_destroy(lbm_server *s);

/* ------------------------------------------------------------ self-test
 * No counterpart in the reference.  Exercises the bounded wait that every
 * device-side wait of the stencil kernels uses (an mbarrier polled a fixed
 * number of times): one block waits on a barrier that expects one arrival.
 * arrive = 0: nothing arrives, the wait gives up, the block records the
 * timeout bit and exits, and the call returns LBM_ERR_TIMEOUT with the
 * device still usable.  arrive = 1: the arrival comes first and the call
 * returns LBM_OK.  Nothing traps or faults either way. */
LBM_API lbm_status lbm_selftest_bounded_wait(int arrive);

/* ------------------------------------------------- allocation-free step
 * No counterpart in the reference.  For callers that cannot call
 * cudaMalloc: an application that owns all device memory through its own
 * pool or arena, or one whose device-memory budget is already spoken for,
 * so that an allocation by a library it calls would fail or break its
 * accounting.  It advances one
 * domain n_steps steps on the FP64 path with every scratch buffer taken
 * from a fixed array that the library reserves on each GPU it is loaded on
 * (about 10.7 MB, held until the process exits) -- nothing is allocated.
 *
 *   cellType  host array [Nx*Ny], the cell type (0 fluid, 1 permanent,
 *             2 solid) of each node in [x*Ny + y] order; any other value
 *             returns LBM_ERR_INVALID before any device work
 *   d_f, d_h  device arrays [(x*Ny + y)*13 + i] (the reference's f_G, h_G
 *             layout) holding the state; updated in place
 *   stream    cudaStream_t to run on (NULL: the default stream); the call
 *             returns after the stream has finished the work
 *
 * Limits: uniform cells only (dx_array/dy_array must be NULL) and
 * Ny * roundup(Nx, 32) <= LBM_NOALLOC_MAX_NODES, e.g. 128 x 128; larger
 * domains return LBM_ERR_INVALID.  The first call on a device looks up the
 * array's device address and sets kernel attributes on that device: make
 * that first call before any stream capture on it.  All calls share the one
 * array and each overwrites what the previous call left in it, so calls that
 * overlap on the GPU (other threads, other streams) race; serialise them.
 * The equilibria of moving walls are whatever d_f, d_h hold at solid nodes. */
#define LBM_NOALLOC_MAX_NODES 16384
LBM_API lbm_status lbm_step_noalloc(const lbm_config *cfg, int Nx, int Ny, const int *cellType, double *d_f,
                                    double *d_h, int n_steps, void *stream);

#ifdef __cplusplus
}
#endif
#endif
