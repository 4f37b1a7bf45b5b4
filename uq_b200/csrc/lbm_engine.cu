// Host engine and C ABI (include/uq_lbm.h) of the D2Q13 thermal LBM step.
//
// A Batch holds any number of samples (a single lbm_handle is a batch of
// one).  Their state lives on the device as structure-of-arrays planes; one
// step is the phase sequence described in lbm_kernels.cu, launched over
// packed tile lists and, when enabled, replayed from a captured CUDA graph.
// Derived run parameters follow cpuLBM::refineInput / setupVars
// (CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp:283-450) and the step driver
// follows runSimStep (main.cpp:32-112).
#include "lbm_common.h"
#include "lbm_hdf5.h"
#include "lbm_mat.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace uqlbm {

thread_local std::string g_last_error;

static int host_bc_index(const HostSample &s, int i, int pm, int axis, int &mir)
{
    i += pm;
    mir = 0;
    const int N = axis == 0 ? s.nx : s.ny;
    if (i < 0) {
        if (s.flags & (axis == 0 ? SF_PERX : SF_PERY)) i = N + i;
        else if (s.flags & (axis == 0 ? SF_MIRW : SF_MIRS)) { i = -i - 1; mir = 1; }
        else i = 0;
    } else if (i > N - 1) {
        if (s.flags & (axis == 0 ? SF_PERX : SF_PERY)) i = i - N;
        else if (s.flags & (axis == 0 ? SF_MIRE : SF_MIRN)) { i = 2 * N - i - 1; mir = 1; }
        else i = N - 1;
    }
    return i;
}

// refineInput (cpuLBM.cpp:283-358) + setupVars (cpuLBM.cpp:360-450) for the
// scalar run parameters.  min_spacing > 0 replaces min(dx, dy) in the CFL
// time step (non-uniform cells, as LBM.py:215-216 does).
void derive_scalars(const lbm_config &c, int Nx, int Ny, double min_spacing, ScalarParams &s)
{
    if (Nx < 3 || Ny < 3) throw LbmError(LBM_ERR_INVALID, "Nx and Ny must be at least 3");
    if (c.RKMETHOD < 0 || c.RKMETHOD > 3) throw LbmError(LBM_ERR_INVALID, "RKMETHOD must be 0..3");
    if (c.FMETHOD < 0 || c.FMETHOD > 1) throw LbmError(LBM_ERR_INVALID, "FMETHOD must be 0 (NND) or 1 (WENO5)");
    if (!(c.gamma > 1.0) || !(c.R > 0.0)) throw LbmError(LBM_ERR_INVALID, "gamma must exceed 1 and R be positive");
    if (c.mu_model < 0 || c.mu_model > 2) throw LbmError(LBM_ERR_INVALID, "mu_model must be 0, 1 or 2");
    s.mu_model = c.mu_model;
    s.upsilon = c.upsilon;
    s.S_v = c.S_v;
    s.rk = c.RKMETHOD;
    s.fm = c.FMETHOD;
    s.flags = (c.periodicX > 0 ? SF_PERX : 0) | (c.periodicY > 0 ? SF_PERY : 0) | (c.mirrorNorth > 0 ? SF_MIRN : 0) |
              (c.mirrorSouth > 0 ? SF_MIRS : 0) | (c.mirrorEast > 0 ? SF_MIRE : 0) | (c.mirrorWest > 0 ? SF_MIRW : 0);
    s.R = c.R;
    s.mu = c.mu;
    s.Pr = c.Pr;
    s.tol = c.tol;
    double dx = c.dx, dy = c.dy, Lx = c.Lx, Ly = c.Ly;
    if (dx == 0) dx = Lx / ((double)Nx - 1); else Lx = dx * (Nx - 1);
    if (dy == 0 && Ly != 0) dy = Ly / ((double)Ny - 1);
    else if (dy == 0 && Ly == 0) { dy = dx; Ly = dy * (Ny - 1); }
    else Ly = dy * (Ny - 1);
    s.dx = dx;
    s.dy = dy;
    double rho_ref = c.rho_ref, p_ref = c.p_ref, T_ref = c.T_ref;
    if (rho_ref == 0) rho_ref = p_ref / (c.R * T_ref);
    else if (p_ref == 0) p_ref = rho_ref * c.R * T_ref;
    else if (T_ref == 0) T_ref = p_ref / (rho_ref * c.R);
    s.rho_ref = rho_ref;
    s.T_ref = T_ref;
    s.b = 2 / (c.gamma - 1);
    s.gamma = c.gamma;
    s.K = s.b - 2;
    s.Tc = c.Tc_Tref * T_ref;
    const double tau_ref = c.mu / p_ref;
    const double u_ref = std::sqrt(c.R * T_ref);
    const double t_ref = std::max(Lx, Ly) / u_ref;
    s.c = std::sqrt(c.R * s.Tc);
    const double mind = min_spacing > 0 ? min_spacing : std::min(dx, dy);
    s.dt = c.dtau == 0 ? (c.CFL * mind) / (2 * s.c) : c.dtau * tau_ref;
    if (!(s.dt > 0) || !std::isfinite(s.dt)) throw LbmError(LBM_ERR_INVALID, "derived dt is not positive");
    double ttotal = 0;
    int need = 0;
    s.nsteps = 0;
    if (c.tt_tref > 0) { ttotal = c.tt_tref * t_ref; need = 1; }
    else if (c.tt_time > 0) { ttotal = c.tt_time; need = 1; }
    else if (c.steps > 0) s.nsteps = c.steps;
    else if (c.tol > 0) s.nsteps = 0;
    if (need) s.nsteps = (int)std::ceil(ttotal / s.dt);
}

HostSample derive(const lbm_config &c, const lbm_init &in)
{
    HostSample s;
    if (!in.bndArray || !in.cellType || !in.density || !in.pressure || !in.temp || !in.velocityX || !in.velocityY ||
        in.numProps < 1)
        throw LbmError(LBM_ERR_INVALID, "lbm_init tables missing");
    const int Nx = in.Nx, Ny = in.Ny;
    if (Nx < 3 || Ny < 3) throw LbmError(LBM_ERR_INVALID, "Nx and Ny must be at least 3");
    // the kernels address a sample's 26 planes with 32-bit offsets
    if ((long long)Ny * (((long long)Nx + 31) / 32 * 32) > (1ll << 26))
        throw LbmError(LBM_ERR_INVALID, "sample too large: Ny * roundup(Nx, 32) must be at most 2^26 nodes");
    s.nx = Nx;
    s.ny = Ny;
    // cell widths first: the CFL step uses their minimum
    ScalarParams sc;
    {
        lbm_config c0 = c;
        c0.dx_array = nullptr;
        c0.dy_array = nullptr;
        ScalarParams tmp;
        derive_scalars(c0, Nx, Ny, 0.0, tmp);  // completes dx, dy
        s.dx.assign(Nx, tmp.dx);
        s.dy.assign(Ny, tmp.dy);
        double mind = 0.0;
        if (c.dx_array || c.dy_array) {
            mind = INFINITY;
            for (int x = 0; x < Nx; ++x) {
                if (c.dx_array) s.dx[x] = c.dx_array[x];
                mind = std::min(mind, s.dx[x]);
            }
            for (int y = 0; y < Ny; ++y) {
                if (c.dy_array) s.dy[y] = c.dy_array[y];
                mind = std::min(mind, s.dy[y]);
            }
        }
        derive_scalars(c, Nx, Ny, mind, sc);
    }
    s.rk = sc.rk;
    s.fm = sc.fm;
    s.flags = sc.flags;
    s.R = sc.R;
    s.mu = sc.mu;
    s.Pr = sc.Pr;
    s.tol = sc.tol;
    s.rho_ref = sc.rho_ref;
    s.T_ref = sc.T_ref;
    s.b = sc.b;
    s.gamma = sc.gamma;
    s.K = sc.K;
    s.Tc = sc.Tc;
    s.c = sc.c;
    s.dt = sc.dt;
    s.nsteps = sc.nsteps;
    s.mu_model = sc.mu_model;
    s.upsilon = sc.upsilon;
    s.S_v = sc.S_v;

    // property tables completed as refineInput does; per-node initial state
    const int np = in.numProps;
    std::vector<double> prho(np), pT(np);
    for (int r = 0; r < np; ++r) {
        double rho = in.density[r], p = in.pressure[r], T = in.temp[r];
        if (rho == 0) rho = p / (c.R * T);
        else if (p == 0) p = rho * c.R * T;
        else if (T == 0) T = p / (rho * c.R);
        prho[r] = rho;
        pT[r] = T;
        if (in.cellType[r] < 0 || in.cellType[r] > 2) throw LbmError(LBM_ERR_INVALID, "cellType must be 0, 1 or 2");
    }
    const size_t N = (size_t)Nx * Ny;
    s.type.resize(N);
    s.rho0.resize(N);
    s.ux0.resize(N);
    s.uy0.resize(N);
    s.T0.resize(N);
    for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y) {
            const int id = in.bndArray[(size_t)x * Ny + y];
            if (id < 0 || id >= np) throw LbmError(LBM_ERR_INVALID, "bndArray holds an unknown property id");
            const size_t k = (size_t)y * Nx + x;
            s.type[k] = (uint8_t)in.cellType[id];
            s.rho0[k] = prho[id];
            s.ux0[k] = in.velocityX[id];
            s.uy0[k] = in.velocityY[id];
            s.T0[k] = pT[id];
        }
    return s;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda needed).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        CU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p)
            throw LbmError(LBM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

void check_tile_shape(int x, int y)
{
    if (x * y > 256 || x < 4 || y < 1 || x * y % 32 != 0 || x % 4 != 0 || y + 6 > 256)
        throw LbmError(LBM_ERR_INVALID, "tile must hold a multiple of 32 and at most 256 nodes, width a multiple of 4");
}

// Sample parameters, rest state, node flags, wall list and spacing tables
// of one sample; layout per sample: 26 planes of ny x pitch, pitch a
// multiple of 32.
void prepare_sample(const HostSample &h, int prec, PreparedSample &out)
{
    SampleParams &p = out.p;
    p = SampleParams{};
    p.nx = h.nx;
    p.ny = h.ny;
    // x-periodic samples wide enough for their images keep ghost columns
    p.gx = (h.flags & SF_PERX) && h.nx >= 2 * GHOST_X ? GHOST_X : 0;
    p.pitch = round_up(h.nx + 2 * p.gx, 32);
    p.flags = h.flags;
    p.rk = h.rk;
    p.fm = h.fm;
    p.plane = (long long)p.ny * p.pitch;
    p.R = h.R;
    p.bR = h.b * h.R;
    p.K = h.K;
    p.Tc = h.Tc;
    p.inv_sRTc = 1.0 / std::sqrt(h.R * h.Tc);
    p.RTc = h.R * h.Tc;
    p.mu = h.mu;
    p.Pr = h.Pr;
    p.dt = h.dt;
    p.c = h.c;
    p.inv_mu = 1.0 / h.mu;
    p.two_over_bR = 2.0 / (h.b * h.R);
    p.visc = h.mu_model;
    p.visc_exp = h.mu_model == 1 ? 0.5 + h.upsilon : 1.5;
    p.visc_S = h.S_v;
    p.visc_T = h.T_ref;
    {
        // FP32 WENO5 weight form: the division-free form spans (eps + b)^4,
        // which stays in the float range when |e| c times the stored values
        // is moderate.  Bound those values by the initial densities and the
        // energy scale rho R Tc (times generous factors for the polynomials).
        double rho_max = 0.0;
        for (double r : h.rho0) rho_max = std::max(rho_max, std::fabs(r));
        const double scale = 2.0 * h.c * rho_max * std::max(2.0, 10.0 * h.R * h.Tc);
        p.wide = (prec == LBM_PREC_F32 && !(scale <= 100.0)) ? 1 : 0;
    }
    // rest state of the stored deviations (FP32 path only)
    if (prec == LBM_PREC_F32) {
        p.rho0 = (h.rho_ref > 0 && std::isfinite(h.rho_ref)) ? h.rho_ref : 1.0;
        p.T0n = (h.T_ref > 0 && std::isfinite(h.T_ref)) ? h.T_ref / h.Tc : 1.0;
    } else {
        p.rho0 = 0.0;
        p.T0n = 1.0;
    }
    {
        // equilibria at rest per family (the polynomials at u = v = 0)
        const double T = p.T0n, K = h.K;
        const double P0[4] = {1 + 2.5 * T * T - 2.5 * T, -T * T + 2.0 * T / 3.0, 0.25 * T * T,
                              0.125 * T * T - T / 24.0};
        const double Q0[4] = {T * T * T * (1.25 * K + 20.0 / 3.0) + T * T * (-1.25 * K - 5) + T * (0.5 * K + 1),
                              T * T * T * (-0.5 * K - 8.0 / 3.0) + T * T * (K / 3.0 + 4.0 / 3.0),
                              T * T * T * (K / 8.0 + 2.0 / 3.0),
                              T * T * T * (K / 16.0 + 1.0 / 3.0) + T * T * (-K / 48.0 - 1.0 / 12.0)};
        double sh = 0;
        for (int i = 0; i < NQ; ++i) {
            const int fam = i == 0 ? 0 : (i <= 4 ? 1 : (i <= 8 ? 2 : 3));
            out.fref[i] = p.rho0 * P0[fam];
        }
        for (int i = 0; i < NQ; ++i) {
            const int fam = i == 0 ? 0 : (i <= 4 ? 1 : (i <= 8 ? 2 : 3));
            const double hv = p.rho0 * h.R * h.Tc * Q0[fam];
            out.fref[NQ + i] = hv;
            sh += hv;
        }
        p.shref = sh;
    }
    out.tdx.resize(h.nx);
    out.dx.resize(h.nx);
    out.tdy.resize(h.ny);
    out.dy.resize(h.ny);
    for (int x = 0; x < h.nx; ++x) { out.tdx[x] = h.dt / h.dx[x]; out.dx[x] = h.dx[x]; }
    for (int y = 0; y < h.ny; ++y) { out.tdy[y] = h.dt / h.dy[y]; out.dy[y] = h.dy[y]; }
    // node flags
    out.flags.assign((size_t)p.plane, 0);
    int m;
    for (int y = 0; y < h.ny; ++y)
        for (int x = 0; x < h.nx; ++x) {
            uint8_t fl = h.type[(size_t)y * h.nx + x];
            for (int d = -2; d <= 2; ++d) {
                const int xr = host_bc_index(h, x, d, 0, m);
                const int yr = host_bc_index(h, y, d, 1, m);
                if (h.type[(size_t)y * h.nx + xr] == 2) fl |= NF_SOLX;
                if (h.type[(size_t)yr * h.nx + x] == 2) fl |= NF_SOLY;
            }
            if (x < 2 || x > h.nx - 3) fl |= (h.flags & SF_PERX) ? NF_WRPX : NF_EDGX;
            if (y < 2 || y > h.ny - 3) fl |= (h.flags & SF_PERY) ? NF_WRPY : NF_EDGY;
            out.flags[(size_t)y * p.pitch + x] = fl;
        }
    // wall nodes: solid with a non-solid 4-neighbour (wallFluxes' test)
    static const int wx[4] = {-1, 1, 0, 0}, wy[4] = {0, 0, -1, 1};
    out.walls.clear();
    for (int y = 0; y < h.ny; ++y)
        for (int x = 0; x < h.nx; ++x) {
            if (h.type[(size_t)y * h.nx + x] != 2) continue;
            bool adj = false;
            for (int j = 0; j < 4; ++j) {
                const int xm = host_bc_index(h, x, wx[j], 0, m);
                const int ym = host_bc_index(h, y, wy[j], 1, m);
                if (h.type[(size_t)ym * h.nx + xm] < 2) adj = true;
            }
            if (adj) out.walls.push_back(WallNode{0, x, y, 0});
        }
}

// Tiles of one sample, each flagged simple when it and its 3-node halo lie
// inside the domain and hold only plain fluid nodes.
void cut_tiles(const uint8_t *flags, int pitch, int nx, int ny, int tx, int ty, int sflags, int gx, int sample,
               std::vector<Tile> &out)
{
    const bool px = (sflags & SF_PERX) != 0, py = (sflags & SF_PERY) != 0;
    for (int y0 = 0; y0 < ny; y0 += ty)
        for (int x0 = 0; x0 < nx; x0 += tx) {
            int gid = (int)out.size();
            const bool in_x = x0 >= 3 && x0 + tx + 3 <= nx, in_y = y0 >= 3 && y0 + ty + 3 <= ny;
            if (in_x && in_y) {
                bool simple = true;
                for (int y = y0 - 3; y < y0 + ty + 3 && simple; ++y)
                    for (int x = x0 - 3; x < x0 + tx + 3; ++x)
                        if (flags[(long long)y * pitch + x] != 0) { simple = false; break; }
                if (simple) gid |= TILE_SIMPLE;
            } else if ((in_x || px) && (in_y || py) && x0 + tx <= nx && y0 + ty <= ny) {
                // a full tile whose halo crosses a periodic edge: plain fluid
                // everywhere in the halo (periodic images included), and no
                // flag but the stencil-wraps bits
                bool wrap = true;
                for (int y = y0 - 3; y < y0 + ty + 3 && wrap; ++y)
                    for (int x = x0 - 3; x < x0 + tx + 3; ++x) {
                        const int xw = ((x % nx) + nx) % nx, yw = ((y % ny) + ny) % ny;
                        if (flags[(long long)yw * pitch + xw] & ~(NF_WRPX | NF_WRPY)) { wrap = false; break; }
                    }
                // crossing only the x edges of a sample with ghost columns,
                // the staged box needs nothing more: a simple tile
                if (wrap) gid |= gx && in_y ? TILE_SIMPLE : TILE_WRAP;
            }
            out.push_back(Tile{sample, x0, y0, gid});
        }
}

// TMA descriptors of a sample, each over the 26 planes as a 3D tensor
// (x, y, plane): stage buffers 2 and 3 with the flux kernels' staged halo
// box (one plane), and the state with the tile's own nodes over
// PREFETCH_PLANES planes (the update's reads of f or of h).
void encode_stage_maps(int prec, const SampleParams &p, unsigned char *state, unsigned char *buf2,
                       unsigned char *buf3, int tx, int ty, CUtensorMap *maps)
{
    auto enc = tensor_map_encoder();
    const size_t es = prec == LBM_PREC_F64 ? 8 : 4;
    for (int b = 0; b < MAPS_PER_SAMPLE; ++b) {
        // with ghost columns the tensor starts at the left ghosts and spans
        // the pitch (boxes at the x edges then read the images); else it is
        // the domain and boxes read zeros beyond it
        unsigned char *base = (b == 0 ? buf2 : b == 1 ? buf3 : state) + (size_t)(p.state_off - p.gx) * es;
        cuuint64_t dims[3] = {(cuuint64_t)(p.gx ? p.pitch : p.nx), (cuuint64_t)p.ny, (cuuint64_t)NPL};
        cuuint64_t strides[2] = {(cuuint64_t)p.pitch * es, (cuuint64_t)p.plane * es};
        cuuint32_t halo[3] = {(cuuint32_t)(tx + 8), (cuuint32_t)(ty + 6), 1};
        cuuint32_t own[3] = {(cuuint32_t)tx, (cuuint32_t)ty, (cuuint32_t)PREFETCH_PLANES};
        cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = enc(&maps[b], prec == LBM_PREC_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         3, base, dims, strides, b < 2 ? halo : own, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw LbmError(LBM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
}

}  // namespace uqlbm

using namespace uqlbm;

struct lbm_batch {
    int prec = LBM_PREC_F64;
    // default tile: the shape the stencil kernels are compiled for, the
    // fastest on the 512-sample UQ ensemble (lbm_batch_autotune re-measures
    // for a given batch)
    int tx = TILE_CX, ty = TILE_CY;
    std::vector<uint8_t> flags_host;
    bool use_graph = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<HostSample> hs;
    std::vector<SampleParams> sp;
    std::vector<Tile> tiles_all, tiles_rk3;
    std::vector<Tile> tiles_by_rk[4], tiles_flux[4];  // by RKMETHOD: sample order; by kind
    // leading simple tiles and the wrap tiles after them in tiles_flux, tiles_rk3
    int ns_by_rk[4] = {0, 0, 0, 0}, nw_by_rk[4] = {0, 0, 0, 0}, ns_rk3 = 0, nw_rk3 = 0;
    std::vector<WallNode> walls_all, walls_rk3;
    std::vector<int> tile_first, tile_count;
    long long total_state = 0, total_nodes = 0, lattice_nodes = 0;
    size_t max_nodes = 0;
    bool any_rk3 = false, any_other = false, any_ghost = false;

    DevBuf<unsigned char> state, buf2, buf3, alpha;  // typed by precision
    DevBuf<uint8_t> nflags;
    DevBuf<double> told, partial, residual, tdx, tdy, dxv, dyv, scratch;
    DevBuf<int> status, d_tile_first, d_tile_count;
    DevBuf<SampleParams> d_sp;
    DevBuf<Tile> d_tiles_all, d_tiles_rk3;
    DevBuf<Tile> d_tiles_by_rk[4], d_tiles_flux[4];
    DevBuf<WallNode> d_walls_all, d_walls_rk3;
    DevBuf<CUtensorMap> d_maps;
    DevBuf<double> d_fref;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [want_residual]
    std::vector<int> host_status;
    std::vector<double> host_residual;

    size_t elem() const { return prec == LBM_PREC_F64 ? 8 : 4; }

    ~lbm_batch()
    {
        for (auto &g : graph)
            if (g) cudaGraphExecDestroy(g);
        if (stream) cudaStreamDestroy(stream);
    }

    // Tile lists for the current tile shape: every sample cut into tx x ty
    // tiles, each flagged simple when it and its 3-node halo lie inside the
    // domain and hold only plain fluid nodes.
    void make_tiles()
    {
        tiles_all.clear();
        tiles_rk3.clear();
        for (auto &v : tiles_by_rk) v.clear();
        tile_first.clear();
        tile_count.clear();
        for (size_t k = 0; k < hs.size(); ++k) {
            const HostSample &h = hs[k];
            SampleParams &p = sp[k];
            p.first_tile = (int)tiles_all.size();
            cut_tiles(flags_host.data() + p.node_off, p.pitch, h.nx, h.ny, tx, ty, p.flags, p.gx, (int)k, tiles_all);
            p.ntile = (int)tiles_all.size() - p.first_tile;
            for (int t = p.first_tile; t < p.first_tile + p.ntile; ++t) {
                tiles_by_rk[h.rk].push_back(tiles_all[t]);
                if (h.rk == 1) tiles_rk3.push_back(tiles_all[t]);
            }
            tile_first.push_back(p.first_tile);
            tile_count.push_back(p.ntile);
        }
        // the stencil phases take the tiles by kind (one kernel per kind);
        // the pointwise phase keeps the sample order
        for (int m = 0; m < 4; ++m) {
            tiles_flux[m] = tiles_by_rk[m];
            order_by_kind(tiles_flux[m], ns_by_rk[m], nw_by_rk[m]);
        }
        order_by_kind(tiles_rk3, ns_rk3, nw_rk3);
    }

    void upload_tiles()
    {
        d_sp.upload(sp, stream);
        d_tiles_all.upload(tiles_all, stream);
        d_tiles_rk3.upload(tiles_rk3, stream);
        for (int m = 0; m < 4; ++m) {
            d_tiles_by_rk[m].upload(tiles_by_rk[m], stream);
            d_tiles_flux[m].upload(tiles_flux[m], stream);
        }
        d_tile_first.upload(tile_first, stream);
        d_tile_count.upload(tile_count, stream);
        partial.alloc(tiles_all.size());
    }

    // TMA descriptors: per sample and stage buffer, the 26 planes as a 3D
    // tensor (x, y, plane) with the staged halo box of the flux kernels
    void make_maps()
    {
        const int n = (int)hs.size();
        std::vector<CUtensorMap> maps(MAPS_PER_SAMPLE * n);
        for (int k = 0; k < n; ++k)
            encode_stage_maps(prec, sp[k], state.p, buf2.p, buf3.p, tx, ty, &maps[MAPS_PER_SAMPLE * k]);
        d_maps.upload(maps, stream);
    }

    static void check_tile(int x, int y) { check_tile_shape(x, y); }

    void drop_graphs()
    {
        for (auto &g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    // switch the tile shape: new tile lists and TMA boxes, no state change
    void retile(int ntx, int nty)
    {
        check_tile(ntx, nty);
        CU(cudaStreamSynchronize(stream));
        tx = ntx;
        ty = nty;
        make_tiles();
        upload_tiles();
        make_maps();
        drop_graphs();
        CU(cudaStreamSynchronize(stream));
    }

    // Autotuner: time `steps` steps for each candidate tile shape (CUDA
    // events, no graph) starting from the same saved state, keep the fastest
    // and restore the state, so tuning leaves the results unchanged.
    void autotune(const int *cand, int ncand, int steps, int *chosen, double *ms_out)
    {
        if (ncand < 1 || !cand || steps < 1) throw LbmError(LBM_ERR_INVALID, "no tile candidates");
        for (int c = 0; c < ncand; ++c) check_tile(cand[2 * c], cand[2 * c + 1]);
        DevBuf<unsigned char> save;
        save.alloc(state.n);
        CU(cudaMemcpyAsync(save.p, state.p, state.n, cudaMemcpyDeviceToDevice, stream));
        std::vector<int> keep_status(host_status);
        std::vector<HostSample> keep_hs_steps(0);
        double best = INFINITY;
        int bx = tx, by = ty;
        for (int c = 0; c < ncand; ++c) {
            retile(cand[2 * c], cand[2 * c + 1]);
            CU(cudaMemcpyAsync(state.p, save.p, state.n, cudaMemcpyDeviceToDevice, stream));
            double ph[6];
            profile(1, ph, 6);  // warm-up (module load, caches)
            CU(cudaMemcpyAsync(state.p, save.p, state.n, cudaMemcpyDeviceToDevice, stream));
            profile(steps, ph, 6);
            double tot = 0;
            for (double v : ph) tot += v;
            if (ms_out) ms_out[c] = tot;
            if (tot < best) { best = tot; bx = cand[2 * c]; by = cand[2 * c + 1]; }
        }
        retile(bx, by);
        CU(cudaMemcpyAsync(state.p, save.p, state.n, cudaMemcpyDeviceToDevice, stream));
        CU(cudaMemsetAsync(status.p, 0, hs.size() * sizeof(int), stream));
        CU(cudaStreamSynchronize(stream));
        host_status = keep_status;
        if (chosen) { chosen[0] = bx; chosen[1] = by; }
    }

    template <class S>
    KArgs<S> args(int want_res) const
    {
        KArgs<S> a{};
        a.samples = d_sp.p;
        a.tiles = d_tiles_all.p;
        a.ntiles = (int)tiles_all.size();
        a.tx = tx;
        a.ty = ty;
        a.state = reinterpret_cast<S *>(state.p);
        a.buf2 = reinterpret_cast<S *>(buf2.p);
        a.buf3 = reinterpret_cast<S *>(buf3.p);
        a.nflags = nflags.p;
        a.alpha_raw = alpha.p;
        a.told = told.p;
        a.partial = partial.p;
        a.status = status.p;
        a.tdx = tdx.p;
        a.tdy = tdy.p;
        a.dxv = dxv.p;
        a.dyv = dyv.p;
        a.tmaps = d_maps.p;
        a.fref = d_fref.p;
        a.want_residual = want_res;
        a.eq_tol = 1e-6;
        return a;
    }

    void build(int n, const lbm_config *cfgs, const lbm_init *inits, const lbm_batch_options *opt)
    {
        if (n < 1 || !cfgs || !inits) throw LbmError(LBM_ERR_INVALID, "empty batch");
        prec = opt ? opt->precision : LBM_PREC_F64;
        if (prec != LBM_PREC_F64 && prec != LBM_PREC_F32) throw LbmError(LBM_ERR_INVALID, "unknown precision");
        if (opt && opt->tile_x > 0) tx = opt->tile_x;
        if (opt && opt->tile_y > 0) ty = opt->tile_y;
        check_tile(tx, ty);
        use_graph = opt ? opt->use_graph != 0 : true;
        hs.reserve(n);
        for (int k = 0; k < n; ++k) hs.push_back(derive(cfgs[k], inits[k]));
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
            throw LbmError(LBM_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
        CU(cudaGetDevice(&device));
        CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

        // layout: per sample 26 planes of ny x pitch, packed one after another
        std::vector<double> v_tdx, v_tdy, v_dx, v_dy, fref_host;
        std::vector<uint8_t> flags;
        long long state_off = 0, node_off = 0;
        PreparedSample ps;
        for (int k = 0; k < n; ++k) {
            const HostSample &h = hs[k];
            prepare_sample(h, prec, ps);
            SampleParams p = ps.p;
            p.state_off = state_off + (p.gx ? GHOST_SLACK : 0);  // the first row's left ghosts before it
            p.node_off = node_off;
            p.xoff = (int)v_tdx.size();
            p.yoff = (int)v_tdy.size();
            fref_host.insert(fref_host.end(), ps.fref, ps.fref + NPL);
            v_tdx.insert(v_tdx.end(), ps.tdx.begin(), ps.tdx.end());
            v_tdy.insert(v_tdy.end(), ps.tdy.begin(), ps.tdy.end());
            v_dx.insert(v_dx.end(), ps.dx.begin(), ps.dx.end());
            v_dy.insert(v_dy.end(), ps.dy.begin(), ps.dy.end());
            flags.insert(flags.end(), ps.flags.begin(), ps.flags.end());
            for (WallNode w : ps.walls) {
                w.sample = k;
                walls_all.push_back(w);
                if (h.rk == 1) walls_rk3.push_back(w);
            }
            state_off += NPL * p.plane + (p.gx ? GHOST_SLACK : 0);
            node_off += p.plane;
            lattice_nodes += (long long)h.nx * h.ny;
            max_nodes = std::max(max_nodes, (size_t)h.nx * h.ny);
            if (h.rk == 1) any_rk3 = true; else any_other = true;
            if (p.gx) any_ghost = true;
            sp.push_back(p);
        }
        total_state = state_off;
        total_nodes = node_off;
        flags_host.swap(flags);
        make_tiles();

        state.alloc(total_state * elem());
        buf2.alloc(total_state * elem());
        buf3.alloc(total_state * elem());
        alpha.alloc(total_nodes * elem());
        CU(cudaMemsetAsync(state.p, 0, state.n, stream));
        CU(cudaMemsetAsync(buf2.p, 0, buf2.n, stream));
        CU(cudaMemsetAsync(buf3.p, 0, buf3.n, stream));
        CU(cudaMemsetAsync(alpha.p, 0, alpha.n, stream));
        nflags.upload(flags_host, stream);
        told.alloc(total_nodes);
        residual.alloc(n);
        status.alloc(n);
        CU(cudaMemsetAsync(status.p, 0, n * sizeof(int), stream));
        tdx.upload(v_tdx, stream);
        tdy.upload(v_tdy, stream);
        dxv.upload(v_dx, stream);
        dyv.upload(v_dy, stream);
        d_fref.upload(fref_host, stream);
        upload_tiles();
        d_walls_all.upload(walls_all, stream);
        d_walls_rk3.upload(walls_rk3, stream);
        scratch.alloc(std::max<size_t>(5 * max_nodes, 2 * 13 * max_nodes));
        host_status.assign(n, 0);
        host_residual.assign(n, 1.0);

        make_maps();
        if (prec == LBM_PREC_F64) CU((prepare_kernels<double, double>()));
        else CU((prepare_kernels<float, float>()));

        // initial state (initialiseFunctions, cpuLBM.cpp:846-875)
        std::vector<double> r0(total_nodes, 1.0), u0(total_nodes, 0.0), v0(total_nodes, 0.0), T0(total_nodes, 1.0);
        for (int k = 0; k < n; ++k) {
            const HostSample &h = hs[k];
            for (int y = 0; y < h.ny; ++y)
                for (int x = 0; x < h.nx; ++x) {
                    const size_t src = (size_t)y * h.nx + x;
                    const long long dst = sp[k].node_off + (long long)y * sp[k].pitch + x;
                    r0[dst] = h.rho0[src];
                    u0[dst] = h.ux0[src];
                    v0[dst] = h.uy0[src];
                    T0[dst] = h.T0[src];
                }
        }
        DevBuf<double> dr, du, dv, dT;
        dr.upload(r0, stream);
        du.upload(u0, stream);
        dv.upload(v0, stream);
        dT.upload(T0, stream);
        if (prec == LBM_PREC_F64) CU(launch_init<double>(args<double>(0), dr.p, du.p, dv.p, dT.p, stream));
        else CU(launch_init<float>(args<float>(0), dr.p, du.p, dv.p, dT.p, stream));
        fill_ghosts(0, n);
        CU(cudaStreamSynchronize(stream));
        // equilibrium failures during initialisation are not reported by the
        // reference (hasFailed is reset by runOne, cpuLBM.cpp:2288)
        CU(cudaMemsetAsync(status.p, 0, n * sizeof(int), stream));
        CU(cudaStreamSynchronize(stream));
    }

    StepLists lists() const
    {
        StepLists l;
        for (int m = 0; m < 4; ++m) {
            l.pointwise[m] = TileRun{d_tiles_by_rk[m].p, (int)tiles_by_rk[m].size()};
            split_runs(d_tiles_flux[m].p, (int)tiles_flux[m].size(), ns_by_rk[m], nw_by_rk[m], l.simple[m], l.wrap[m],
                       l.general[m]);
        }
        if (any_rk3)
            split_runs(d_tiles_rk3.p, (int)tiles_rk3.size(), ns_rk3, nw_rk3, l.rk3_simple, l.rk3_wrap, l.rk3_general);
        l.samples = d_sp.p;
        l.nsamples = (int)hs.size();
        l.any_ghost = any_ghost;
        l.walls_all = d_walls_all.p;
        l.n_walls_all = (int)walls_all.size();
        l.walls_rk3 = d_walls_rk3.p;
        l.n_walls_rk3 = (int)walls_rk3.size();
        return l;
    }

    // One step.  ev (optional) receives 7 events around the phases:
    // [0] start, then after pointwise, walls 2, phase 1, walls 3, phase 2,
    // residual.
    template <class S, class C>
    void enqueue_step_t(int want_res, cudaEvent_t *ev = nullptr)
    {
        enqueue_step_phases<S, C>(args<S>(want_res), lists(), stream, ev);
        if (want_res)
            CU(launch_residual(d_sp.p, (int)hs.size(), partial.p, d_tile_first.p, d_tile_count.p, residual.p, stream));
        if (ev) CU(cudaEventRecord(ev[6], stream));
    }

    int launches_per_step(int want_res) const { return step_launches(lists()) + (want_res ? 1 : 0); }

    void profile(int n, double *ms, int nph)
    {
        cudaEvent_t ev[7];
        for (auto &e : ev) CU(cudaEventCreate(&e));
        std::vector<double> acc(6, 0.0);
        for (int k = 0; k < n; ++k) {
            if (prec == LBM_PREC_F64) enqueue_step_t<double, double>(1, ev);
            else enqueue_step_t<float, float>(1, ev);
            CU(cudaEventSynchronize(ev[6]));
            for (int p = 0; p < 6; ++p) {
                float t = 0;
                CU(cudaEventElapsedTime(&t, ev[p], ev[p + 1]));
                acc[p] += t;
            }
        }
        for (auto &e : ev) cudaEventDestroy(e);
        for (int p = 0; p < nph && p < 6; ++p) ms[p] = n ? acc[p] / n : 0.0;
    }

    // the ghost columns of samples s0 .. s0 + ns - 1 after their state was set
    void fill_ghosts(int s0, int ns)
    {
        if (!any_ghost) return;
        if (prec == LBM_PREC_F64)
            CU(launch_fill_ghosts<double>(d_sp.p, s0, ns, reinterpret_cast<double *>(buf2.p),
                                          reinterpret_cast<double *>(buf3.p), stream));
        else
            CU(launch_fill_ghosts<float>(d_sp.p, s0, ns, reinterpret_cast<float *>(buf2.p),
                                         reinterpret_cast<float *>(buf3.p), stream));
    }

    void set_macro(int s, const double *rho, const double *ux, const double *uy, const double *T)
    {
        const long long n = (long long)hs[s].nx * hs[s].ny;
        const double *src[4] = {rho, ux, uy, T};
        for (int k = 0; k < 4; ++k)
            CU(cudaMemcpyAsync(scratch.p + k * n, src[k], n * sizeof(double), cudaMemcpyHostToDevice, stream));
        if (prec == LBM_PREC_F64)
            CU(launch_set_macro<double>(d_sp.p, s, reinterpret_cast<double *>(state.p), reinterpret_cast<double *>(buf2.p),
                                        reinterpret_cast<double *>(buf3.p), scratch.p, nflags.p, d_fref.p, n, stream));
        else
            CU(launch_set_macro<float>(d_sp.p, s, reinterpret_cast<float *>(state.p), reinterpret_cast<float *>(buf2.p),
                                       reinterpret_cast<float *>(buf3.p), scratch.p, nflags.p, d_fref.p, n, stream));
        fill_ghosts(s, 1);
    }

    // all samples' fields in one device buffer (5 fields x lattice nodes,
    // made on first use): per field one copy to or from the host
    DevBuf<double> all_fields;
    std::vector<long long> lattice_off;  // per sample: first value in the concatenated fields

    void ensure_all_fields()
    {
        if (lattice_off.empty()) {
            long long off = 0;
            for (const HostSample &h : hs) {
                lattice_off.push_back(off);
                off += (long long)h.nx * h.ny;
            }
        }
        if (all_fields.n < (size_t)(5 * lattice_nodes)) all_fields.alloc(5 * lattice_nodes);
    }

    void set_macro_all(const double *rho, const double *ux, const double *uy, const double *T)
    {
        ensure_all_fields();
        const double *src[4] = {rho, ux, uy, T};
        for (int k = 0; k < 4; ++k)
            CU(cudaMemcpyAsync(all_fields.p + k * lattice_nodes, src[k], lattice_nodes * sizeof(double),
                               cudaMemcpyHostToDevice, stream));
        for (size_t s = 0; s < hs.size(); ++s) {
            const long long n = (long long)hs[s].nx * hs[s].ny;
            // the four fields of sample s, each n values, lattice_nodes apart
            double *f0 = all_fields.p + lattice_off[s];
            if (prec == LBM_PREC_F64)
                CU(launch_set_macro_strided<double>(d_sp.p, (int)s, reinterpret_cast<double *>(state.p),
                                                    reinterpret_cast<double *>(buf2.p),
                                                    reinterpret_cast<double *>(buf3.p), f0, lattice_nodes, nflags.p,
                                                    d_fref.p, n, stream));
            else
                CU(launch_set_macro_strided<float>(d_sp.p, (int)s, reinterpret_cast<float *>(state.p),
                                                   reinterpret_cast<float *>(buf2.p), reinterpret_cast<float *>(buf3.p),
                                                   f0, lattice_nodes, nflags.p, d_fref.p, n, stream));
        }
        fill_ghosts(0, (int)hs.size());
    }

    void get_macro_all(double *rho, double *ux, double *uy, double *T, double *p)
    {
        ensure_all_fields();
        for (size_t s = 0; s < hs.size(); ++s) {
            const long long n = (long long)hs[s].nx * hs[s].ny;
            double *out = all_fields.p + lattice_off[s];
            if (prec == LBM_PREC_F64)
                CU(launch_macro_out_strided<double>(d_sp.p, (int)s, reinterpret_cast<double *>(state.p), out,
                                                    lattice_nodes, n, stream));
            else
                CU(launch_macro_out_strided<float>(d_sp.p, (int)s, reinterpret_cast<float *>(state.p), out,
                                                   lattice_nodes, n, stream));
        }
        double *dst[5] = {rho, ux, uy, T, p};
        for (int k = 0; k < 5; ++k)
            if (dst[k])
                CU(cudaMemcpyAsync(dst[k], all_fields.p + k * lattice_nodes, lattice_nodes * sizeof(double),
                                   cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
    }

    void enqueue_step(int want_res)
    {
        if (prec == LBM_PREC_F64) enqueue_step_t<double, double>(want_res);
        else enqueue_step_t<float, float>(want_res);
    }

    void launch_steps(int n, int want_res)
    {
        const int g = want_res ? 1 : 0;
        if (use_graph && !graph[g]) {
            cudaGraph_t gr;
            CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_step(want_res);
            } catch (...) {
                cudaStreamEndCapture(stream, &gr);
                throw;
            }
            CU(cudaStreamEndCapture(stream, &gr));
            CU(cudaGraphInstantiate(&graph[g], gr, 0));
            cudaGraphDestroy(gr);
        }
        for (int k = 0; k < n; ++k) {
            if (use_graph) CU(cudaGraphLaunch(graph[g], stream));
            else enqueue_step(want_res);
        }
    }

    // collect and clear the per-sample status words
    void fetch_status()
    {
        std::vector<int> st(hs.size());
        CU(cudaMemcpyAsync(st.data(), status.p, st.size() * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CU(cudaMemsetAsync(status.p, 0, st.size() * sizeof(int), stream));
        CU(cudaStreamSynchronize(stream));
        for (size_t k = 0; k < st.size(); ++k) host_status[k] |= st[k];
    }

    void fetch_residual()
    {
        CU(cudaMemcpyAsync(host_residual.data(), residual.p, host_residual.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
    }

    static lbm_status to_status(int bits)
    {
        if (bits & STATUS_TIMEOUT) return LBM_ERR_TIMEOUT;
        if (bits & STATUS_EQ) return LBM_ERR_EQUILIBRIUM;
        if (bits & STATUS_NONFINITE) return LBM_ERR_NONFINITE;
        return LBM_OK;
    }

    void get_macro(int s, double *rho, double *ux, double *uy, double *T, double *p)
    {
        const long long n = (long long)hs[s].nx * hs[s].ny;
        if (prec == LBM_PREC_F64)
            CU(launch_macro_out<double>(d_sp.p, s, reinterpret_cast<double *>(state.p), scratch.p, n, stream));
        else
            CU(launch_macro_out<float>(d_sp.p, s, reinterpret_cast<float *>(state.p), scratch.p, n, stream));
        double *dst[5] = {rho, ux, uy, T, p};
        for (int k = 0; k < 5; ++k)
            if (dst[k]) CU(cudaMemcpyAsync(dst[k], scratch.p + k * n, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
    }

    void dist_io(int s, double *f, double *h, const double *fin, const double *hin)
    {
        const long long n = (long long)hs[s].nx * hs[s].ny;
        const long long n3 = n * NQ;
        const bool to_aos = fin == nullptr;
        if (!to_aos) {
            CU(cudaMemcpyAsync(scratch.p, fin, n3 * sizeof(double), cudaMemcpyHostToDevice, stream));
            CU(cudaMemcpyAsync(scratch.p + n3, hin, n3 * sizeof(double), cudaMemcpyHostToDevice, stream));
        }
        if (prec == LBM_PREC_F64)
            CU(launch_dist_io<double>(d_sp.p, s, reinterpret_cast<double *>(state.p), reinterpret_cast<double *>(buf2.p),
                                      reinterpret_cast<double *>(buf3.p), scratch.p, to_aos ? 1 : 0, nflags.p, d_fref.p, n,
                                      stream));
        else
            CU(launch_dist_io<float>(d_sp.p, s, reinterpret_cast<float *>(state.p), reinterpret_cast<float *>(buf2.p),
                                     reinterpret_cast<float *>(buf3.p), scratch.p, to_aos ? 1 : 0, nflags.p, d_fref.p, n,
                                     stream));
        if (to_aos) {
            if (f) CU(cudaMemcpyAsync(f, scratch.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
            if (h) CU(cudaMemcpyAsync(h, scratch.p + n3, n3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        } else {
            fill_ghosts(s, 1);
        }
        CU(cudaStreamSynchronize(stream));
    }

    size_t device_bytes() const
    {
        return state.n + buf2.n + buf3.n + alpha.n + nflags.n + sizeof(double) * (told.n + partial.n + scratch.n);
    }
};

struct lbm_handle {
    lbm_batch b;
};

// ---------------------------------------------------------------- C ABI
#define API_BEGIN try {
#define API_END                                          \
    }                                                    \
    catch (const LbmError &e)                            \
    {                                                    \
        g_last_error = e.what();                         \
        return e.code;                                   \
    }                                                    \
    catch (const std::bad_alloc &)                       \
    {                                                    \
        g_last_error = "host allocation failed";         \
        return LBM_ERR_NOMEM;                            \
    }                                                    \
    catch (const std::exception &e)                      \
    {                                                    \
        g_last_error = e.what();                         \
        return LBM_ERR_INVALID;                          \
    }

extern "C" {

const char *lbm_last_error(void) { return g_last_error.c_str(); }

lbm_status lbm_create(const lbm_config *cfg, const lbm_init *init, int precision, lbm_handle **out)
{
    API_BEGIN
    if (!cfg || !init || !out) throw LbmError(LBM_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<lbm_handle> h(new lbm_handle);
    lbm_batch_options o{precision, 0, 0, 1};
    h->b.build(1, cfg, init, &o);
    *out = h.release();
    return LBM_OK;
    API_END
}

lbm_status lbm_create_from_mat(const char *path, int precision, lbm_handle **out)
{
    API_BEGIN
    if (!path || !out) throw LbmError(LBM_ERR_INVALID, "null argument");
    *out = nullptr;
    MatCase c;
    mat_read_case(path, c);
    std::unique_ptr<lbm_handle> h(new lbm_handle);
    lbm_batch_options o{precision, 0, 0, 1};
    h->b.build(1, &c.cfg, &c.init, &o);
    *out = h.release();
    return LBM_OK;
    API_END
}

lbm_status lbm_write_mat(lbm_handle *h, const char *path, int with_dist)
{
    API_BEGIN
    if (!h || !path) throw LbmError(LBM_ERR_INVALID, "null argument");
    lbm_batch &b = h->b;
    const HostSample &s = b.hs[0];
    const size_t n = (size_t)s.nx * s.ny;
    std::vector<double> rho(n), ux(n), uy(n), T(n), p(n);
    b.get_macro(0, rho.data(), ux.data(), uy.data(), T.data(), p.data());
    std::vector<double> f, hh, ex(NQ), ey(NQ);
    if (with_dist) {
        f.resize(n * NQ);
        hh.resize(n * NQ);
        b.dist_io(0, f.data(), hh.data(), nullptr, nullptr);
        for (int i = 0; i < NQ; ++i) {
            ex[i] = s.c * kEX[i];
            ey[i] = s.c * kEY[i];
        }
    }
    mat_write_fields(path, s.nx, s.ny, rho.data(), ux.data(), uy.data(), p.data(), T.data(), s.step * s.dt, s.dx[0],
                     s.dy[0], with_dist ? f.data() : nullptr, with_dist ? hh.data() : nullptr,
                     with_dist ? ex.data() : nullptr, with_dist ? ey.data() : nullptr);
    return LBM_OK;
    API_END
}

lbm_status lbm_write_hdf5(lbm_handle *h, const char *path, int with_dist)
{
    API_BEGIN
    if (!h || !path) throw LbmError(LBM_ERR_INVALID, "null argument");
    lbm_batch &b = h->b;
    const HostSample &s = b.hs[0];
    const size_t n = (size_t)s.nx * s.ny;
    std::vector<double> rho(n), ux(n), uy(n), T(n), p(n), f, hh;
    b.get_macro(0, rho.data(), ux.data(), uy.data(), T.data(), p.data());
    if (with_dist) {
        f.resize(n * NQ);
        hh.resize(n * NQ);
        b.dist_io(0, f.data(), hh.data(), nullptr, nullptr);
    }
    // dx, dy: one value for uniform cells (as the reference's scalars)
    const bool ux1 = std::all_of(s.dx.begin(), s.dx.end(), [&](double v) { return v == s.dx[0]; });
    const bool uy1 = std::all_of(s.dy.begin(), s.dy.end(), [&](double v) { return v == s.dy[0]; });
    hdf5_write_fields(path, s.nx, s.ny, rho.data(), ux.data(), uy.data(), T.data(), s.step * s.dt, s.gamma, s.R,
                      s.T_ref, s.rho_ref, s.dx.data(), ux1 ? 1 : (int)s.dx.size(), s.dy.data(),
                      uy1 ? 1 : (int)s.dy.size(), with_dist ? f.data() : nullptr, with_dist ? hh.data() : nullptr);
    return LBM_OK;
    API_END
}

lbm_status lbm_restore_mat(lbm_handle *h, const char *path)
{
    API_BEGIN
    if (!h || !path) throw LbmError(LBM_ERR_INVALID, "null argument");
    lbm_batch &b = h->b;
    HostSample &s = b.hs[0];
    const size_t n = (size_t)s.nx * s.ny * NQ;
    std::vector<double> f(n), hh(n);
    double t = 0.0;
    mat_read_dist(path, s.nx, s.ny, f.data(), hh.data(), &t);
    b.dist_io(0, nullptr, nullptr, f.data(), hh.data());
    s.step = (int)std::lround(t / s.dt);
    return LBM_OK;
    API_END
}

void lbm_destroy(lbm_handle *h) { delete h; }

void *lbm_stream(lbm_handle *h) { return h ? (void *)h->b.stream : nullptr; }

lbm_status lbm_step(lbm_handle *h, int n_steps, int want_residual, double *residual_out)
{
    API_BEGIN
    if (!h || n_steps < 0) throw LbmError(LBM_ERR_INVALID, "bad argument");
    lbm_batch &b = h->b;
    HostSample &s = b.hs[0];
    b.host_status[0] = 0;
    if (want_residual) {
        // the residual belongs to each step; step one at a time
        for (int k = 0; k < n_steps; ++k) {
            s.step += 1;
            b.launch_steps(1, 1);
            b.fetch_residual();
            s.residual = b.host_residual[0];
        }
    } else {
        b.launch_steps(n_steps, 0);
        s.step += n_steps;
    }
    b.fetch_status();
    if (residual_out) *residual_out = s.residual;
    return lbm_batch::to_status(b.host_status[0]);
    API_END
}

lbm_status lbm_run(lbm_handle *h, int max_steps, int *stop_out, double *trace, int trace_len)
{
    API_BEGIN
    if (!h) throw LbmError(LBM_ERR_INVALID, "null handle");
    lbm_batch &b = h->b;
    HostSample &s = b.hs[0];
    const int numRes = 20;
    int stop = 0, k = 0;
    lbm_status last = LBM_OK;
    while (stop == 0 && (max_steps < 0 || k < max_steps)) {
        s.step += 1;
        b.host_status[0] = 0;
        if (s.tol != 0) {
            b.launch_steps(1, 1);
            b.fetch_residual();
            b.fetch_status();
            s.residual = b.host_residual[0];
            stop = (b.host_status[0] & STATUS_EQ) ? 1 : 0;
            if (s.step >= 2 && s.step <= numRes) {
                s.initRes[s.step - 2] = s.residual;
                s.residual = 1;
            } else if (s.step == numRes + 1) {
                for (int i = 0; i < numRes - 1; ++i) s.resNorm = std::max(s.initRes[i], s.resNorm);
                s.residual = s.residual / s.resNorm;
            } else if (s.step >= numRes + 1) {
                s.residual = s.residual / s.resNorm;
            }
        } else {
            b.launch_steps(1, 0);
            b.fetch_status();
            stop = (b.host_status[0] & STATUS_EQ) ? 1 : 0;
        }
        if (b.host_status[0] & STATUS_NONFINITE) last = LBM_ERR_NONFINITE;
        if (trace && k < trace_len) trace[k] = s.residual;
        if (s.step >= s.nsteps && s.nsteps != 0) stop = 2;
        if (s.tol != 0 && s.residual <= s.tol && s.step >= numRes + 1) stop = 2;
        ++k;
    }
    if (stop_out) *stop_out = stop;
    return stop == 1 ? LBM_ERR_EQUILIBRIUM : last;
    API_END
}

lbm_status lbm_get_macro(lbm_handle *h, double *rho, double *ux, double *uy, double *T, double *p)
{
    API_BEGIN
    if (!h) throw LbmError(LBM_ERR_INVALID, "null handle");
    h->b.get_macro(0, rho, ux, uy, T, p);
    return LBM_OK;
    API_END
}

lbm_status lbm_get_dist(lbm_handle *h, double *f, double *hh)
{
    API_BEGIN
    if (!h) throw LbmError(LBM_ERR_INVALID, "null handle");
    h->b.dist_io(0, f, hh, nullptr, nullptr);
    return LBM_OK;
    API_END
}

lbm_status lbm_set_dist(lbm_handle *h, const double *f, const double *hh)
{
    API_BEGIN
    if (!h || !f || !hh) throw LbmError(LBM_ERR_INVALID, "null argument");
    h->b.dist_io(0, nullptr, nullptr, f, hh);
    return LBM_OK;
    API_END
}

lbm_status lbm_get_info(lbm_handle *h, lbm_info *info)
{
    API_BEGIN
    if (!h || !info) throw LbmError(LBM_ERR_INVALID, "null argument");
    const HostSample &s = h->b.hs[0];
    info->Nx = s.nx;
    info->Ny = s.ny;
    info->step = s.step;
    info->nsteps = s.nsteps;
    info->dt = s.dt;
    info->tstep = s.step * s.dt;
    info->residual = s.residual;
    info->precision = h->b.prec;
    info->rkmethod = s.rk;
    info->fmethod = s.fm;
    info->device_bytes = h->b.device_bytes();
    return LBM_OK;
    API_END
}

// ---------------------------------------------------------------- batches
lbm_status lbm_batch_create(int n, const lbm_config *cfgs, const lbm_init *inits, const lbm_batch_options *opt,
                            lbm_batch **out)
{
    API_BEGIN
    if (!out) throw LbmError(LBM_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<lbm_batch> b(new lbm_batch);
    b->build(n, cfgs, inits, opt);
    *out = b.release();
    return LBM_OK;
    API_END
}

void lbm_batch_destroy(lbm_batch *b) { delete b; }

void *lbm_batch_stream(lbm_batch *b) { return b ? (void *)b->stream : nullptr; }

long long lbm_batch_nodes(lbm_batch *b) { return b ? b->lattice_nodes : 0; }

lbm_status lbm_selftest_bounded_wait(int arrive)
{
    API_BEGIN
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        throw LbmError(LBM_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
    DevBuf<int> st;
    st.alloc(1);
    CU(cudaMemset(st.p, 0, sizeof(int)));
    CU(launch_wait_selftest(st.p, arrive ? 1 : 0, nullptr));
    int bits = 0;
    CU(cudaMemcpy(&bits, st.p, sizeof(int), cudaMemcpyDeviceToHost));
    const lbm_status r = lbm_batch::to_status(bits);
    if (r != LBM_OK) g_last_error = "bounded device wait ran out";
    return r;
    API_END
}

lbm_status lbm_batch_step(lbm_batch *b, int n_steps, int want_residual)
{
    API_BEGIN
    if (!b || n_steps < 0) throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->launch_steps(n_steps, want_residual ? 1 : 0);
    for (auto &s : b->hs) s.step += n_steps;
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_status(lbm_batch *b, int *status)
{
    API_BEGIN
    if (!b || !status) throw LbmError(LBM_ERR_INVALID, "null argument");
    b->fetch_status();
    for (size_t k = 0; k < b->hs.size(); ++k) {
        status[k] = (int)lbm_batch::to_status(b->host_status[k]);
        b->host_status[k] = 0;
    }
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_residuals(lbm_batch *b, double *residual)
{
    API_BEGIN
    if (!b || !residual) throw LbmError(LBM_ERR_INVALID, "null argument");
    b->fetch_residual();
    std::copy(b->host_residual.begin(), b->host_residual.end(), residual);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_get_macro(lbm_batch *b, int sample, double *rho, double *ux, double *uy, double *T, double *p)
{
    API_BEGIN
    if (!b || sample < 0 || sample >= (int)b->hs.size()) throw LbmError(LBM_ERR_INVALID, "bad sample");
    b->get_macro(sample, rho, ux, uy, T, p);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_get_dist(lbm_batch *b, int sample, double *f, double *hh)
{
    API_BEGIN
    if (!b || sample < 0 || sample >= (int)b->hs.size()) throw LbmError(LBM_ERR_INVALID, "bad sample");
    b->dist_io(sample, f, hh, nullptr, nullptr);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_set_macro(lbm_batch *b, int sample, const double *rho, const double *ux, const double *uy,
                               const double *T)
{
    API_BEGIN
    if (!b || !rho || !ux || !uy || !T || sample < 0 || sample >= (int)b->hs.size())
        throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->set_macro(sample, rho, ux, uy, T);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_set_macro_all(lbm_batch *b, const double *rho, const double *ux, const double *uy,
                                   const double *T)
{
    API_BEGIN
    if (!b || !rho || !ux || !uy || !T) throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->set_macro_all(rho, ux, uy, T);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_get_macro_all(lbm_batch *b, double *rho, double *ux, double *uy, double *T, double *p)
{
    API_BEGIN
    if (!b) throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->get_macro_all(rho, ux, uy, T, p);
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_profile(lbm_batch *b, int n_steps, double *phase_ms, int n_phases)
{
    API_BEGIN
    if (!b || !phase_ms || n_steps < 1) throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->profile(n_steps, phase_ms, n_phases);
    for (auto &s : b->hs) s.step += n_steps;
    return LBM_OK;
    API_END
}

lbm_status lbm_batch_autotune(lbm_batch *b, const int *candidates, int n_candidates, int steps, int *chosen,
                              double *ms_per_step)
{
    API_BEGIN
    if (!b) throw LbmError(LBM_ERR_INVALID, "null batch");
    static const int defaults[] = {32, 8, 16, 16, 64, 4, 8, 32, 32, 4, 16, 8};
    if (!candidates || n_candidates <= 0) {
        candidates = defaults;
        n_candidates = 6;
    }
    b->autotune(candidates, n_candidates, steps, chosen, ms_per_step);
    return LBM_OK;
    API_END
}

int lbm_batch_launches_per_step(lbm_batch *b, int want_residual) { return b ? b->launches_per_step(want_residual) : 0; }

lbm_status lbm_batch_set_dist(lbm_batch *b, int sample, const double *f, const double *hh)
{
    API_BEGIN
    if (!b || !f || !hh || sample < 0 || sample >= (int)b->hs.size()) throw LbmError(LBM_ERR_INVALID, "bad argument");
    b->dist_io(sample, nullptr, nullptr, f, hh);
    return LBM_OK;
    API_END
}

}  // extern "C"
