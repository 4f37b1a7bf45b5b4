// lbm_step_noalloc: the FP64 step of one small domain with no device
// allocation.  Some callers cannot call cudaMalloc: a host application that
// owns all device memory through its own pool or arena, or one whose
// device-memory budget is already spoken for, so that a library's own
// allocation would fail or break its accounting.  For them the stage
// buffers, wall factors, node flags, tile list and TMA descriptors that
// lbm_create would cudaMalloc live in one file-scope device array of fixed
// size instead, and the caller passes only its own f and h arrays (device
// memory it already owns).
//
// The array is reserved on every GPU that loads this library, until the
// process exits.  Every call shares it and overwrites what the last call
// left; calls that overlap on the GPU (two streams, two threads) race on it.
#include "lbm_device.cuh"
#include "lbm_host.h"
#include "lbm_kernels.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

namespace uqlbm {

// capacity: padded nodes Ny * roundup(Nx, 32)
constexpr long long NA_MAX_NODES = LBM_NOALLOC_MAX_NODES;
constexpr int NA_MAX_LINE = 8192;  // longest row or column (Nx, Ny <= 16384 / 3)
constexpr int NA_MAX_TILES = 1024;
constexpr int NA_TX = 32, NA_TY = 8;

constexpr size_t na_align(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t NA_STATE = na_align(NPL * NA_MAX_NODES * sizeof(double));
constexpr size_t NA_OFF_STATE = 0;
constexpr size_t NA_OFF_BUF2 = NA_OFF_STATE + NA_STATE;
constexpr size_t NA_OFF_BUF3 = NA_OFF_BUF2 + NA_STATE;
constexpr size_t NA_OFF_ALPHA = NA_OFF_BUF3 + NA_STATE;
constexpr size_t NA_OFF_FLAGS = NA_OFF_ALPHA + na_align(NA_MAX_NODES * sizeof(double));
constexpr size_t NA_OFF_CTYPE = NA_OFF_FLAGS + na_align(NA_MAX_NODES);
constexpr size_t NA_OFF_LINES = NA_OFF_CTYPE + na_align(NA_MAX_NODES * sizeof(int));
constexpr size_t NA_OFF_TILES = NA_OFF_LINES + na_align(4 * NA_MAX_LINE * sizeof(double));
constexpr size_t NA_OFF_SP = NA_OFF_TILES + na_align(NA_MAX_TILES * sizeof(Tile));
constexpr size_t NA_OFF_STATUS = NA_OFF_SP + na_align(sizeof(SampleParams));
constexpr size_t NA_OFF_FREF = NA_OFF_STATUS + na_align(sizeof(int));
constexpr size_t NA_OFF_MAPS = NA_OFF_FREF + na_align(NPL * sizeof(double));
constexpr size_t NA_BYTES = NA_OFF_MAPS + na_align(2 * sizeof(CUtensorMap));

// the scratch: reserved per device by loading the module, never cudaMalloc'd
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// node flags (as the engine computes them on the host), tile list, spacing
// tables and cleared status / wall factors / rest state
__global__ void k_na_setup(int nx, int ny, int pitch, int flags, double dx, double dy, double dt, unsigned char *base)
{
    SampleParams sp{};
    sp.nx = nx;
    sp.ny = ny;
    sp.pitch = pitch;
    sp.flags = flags;
    const int *ct = reinterpret_cast<const int *>(base + NA_OFF_CTYPE);  // [x*ny + y]
    uint8_t *nf = base + NA_OFF_FLAGS;
    double *alpha = reinterpret_cast<double *>(base + NA_OFF_ALPHA);
    const long long n = (long long)ny * pitch;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (long long k = tid; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / pitch), x = (int)(k % pitch);
        alpha[k] = 0.0;
        if (x >= nx) { nf[k] = 0; continue; }
        uint8_t fl = (uint8_t)ct[(long long)x * ny + y];
        int m;
        for (int d = -2; d <= 2; ++d) {
            const int xr = bc_index(sp, x, d, 0, m), yr = bc_index(sp, y, d, 1, m);
            if (ct[(long long)xr * ny + y] == 2) fl |= NF_SOLX;
            if (ct[(long long)x * ny + yr] == 2) fl |= NF_SOLY;
        }
        if (x < 2 || x > nx - 3) fl |= (flags & SF_PERX) ? NF_WRPX : NF_EDGX;
        if (y < 2 || y > ny - 3) fl |= (flags & SF_PERY) ? NF_WRPY : NF_EDGY;
        nf[k] = fl;
    }
    double *lines = reinterpret_cast<double *>(base + NA_OFF_LINES);  // tdx | tdy | dxv | dyv
    for (long long k = tid; k < NA_MAX_LINE; k += (long long)gridDim.x * blockDim.x) {
        lines[k] = dt / dx;
        lines[NA_MAX_LINE + k] = dt / dy;
        lines[2 * NA_MAX_LINE + k] = dx;
        lines[3 * NA_MAX_LINE + k] = dy;
    }
    const int tiles_x = (nx + NA_TX - 1) / NA_TX, tiles_y = (ny + NA_TY - 1) / NA_TY;
    Tile *tiles = reinterpret_cast<Tile *>(base + NA_OFF_TILES);
    for (long long t = tid; t < (long long)tiles_x * tiles_y; t += (long long)gridDim.x * blockDim.x)
        tiles[t] = Tile{0, (int)(t % tiles_x) * NA_TX, (int)(t / tiles_x) * NA_TY, (int)t};
    double *fref = reinterpret_cast<double *>(base + NA_OFF_FREF);
    if (tid < NPL) fref[tid] = 0.0;  // the FP64 path stores f and h in full
    if (tid == 0) *reinterpret_cast<int *>(base + NA_OFF_STATUS) = 0;
}

// caller's reference-layout f, h [(x*Ny + y)*13 + i] <-> planes; fixed nodes
// also seed the stage buffers
__global__ void k_na_io(int nx, int ny, int pitch, double *f, double *h, unsigned char *base, int to_caller)
{
    double *st = reinterpret_cast<double *>(base + NA_OFF_STATE);
    double *b2 = reinterpret_cast<double *>(base + NA_OFF_BUF2);
    double *b3 = reinterpret_cast<double *>(base + NA_OFF_BUF3);
    const uint8_t *nf = base + NA_OFF_FLAGS;
    const long long plane = (long long)ny * pitch;
    const long long n = (long long)nx * ny * NQ;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % NQ);
        const long long xy = k / NQ;
        const int y = (int)(xy % ny), x = (int)(xy / ny);
        const long long o = (long long)y * pitch + x;
        const long long of = i * plane + o, oh = (NQ + i) * plane + o;
        if (to_caller) {
            f[k] = st[of];
            h[k] = st[oh];
        } else {
            st[of] = f[k];
            st[oh] = h[k];
            if (nf[o] & NF_TYPE) {
                b2[of] = f[k]; b3[of] = f[k];
                b2[oh] = h[k]; b3[oh] = h[k];
            }
        }
    }
}

// wall factors for every solid node next to fluid (the engine keeps a list;
// here every node checks itself)
__global__ void k_na_wall(const unsigned char *base, size_t stage_off)
{
    const SampleParams &sp = *reinterpret_cast<const SampleParams *>(base + NA_OFF_SP);
    const StageView<double> v{reinterpret_cast<const double *>(base + stage_off), base + NA_OFF_FLAGS, (int)sp.plane,
                              sp.pitch};
    const long long n = (long long)sp.ny * sp.pitch;
    double *alpha = reinterpret_cast<double *>(const_cast<unsigned char *>(base) + NA_OFF_ALPHA);
    const double *lines = reinterpret_cast<const double *>(base + NA_OFF_LINES);
    const double *fref = reinterpret_cast<const double *>(base + NA_OFF_FREF);
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / sp.pitch), x = (int)(k % sp.pitch);
        if (x >= sp.nx || (v.nf[k] & NF_TYPE) != 2) continue;
        bool adj = false;
        for (int j = 0; j < 4; ++j) {
            int m;
            const int xm = bc_index(sp, x, c_WXX[j], 0, m), ym = bc_index(sp, y, c_WYY[j], 1, m);
            if ((v.nf[ym * sp.pitch + xm] & NF_TYPE) < 2) adj = true;
        }
        if (adj)
            alpha[k] = wall_alpha_m1<double, double>(sp, v, x, y, lines[2 * NA_MAX_LINE + x], lines[3 * NA_MAX_LINE + y],
                                                    fref);
    }
}

namespace {
struct DeviceScratch {
    unsigned char *ptr = nullptr;
    bool ready = false;
};
DeviceScratch g_dev[64];
std::mutex g_dev_mutex;

// once per device, with that device current: the scratch's device address
// (the host-side symbol is only a stand-in) and the flux kernels' shared
// memory opt-in
unsigned char *scratch_for_current_device()
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw LbmError(LBM_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    DeviceScratch &d = g_dev[dev];
    if (!d.ready) {
        void *p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        CU((prepare_kernels<double, double>()));
        d.ptr = static_cast<unsigned char *>(p);
        d.ready = true;
    }
    return d.ptr;
}

PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        CU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw LbmError(LBM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
}  // namespace

static lbm_status step_noalloc(const lbm_config *cfg, int Nx, int Ny, const int *cellType, double *d_f, double *d_h,
                               int n_steps, cudaStream_t st)
{
    if (!cfg || !cellType || !d_f || !d_h || n_steps < 0) throw LbmError(LBM_ERR_INVALID, "bad argument");
    if (cfg->dx_array || cfg->dy_array)
        throw LbmError(LBM_ERR_INVALID, "lbm_step_noalloc supports uniform cells only");
    if (Nx < 3 || Ny < 3) throw LbmError(LBM_ERR_INVALID, "Nx and Ny must be at least 3");
    // the node flags keep the cell type in two bits next to the stencil
    // bits: a value outside 0..2 would mark interior nodes as boundaries
    for (long long k = 0; k < (long long)Nx * Ny; ++k)
        if (cellType[k] < 0 || cellType[k] > 2) throw LbmError(LBM_ERR_INVALID, "cellType must be 0, 1 or 2");
    const int pitch = (Nx + 31) / 32 * 32;
    if ((long long)Ny * pitch > NA_MAX_NODES || Nx > NA_MAX_LINE || Ny > NA_MAX_LINE)
        throw LbmError(LBM_ERR_INVALID, "domain exceeds lbm_step_noalloc's fixed scratch: Ny * roundup(Nx, 32) must be <= " +
                                            std::to_string(NA_MAX_NODES));
    ScalarParams sc;
    derive_scalars(*cfg, Nx, Ny, 0.0, sc);
    unsigned char *base = scratch_for_current_device();

    SampleParams sp{};
    sp.nx = Nx;
    sp.ny = Ny;
    sp.pitch = pitch;
    sp.flags = sc.flags;
    sp.rk = sc.rk;
    sp.fm = sc.fm;
    const int tiles_x = (Nx + NA_TX - 1) / NA_TX, tiles_y = (Ny + NA_TY - 1) / NA_TY;
    sp.ntile = tiles_x * tiles_y;
    sp.plane = (long long)Ny * pitch;
    sp.R = sc.R;
    sp.bR = sc.b * sc.R;
    sp.K = sc.K;
    sp.Tc = sc.Tc;
    sp.inv_sRTc = 1.0 / std::sqrt(sc.R * sc.Tc);
    sp.RTc = sc.R * sc.Tc;
    sp.mu = sc.mu;
    sp.Pr = sc.Pr;
    sp.dt = sc.dt;
    sp.c = sc.c;
    sp.inv_mu = 1.0 / sc.mu;
    sp.two_over_bR = 2.0 / (sc.b * sc.R);
    sp.visc = sc.mu_model;
    sp.visc_exp = sc.mu_model == 1 ? 0.5 + sc.upsilon : 1.5;
    sp.visc_S = sc.S_v;
    sp.visc_T = sc.T_ref;
    sp.rho0 = 0.0;
    sp.T0n = 1.0;
    sp.shref = 0.0;

    CUtensorMap maps[2];
    for (int b = 0; b < 2; ++b) {
        cuuint64_t dims[3] = {(cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)NPL};
        cuuint64_t strides[2] = {(cuuint64_t)pitch * sizeof(double), (cuuint64_t)sp.plane * sizeof(double)};
        cuuint32_t box[3] = {(cuuint32_t)(NA_TX + 8), (cuuint32_t)(NA_TY + 6), 1};
        cuuint32_t estr[3] = {1, 1, 1};
        if (encoder()(&maps[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base + (b == 0 ? NA_OFF_BUF2 : NA_OFF_BUF3), dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            throw LbmError(LBM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
    // small host-to-device copies of values on this stack frame (staged by
    // the driver before the call returns)
    CU(cudaMemcpyAsync(base + NA_OFF_SP, &sp, sizeof(sp), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(base + NA_OFF_MAPS, maps, sizeof(maps), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(base + NA_OFF_CTYPE, cellType, sizeof(int) * (size_t)Nx * Ny, cudaMemcpyHostToDevice, st));
    k_na_setup<<<64, 256, 0, st>>>(Nx, Ny, pitch, sc.flags, sc.dx, sc.dy, sc.dt, base);
    CU(cudaGetLastError());
    k_na_io<<<128, 256, 0, st>>>(Nx, Ny, pitch, d_f, d_h, base, 0);
    CU(cudaGetLastError());

    KArgs<double> a{};
    a.samples = reinterpret_cast<const SampleParams *>(base + NA_OFF_SP);
    a.tiles = reinterpret_cast<const Tile *>(base + NA_OFF_TILES);
    a.ntiles = sp.ntile;
    a.tx = NA_TX;
    a.ty = NA_TY;
    a.state = reinterpret_cast<double *>(base + NA_OFF_STATE);
    a.buf2 = reinterpret_cast<double *>(base + NA_OFF_BUF2);
    a.buf3 = reinterpret_cast<double *>(base + NA_OFF_BUF3);
    a.nflags = base + NA_OFF_FLAGS;
    a.alpha_raw = base + NA_OFF_ALPHA;
    a.told = nullptr;
    a.partial = nullptr;
    a.status = reinterpret_cast<int *>(base + NA_OFF_STATUS);
    const double *lines = reinterpret_cast<const double *>(base + NA_OFF_LINES);
    a.tdx = lines;
    a.tdy = lines + NA_MAX_LINE;
    a.dxv = lines + 2 * NA_MAX_LINE;
    a.dyv = lines + 3 * NA_MAX_LINE;
    a.tmaps = reinterpret_cast<const CUtensorMap *>(base + NA_OFF_MAPS);
    a.fref = reinterpret_cast<const double *>(base + NA_OFF_FREF);
    a.want_residual = 0;
    a.eq_tol = 1e-6;
    for (int k = 0; k < n_steps; ++k) {
        CU((launch_phase<double, double>(a, 0, sc.rk, a.tiles, sp.ntile, nullptr, 0, st)));
        k_na_wall<<<64, 256, 0, st>>>(base, NA_OFF_BUF2);
        CU(cudaGetLastError());
        CU((launch_phase<double, double>(a, 1, sc.rk, a.tiles, sp.ntile, nullptr, 0, st)));
        if (sc.rk == 1) {
            k_na_wall<<<64, 256, 0, st>>>(base, NA_OFF_BUF3);
            CU(cudaGetLastError());
            CU((launch_phase<double, double>(a, 2, 1, a.tiles, sp.ntile, nullptr, 0, st)));
        }
    }
    k_na_io<<<128, 256, 0, st>>>(Nx, Ny, pitch, d_f, d_h, base, 1);
    CU(cudaGetLastError());
    int status = 0;
    CU(cudaMemcpyAsync(&status, base + NA_OFF_STATUS, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (status & STATUS_TIMEOUT) return LBM_ERR_TIMEOUT;
    if (status & STATUS_EQ) return LBM_ERR_EQUILIBRIUM;
    if (status & STATUS_NONFINITE) return LBM_ERR_NONFINITE;
    return LBM_OK;
}

}  // namespace uqlbm

extern "C" lbm_status lbm_step_noalloc(const lbm_config *cfg, int Nx, int Ny, const int *cellType, double *d_f,
                                       double *d_h, int n_steps, void *stream)
{
    try {
        return uqlbm::step_noalloc(cfg, Nx, Ny, cellType, d_f, d_h, n_steps, static_cast<cudaStream_t>(stream));
    } catch (const uqlbm::LbmError &e) {
        uqlbm::g_last_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        uqlbm::g_last_error = e.what();
        return LBM_ERR_INVALID;
    }
}
