// Host-visible kernel interface of the D2Q13 LBM step (see lbm_kernels.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace uqlbm {

struct SampleParams;
struct Tile;

constexpr int STATUS_EQ = 1;         // equilibrium mass check (cpuLBM.cpp:839-843)
constexpr int STATUS_NONFINITE = 2;  // NaN / Inf / rho <= 0 in the state
constexpr int STATUS_TIMEOUT = 4;    // a bounded device-side wait ran out

// tensor maps per sample: the stage buffers 2 and 3 with the stencil
// kernels' halo box, and the state with a box of the tile's own nodes over
// 13 planes (the f or the h half of the state, prefetched for the update)
constexpr int MAPS_PER_SAMPLE = 3;
constexpr int PREFETCH_PLANES = 13;
// the default tile shape, also compiled into the stencil kernels (box
// widths, strides and the thread-to-node map become constants); other shapes
// run the same kernels with the shape read at run time.  A tile row of 32 is
// one warp: a row's x neighbours sit in the same warp and its staged-box
// reads are unit-stride across the warp.
constexpr int TILE_CX = 32, TILE_CY = 8;

struct WallNode {
    int sample, x, y, pad;
};

// Everything a phase kernel needs, passed by value.
template <class S>
struct KArgs {
    const SampleParams *samples;
    const Tile *tiles;
    int ntiles;
    int tx, ty;  // tile shape (threads = tx * ty)
    S *state;    // f, h (and, between P1 and P2 of RK3, the update partial sum)
    S *buf2;     // stage buffer 2 (f1 or f2)
    S *buf3;     // stage buffer 3 (f3)
    const uint8_t *nflags;
    void *alpha_raw;  // per node: wall correction factor alpha - 1
    double *told;     // T at the start of the step (residual)
    double *partial;  // per-tile residual partial sums
    int *status;      // per-sample status bits
    const double *tdx, *tdy, *dxv, *dyv;
    const CUtensorMap *tmaps;  // per sample MAPS_PER_SAMPLE maps: [buffer 2, buffer 3, state]
    const double *fref;        // per sample: 26 rest-state values subtracted from the stored state
    int want_residual;
    double eq_tol;
#ifdef __CUDACC__
    // alpha is stored in the compute type of the kernel instantiation
    template <class C>
    __device__ __forceinline__ C *alpha_as() const { return reinterpret_cast<C *>(alpha_raw); }
#endif
};

// Which tiles a stencil-phase launch covers: FLUX_SIMPLE, FLUX_WRAP and
// FLUX_GENERAL run the kernel compiled for that kind alone over a list
// holding only that kind; FLUX_BOTH runs the simple and the general kernel
// over a list of those two kinds (each skips the other kind's tiles).
enum FluxPath { FLUX_BOTH = 0, FLUX_SIMPLE = 1, FLUX_GENERAL = 2, FLUX_WRAP = 3 };

template <class S, class C>
cudaError_t launch_phase(const KArgs<S> &a, int phase, int rk, const Tile *tiles, int ntiles, const WallNode *walls,
                         int nwalls, cudaStream_t st, int path = FLUX_BOTH);
template <class S, class C>
cudaError_t prepare_kernels();
size_t flux_smem_bytes(int prec, int tx, int ty);
template <class S>
cudaError_t launch_init(const KArgs<S> &a, const double *rho, const double *ux, const double *uy, const double *T,
                        cudaStream_t st);
template <class S>
cudaError_t launch_macro_out(const SampleParams *samples, int s, const S *state, double *out, long long nodes,
                             cudaStream_t st);
// the same with the fields `stride` values apart (several samples' fields
// in one buffer)
template <class S>
cudaError_t launch_macro_out_strided(const SampleParams *samples, int s, const S *state, double *out,
                                     long long stride, long long nodes, cudaStream_t st);
template <class S>
cudaError_t launch_set_macro_strided(const SampleParams *samples, int s, S *state, S *buf2, S *buf3,
                                     const double *fields, long long stride, const uint8_t *nflags, const double *fref,
                                     long long nodes, cudaStream_t st);
template <class S>
cudaError_t launch_dist_io(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, double *aos, int to_aos,
                           const uint8_t *nflags, const double *fref, long long nodes, cudaStream_t st);
template <class S>
cudaError_t launch_set_macro(const SampleParams *samples, int s, S *state, S *buf2, S *buf3, const double *fields,
                             const uint8_t *nflags, const double *fref, long long nodes, cudaStream_t st);
cudaError_t launch_wait_selftest(int *status, int arrive, cudaStream_t st);
// copy the edge columns of stage buffers 2 and 3 into the ghost columns
// (SampleParams::gx) of samples s0 .. s0 + ns - 1 (after their state was set)
template <class S>
cudaError_t launch_fill_ghosts(const SampleParams *samples, int s0, int ns, S *buf2, S *buf3, cudaStream_t st);
cudaError_t launch_residual(const SampleParams *samples, int nsamples, const double *partial, const int *tile_first,
                            const int *tile_count, double *residual, cudaStream_t st);

}  // namespace uqlbm
