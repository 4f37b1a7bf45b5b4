// Host-side pieces shared by batches (lbm_engine.cu) and the request server
// (lbm_server.cu): device buffers, the derived per-sample description, the
// per-sample preparation that does not depend on where a sample is packed,
// and the launch sequence of one step over packed tile and wall lists.
#pragma once

#include "lbm_device.cuh"
#include "lbm_host.h"
#include "lbm_kernels.h"
#include "../../include/uq_lbm.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace uqlbm {

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;    // elements in use
    size_t cap = 0;  // elements allocated
    void alloc(size_t count)
    {
        free();
        if (count == 0) return;
        CU(cudaMalloc(&p, count * sizeof(T)));
        n = cap = count;
    }
    void upload(const std::vector<T> &v, cudaStream_t s)
    {
        alloc(v.size());
        if (!v.empty()) CU(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    // keep the allocation when it is large enough (grows by half again
    // otherwise), so repeated repacks do not reallocate
    void upload_keep(const std::vector<T> &v, cudaStream_t s)
    {
        if (v.size() > cap) {
            const size_t c = std::max(v.size(), cap + cap / 2);
            free();
            CU(cudaMalloc(&p, c * sizeof(T)));
            cap = c;
        }
        n = v.size();
        if (!v.empty()) CU(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void free()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = cap = 0;
    }
    ~DevBuf() { free(); }
};

// Host-side description of one sample after refineInput / setupVars.
struct HostSample {
    int nx = 0, ny = 0, rk = 1, fm = 1;
    int flags = 0;
    double R = 1, b = 5, K = 3, Tc = 1, c = 1, mu = 0, Pr = 1, dt = 0, tol = 0;
    double rho_ref = 1, T_ref = 1;  // completed reference state (refineInput)
    double gamma = 1.4;
    int mu_model = 0;               // viscosity law (lbm_config::mu_model)
    double upsilon = 0, S_v = 0;
    int nsteps = 0;
    std::vector<double> dx, dy;
    std::vector<uint8_t> type;  // [y*nx + x]
    std::vector<double> rho0, ux0, uy0, T0;  // [y*nx + x] initial node state
    // driver state (cpuLBM::step, residual, initRes, resNorm; main.cpp:34-70)
    int step = 0;
    double residual = 1, resNorm = 0, initRes[100] = {0};
};

// What a sample needs on the device apart from its place in a packing.
struct PreparedSample {
    SampleParams p{};  // offsets, first_tile and ntile are set when packed
    double fref[NPL] = {};
    std::vector<uint8_t> flags;  // node flags, ny rows of pitch bytes
    std::vector<WallNode> walls; // solid nodes next to fluid; sample field 0
    std::vector<double> tdx, tdy, dx, dy;
};

HostSample derive(const lbm_config &c, const lbm_init &in);
void prepare_sample(const HostSample &h, int prec, PreparedSample &out);
// append the tx x ty tiles of one sample (flags in pitch layout, sample
// flags sflags for its periodic axes) with the given sample index; gid
// numbers continue from out.size()
void cut_tiles(const uint8_t *flags, int pitch, int nx, int ny, int tx, int ty, int sflags, int gx, int sample,
               std::vector<Tile> &out);
// TMA descriptors of one sample (MAPS_PER_SAMPLE of them): stage buffers 2
// and 3 with the stencil halo box, and the state with the tile's own box
void encode_stage_maps(int prec, const SampleParams &p, unsigned char *state, unsigned char *buf2,
                       unsigned char *buf3, int tx, int ty, CUtensorMap *maps);
void check_tile_shape(int x, int y);
int round_up(int v, int m);

// A run of tiles in a device list.
struct TileRun {
    const Tile *p = nullptr;
    int n = 0;
};

// Device pointers and lengths of the packed lists one step launches over.
// The pointwise phase runs over the tiles of each RKMETHOD in sample order;
// the stencil phases over the same tiles as three runs, the simple tiles,
// the wrap tiles and the rest, one kernel per run, each compiled for its
// kind of tile alone.
struct StepLists {
    TileRun pointwise[4];                           // tiles by RKMETHOD, sample order
    TileRun simple[4], wrap[4], general[4];         // the same tiles by kind
    TileRun rk3_simple, rk3_wrap, rk3_general;      // RK3 tiles (final stencil phase)
    const WallNode *walls_all = nullptr, *walls_rk3 = nullptr;
    int n_walls_all = 0, n_walls_rk3 = 0;
    // the samples, for copying buffer 2's ghost columns (SampleParams::gx)
    // after the pointwise phase
    const SampleParams *samples = nullptr;
    int nsamples = 0;
    bool any_ghost = false;
};

// A device list of n tiles whose first ns are simple and next nw wrap
// tiles, as three runs.
inline void split_runs(const Tile *p, int n, int ns, int nw, TileRun &simple, TileRun &wrap, TileRun &general)
{
    simple.p = p;
    simple.n = ns;
    wrap.p = p ? p + ns : nullptr;
    wrap.n = nw;
    general.p = p ? p + ns + nw : nullptr;
    general.n = n - ns - nw;
}

// Reorder a host tile list by kind, simple tiles first, then wrap tiles,
// then the rest (each kind keeps its order); ns, nw: how many are simple
// and wrap tiles.
inline void order_by_kind(std::vector<Tile> &v, int &ns, int &nw)
{
    auto mid = std::stable_partition(v.begin(), v.end(), [](const Tile &t) { return tile_simple(t); });
    auto end = std::stable_partition(mid, v.end(), [](const Tile &t) { return tile_wrap(t); });
    ns = (int)(mid - v.begin());
    nw = (int)(end - mid);
}

template <class S, class C>
void stencil_runs(const KArgs<S> &a, int phase, int m, const TileRun &s, const TileRun &w, const TileRun &g,
                  cudaStream_t st)
{
    if (s.n) CU((launch_phase<S, C>(a, phase, m, s.p, s.n, nullptr, 0, st, FLUX_SIMPLE)));
    if (w.n) CU((launch_phase<S, C>(a, phase, m, w.p, w.n, nullptr, 0, st, FLUX_WRAP)));
    if (g.n) CU((launch_phase<S, C>(a, phase, m, g.p, g.n, nullptr, 0, st, FLUX_GENERAL)));
}

// One step: pointwise stages, walls, first stencil phase, and for RK3 the
// walls of buffer 3 and the final stencil phase.  ev (optional) receives
// events [0] start, after pointwise, walls 2, phase 1, walls 3, phase 2.
template <class S, class C>
void enqueue_step_phases(const KArgs<S> &a, const StepLists &l, cudaStream_t st, cudaEvent_t *ev = nullptr)
{
    if (ev) CU(cudaEventRecord(ev[0], st));
    for (int m = 0; m < 4; ++m)
        if (l.pointwise[m].n) CU((launch_phase<S, C>(a, 0, m, l.pointwise[m].p, l.pointwise[m].n, nullptr, 0, st)));
    if (l.any_ghost) CU(launch_fill_ghosts<S>(l.samples, 0, l.nsamples, a.buf2, nullptr, st));
    if (ev) CU(cudaEventRecord(ev[1], st));
    CU((launch_phase<S, C>(a, 3, 0, nullptr, 0, l.walls_all, l.n_walls_all, st)));
    if (ev) CU(cudaEventRecord(ev[2], st));
    for (int m = 0; m < 4; ++m) stencil_runs<S, C>(a, 1, m, l.simple[m], l.wrap[m], l.general[m], st);
    const bool rk3 = l.rk3_simple.n || l.rk3_wrap.n || l.rk3_general.n;
    if (ev) CU(cudaEventRecord(ev[3], st));
    if (rk3) CU((launch_phase<S, C>(a, 4, 1, nullptr, 0, l.walls_rk3, l.n_walls_rk3, st)));
    if (ev) CU(cudaEventRecord(ev[4], st));
    if (rk3) stencil_runs<S, C>(a, 2, 1, l.rk3_simple, l.rk3_wrap, l.rk3_general, st);
    if (ev) CU(cudaEventRecord(ev[5], st));
}

inline int step_launches(const StepLists &l)
{
    int n = l.any_ghost ? 1 : 0;
    for (int m = 0; m < 4; ++m)
        n += (l.pointwise[m].n ? 1 : 0) + (l.simple[m].n ? 1 : 0) + (l.wrap[m].n ? 1 : 0) + (l.general[m].n ? 1 : 0);
    n += l.n_walls_all ? 1 : 0;
    if (l.rk3_simple.n || l.rk3_wrap.n || l.rk3_general.n)
        n += (l.n_walls_rk3 ? 1 : 0) + (l.rk3_simple.n ? 1 : 0) + (l.rk3_wrap.n ? 1 : 0) + (l.rk3_general.n ? 1 : 0);
    return n;
}

}  // namespace uqlbm
