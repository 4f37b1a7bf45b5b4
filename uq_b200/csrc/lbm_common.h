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
// append the tx x ty tiles of one sample (flags in pitch layout) with the
// given sample index; gid numbers continue from out.size()
void cut_tiles(const uint8_t *flags, int pitch, int nx, int ny, int tx, int ty, int sample, std::vector<Tile> &out);
// TMA descriptors of one sample's stage buffers 2 and 3
void encode_stage_maps(int prec, const SampleParams &p, unsigned char *buf2, unsigned char *buf3, int tx, int ty,
                       CUtensorMap *maps2);
void check_tile_shape(int x, int y);
int round_up(int v, int m);

// Device pointers and lengths of the packed lists one step launches over.
struct StepLists {
    const Tile *by_rk[4] = {nullptr, nullptr, nullptr, nullptr};
    int n_by_rk[4] = {0, 0, 0, 0};
    const Tile *rk3 = nullptr;
    int n_rk3 = 0;
    const WallNode *walls_all = nullptr, *walls_rk3 = nullptr;
    int n_walls_all = 0, n_walls_rk3 = 0;
};

// One step: pointwise stages, walls, first stencil phase, and for RK3 the
// walls of buffer 3 and the final stencil phase.  ev (optional) receives
// events [0] start, after pointwise, walls 2, phase 1, walls 3, phase 2.
template <class S, class C>
void enqueue_step_phases(const KArgs<S> &a, const StepLists &l, cudaStream_t st, cudaEvent_t *ev = nullptr)
{
    if (ev) CU(cudaEventRecord(ev[0], st));
    for (int m = 0; m < 4; ++m)
        if (l.n_by_rk[m]) CU((launch_phase<S, C>(a, 0, m, l.by_rk[m], l.n_by_rk[m], nullptr, 0, st)));
    if (ev) CU(cudaEventRecord(ev[1], st));
    CU((launch_phase<S, C>(a, 3, 0, nullptr, 0, l.walls_all, l.n_walls_all, st)));
    if (ev) CU(cudaEventRecord(ev[2], st));
    for (int m = 0; m < 4; ++m)
        if (l.n_by_rk[m]) CU((launch_phase<S, C>(a, 1, m, l.by_rk[m], l.n_by_rk[m], nullptr, 0, st)));
    if (ev) CU(cudaEventRecord(ev[3], st));
    if (l.n_rk3) CU((launch_phase<S, C>(a, 4, 1, nullptr, 0, l.walls_rk3, l.n_walls_rk3, st)));
    if (ev) CU(cudaEventRecord(ev[4], st));
    if (l.n_rk3) CU((launch_phase<S, C>(a, 2, 1, l.rk3, l.n_rk3, nullptr, 0, st)));
    if (ev) CU(cudaEventRecord(ev[5], st));
}

inline int step_launches(const StepLists &l)
{
    int n = 0;
    for (int m = 0; m < 4; ++m) n += l.n_by_rk[m] ? 2 : 0;  // pointwise + stencil
    n += l.n_walls_all ? 1 : 0;
    if (l.n_rk3) n += (l.n_walls_rk3 ? 1 : 0) + 1;
    return n;
}

}  // namespace uqlbm
