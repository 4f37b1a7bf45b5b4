// Request server of the D2Q13 thermal LBM step (lbm_server_* in
// include/uq_lbm.h): continuous batching of independent solves.
//
// Threads.  The caller's threads submit solves and collect results.  The
// loop thread owns the device work: at every step boundary it retires
// finished / failed / cancelled solves, admits queued ones into free arena
// regions (moving the resident regions together when the free space is
// fragmented), repacks the tile and wall lists, and enqueues one step of all
// resident solves on its stream, at most kRunAhead steps ahead of the GPU.
// The collector thread waits for each retired solve's macroscopic fields,
// copies them to host memory and frees the region.
//
// Device memory.  One arena of cap_nodes node slots; a solve holds
// ny * pitch consecutive slots (pitch = nx rounded up to 32), which address
// its 26 planes in each of the state, stage-2 and stage-3 buffers, its wall
// factors and its node flags exactly as a batch lays out one sample.  When a
// solve retires its fields are written into its own stage-2 planes, which no
// later step reads, and copied out from there.
#include "lbm_common.h"

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace uqlbm {
namespace {

constexpr int kRunAhead = 3;      // steps the loop may enqueue ahead of the GPU
constexpr int kSnapRing = 64;     // pinned status snapshots in flight (> kRunAhead + 1)

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    int nx = 0, ny = 0;
    int steps_total = 0, steps_done = 0;
    PreparedSample ps;
    std::vector<Tile> tiles;     // local: sample 0, gid = local index | simple bit
    std::vector<double> fields;  // rho, ux, uy, T in [x*Ny + y] order until admitted
    std::vector<double> result;  // rho, ux, uy, T, p in [x*Ny + y] order when done
    long long nodes = 0;         // arena slots
    long long node_off = -1;
    int state = LBM_REQ_QUEUED;
    int bits = 0;                // device status bits gathered so far
    bool cancel = false;
    bool returned_any = false;   // reported by wait_any
    lbm_status status = LBM_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    long long step_admit = 0, step_done = 0;
};

// first-fit allocator over node slots
struct Arena {
    long long cap = 0, used = 0;
    std::map<long long, long long> holes;  // offset -> length
    void reset(long long c)
    {
        cap = c;
        used = 0;
        holes.clear();
        if (c > 0) holes[0] = c;
    }
    bool alloc(long long len, long long &off)
    {
        for (auto it = holes.begin(); it != holes.end(); ++it)
            if (it->second >= len) {
                off = it->first;
                const long long rest = it->second - len;
                holes.erase(it);
                if (rest) holes[off + len] = rest;
                used += len;
                return true;
            }
        return false;
    }
    void release(long long off, long long len)
    {
        used -= len;
        auto it = holes.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != holes.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            holes.erase(nx);
        }
        if (it != holes.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                holes.erase(it);
            }
        }
    }
    long long free_slots() const { return cap - used; }
};

// status words of one packing, read back after the steps before it
struct Snapshot {
    int *bits = nullptr;  // pinned, one per packed solve
    std::vector<Request *> pack;
    cudaEvent_t ev = nullptr;
    bool applied = false;
    ~Snapshot()
    {
        if (ev) cudaEventDestroy(ev);
    }
};

// a retired solve whose fields are being copied out
struct Retired {
    Request *r;
    std::shared_ptr<Snapshot> snap;
};

}  // namespace
}  // namespace uqlbm

using namespace uqlbm;

struct lbm_server {
    int prec = LBM_PREC_F32;
    int tx = TILE_CX, ty = TILE_CY;
    int device = 0;
    bool use_graph = true;
    int max_resident = 1024, max_queued = 0, poll_steps = 32;
    int fast_k = 4;  // steps per server step of the fast set
    size_t es = 4;
    size_t arena_bytes = 0;
    Clock::time_point t0;

    cudaStream_t stream = nullptr, copy_stream = nullptr;
    // arena
    Arena arena;
    DevBuf<unsigned char> state, buf2, buf3, alpha;
    DevBuf<uint8_t> nflags;
    DevBuf<double> scratch;  // admission fields
    // packing (loop thread only)
    std::vector<Request *> packed;
    std::vector<SampleParams> sp;
    std::vector<Tile> tiles_all, tiles_rk3, tiles_by_rk[4];
    // stencil-phase lists: the simple tiles of every solve, then the others
    // stencil runs being built: simple tiles (flux_by_rk, tiles_rk3), wrap
    // tiles and the rest, concatenated in that order
    std::vector<Tile> flux_by_rk[4], gen_rk3, gen_by_rk[4], wrap_rk3, wrap_by_rk[4];
    std::vector<WallNode> walls_all, walls_rk3;
    std::vector<double> v_tdx, v_tdy, v_dx, v_dy, v_fref;
    std::vector<CUtensorMap> maps;
    DevBuf<SampleParams> d_sp;
    DevBuf<Tile> d_tiles_rk3, d_tiles_by_rk[4], d_flux_by_rk[4];
    DevBuf<WallNode> d_walls_all, d_walls_rk3;
    DevBuf<double> d_tdx, d_tdy, d_dx, d_dy, d_fref;
    DevBuf<CUtensorMap> d_maps;
    DevBuf<int> d_status;
    StepLists lists;
    long long packed_nodes = 0;  // lattice nodes of the resident set
    // fast set: the first n_fast packed solves, whose tiles and walls are
    // prefixes of every list (of both tile runs); fast_lists holds those
    // prefixes
    int n_fast = 0;
    StepLists fast_lists;
    long long fast_nodes = 0;
    cudaGraphExec_t graph = nullptr;
    int stable_steps = 0;
    int *pinned_bits = nullptr;  // kSnapRing x max_resident
    int snap_slot = 0;
    std::deque<std::shared_ptr<Snapshot>> snaps;  // not yet applied, oldest first
    cudaEvent_t ev_step[kRunAhead] = {};
    long long steps_enqueued = 0;

    // shared state
    std::mutex mu;
    std::condition_variable cv_loop, cv_done, cv_collect;
    std::deque<Request *> queue;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::deque<Retired> to_collect;
    std::deque<long long> finished;  // for wait_any
    long long next_id = 1;
    bool stopping = false;
    lbm_status fatal = LBM_OK;
    std::string fatal_msg;
    int awaiting_copy = 0;
    lbm_server_stats stats{};
    Clock::time_point busy_since;
    bool busy = false;

    std::thread loop_thread, collect_thread;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    // ------------------------------------------------------------ set-up
    void create(const lbm_server_options *opt)
    {
        prec = opt ? opt->precision : LBM_PREC_F32;
        if (prec != LBM_PREC_F64 && prec != LBM_PREC_F32) throw LbmError(LBM_ERR_INVALID, "unknown precision");
        es = prec == LBM_PREC_F64 ? 8 : 4;
        if (opt && opt->tile_x > 0) tx = opt->tile_x;
        if (opt && opt->tile_y > 0) ty = opt->tile_y;
        check_tile_shape(tx, ty);
        use_graph = opt ? opt->use_graph != 0 : true;
        if (opt && opt->max_resident > 0) max_resident = opt->max_resident;
        if (opt && opt->max_queued > 0) max_queued = opt->max_queued;
        if (opt && opt->status_poll_steps > 0) poll_steps = opt->status_poll_steps;
        if (opt && opt->fast_lane_steps > 0) fast_k = opt->fast_lane_steps;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
            throw LbmError(LBM_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
        CU(cudaGetDevice(&device));
        size_t free_b = 0, total_b = 0;
        CU(cudaMemGetInfo(&free_b, &total_b));
        arena_bytes = opt ? opt->arena_bytes : 0;
        if (arena_bytes == 0) {
            double frac = opt && opt->hbm_fraction > 0 ? opt->hbm_fraction : 0.6;
            if (frac > 0.9) frac = 0.9;
            arena_bytes = (size_t)(frac * (double)free_b);
        }
        // per node slot: 26 planes in three buffers, the wall factor, the flags
        const size_t per_node = 3 * NPL * es + es + 1;
        const long long cap = (long long)(arena_bytes / per_node) / 32 * 32;
        if (cap < 32 * 32) throw LbmError(LBM_ERR_NOMEM, "arena too small");
        if ((size_t)cap * per_node > free_b) throw LbmError(LBM_ERR_NOMEM, "arena larger than the free device memory");
        arena.reset(cap);
        state.alloc((size_t)cap * NPL * es);
        buf2.alloc((size_t)cap * NPL * es);
        buf3.alloc((size_t)cap * NPL * es);
        alpha.alloc((size_t)cap * es);
        nflags.alloc((size_t)cap);
        scratch.alloc((size_t)4 * 1024 * 1024);
        d_status.alloc(max_resident);
        CU(cudaMemset(d_status.p, 0, sizeof(int) * max_resident));
        CU(cudaHostAlloc(&pinned_bits, sizeof(int) * (size_t)kSnapRing * max_resident, cudaHostAllocDefault));
        CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CU(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
        for (auto &e : ev_step) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        if (prec == LBM_PREC_F64) CU((prepare_kernels<double, double>()));
        else CU((prepare_kernels<float, float>()));
        stats.arena_nodes = cap;
        stats.arena_bytes = (size_t)cap * per_node;
        t0 = Clock::now();
        loop_thread = std::thread([this] { run_loop(); });
        collect_thread = std::thread([this] { run_collector(); });
    }

    void shutdown()
    {
        {
            std::lock_guard<std::mutex> g(mu);
            stopping = true;
        }
        cv_loop.notify_all();
        cv_collect.notify_all();
        cv_done.notify_all();
        if (loop_thread.joinable()) loop_thread.join();
        if (collect_thread.joinable()) collect_thread.join();
        if (stream) cudaStreamSynchronize(stream);
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        snaps.clear();
        to_collect.clear();
        for (auto &e : ev_step)
            if (e) cudaEventDestroy(e);
        if (pinned_bits) cudaFreeHost(pinned_bits);
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }

    // ------------------------------------------------------------ submit
    long long submit(const lbm_config &cfg, const lbm_init &init)
    {
        std::unique_ptr<Request> r(new Request);
        HostSample h = derive(cfg, init);
        if (h.nsteps < 1) throw LbmError(LBM_ERR_INVALID, "a served solve needs a step count (steps, tt_tref or tt_time)");
        prepare_sample(h, prec, r->ps);
        r->nx = h.nx;
        r->ny = h.ny;
        r->steps_total = h.nsteps;
        // node slots: the planes, and room for GHOST_SLACK state elements
        r->nodes = r->ps.p.plane + (r->ps.p.gx ? (GHOST_SLACK + NPL - 1) / NPL : 0);
        cut_tiles(r->ps.flags.data(), r->ps.p.pitch, h.nx, h.ny, tx, ty, r->ps.p.flags, r->ps.p.gx, 0, r->tiles);
        const long long n = (long long)h.nx * h.ny;
        r->fields.resize(4 * n);
        for (int x = 0; x < h.nx; ++x)
            for (int y = 0; y < h.ny; ++y) {
                const size_t src = (size_t)y * h.nx + x;
                const long long k = (long long)x * h.ny + y;
                r->fields[k] = h.rho0[src];
                r->fields[n + k] = h.ux0[src];
                r->fields[2 * n + k] = h.uy0[src];
                r->fields[3 * n + k] = h.T0[src];
            }
        std::lock_guard<std::mutex> g(mu);
        if (fatal != LBM_OK) throw LbmError(fatal, fatal_msg);
        if (stopping) throw LbmError(LBM_ERR_INVALID, "server is stopping");
        if (r->nodes > arena.cap) throw LbmError(LBM_ERR_NOMEM, "solve larger than the server's arena");
        if (max_queued > 0 && (int)queue.size() >= max_queued) throw LbmError(LBM_ERR_BUSY, "queue full");
        r->id = next_id++;
        r->t_submit = now();
        const long long id = r->id;
        queue.push_back(r.get());
        reqs[id] = std::move(r);
        stats.submitted++;
        cv_loop.notify_all();
        return id;
    }

    // ------------------------------------------------------------ snapshots
    // fold device status bits into their solves (mu held)
    static void apply(Snapshot &s)
    {
        if (s.applied) return;
        for (size_t k = 0; k < s.pack.size(); ++k) s.pack[k]->bits |= s.bits[k];
        s.applied = true;
    }

    void poll_snaps_locked()
    {
        while (!snaps.empty()) {
            Snapshot &s = *snaps.front();
            if (!s.applied) {
                const cudaError_t e = cudaEventQuery(s.ev);
                if (e == cudaErrorNotReady) break;
                CU(e);
                apply(s);
            }
            snaps.pop_front();
        }
    }

    // copy the status words of the current packing and clear them
    std::shared_ptr<Snapshot> enqueue_snapshot()
    {
        auto s = std::make_shared<Snapshot>();
        s->bits = pinned_bits + (size_t)snap_slot * max_resident;
        snap_slot = (snap_slot + 1) % kSnapRing;
        s->pack = packed;
        if (!packed.empty()) {
            CU(cudaMemcpyAsync(s->bits, d_status.p, sizeof(int) * packed.size(), cudaMemcpyDeviceToHost, stream));
            CU(cudaMemsetAsync(d_status.p, 0, sizeof(int) * packed.size(), stream));
        }
        CU(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming));
        CU(cudaEventRecord(s->ev, stream));
        return s;
    }

    // ------------------------------------------------------------ packing
    void repack()
    {
        sp.clear();
        tiles_all.clear();
        tiles_rk3.clear();
        for (auto &v : tiles_by_rk) v.clear();
        gen_rk3.clear();
        wrap_rk3.clear();
        for (auto &v : gen_by_rk) v.clear();
        for (auto &v : wrap_by_rk) v.clear();
        for (auto &v : flux_by_rk) v.clear();
        walls_all.clear();
        walls_rk3.clear();
        v_tdx.clear();
        v_tdy.clear();
        v_dx.clear();
        v_dy.clear();
        v_fref.clear();
        maps.resize(MAPS_PER_SAMPLE * packed.size());
        packed_nodes = 0;
        for (size_t k = 0; k < packed.size(); ++k) {
            Request *r = packed[k];
            SampleParams p = r->ps.p;
            p.node_off = r->node_off;
            // the first row's left ghosts (SampleParams::gx) before plane 0
            p.state_off = (long long)NPL * r->node_off + (p.gx ? GHOST_SLACK : 0);
            p.xoff = (int)v_tdx.size();
            p.yoff = (int)v_tdy.size();
            p.first_tile = (int)tiles_all.size();
            p.ntile = (int)r->tiles.size();
            for (const Tile &lt : r->tiles) {
                Tile t = lt;
                t.sample = (int)k;
                t.gid = (int)tiles_all.size() | (lt.gid & (TILE_SIMPLE | TILE_WRAP));
                tiles_all.push_back(t);
                tiles_by_rk[p.rk].push_back(t);
                const bool simple = tile_simple(t), wrap = tile_wrap(t);
                (simple ? flux_by_rk[p.rk] : wrap ? wrap_by_rk[p.rk] : gen_by_rk[p.rk]).push_back(t);
                if (p.rk == 1) (simple ? tiles_rk3 : wrap ? wrap_rk3 : gen_rk3).push_back(t);
            }
            for (WallNode w : r->ps.walls) {
                w.sample = (int)k;
                walls_all.push_back(w);
                if (p.rk == 1) walls_rk3.push_back(w);
            }
            v_tdx.insert(v_tdx.end(), r->ps.tdx.begin(), r->ps.tdx.end());
            v_tdy.insert(v_tdy.end(), r->ps.tdy.begin(), r->ps.tdy.end());
            v_dx.insert(v_dx.end(), r->ps.dx.begin(), r->ps.dx.end());
            v_dy.insert(v_dy.end(), r->ps.dy.begin(), r->ps.dy.end());
            v_fref.insert(v_fref.end(), r->ps.fref, r->ps.fref + NPL);
            encode_stage_maps(prec, p, state.p, buf2.p, buf3.p, tx, ty, &maps[MAPS_PER_SAMPLE * k]);
            sp.push_back(p);
            packed_nodes += (long long)r->nx * r->ny;
        }
        int ns_by_rk[4], nw_by_rk[4], ns_rk3 = (int)tiles_rk3.size(), nw_rk3 = (int)wrap_rk3.size();
        for (int m = 0; m < 4; ++m) {
            ns_by_rk[m] = (int)flux_by_rk[m].size();
            nw_by_rk[m] = (int)wrap_by_rk[m].size();
            flux_by_rk[m].insert(flux_by_rk[m].end(), wrap_by_rk[m].begin(), wrap_by_rk[m].end());
            flux_by_rk[m].insert(flux_by_rk[m].end(), gen_by_rk[m].begin(), gen_by_rk[m].end());
        }
        tiles_rk3.insert(tiles_rk3.end(), wrap_rk3.begin(), wrap_rk3.end());
        tiles_rk3.insert(tiles_rk3.end(), gen_rk3.begin(), gen_rk3.end());
        d_sp.upload_keep(sp, stream);
        for (int m = 0; m < 4; ++m) {
            d_tiles_by_rk[m].upload_keep(tiles_by_rk[m], stream);
            d_flux_by_rk[m].upload_keep(flux_by_rk[m], stream);
        }
        d_tiles_rk3.upload_keep(tiles_rk3, stream);
        d_walls_all.upload_keep(walls_all, stream);
        d_walls_rk3.upload_keep(walls_rk3, stream);
        d_tdx.upload_keep(v_tdx, stream);
        d_tdy.upload_keep(v_tdy, stream);
        d_dx.upload_keep(v_dx, stream);
        d_dy.upload_keep(v_dy, stream);
        d_fref.upload_keep(v_fref, stream);
        d_maps.upload_keep(maps, stream);
        lists = StepLists{};
        for (int m = 0; m < 4; ++m) {
            lists.pointwise[m] = TileRun{d_tiles_by_rk[m].p, (int)tiles_by_rk[m].size()};
            split_runs(d_flux_by_rk[m].p, (int)flux_by_rk[m].size(), ns_by_rk[m], nw_by_rk[m], lists.simple[m],
                       lists.wrap[m], lists.general[m]);
        }
        split_runs(d_tiles_rk3.p, (int)tiles_rk3.size(), ns_rk3, nw_rk3, lists.rk3_simple, lists.rk3_wrap,
                   lists.rk3_general);
        lists.samples = d_sp.p;
        lists.nsamples = (int)sp.size();
        lists.any_ghost = std::any_of(sp.begin(), sp.end(), [](const SampleParams &q) { return q.gx != 0; });
        lists.walls_all = d_walls_all.p;
        lists.n_walls_all = (int)walls_all.size();
        lists.walls_rk3 = d_walls_rk3.p;
        lists.n_walls_rk3 = (int)walls_rk3.size();
        fast_lists = lists;
        for (int m = 0; m < 4; ++m)
            fast_lists.pointwise[m].n = fast_lists.simple[m].n = fast_lists.wrap[m].n = fast_lists.general[m].n = 0;
        fast_lists.rk3_simple.n = fast_lists.rk3_wrap.n = fast_lists.rk3_general.n = 0;
        fast_lists.n_walls_all = fast_lists.n_walls_rk3 = 0;
        fast_nodes = 0;
        for (int k = 0; k < n_fast; ++k) {
            const Request *r = packed[k];
            int ns = 0, nwr = 0;
            for (const Tile &t : r->tiles) {
                ns += tile_simple(t) ? 1 : 0;
                nwr += tile_wrap(t) ? 1 : 0;
            }
            const int ng = (int)r->tiles.size() - ns - nwr, nw = (int)r->ps.walls.size();
            const int m = r->ps.p.rk;
            fast_lists.pointwise[m].n += ns + nwr + ng;
            fast_lists.simple[m].n += ns;
            fast_lists.wrap[m].n += nwr;
            fast_lists.general[m].n += ng;
            fast_lists.n_walls_all += nw;
            if (m == 1) {
                fast_lists.rk3_simple.n += ns;
                fast_lists.rk3_wrap.n += nwr;
                fast_lists.rk3_general.n += ng;
                fast_lists.n_walls_rk3 += nw;
            }
            fast_nodes += (long long)r->nx * r->ny;
        }
        if (graph) {
            CU(cudaGraphExecDestroy(graph));
            graph = nullptr;
        }
        stable_steps = 0;
        stats.repacks++;
    }

    template <class S>
    KArgs<S> args() const
    {
        KArgs<S> a{};
        a.samples = d_sp.p;
        a.tiles = nullptr;
        a.ntiles = 0;
        a.tx = tx;
        a.ty = ty;
        a.state = reinterpret_cast<S *>(state.p);
        a.buf2 = reinterpret_cast<S *>(buf2.p);
        a.buf3 = reinterpret_cast<S *>(buf3.p);
        a.nflags = nflags.p;
        a.alpha_raw = alpha.p;
        a.told = nullptr;
        a.partial = nullptr;
        a.status = d_status.p;
        a.tdx = d_tdx.p;
        a.tdy = d_tdy.p;
        a.dxv = d_dx.p;
        a.dyv = d_dy.p;
        a.tmaps = d_maps.p;
        a.fref = d_fref.p;
        a.want_residual = 0;
        a.eq_tol = 1e-6;
        return a;
    }

    // one server step: every resident solve one step, then the fast set
    // fast_k - 1 more (the same launches over the lists' prefixes)
    void enqueue_one_step()
    {
        if (prec == LBM_PREC_F64) {
            enqueue_step_phases<double, double>(args<double>(), lists, stream);
            for (int j = 1; n_fast && j < fast_k; ++j)
                enqueue_step_phases<double, double>(args<double>(), fast_lists, stream);
        } else {
            enqueue_step_phases<float, float>(args<float>(), lists, stream);
            for (int j = 1; n_fast && j < fast_k; ++j)
                enqueue_step_phases<float, float>(args<float>(), fast_lists, stream);
        }
    }

    void step_once()
    {
        // bound how far the host runs ahead of the GPU
        const int slot = (int)(steps_enqueued % kRunAhead);
        if (steps_enqueued >= kRunAhead) CU(cudaEventSynchronize(ev_step[slot]));
        if (use_graph && !graph && stable_steps >= 2) {
            const auto t0 = Clock::now();
            cudaGraph_t g;
            CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_one_step();
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                throw;
            }
            CU(cudaStreamEndCapture(stream, &g));
            CU(cudaGraphInstantiate(&graph, g, 0));
            cudaGraphDestroy(g);
            stats.graph_captures++;
            stats.capture_seconds += std::chrono::duration<double>(Clock::now() - t0).count();
        }
        if (graph) {
            CU(cudaGraphLaunch(graph, stream));
            stats.steps_graph++;
        } else {
            enqueue_one_step();
            stats.steps_eager++;
        }
        CU(cudaEventRecord(ev_step[slot], stream));
        steps_enqueued++;
        stable_steps++;
    }

    // ------------------------------------------------------------ regions
    // device-to-device move of one solve's planes and flags via a bounce
    // buffer (source and destination may overlap)
    void move_region(Request *r, long long new_off, DevBuf<unsigned char> &bounce)
    {
        const size_t pbytes = (size_t)NPL * r->nodes * es;
        const size_t so = (size_t)NPL * r->node_off * es, sn = (size_t)NPL * new_off * es;
        DevBuf<unsigned char> *arrs[3] = {&state, &buf2, &buf3};
        for (auto *a : arrs) {
            CU(cudaMemcpyAsync(bounce.p, a->p + so, pbytes, cudaMemcpyDeviceToDevice, stream));
            CU(cudaMemcpyAsync(a->p + sn, bounce.p, pbytes, cudaMemcpyDeviceToDevice, stream));
        }
        CU(cudaMemcpyAsync(bounce.p, nflags.p + r->node_off, r->nodes, cudaMemcpyDeviceToDevice, stream));
        CU(cudaMemcpyAsync(nflags.p + new_off, bounce.p, r->nodes, cudaMemcpyDeviceToDevice, stream));
    }

    // pack the resident regions at the start of the arena (mu held; no
    // region is waiting to be copied out)
    void compact_locked()
    {
        std::vector<Request *> order(packed);
        std::sort(order.begin(), order.end(), [](Request *a, Request *b) { return a->node_off < b->node_off; });
        long long biggest = 0;
        for (Request *r : order) biggest = std::max(biggest, r->nodes);
        DevBuf<unsigned char> bounce;
        bounce.alloc((size_t)NPL * biggest * es);
        long long off = 0;
        for (Request *r : order) {
            if (r->node_off != off) move_region(r, off, bounce);
            r->node_off = off;
            off += r->nodes;
        }
        CU(cudaStreamSynchronize(stream));
        arena.reset(arena.cap);
        long long dummy;
        if (off > 0) arena.alloc(off, dummy);
        stats.compactions++;
    }

    // zero a new solve's region, upload its flags and initial state
    // (initialiseFunctions, cpuLBM.cpp:846-875)
    void init_solve(Request *r, int k)
    {
        const size_t pbytes = (size_t)NPL * r->nodes * es, so = (size_t)NPL * r->node_off * es;
        CU(cudaMemsetAsync(state.p + so, 0, pbytes, stream));
        CU(cudaMemsetAsync(buf2.p + so, 0, pbytes, stream));
        CU(cudaMemsetAsync(buf3.p + so, 0, pbytes, stream));
        CU(cudaMemsetAsync(alpha.p + (size_t)r->node_off * es, 0, (size_t)r->nodes * es, stream));
        CU(cudaMemcpyAsync(nflags.p + r->node_off, r->ps.flags.data(), r->nodes, cudaMemcpyHostToDevice, stream));
        const long long n = (long long)r->nx * r->ny;
        if ((size_t)(4 * n) > scratch.n) {
            CU(cudaStreamSynchronize(stream));
            scratch.alloc((size_t)4 * n);
        }
        CU(cudaMemcpyAsync(scratch.p, r->fields.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice, stream));
        if (prec == LBM_PREC_F64)
            CU(launch_set_macro<double>(d_sp.p, k, reinterpret_cast<double *>(state.p), reinterpret_cast<double *>(buf2.p),
                                        reinterpret_cast<double *>(buf3.p), scratch.p, nflags.p, d_fref.p, n, stream));
        else
            CU(launch_set_macro<float>(d_sp.p, k, reinterpret_cast<float *>(state.p), reinterpret_cast<float *>(buf2.p),
                                       reinterpret_cast<float *>(buf3.p), scratch.p, nflags.p, d_fref.p, n, stream));
        // the ghost columns of the new solve's stage buffers (SampleParams::gx)
        if (r->ps.p.gx) {
            if (prec == LBM_PREC_F64)
                CU(launch_fill_ghosts<double>(d_sp.p, k, 1, reinterpret_cast<double *>(buf2.p),
                                              reinterpret_cast<double *>(buf3.p), stream));
            else
                CU(launch_fill_ghosts<float>(d_sp.p, k, 1, reinterpret_cast<float *>(buf2.p),
                                             reinterpret_cast<float *>(buf3.p), stream));
        }
    }

    double *result_ptr(const Request *r) const
    {
        return reinterpret_cast<double *>(buf2.p + (size_t)NPL * r->node_off * es);
    }

    // ------------------------------------------------------------ loop
    void run_loop()
    {
        try {
            CU(cudaSetDevice(device));
            loop_body();
        } catch (const LbmError &e) {
            fail_all(e.code, e.what());
        } catch (const std::exception &e) {
            fail_all(LBM_ERR_CUDA, e.what());
        }
    }

    void fail_all(lbm_status code, const std::string &msg)
    {
        std::lock_guard<std::mutex> g(mu);
        fatal = code;
        fatal_msg = msg;
        stopping = true;
        const double t = now();
        for (auto &kv : reqs) {
            Request *r = kv.second.get();
            if (r->state != LBM_REQ_DONE) {
                r->state = LBM_REQ_DONE;
                r->status = code;
                r->t_done = t;
                finished.push_back(r->id);
            }
        }
        queue.clear();
        cv_done.notify_all();
        cv_collect.notify_all();
    }

    void loop_body()
    {
        for (;;) {
            std::vector<Request *> leaving, joining, staying;
            {
                std::unique_lock<std::mutex> lk(mu);
                poll_snaps_locked();
                if (packed.empty() && queue.empty()) {
                    set_busy_locked(false);
                    if (stopping) return;
                    cv_loop.wait(lk, [&] { return stopping || !queue.empty(); });
                    continue;
                }
                if (stopping) return;
                for (Request *r : packed) {
                    if (r->steps_done >= r->steps_total || r->bits != 0 || r->cancel) leaving.push_back(r);
                    else staying.push_back(r);
                }
                // a fast solve with fewer than fast_k steps left must leave
                // the fast set before the next server step
                for (int k = 0; k < n_fast; ++k)
                    if (packed[k]->steps_total - packed[k]->steps_done < fast_k) rebuild_needed = true;
                // FIFO admission into free arena regions
                bool compacted = false;
                while (!queue.empty() && (int)(staying.size() + joining.size()) < max_resident) {
                    Request *r = queue.front();
                    if (r->cancel) {
                        queue.pop_front();
                        finish_locked(r, LBM_ERR_CANCELLED);
                        continue;
                    }
                    long long off = 0;
                    bool got = arena.alloc(r->nodes, off);
                    if (!got && !compacted && awaiting_copy == 0 && leaving.empty() && joining.empty() &&
                        arena.free_slots() >= r->nodes) {
                        // fragmented: move the resident regions together
                        // (their offsets change, so the packing is rebuilt)
                        compact_locked();
                        compacted = true;
                        rebuild_needed = true;
                        got = arena.alloc(r->nodes, off);
                    }
                    if (!got) break;
                    queue.pop_front();
                    r->node_off = off;
                    r->state = LBM_REQ_RESIDENT;
                    r->t_admit = now();
                    r->step_admit = stats.steps;
                    stats.admitted++;
                    joining.push_back(r);
                }
                set_busy_locked(!staying.empty() || !joining.empty());
                if (staying.empty() && joining.empty() && leaving.empty()) {
                    // nothing resident and the queue head does not fit yet:
                    // wait for the collector to free a region
                    cv_loop.wait_for(lk, std::chrono::milliseconds(2));
                    continue;
                }
            }
            if (!leaving.empty() || !joining.empty() || rebuild_needed) {
                const auto t0 = Clock::now();
                boundary(leaving, staying, joining);
                stats.boundary_seconds += std::chrono::duration<double>(Clock::now() - t0).count();
            }
            rebuild_needed = false;
            if (packed.empty()) continue;
            step_once();
            {
                std::lock_guard<std::mutex> g(mu);
                for (size_t k = 0; k < packed.size(); ++k) packed[k]->steps_done += (int)k < n_fast ? fast_k : 1;
                stats.steps++;
                stats.lattice_updates += packed_nodes + (long long)(fast_k - 1) * fast_nodes;
            }
            if (stats.steps % poll_steps == 0) {
                auto s = enqueue_snapshot();
                std::lock_guard<std::mutex> g(mu);
                snaps.push_back(s);
            }
        }
    }
    bool rebuild_needed = false;

    void set_busy_locked(bool b)
    {
        const auto t = Clock::now();
        if (b && !busy) busy_since = t;
        if (!b && busy) stats.busy_seconds += std::chrono::duration<double>(t - busy_since).count();
        busy = b;
    }

    // mu held
    void finish_locked(Request *r, lbm_status st)
    {
        r->state = LBM_REQ_DONE;
        r->status = st;
        r->t_done = now();
        r->step_done = stats.steps;
        r->fields.clear();
        r->fields.shrink_to_fit();
        if (st == LBM_ERR_CANCELLED) stats.cancelled++;
        else if (st != LBM_OK) stats.failed++;
        else stats.completed++;
        finished.push_back(r->id);
        cv_done.notify_all();
    }

    // Order the packing smallest first and choose the fast set: the leading
    // solves with at least fast_k steps left, each at most 1/16 of the
    // resident nodes and together at most 1/4 (mu held).
    void order_fast_locked()
    {
        n_fast = 0;
        if (fast_k <= 1 || packed.size() < 2) return;
        long long total = 0;
        for (const Request *r : packed) total += r->nodes;
        auto eligible = [&](const Request *r) {
            return r->steps_total - r->steps_done >= fast_k && r->nodes * 16 <= total;
        };
        std::stable_sort(packed.begin(), packed.end(), [&](const Request *a, const Request *b) {
            const bool ea = eligible(a), eb = eligible(b);
            if (ea != eb) return ea;
            return a->nodes < b->nodes;
        });
        long long sum = 0;
        while (n_fast < (int)packed.size() && eligible(packed[n_fast]) && (sum + packed[n_fast]->nodes) * 4 <= total)
            sum += packed[n_fast++]->nodes;
    }

    // step boundary with a membership change: fields of leaving solves into
    // their stage-2 planes, status words of the old packing, the new
    // packing, then the initial state of joining solves
    void boundary(const std::vector<Request *> &leaving, const std::vector<Request *> &staying,
                  const std::vector<Request *> &joining)
    {
        for (Request *r : leaving) {
            size_t k = 0;
            while (packed[k] != r) ++k;
            const long long n = (long long)r->nx * r->ny;
            if (prec == LBM_PREC_F64)
                CU(launch_macro_out<double>(d_sp.p, (int)k, reinterpret_cast<double *>(state.p), result_ptr(r), n, stream));
            else
                CU(launch_macro_out<float>(d_sp.p, (int)k, reinterpret_cast<float *>(state.p), result_ptr(r), n, stream));
        }
        std::shared_ptr<Snapshot> snap = enqueue_snapshot();
        {
            std::lock_guard<std::mutex> g(mu);
            snaps.push_back(snap);
            for (Request *r : leaving) {
                r->step_done = stats.steps;
                to_collect.push_back(Retired{r, snap});
                awaiting_copy++;
            }
        }
        if (!leaving.empty()) cv_collect.notify_all();
        {
            std::lock_guard<std::mutex> g(mu);
            packed = staying;
            packed.insert(packed.end(), joining.begin(), joining.end());
            order_fast_locked();
        }
        repack();
        for (Request *r : joining) {
            int k = 0;
            while (packed[k] != r) ++k;
            init_solve(r, k);
            // pageable sources are staged when the copy call returns
            std::lock_guard<std::mutex> g(mu);
            r->fields.clear();
            r->fields.shrink_to_fit();
            r->ps.flags.clear();
            r->ps.flags.shrink_to_fit();
        }
    }

    // ------------------------------------------------------------ collector
    void run_collector()
    {
        try {
            CU(cudaSetDevice(device));
            for (;;) {
                Retired job;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv_collect.wait(lk, [&] { return stopping || !to_collect.empty(); });
                    if (to_collect.empty()) return;  // stopping
                    job = to_collect.front();
                    to_collect.pop_front();
                }
                Request *r = job.r;
                CU(cudaEventSynchronize(job.snap->ev));
                const long long n = (long long)r->nx * r->ny;
                std::vector<double> out(5 * n);
                CU(cudaMemcpyAsync(out.data(), result_ptr(r), sizeof(double) * 5 * n, cudaMemcpyDeviceToHost,
                                   copy_stream));
                CU(cudaStreamSynchronize(copy_stream));
                std::lock_guard<std::mutex> g(mu);
                // fold in every earlier snapshot too: none may still point
                // at this request once the caller can release it
                poll_snaps_locked();
                apply(*job.snap);
                r->result.swap(out);
                arena.release(r->node_off, r->nodes);
                awaiting_copy--;
                lbm_status st = LBM_OK;
                if (r->cancel && r->steps_done < r->steps_total) st = LBM_ERR_CANCELLED;
                else if (r->bits & STATUS_TIMEOUT) st = LBM_ERR_TIMEOUT;
                else if (r->bits & STATUS_EQ) st = LBM_ERR_EQUILIBRIUM;
                else if (r->bits & STATUS_NONFINITE) st = LBM_ERR_NONFINITE;
                finish_locked(r, st);
                cv_loop.notify_all();
            }
        } catch (const LbmError &e) {
            fail_all(e.code, e.what());
        } catch (const std::exception &e) {
            fail_all(LBM_ERR_CUDA, e.what());
        }
    }

    // ------------------------------------------------------------ queries
    Request *find_locked(long long id)
    {
        auto it = reqs.find(id);
        if (it == reqs.end()) throw LbmError(LBM_ERR_NOT_FOUND, "unknown request id");
        return it->second.get();
    }
};

// ---------------------------------------------------------------- C ABI
#define SRV_BEGIN try {
#define SRV_END                                          \
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

LBM_API lbm_status lbm_server_create(const lbm_server_options *opt, lbm_server **out)
{
    SRV_BEGIN
    if (!out) throw LbmError(LBM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    std::unique_ptr<lbm_server> s(new lbm_server);
    try {
        s->create(opt);
    } catch (...) {
        s->shutdown();
        throw;
    }
    *out = s.release();
    return LBM_OK;
    SRV_END
}

LBM_API lbm_status lbm_server_submit(lbm_server *s, const lbm_config *cfg, const lbm_init *init, long long *id)
{
    SRV_BEGIN
    if (!s || !cfg || !init || !id) throw LbmError(LBM_ERR_INVALID, "NULL argument");
    *id = s->submit(*cfg, *init);
    return LBM_OK;
    SRV_END
}

static bool wait_pred(lbm_server *s, std::unique_lock<std::mutex> &lk, double timeout_s,
                      const std::function<bool()> &pred)
{
    if (timeout_s < 0) {
        s->cv_done.wait(lk, pred);
        return true;
    }
    return s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
}

LBM_API lbm_status lbm_server_wait(lbm_server *s, long long id, double timeout_s)
{
    SRV_BEGIN
    if (!s) throw LbmError(LBM_ERR_INVALID, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    Request *r = s->find_locked(id);
    const bool ok = wait_pred(s, lk, timeout_s, [&] { return r->state == LBM_REQ_DONE; });
    if (!ok) throw LbmError(LBM_ERR_TIMEOUT, "request not done yet");
    return LBM_OK;
    SRV_END
}

LBM_API lbm_status lbm_server_wait_any(lbm_server *s, double timeout_s, long long *id)
{
    SRV_BEGIN
    if (!s || !id) throw LbmError(LBM_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        const bool ok = wait_pred(s, lk, timeout_s, [&] { return !s->finished.empty() || s->stopping; });
        if (!ok) throw LbmError(LBM_ERR_TIMEOUT, "no request finished in time");
        if (s->finished.empty()) throw LbmError(s->fatal != LBM_OK ? s->fatal : LBM_ERR_INVALID, "server stopped");
        const long long f = s->finished.front();
        s->finished.pop_front();
        auto it = s->reqs.find(f);
        if (it == s->reqs.end() || it->second->returned_any) continue;  // released meanwhile
        it->second->returned_any = true;
        *id = f;
        return LBM_OK;
    }
    SRV_END
}

LBM_API lbm_status lbm_server_info(lbm_server *s, long long id, lbm_request_info *info)
{
    SRV_BEGIN
    if (!s || !info) throw LbmError(LBM_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> g(s->mu);
    const Request *r = s->find_locked(id);
    info->id = r->id;
    info->Nx = r->nx;
    info->Ny = r->ny;
    info->steps_total = r->steps_total;
    info->steps_done = r->steps_done;
    info->state = r->state;
    info->status = r->status;
    info->t_submit = r->t_submit;
    info->t_admit = r->t_admit;
    info->t_done = r->t_done;
    info->step_admit = r->step_admit;
    info->step_done = r->step_done;
    return LBM_OK;
    SRV_END
}

LBM_API lbm_status lbm_server_result(lbm_server *s, long long id, double *rho, double *ux, double *uy, double *T,
                                     double *p)
{
    SRV_BEGIN
    if (!s) throw LbmError(LBM_ERR_INVALID, "NULL server");
    std::lock_guard<std::mutex> g(s->mu);
    const Request *r = s->find_locked(id);
    if (r->state != LBM_REQ_DONE) throw LbmError(LBM_ERR_BUSY, "request not done");
    const size_t n = (size_t)r->nx * r->ny;
    if (r->result.size() == 5 * n) {
        double *dst[5] = {rho, ux, uy, T, p};
        for (int k = 0; k < 5; ++k)
            if (dst[k]) std::copy(r->result.begin() + k * n, r->result.begin() + (k + 1) * n, dst[k]);
    } else if (r->status == LBM_OK) {
        throw LbmError(LBM_ERR_INVALID, "no result stored");
    }
    if (r->status != LBM_OK) g_last_error = "request finished with an error status";
    return r->status;
    SRV_END
}

LBM_API lbm_status lbm_server_cancel(lbm_server *s, long long id)
{
    SRV_BEGIN
    if (!s) throw LbmError(LBM_ERR_INVALID, "NULL server");
    std::lock_guard<std::mutex> g(s->mu);
    Request *r = s->find_locked(id);
    if (r->state == LBM_REQ_DONE) return LBM_OK;
    r->cancel = true;
    if (r->state == LBM_REQ_QUEUED) {
        for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
            if (*it == r) {
                s->queue.erase(it);
                break;
            }
        s->finish_locked(r, LBM_ERR_CANCELLED);
    }
    s->cv_loop.notify_all();
    return LBM_OK;
    SRV_END
}

LBM_API lbm_status lbm_server_release(lbm_server *s, long long id)
{
    SRV_BEGIN
    if (!s) throw LbmError(LBM_ERR_INVALID, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    Request *r = s->find_locked(id);
    if (r->state != LBM_REQ_DONE) {
        lk.unlock();
        lbm_server_cancel(s, id);
        lk.lock();
        r = s->find_locked(id);
        s->cv_done.wait(lk, [&] { return r->state == LBM_REQ_DONE; });
    }
    s->reqs.erase(id);
    return LBM_OK;
    SRV_END
}

LBM_API lbm_status lbm_server_get_stats(lbm_server *s, lbm_server_stats *st)
{
    SRV_BEGIN
    if (!s || !st) throw LbmError(LBM_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> g(s->mu);
    *st = s->stats;
    st->resident = (int)s->packed.size();
    st->queued = (int)s->queue.size();
    st->arena_nodes_used = s->arena.used;
    if (s->busy) st->busy_seconds += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
    st->uptime_seconds = s->now();
    return LBM_OK;
    SRV_END
}

LBM_API void lbm_server_destroy(lbm_server *s)
{
    if (!s) return;
    try {
        s->shutdown();
    } catch (...) {
    }
    delete s;
}

}  // extern "C"
