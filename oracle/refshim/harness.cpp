// Driver for the reference solver, compiled unmodified from
// CODE/C++/VS2010/simLB/simLB/{cpuLBM,fileHandling,main}.cpp.
//
// Test infrastructure: this binary is the parity oracle ("oracle/_ref") and
// the timed CPU baseline.  It never ships in the product path.
//
//   simlb_ref <input.lbmv> <output.lbmv> [max_steps]
//
// The input container holds the MAT variables that cpuLBM::loadInput reads
// (cpuLBM.cpp:113-265).  The harness writes input.txt for the reference's
// folderSystem (fileHandling.cpp:131-147), builds cpuLBM exactly as main()
// does (main.cpp:12-14) and calls the reference's own runSimStep()
// (main.cpp:32-112) until the solver sets stop, or max_steps steps ran.
// It then writes rho, ux, uy, T, p, f, h in the reference's AoS order plus
// the step count, dt, per-step residual trace and the timed loop's seconds.
#include "cpuLBM.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>
#include <string>
#include <vector>

// main.cpp (compiled with -Dmain=simlb_reference_main) defines these.
extern cpuLBM *lbm;
void runSimStep();

// Zero-fill every heap allocation.  cpuLBM leaves several members
// uninitialised (e.g. resNorm, read at main.cpp:64); zeroed memory makes the
// reference's runs deterministic, matching a fresh process heap.
void *operator new(size_t n)
{
    void *p = calloc(1, n ? n : 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void *operator new[](size_t n) { return operator new(n); }
void operator delete(void *p) noexcept { free(p); }
void operator delete[](void *p) noexcept { free(p); }
void operator delete(void *p, size_t) noexcept { free(p); }
void operator delete[](void *p, size_t) noexcept { free(p); }

struct Var {
    std::string name;
    std::vector<uint64_t> dims;
    std::vector<double> data;
};

static void put(std::vector<Var> &out, const char *name, std::vector<uint64_t> dims, const double *src)
{
    Var v;
    v.name = name;
    v.dims = dims;
    size_t n = 1;
    for (auto d : dims) n *= d;
    v.data.assign(src, src + n);
    out.push_back(v);
}

static int write_container(const char *path, const std::vector<Var> &vars)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return 1;
    fwrite("LBMV1\0\0\0", 1, 8, fp);
    uint32_t n = (uint32_t)vars.size();
    fwrite(&n, 4, 1, fp);
    for (const auto &v : vars) {
        uint32_t nl = (uint32_t)v.name.size(), nd = (uint32_t)v.dims.size();
        fwrite(&nl, 4, 1, fp);
        fwrite(v.name.data(), 1, nl, fp);
        fwrite(&nd, 4, 1, fp);
        fwrite(v.dims.data(), 8, nd, fp);
        fwrite(v.data.data(), 8, v.data.size(), fp);
    }
    fclose(fp);
    return 0;
}

static double now_s()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <input.lbmv> <output.lbmv> [max_steps]\n", argv[0]);
        return 2;
    }
    long max_steps = argc > 3 ? atol(argv[3]) : -1;
    {
        FILE *fp = fopen("input.txt", "w");
        if (!fp) { fprintf(stderr, "cannot write input.txt\n"); return 2; }
        fprintf(fp, "%send\n", argv[1]);
        fclose(fp);
    }
    // The reference prints every step; keep the harness quiet.
    if (!freopen("/dev/null", "w", stdout)) return 2;

    folderSystem *files = new folderSystem;
    lbm = new cpuLBM(files);

    std::vector<double> res_trace, fail_trace;
    double t0 = now_s();
    while (lbm->stop == 0 && (max_steps < 0 || lbm->step < max_steps)) {
        runSimStep();
        res_trace.push_back(lbm->residual);
        fail_trace.push_back((double)lbm->stop);
    }
    double elapsed = now_s() - t0;

    const int Nx = lbm->Nx, Ny = lbm->Ny;
    const size_t N = (size_t)Nx * Ny;
    std::vector<double> ux(N), uy(N);
    for (size_t k = 0; k < N; ++k) { ux[k] = lbm->u_G[k].x; uy[k] = lbm->u_G[k].y; }

    std::vector<Var> out;
    put(out, "rho", {N}, lbm->rho_G);
    put(out, "ux", {N}, ux.data());
    put(out, "uy", {N}, uy.data());
    put(out, "T", {N}, lbm->T_G);
    put(out, "p", {N}, lbm->p_G);
    put(out, "f", {N * 13}, lbm->f_G);
    put(out, "h", {N * 13}, lbm->h_G);
    double scal[8] = {(double)Nx, (double)Ny, (double)lbm->step, (double)lbm->nsteps,
                      lbm->dt, (double)lbm->stop, lbm->residual, elapsed};
    put(out, "scalars", {8}, scal);
    put(out, "residual_trace", {res_trace.size()}, res_trace.data());
    put(out, "stop_trace", {fail_trace.size()}, fail_trace.data());
    double ev[26];
    for (int i = 0; i < 13; ++i) { ev[i] = lbm->e[i].x; ev[13 + i] = lbm->e[i].y; }
    put(out, "e", {26}, ev);
    if (write_container(argv[2], out)) {
        fprintf(stderr, "cannot write %s\n", argv[2]);
        return 2;
    }
    return 0;
}
