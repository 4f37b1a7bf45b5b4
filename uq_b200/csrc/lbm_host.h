// Host-side pieces shared by the engine (lbm_engine.cu) and the
// allocation-free entry point (lbm_noalloc.cu).
#pragma once

#include "../../include/uq_lbm.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace uqlbm {

extern thread_local std::string g_last_error;

struct LbmError : std::runtime_error {
    lbm_status code;
    LbmError(lbm_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CU(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            throw ::uqlbm::LbmError(e_ == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,       \
                                    std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

// Scalar run parameters after refineInput / setupVars (cpuLBM.cpp:283-450).
struct ScalarParams {
    int rk = 1, fm = 1, flags = 0, nsteps = 0;
    double R = 1, b = 5, K = 3, Tc = 1, c = 1, mu = 0, Pr = 1, dt = 0, tol = 0;
    double dx = 1, dy = 1, rho_ref = 1, T_ref = 1, gamma = 1.4;
    int mu_model = 0;  // 0 constant, 1 VHS, 2 Sutherland
    double upsilon = 0, S_v = 0;
};

void derive_scalars(const lbm_config &c, int Nx, int Ny, double min_spacing, ScalarParams &s);

}  // namespace uqlbm
