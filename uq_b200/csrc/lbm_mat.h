// MATLAB Level-5 MAT input and output at the boundary (lbm_mat.cpp).
#pragma once

#include "../../include/uq_lbm.h"

#include <vector>

namespace uqlbm {

// An input case read from a MAT file: the lbm_config / lbm_init pair and
// the arrays lbm_init points into.
struct MatCase {
    lbm_config cfg{};
    lbm_init init{};
    std::vector<int> bnd, cellType;
    std::vector<double> density, pressure, temp, velocityX, velocityY;
};

// cpuLBM::loadInput semantics: same variable names, tables of max(dims)
// entries, bndArray with Nx = dims[1], Ny = dims[0] and y flipped.
void mat_read_case(const char *path, MatCase &c);

// f and h ({13, Ny, Nx}, i.e. [(x*Ny + y)*13 + i]) and t of a file that
// mat_write_fields wrote with distributions: the checkpoint to resume from.
void mat_read_dist(const char *path, int Nx, int Ny, double *f, double *h, double *t);

// cpuLBM::createMAT's variables; f, h, ex, ey all non-null adds the
// distributions.
void mat_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux, const double *uy,
                      const double *p, const double *T, double t, double dx, double dy, const double *f,
                      const double *h, const double *ex, const double *ey);

}  // namespace uqlbm
