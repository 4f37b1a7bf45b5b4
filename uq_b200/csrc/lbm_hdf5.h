// HDF5 output at the boundary (lbm_hdf5.cpp).
#pragma once

namespace uqlbm {

// The datasets of the Python reference's saveHDF5 (LBM.py:516-567): rho,
// T, ux, uy over [x*Ny + y]; t, gamma, R, T_ref, rho_ref; dx (ndx values)
// and dy (ndy values), scalars when one value; Nx, Ny; f and h over
// [(x*Ny + y)*13 + i] when both are given.
void hdf5_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux, const double *uy,
                       const double *T, double t, double gamma, double R, double T_ref, double rho_ref,
                       const double *dx, int ndx, const double *dy, int ndy, const double *f, const double *h);

}  // namespace uqlbm
