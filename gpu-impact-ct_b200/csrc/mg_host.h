// mg_host.h -- host-side multigrid hierarchy of a periodic grid (internal).
#pragma once
#include <vector>

namespace impact {

struct MGHostLevel {
  int M[3];      // points per axis (NN of the level)
  int ratio[3];  // coarsening factor to the next level (2, or 1 for an axis that stopped)
  std::vector<double> cdg[3];  // cdg(-1:1, 1:M)
  std::vector<double> cI[3];   // cI(1:2, 0:M), weights at the even points (interpolation to this level)
};

// Level sizes (mod_setup.f90:95-143), level coordinates (mod_geometry.f90:66-103), compact
// Laplacians (get_stencil, mod_coeffs.f90:1048-1259) and interpolation weights (interp_coeffs,
// mod_coeffs.f90:1683-1746) from the finest coordinates xp/xu (indices -3..N+3, offset 3).
std::vector<MGHostLevel> build_mg_hierarchy(const int N[3], const double* const xp[3], const double* const xu[3],
                                            const double L[3], int n_grids_limit);

}  // namespace impact
