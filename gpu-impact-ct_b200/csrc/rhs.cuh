// rhs.cuh -- rhs_vel of one velocity component (z-marching stencil pass, rhs.cu; internal).
#pragma once
#include "common.cuh"

namespace impact {

// nl_m = upwind advection by the interpolated velocities work[0..2] + explicit Helmholtz of
// vel_m; rhs_m = vel_m - mult_b nl_m(old) (use_old) - mult_a nl_m (mod_rhs.f90:35-140)
void launch_rhs_march(int m, const Geom& g, const Coeffs<double>& c, double multL, double mult_b, double mult_a,
                      int use_old, const double* vel, const double* const work[3], double* nl, double* rhs,
                      cudaStream_t s);
// z planes per block of that pass for grid g
int rhs_march_kz(const Geom& g);

}  // namespace impact
