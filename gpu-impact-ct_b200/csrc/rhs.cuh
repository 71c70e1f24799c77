// rhs.cuh -- rhs_vel of one velocity component (z-marching stencil pass, rhs.cu; internal).
#pragma once
#include "common.cuh"

namespace impact {

// nl_m = upwind advection by the interpolated velocities work[0..2] + explicit Helmholtz of
// vel_m; rhs_m = vel_m - mult_b nl_m(old) (use_old) - mult_a nl_m (mod_rhs.f90:35-140)
void launch_rhs_march(int m, const Geom& g, const Coeffs<double>& c, double multL, double mult_b, double mult_a,
                      int use_old, const double* vel, const double* const work[3], double* nl, double* rhs,
                      cudaStream_t s);
// the same pass in FP32 (mixed-precision cases): work fields, nl_m, coefficients and arithmetic
// in FP32; the velocity and rhs_m FP64
void launch_rhs_march32(int m, const Geom& g, const Coeffs<float>& c, double multL, double mult_b, double mult_a,
                        int use_old, const double* vel, const float* const work[3], float* nl, double* rhs,
                        cudaStream_t s);
// z planes per block of that pass for grid g
int rhs_march_kz(const Geom& g);

// one case of the batched pass: its fields, coefficients and 1/Re, its time step (device), and
// its grid of blocks (gx x gy x gz, planes kz per block) starting at block b0 of the launch
struct RhsJob {
  Geom g;
  Coeffs<double> c;
  Coeffs<float> c32;
  const double* Re;  // Reynolds number of the step (device): 1/Re multiplies the Helmholtz term
  const double* dt;
  const double* vel[3];
  const double* work[3];
  double* nl[3];
  const float* work32[3];  // FP32 passes (mixed precision)
  float* nl32[3];
  double* rhs[3];
  int kz, gx, gy, gz, b0;
};
// kz, gx, gy, gz of a case of grid g (b0 and the rest are the caller's)
// kz: planes per block (0: the grid's own choice); a batch passes the choice for all its grids
void rhs_march_job_grid(const Geom& g, RhsJob& J, int kz = 0);
int rhs_march_kz_for(long long column_planes);
long long rhs_march_column_planes(const Geom& g);
// component m of every job in one launch of `blocks` blocks (the sum of the jobs' grids), RK
// substep sub, FP64 or (f32) FP32 pass; job j's blocks start at jobs[j].b0 (increasing)
void launch_rhs_march_batch(int m, const RhsJob* jobs, int nj, int blocks, int sub, int f32, cudaStream_t s);

}  // namespace impact
