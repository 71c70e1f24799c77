// step.cu -- one RK3 fractional time step of IMPACT on resident device fields, and the case
// life cycle (the GPU_setup / GPU_malloc / GPU_memcopy / GPU_memfree of mod_mem_GPU.f90:18-437).
//
// The substep (mod_timeint.f90:275-377) is reorganised into fused passes:
//   interpolate_vel  -> k_interp_vel3   (3 interpolations, one pass)
//   rhs_vel          -> k_rhs_march     (pp interpolation, 3 upwind terms, explicit Helmholtz and
//                                        both RK updates of one component in one z-marching pass,
//                                        rhs.cu)
//   explicit         -> divergence2 of rhs, Poisson solve, k_project (vel = rhs - G pre, 3 comps)
// Every pass keeps the reference's order of floating-point operations per point.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "case.cuh"
#include "mg_host.h"
#include "kernels.cuh"
#include "prof.cuh"
#include "rhs.cuh"
#include "solver.cuh"

namespace impact {

constexpr int BX = 32, BY = 8, NT = BX * BY;
static inline dim3 grid3(const Geom& g) { return dim3((g.n1 + BX - 1) / BX, (g.n2 + BY - 1) / BY, g.n3); }

// RK3 coefficients (mod_vars.f90:774-775)
static const double aRK[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double bRK[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

#define PT                                                  \
  const int i = blockIdx.x * BX + threadIdx.x + 1;          \
  const int j = blockIdx.y * BY + threadIdx.y + 1;          \
  const int k = blockIdx.z + 1;                             \
  if (i > g.n1 || j > g.n2) return;                         \
  const long long p = off(g, i, j, k);

__device__ __forceinline__ int crd(int a, int i, int j, int k) { return a == 0 ? i : (a == 1 ? j : k); }
__device__ __forceinline__ int ext(const Geom& g, int a) { return a == 0 ? g.n1 : (a == 1 ? g.n2 : g.n3); }
__device__ __forceinline__ long long strd(const Geom& g, int a) { return a == 0 ? 1LL : (a == 1 ? (long long)g.nx : g.nxy); }

// WRAP = false: the whole block lies at least 3 points inside the periodic box, so the stencil
// points are p + l * stride without any index wrapping (same values, same operation order)
template <int LO, int CNT, bool WRAP>
__device__ __forceinline__ double st1w(const double* __restrict__ c, const double* __restrict__ f, const Geom& g, int a,
                                       int i, int j, int k, long long p) {
  if (WRAP) {
    const int q = crd(a, i, j, k), n = ext(g, a);
    const long long s = strd(g, a);
    const long long base = p - (long long)q * s;
    const double* cr = c + (long long)q * CNT;
    double v = cr[0] * __ldg(f + base + (long long)wrapi(q + LO, n) * s);
#pragma unroll
    for (int l = 1; l < CNT; ++l) v = v + cr[l] * __ldg(f + base + (long long)wrapi(q + LO + l, n) * s);
    return v;
  }
  const int q = crd(a, i, j, k);
  const long long s = strd(g, a);
  const double* cr = c + (long long)q * CNT;
  const double* fp = f + p + (long long)LO * s;
  double v = cr[0] * __ldg(fp);
#pragma unroll
  for (int l = 1; l < CNT; ++l) v = v + cr[l] * __ldg(fp + l * s);
  return v;
}
template <int LO, int CNT, bool WRAP>
__device__ __forceinline__ double st1w_acc(double v, const double* __restrict__ c, const double* __restrict__ f,
                                           const Geom& g, int a, int i, int j, int k, long long p) {
  if (WRAP) {
    const int q = crd(a, i, j, k), n = ext(g, a);
    const long long s = strd(g, a);
    const long long base = p - (long long)q * s;
    const double* cr = c + (long long)q * CNT;
#pragma unroll
    for (int l = 0; l < CNT; ++l) v = v + cr[l] * __ldg(f + base + (long long)wrapi(q + LO + l, n) * s);
    return v;
  }
  const int q = crd(a, i, j, k);
  const long long s = strd(g, a);
  const double* cr = c + (long long)q * CNT;
  const double* fp = f + p + (long long)LO * s;
#pragma unroll
  for (int l = 0; l < CNT; ++l) v = v + cr[l] * __ldg(fp + l * s);
  return v;
}
// the points of block (bx, by) on plane k and their 3-point halos stay inside 1..n on every axis
__device__ __forceinline__ bool block_interior(const Geom& g, int bx, int by, int k) {
  const int i0 = bx * BX + 1, j0 = by * BY + 1;
  return i0 - 3 >= 1 && i0 + BX - 1 + 3 <= g.n1 && j0 - 3 >= 1 && j0 + BY - 1 + 3 <= g.n2 && k - 3 >= 1 &&
         k + 3 <= g.n3;
}
// the point of this thread in block (bx, by, bz) of a grid3 launch; returns false outside the grid
#define PTB(bx, by, bz)                                      \
  const int i = (bx) * BX + threadIdx.x + 1;                 \
  const int j = (by) * BY + threadIdx.y + 1;                 \
  const int k = (bz) + 1;                                    \
  if (i > g.n1 || j > g.n2) return;                          \
  const long long p = off(g, i, j, k);

// interpolate_vel (mod_diff.f90:1436-1472): work_m = I_{u_m -> p} vel_m, three components, in
// FP64 from the FP64 velocity; TO = float stores the FP32 work fields of a mixed-precision case
template <typename TO>
__device__ __forceinline__ void interp_vel3_block(const Geom& g, const Coeffs<double>& c, const double* __restrict__ u,
                                                  const double* __restrict__ v, const double* __restrict__ w,
                                                  TO* __restrict__ w1, TO* __restrict__ w2, TO* __restrict__ w3,
                                                  int bx, int by, int bz) {
  const bool wrap = !block_interior(g, bx, by, bz + 1);
  PTB(bx, by, bz)
  if (wrap) {
    w1[p] = (TO)st1w<D_LO, ND, true>(c.cIup[0], u, g, 0, i, j, k, p);
    w2[p] = (TO)st1w<D_LO, ND, true>(c.cIup[1], v, g, 1, i, j, k, p);
    w3[p] = (TO)st1w<D_LO, ND, true>(c.cIup[2], w, g, 2, i, j, k, p);
  } else {
    w1[p] = (TO)st1w<D_LO, ND, false>(c.cIup[0], u, g, 0, i, j, k, p);
    w2[p] = (TO)st1w<D_LO, ND, false>(c.cIup[1], v, g, 1, i, j, k, p);
    w3[p] = (TO)st1w<D_LO, ND, false>(c.cIup[2], w, g, 2, i, j, k, p);
  }
}
__global__ void __launch_bounds__(NT) k_interp_vel3_32(Geom g, Coeffs<double> c, const double* __restrict__ u,
                                                       const double* __restrict__ v, const double* __restrict__ w,
                                                       float* __restrict__ w1, float* __restrict__ w2,
                                                       float* __restrict__ w3) {
  interp_vel3_block<float>(g, c, u, v, w, w1, w2, w3, blockIdx.x, blockIdx.y, blockIdx.z);
}
__global__ void __launch_bounds__(NT) k_interp_vel3(Geom g, Coeffs<double> c, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    double* __restrict__ w1, double* __restrict__ w2,
                                                    double* __restrict__ w3) {
  interp_vel3_block<double>(g, c, u, v, w, w1, w2, w3, blockIdx.x, blockIdx.y, blockIdx.z);
}

// pre = pre * ab * dt  (mod_timeint.f90:318)  /  pre = pre / ab / dt  (:372)
__device__ __forceinline__ void scale_pre_block(const Geom& g, double ab, double dt, int divide,
                                                double* __restrict__ pre, int bx, int by, int bz) {
  PTB(bx, by, bz)
  pre[p] = divide ? pre[p] / ab / dt : pre[p] * ab * dt;
}
__global__ void __launch_bounds__(NT) k_scale_pre(Geom g, double ab, double dt, int divide, double* __restrict__ pre) {
  scale_pre_block(g, ab, dt, divide, pre, blockIdx.x, blockIdx.y, blockIdx.z);
}

// explicit (mod_solvers.f90:180-330): vel_m = rhs_m - G_m pre for the three components
__device__ __forceinline__ void project_block(const Geom& g, const Coeffs<double>& c, const double* __restrict__ pre,
                                              const double* __restrict__ r1, const double* __restrict__ r2,
                                              const double* __restrict__ r3, double* __restrict__ u,
                                              double* __restrict__ v, double* __restrict__ w, int bx, int by, int bz) {
  const bool wrap = !block_interior(g, bx, by, bz + 1);
  PTB(bx, by, bz)
  if (wrap) {
    u[p] = 1.0 * r1[p] + (-1.0) * st1w<G_LO, NG, true>(c.cG[0], pre, g, 0, i, j, k, p);
    v[p] = 1.0 * r2[p] + (-1.0) * st1w<G_LO, NG, true>(c.cG[1], pre, g, 1, i, j, k, p);
    w[p] = 1.0 * r3[p] + (-1.0) * st1w<G_LO, NG, true>(c.cG[2], pre, g, 2, i, j, k, p);
  } else {
    u[p] = 1.0 * r1[p] + (-1.0) * st1w<G_LO, NG, false>(c.cG[0], pre, g, 0, i, j, k, p);
    v[p] = 1.0 * r2[p] + (-1.0) * st1w<G_LO, NG, false>(c.cG[1], pre, g, 1, i, j, k, p);
    w[p] = 1.0 * r3[p] + (-1.0) * st1w<G_LO, NG, false>(c.cG[2], pre, g, 2, i, j, k, p);
  }
}
__global__ void __launch_bounds__(NT) k_project(Geom g, Coeffs<double> c, const double* __restrict__ pre,
                                                const double* __restrict__ r1, const double* __restrict__ r2,
                                                const double* __restrict__ r3, double* __restrict__ u,
                                                double* __restrict__ v, double* __restrict__ w) {
  project_block(g, c, pre, r1, r2, r3, u, v, w, blockIdx.x, blockIdx.y, blockIdx.z);
}

// divergence2 (mod_diff.f90:130-215) of the provisional velocity into the pressure equation's
// right-hand side: x stencil, then y and z added in table order
__device__ __forceinline__ void div2_block(const Geom& g, const Coeffs<double>& c, const double* __restrict__ u,
                                           const double* __restrict__ v, const double* __restrict__ w,
                                           double* __restrict__ div, int bx, int by, int bz) {
  const bool wrap = !block_interior(g, bx, by, bz + 1);
  PTB(bx, by, bz)
  double d;
  if (wrap) {
    d = st1w<D_LO, ND, true>(c.cD[0], u, g, 0, i, j, k, p);
    d = st1w_acc<D_LO, ND, true>(d, c.cD[1], v, g, 1, i, j, k, p);
    d = st1w_acc<D_LO, ND, true>(d, c.cD[2], w, g, 2, i, j, k, p);
  } else {
    d = st1w<D_LO, ND, false>(c.cD[0], u, g, 0, i, j, k, p);
    d = st1w_acc<D_LO, ND, false>(d, c.cD[1], v, g, 1, i, j, k, p);
    d = st1w_acc<D_LO, ND, false>(d, c.cD[2], w, g, 2, i, j, k, p);
  }
  div[p] = d;
}
__global__ void __launch_bounds__(NT) k_div2(Geom g, Coeffs<double> c, const double* __restrict__ u,
                                             const double* __restrict__ v, const double* __restrict__ w,
                                             double* __restrict__ div) {
  div2_block(g, c, u, v, w, div, blockIdx.x, blockIdx.y, blockIdx.z);
}


// get_dtime (mod_lib.f90:46-250), timeint_mode 1: block max of radius / stabilitylimit(angle)
__constant__ double c_stab[41];

__device__ __forceinline__ double wmax_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double wsum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void dtime_block(const Geom& g, const Coeffs<double>& c, const DtRows& dr, double Re,
                                            const double* __restrict__ u, const double* __restrict__ v,
                                            const double* __restrict__ w, double* __restrict__ partial, int bx,
                                            int by, int bz, int gx, int gy) {
  const int i = bx * BX + threadIdx.x + 1;
  const int j = by * BY + threadIdx.y + 1;
  const int k = bz + 1;
  double beta = 0.0;
  const bool wrap = !block_interior(g, bx, by, k);
  if (i <= g.n1 && j <= g.n2) {
    const long long p = off(g, i, j, k);
    double w1, w2, w3;
    if (wrap) {
      w1 = st1w<D_LO, ND, true>(c.cIup[0], u, g, 0, i, j, k, p);
      w2 = st1w<D_LO, ND, true>(c.cIup[1], v, g, 1, i, j, k, p);
      w3 = st1w<D_LO, ND, true>(c.cIup[2], w, g, 2, i, j, k, p);
    } else {
      w1 = st1w<D_LO, ND, false>(c.cIup[0], u, g, 0, i, j, k, p);
      w2 = st1w<D_LO, ND, false>(c.cIup[1], v, g, 1, i, j, k, p);
      w3 = st1w<D_LO, ND, false>(c.cIup[2], w, g, 2, i, j, k, p);
    }
    double are = dr.spp[0][i] + dr.spp[1][j];
    are = are + dr.spp[2][k];
    are = are / Re;
    double aim = dr.sp1[0][i] * fabs(w1);
    aim = aim + dr.sp1[1][j] * fabs(w2);
    aim = aim + dr.sp1[2][k] * fabs(w3);
    const double pi = 3.14159265358979323846;
    const double angle = (fabs(aim) < 1e-16) ? pi / 2.0 : atan(are / aim);
    const double radius = sqrt(are * are + aim * aim);
    long long idx = llround(2.0 * 40.0 * angle / pi);
    idx = idx < 0 ? 0 : (idx > 40 ? 40 : idx);
    beta = radius / c_stab[idx];
  }
  __shared__ double sh[NT / 32];
  const int tid = threadIdx.x + BX * threadIdx.y;
  beta = wmax_d(beta);
  if ((tid & 31) == 0) sh[tid >> 5] = beta;
  __syncthreads();
  if (tid < 32) {
    double x = tid < NT / 32 ? sh[tid] : 0.0;
    x = wmax_d(x);
    if (tid == 0) partial[bx + (long long)gx * (by + (long long)gy * bz)] = x;
  }
}
__global__ void __launch_bounds__(NT) k_dtime(Geom g, Coeffs<double> c, DtRows dr, double Re, const double* __restrict__ u,
                                              const double* __restrict__ v, const double* __restrict__ w,
                                              double* __restrict__ partial) {
  dtime_block(g, c, dr, Re, u, v, w, partial, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
}

// fixed-order max / sum over n partials (single block)
__device__ __forceinline__ void reduce_partials_block(const double* __restrict__ partial, long long n, int is_max,
                                                      double* __restrict__ out) {
  __shared__ double sh[32];
  double v = 0.0;
  for (long long b = threadIdx.x; b < n; b += blockDim.x) v = is_max ? fmax(v, partial[b]) : v + partial[b];
  v = is_max ? wmax_d(v) : wsum_d(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = sh[threadIdx.x];
    x = is_max ? wmax_d(x) : wsum_d(x);
    if (threadIdx.x == 0) *out = x;
  }
}
__global__ void __launch_bounds__(1024) k_reduce_partials(const double* __restrict__ partial, long long n, int is_max,
                                                          double* __restrict__ out) {
  reduce_partials_block(partial, n, is_max, out);
}

// sum of pre over the unique points, block partials (level_pressure, mod_lib.f90:507-537)
// FP64 -> FP32 and back, whole padded fields
__global__ void k_narrow(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (float)a[q];
}
__global__ void k_widen(const float* __restrict__ a, double* __restrict__ b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (double)a[q];
}
__device__ __forceinline__ void sum_block(const Geom& g, const double* __restrict__ a, double* __restrict__ partial,
                                          int bx, int by, int bz, int gx, int gy) {
  const int i = bx * BX + threadIdx.x + 1;
  const int j = by * BY + threadIdx.y + 1;
  const int k = bz + 1;
  double s = (i <= g.n1 && j <= g.n2) ? a[off(g, i, j, k)] : 0.0;
  __shared__ double sh[NT / 32];
  const int tid = threadIdx.x + BX * threadIdx.y;
  s = wsum_d(s);
  if ((tid & 31) == 0) sh[tid >> 5] = s;
  __syncthreads();
  if (tid < 32) {
    double x = tid < NT / 32 ? sh[tid] : 0.0;
    x = wsum_d(x);
    if (tid == 0) partial[bx + (long long)gx * (by + (long long)gy * bz)] = x;
  }
}
__global__ void __launch_bounds__(NT) k_sum(Geom g, const double* __restrict__ a, double* __restrict__ partial) {
  sum_block(g, a, partial, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
}
__device__ __forceinline__ void sub_mean_block(const Geom& g, const double* __restrict__ sum, double* __restrict__ pre,
                                               int bx, int by, int bz) {
  PTB(bx, by, bz)
  const double m = *sum / (double)g.n1 / (double)g.n2 / (double)g.n3;
  pre[p] = pre[p] - m;
}
__global__ void __launch_bounds__(NT) k_sub_mean(Geom g, const double* __restrict__ sum, double* __restrict__ pre) {
  sub_mean_block(g, sum, pre, blockIdx.x, blockIdx.y, blockIdx.z);
}

// apply_CT_forcing (usr_func.f90:909-1049, idealized branch): label 0/7 -> u = 0; 5 -> inflow
// inflow_on = 0: the inflow voxels keep their velocity (a measured waveform without an interval
// that holds the current time, as in apply_CT_forcing)
__device__ __forceinline__ void mask_block(const Geom& g, const uint8_t* __restrict__ label, double u_in, int inflow_on,
                                           double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                                           int bx, int by, int bz) {
  PTB(bx, by, bz)
  const uint8_t lb = label[p];
  if (lb == 0 || lb == 7) {
    u[p] = 0.0;
    v[p] = 0.0;
    w[p] = 0.0;
  } else if (lb == 5 && inflow_on) {
    w[p] = u_in;
    v[p] = 0.0;
    u[p] = 0.0;
  }
}
__global__ void __launch_bounds__(NT) k_mask(Geom g, const uint8_t* __restrict__ label, double u_in, int inflow_on,
                                             double* __restrict__ u, double* __restrict__ v, double* __restrict__ w) {
  mask_block(g, label, u_in, inflow_on, u, v, w, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------------------
// the explicit part of a batch step: one launch per kernel over all cases.  Block b of a
// reduction launch is block b - job.b0 of its case's grid3 grid (gx x gy x gz), block b of a
// point-kernel launch covers XPL planes of that grid from block b - job.pb0 on; every block runs
// the body of the single-case kernel for each of its planes, so a case's bits do not depend on
// the batch.
// ---------------------------------------------------------------------------------------
struct StepScal {  // per case and step: time step, Reynolds number, inflow at the step's end
  double dt, Re, u_in;
  int inflow_on, level_pressure;
};
struct ExJob {
  Geom g;
  Coeffs<double> c;
  DtRows dr;
  double* vel[3];
  double* nl[3];
  double* rhs[3];
  double* work[3];
  float* work32[3];  // mixed precision: the FP32 interpolated velocities (null in FP64)
  double* pre;
  double* res;
  const uint8_t* label;
  double* partial;
  double* dscal;
  const StepScal* sc;  // this case's scalars of the current step
  int gx, gy, gz, b0;  // grid3 blocks (one plane each) of the case, from block b0 on
  int pb0;             // blocks of XPL planes (the point kernels), from block pb0 on
};

__device__ __forceinline__ int ex_job(const ExJob* __restrict__ jobs, int nj, int b) {
  int lo = 0, hi = nj - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].b0 <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}
#define EX_BLOCK                                                         \
  const ExJob& J = jobs[ex_job(jobs, nj, blockIdx.x)];                   \
  const int lb = blockIdx.x - J.b0;                                      \
  const int bx = lb % J.gx, by = (lb / J.gx) % J.gy, bz = lb / (J.gx * J.gy); \
  const Geom& g = J.g;                                                   \
  (void)g;
// The point kernels (no reduction) give each block XPL planes of its 32 x 8 columns, so that the
// search for the block's case and its set-up are paid once per XPL planes; the planes
// bz = kb0 .. kb1-1 of the case's grid3 blocks.
constexpr int XPL = 8;
__device__ __forceinline__ int ex_pjob(const ExJob* __restrict__ jobs, int nj, int b) {
  int lo = 0, hi = nj - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].pb0 <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}
#define EX_PBLOCK                                                        \
  const ExJob& J = jobs[ex_pjob(jobs, nj, blockIdx.x)];                  \
  const int lb = blockIdx.x - J.pb0;                                     \
  const int bx = lb % J.gx, by = (lb / J.gx) % J.gy, bq = lb / (J.gx * J.gy); \
  const int kb0 = bq * XPL, kb1 = min(J.gz, kb0 + XPL);                  \
  const Geom& g = J.g;

__constant__ double RKA_D[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
__constant__ double RKB_D[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

__global__ void __launch_bounds__(NT) k_b_dtime(const ExJob* __restrict__ jobs, int nj) {
  EX_BLOCK
  dtime_block(g, J.c, J.dr, J.sc->Re, J.vel[0], J.vel[1], J.vel[2], J.partial, bx, by, bz, J.gx, J.gy);
}
// one block per case: out = dscal[slot] of the case
// one block per case: the case's dscal[slot], or out[case] when out is given
__global__ void __launch_bounds__(1024) k_b_reduce(const ExJob* __restrict__ jobs, int is_max, int slot, int only_lp,
                                                   double* __restrict__ out) {
  const ExJob& J = jobs[blockIdx.x];
  if (only_lp && !J.sc->level_pressure) return;
  reduce_partials_block(J.partial, (long long)J.gx * J.gy * J.gz, is_max, out ? out + blockIdx.x : J.dscal + slot);
}
__global__ void __launch_bounds__(NT) k_b_interp(const ExJob* __restrict__ jobs, int nj, int f32) {
  EX_PBLOCK
  for (int bz = kb0; bz < kb1; ++bz) {
    if (f32)
      interp_vel3_block<float>(g, J.c, J.vel[0], J.vel[1], J.vel[2], J.work32[0], J.work32[1], J.work32[2], bx, by,
                               bz);
    else
      interp_vel3_block<double>(g, J.c, J.vel[0], J.vel[1], J.vel[2], J.work[0], J.work[1], J.work[2], bx, by, bz);
  }
}
__global__ void __launch_bounds__(NT) k_b_scale_pre(const ExJob* __restrict__ jobs, int nj, int sub, int divide) {
  EX_PBLOCK
  for (int bz = kb0; bz < kb1; ++bz) scale_pre_block(g, RKA_D[sub] + RKB_D[sub], J.sc->dt, divide, J.pre, bx, by, bz);
}
__global__ void __launch_bounds__(NT) k_b_div2(const ExJob* __restrict__ jobs, int nj) {
  EX_PBLOCK
  for (int bz = kb0; bz < kb1; ++bz) div2_block(g, J.c, J.rhs[0], J.rhs[1], J.rhs[2], J.res, bx, by, bz);
}
__global__ void __launch_bounds__(NT) k_b_project(const ExJob* __restrict__ jobs, int nj) {
  EX_PBLOCK
  for (int bz = kb0; bz < kb1; ++bz)
    project_block(g, J.c, J.pre, J.rhs[0], J.rhs[1], J.rhs[2], J.vel[0], J.vel[1], J.vel[2], bx, by, bz);
}
__global__ void __launch_bounds__(NT) k_b_mask(const ExJob* __restrict__ jobs, int nj) {
  EX_PBLOCK
  for (int bz = kb0; bz < kb1; ++bz)
    mask_block(g, J.label, J.sc->u_in, J.sc->inflow_on, J.vel[0], J.vel[1], J.vel[2], bx, by, bz);
}
__global__ void __launch_bounds__(NT) k_b_sum(const ExJob* __restrict__ jobs, int nj) {
  EX_BLOCK
  if (!J.sc->level_pressure) return;
  sum_block(g, J.pre, J.partial, bx, by, bz, J.gx, J.gy);
}
__global__ void __launch_bounds__(NT) k_b_sub_mean(const ExJob* __restrict__ jobs, int nj) {
  EX_PBLOCK
  if (!J.sc->level_pressure) return;
  for (int bz = kb0; bz < kb1; ++bz) sub_mean_block(g, J.dscal + 1, J.pre, bx, by, bz);
}

}  // namespace impact

using namespace impact;

// =========================================================================================
// case life cycle
// =========================================================================================
static long long nblocks(const Geom& g) {
  const dim3 d = grid3(g);
  return (long long)d.x * d.y * d.z;
}

extern "C" long long impact_b200_case_bytes(int N1, int N2, int N3, int precision) {
  const Geom g = make_geom(N1, N2, N3);
  const long long f = g.nfield * 8;
  long long b = f * (IMPACT_B200_NFIELDS + 3);            // fields + work
  b += g.nfield;                                          // labels
  if (precision == 0)
    b += 8 * f;                                           // FP64 Krylov set
  else
    b += f + 10 * (f / 2);                                // r64 + FP32 r, e + 8 inner fields
  b += 2 * reduce_partial_doubles(g, 4) * 8 + (1 << 20);  // reduction scratch, coefficients
  // multigrid levels >= 1 (three fields each, at most 1/8 of the previous level, padded)
  const long long elt = precision == 0 ? 8 : 4;
  long long lvl = 0;
  int m[3] = {N1 - 1, N2 - 1, N3 - 1};
  for (int q = 1; q < MG_MAX_LEVELS; ++q) {
    bool any = false;
    for (int a = 0; a < 3; ++a)
      if (m[a] % 2 == 0 && m[a] >= 4) {
        m[a] /= 2;
        any = true;
      }
    if (!any) break;
    lvl += (long long)(m[0] + 8) * (m[1] + 8) * (m[2] + 8);
  }
  b += 3 * elt * lvl;
  b += 12LL * 11 * (N1 + N2 + N3);  // collapsed operator weights
  b += 4LL * 8 * (g.nfield / 16 + 1024);  // engine tile partials
  return b;
}

// Case memory comes from one stream-ordered pool per device that keeps what cases free (release
// threshold: never), so that a serving loop which creates and destroys cases reuses device
// memory without cudaMalloc / cudaFree and the device-wide synchronisation they can cause.
static cudaMemPool_t case_pool(int dev) {
  static cudaMemPool_t pools[64] = {};
  if (dev < 0 || dev >= 64) return nullptr;
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    unsigned long long keep = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = pool;
  }
  return pools[dev];
}

int case_alloc(CaseState& s, void** p, size_t bytes) {
  cudaMemPool_t pool = case_pool(s.device);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, s.stream) : cudaMalloc(p, bytes);
  // usable by any stream and by the synchronous copies of case creation from here on
  if (e == cudaSuccess && pool) e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) return impact_set_error(e, "cudaMalloc (case)", __FILE__, __LINE__);
  s.allocs.push_back(*p);
  s.pooled = pool != nullptr;
  return 0;
}

extern "C" int impact_b200_case_destroy(impact_b200_case* c) {
  if (!c) return 0;
  CaseState& s = c->s;
  cudaSetDevice(s.device);
  if (s.stream) cudaStreamSynchronize(s.stream);
  delete s.e64;
  delete s.emx;
  s.e64 = nullptr;
  s.emx = nullptr;
  if (s.pooled) {
    for (void* p : s.allocs) cudaFreeAsync(p, s.stream);
    cudaStreamSynchronize(s.stream);
  } else {
    for (void* p : s.allocs) cudaFree(p);
  }
  if (s.snap_taken) cudaEventDestroy(s.snap_taken);
  if (s.snap_read) cudaEventDestroy(s.snap_read);
  if (s.hscal) cudaFreeHost(s.hscal);
  if (s.scal_host) cudaFreeHost(s.scal_host);
  if (s.mw.scal64_host) cudaFreeHost(s.mw.scal64_host);
  if (s.own_stream && s.stream) cudaStreamDestroy(s.stream);
  delete c;
  return 0;
}

// 1 when the rows of a table (width w, `rows` rows) agree to 1e-12 of its largest entry.  The
// tables of an equidistant axis differ row to row only by the rounding of the coordinates
// (about 1e-13 of the largest entry); kernels then use the first row for the whole axis.  This is
// applied to the multigrid smoother's compact Laplacians and to the FP32 operator of the inner
// solve, never to the FP64 operator A that defines the residual.
static int rows_uniform(const double* t, size_t rows, int w) {
  double mx = 0.0, dev = 0.0;
  for (size_t q = 0; q < rows * w; ++q) mx = std::fmax(mx, std::fabs(t[q]));
  for (size_t r = 1; r < rows; ++r)
    for (int l = 0; l < w; ++l) dev = std::fmax(dev, std::fabs(t[r * w + l] - t[l]));
  return dev <= 1e-12 * mx ? 1 : 0;
}

// Estimate of the smallest nonzero eigenvalue of diag(A)^-1 A for the compact periodic Laplacian
// A of one multigrid level (the Chebyshev bottom's lower bound): on an equidistant axis the
// lowest mode exp(2 pi i x / L) of axis m gives w_m (1 - cos(2 pi / n_m)), w_m = the axis's share
// of the diagonal; stretched axes use their mean centre weight.  Axes of one cell are skipped.
static double level_lmin(const MGHostLevel& L) {
  double c[3] = {0, 0, 0}, diag = 0;
  for (int m = 0; m < 3; ++m) {
    const int n = L.M[m] - 1;
    for (int i = 0; i < n; ++i) c[m] += L.cdg[m][3 * i + 1];
    c[m] /= n > 0 ? n : 1;
    diag += c[m];
  }
  double lo = 2.0;
  for (int m = 0; m < 3; ++m) {
    const int n = L.M[m] - 1;
    if (n < 2 || diag == 0.0) continue;
    lo = std::min(lo, c[m] / diag * (1.0 - std::cos(2.0 * M_PI / n)));
  }
  return lo;
}

extern "C" int impact_b200_case_create(const impact_b200_case_desc* desc, const impact_b200_coeffs* co,
                                       impact_b200_case** out) {
  if (!desc || !co || !out) return impact_set_error_msg(-1, "impact_b200_case_create: null argument");
  *out = nullptr;
  if (desc->N1 < 9 || desc->N2 < 9 || desc->N3 < 9)
    return impact_set_error_msg(-1, "impact_b200_case_create: need at least 8 unique points per axis");
  if (desc->precision != 0 && desc->precision != 1)
    return impact_set_error_msg(-1, "impact_b200_case_create: precision must be 0 (FP64) or 1 (mixed)");
  for (int a = 0; a < 3; ++a)
    if (!co->axis[a]) return impact_set_error_msg(-1, "impact_b200_case_create: missing coefficient tables");
  IMPACT_CUDA_CHECK(cudaSetDevice(desc->device));
  impact_b200_case* c = new impact_b200_case();
  CaseState& s = c->s;
  s.device = desc->device;
  s.precision = desc->precision;
  s.g = make_geom(desc->N1, desc->N2, desc->N3);
  const Geom& g = s.g;
  int rc = 0;
  if (desc->stream) {
    s.stream = static_cast<cudaStream_t>(desc->stream);
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      return impact_set_error(e, "cudaStreamCreate", __FILE__, __LINE__);
    }
    s.own_stream = true;
  }
  const int Nax[3] = {desc->N1, desc->N2, desc->N3};
  // ---- coefficients: 12 tables per axis + 2 dt row-sum tables per axis ----
  size_t total = 0;
  size_t sz[3][14];
  for (int a = 0; a < 3; ++a) {
    const size_t M = Nax[a];
    const size_t t6 = 6 * (M + 1), t7 = 7 * (M + 1), t3 = 3 * M, tr = M + 1;
    const size_t tmp[14] = {t6, t6, t6, t6, t7, t7, t7, t7, t7, t7, t7, t3, tr, tr};
    for (int q = 0; q < 14; ++q) {
      sz[a][q] = tmp[q];
      total += tmp[q];
    }
  }
  std::vector<double> h64(total);
  std::vector<float> h32(total);
  size_t o = 0;
  size_t offs[3][14];
  for (int a = 0; a < 3; ++a) {
    const impact_b200_axis_tables* t = co->axis[a];
    const double* src[12] = {t->cG, t->cD, t->cIpu, t->cIup, t->cNpU, t->cNpD, t->cNuU, t->cNuD, t->cp1, t->cpp, t->cuu, t->cdg};
    for (int q = 0; q < 12; ++q) {
      if (!src[q]) {
        impact_b200_case_destroy(c);
        return impact_set_error_msg(-1, "impact_b200_case_create: null coefficient table");
      }
      offs[a][q] = o;
      std::memcpy(&h64[o], src[q], sz[a][q] * sizeof(double));
      o += sz[a][q];
    }
    // row sums of |cpp| and |cp1| (get_dtime), in the reference's summation order
    offs[a][12] = o;
    offs[a][13] = o + sz[a][12];
    const size_t M = Nax[a];
    for (size_t r = 0; r <= M; ++r) {
      double spp = 0.0, sp1 = 0.0;
      for (int l = 0; l < 7; ++l) {
        spp = spp + std::fabs(t->cpp[r * 7 + l]);
        sp1 = sp1 + std::fabs(t->cp1[r * 7 + l]);
      }
      h64[o + r] = spp;
      h64[o + sz[a][12] + r] = sp1;
    }
    o += sz[a][12] + sz[a][13];
  }
  for (size_t q = 0; q < total; ++q) h32[q] = static_cast<float>(h64[q]);
  rc |= case_alloc(s, (void**)&s.coef64, total * sizeof(double));
  rc |= case_alloc(s, (void**)&s.coef32, total * sizeof(float));
  if (rc) {
    impact_b200_case_destroy(c);
    return -1;
  }
  cudaMemcpy(s.coef64, h64.data(), total * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(s.coef32, h32.data(), total * sizeof(float), cudaMemcpyHostToDevice);
  for (int a = 0; a < 3; ++a) {
    const double* b = s.coef64;
    const float* f = s.coef32;
#define SETC(fld, q)                 \
  s.c64.fld[a] = b + offs[a][q];     \
  s.c32.fld[a] = f + offs[a][q];
    SETC(cG, 0) SETC(cD, 1) SETC(cIpu, 2) SETC(cIup, 3) SETC(cNpU, 4) SETC(cNpD, 5) SETC(cNuU, 6) SETC(cNuD, 7)
    SETC(cp1, 8) SETC(cpp, 9) SETC(cuu, 10) SETC(cdg, 11)
#undef SETC
    s.dt.spp[a] = b + offs[a][12];
    s.dt.sp1[a] = b + offs[a][13];
  }
  // ---- collapsed operator weights of product_div_grad ----
  {
    std::vector<double> w[3];
    size_t tot = 0;
    for (int a = 0; a < 3; ++a) {
      collapse_divgrad(Nax[a], co->axis[a]->cG, co->axis[a]->cD, w[a]);
      tot += w[a].size();
    }
    double* d64 = nullptr;
    float* d32 = nullptr;
    rc |= case_alloc(s, (void**)&d64, tot * sizeof(double));
    rc |= case_alloc(s, (void**)&d32, tot * sizeof(float));
    if (rc) {
      impact_b200_case_destroy(c);
      return -1;
    }
    std::vector<double> all;
    all.reserve(tot);
    for (int a = 0; a < 3; ++a) {
      s.W64[a] = d64 + all.size();
      s.W32[a] = d32 + all.size();
      all.insert(all.end(), w[a].begin(), w[a].end());
    }
    // uniform z spacing: all z rows equal up to rounding of the table construction (1e-14 of the
    // largest weight), then the kernels keep one row in registers
    s.zuni = rows_uniform(w[2].data(), w[2].size() / AXW, AXW);
    s.xuni = rows_uniform(w[0].data(), w[0].size() / AXW, AXW);
    s.cdg_zuni = rows_uniform(co->axis[2]->cdg, (size_t)(desc->N3 - 1), 3);
    std::vector<float> all32(all.begin(), all.end());
    cudaMemcpy(d64, all.data(), tot * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d32, all32.data(), tot * sizeof(float), cudaMemcpyHostToDevice);
  }
  // ---- fields ----
  const size_t fb = (size_t)g.nfield * sizeof(double);
  for (int q = 0; q < IMPACT_B200_NFIELDS; ++q) rc |= case_alloc(s, (void**)&s.f[q], fb);
  for (int q = 0; q < 3; ++q) rc |= case_alloc(s, (void**)&s.work[q], fb);
  if (s.precision == 1)
    for (int q = 0; q < 3; ++q) {
      rc |= case_alloc(s, (void**)&s.work32[q], (size_t)g.nfield * sizeof(float));
      rc |= case_alloc(s, (void**)&s.nl32[q], (size_t)g.nfield * sizeof(float));
    }
  rc |= case_alloc(s, (void**)&s.label, (size_t)g.nfield);
  const size_t pd = (size_t)reduce_partial_doubles(g, 4) * sizeof(double);
  rc |= case_alloc(s, (void**)&s.partial, pd);
  rc |= case_alloc(s, (void**)&s.dscal, 64 * sizeof(double));
  if (s.precision == 0) {
    KrylovWork<double>& w = s.kw64;
    double** pf[8] = {&w.rr, &w.rh, &w.pp, &w.Ap, &w.Ar, &w.z1, &w.z2, &w.comp};
    for (double** q : pf) rc |= case_alloc(s, (void**)q, fb);
    w.partial = s.partial;
    w.partial_capacity = pd / sizeof(double);
    rc |= case_alloc(s, (void**)&w.scal, sizeof(SolverScalars));
  } else {
    MixedWork& w = s.mw;
    const size_t fb32 = (size_t)g.nfield * sizeof(float);
    rc |= case_alloc(s, (void**)&w.r64, fb);
    rc |= case_alloc(s, (void**)&w.r32, fb32);
    rc |= case_alloc(s, (void**)&w.e32, fb32);
    float** pf[8] = {&w.inner.rr, &w.inner.rh, &w.inner.pp, &w.inner.Ap, &w.inner.Ar, &w.inner.z1, &w.inner.z2, &w.inner.comp};
    for (float** q : pf) rc |= case_alloc(s, (void**)q, fb32);
    w.inner.partial = s.partial;
    w.inner.partial_capacity = pd / sizeof(double);
    rc |= case_alloc(s, (void**)&w.inner.scal, sizeof(SolverScalars));
    rc |= case_alloc(s, (void**)&w.partial64, pd);
  }
  if (rc) {
    impact_b200_case_destroy(c);
    return -1;
  }
  // ---- multigrid hierarchy ----
  if (co->xp[0] && co->xp[1] && co->xp[2] && co->xu[0] && co->xu[1] && co->xu[2]) {
    const int N[3] = {desc->N1, desc->N2, desc->N3};
    for (int a = 0; a < 3; ++a) {
      s.xp[a].assign(co->xp[a], co->xp[a] + N[a] + 7);
      s.xu[a].assign(co->xu[a], co->xu[a] + N[a] + 7);
    }
    std::vector<MGHostLevel> lv = build_mg_hierarchy(N, co->xp, co->xu, co->L, MG_MAX_LEVELS);
    s.mg_levels = (int)lv.size();
    // tables of every level in one FP64 and one FP32 allocation
    size_t tot = 0;
    for (auto& L : lv)
      for (int m = 0; m < 3; ++m) tot += L.cdg[m].size() + L.cI[m].size();
    std::vector<double> t64;
    t64.reserve(tot);
    std::vector<size_t> o_cdg(lv.size() * 3), o_cI(lv.size() * 3);
    for (size_t g = 0; g < lv.size(); ++g)
      for (int m = 0; m < 3; ++m) {
        o_cdg[g * 3 + m] = t64.size();
        t64.insert(t64.end(), lv[g].cdg[m].begin(), lv[g].cdg[m].end());
        o_cI[g * 3 + m] = t64.size();
        t64.insert(t64.end(), lv[g].cI[m].begin(), lv[g].cI[m].end());
      }
    std::vector<float> t32(t64.begin(), t64.end());
    double* d64 = nullptr;
    float* d32 = nullptr;
    rc |= case_alloc(s, (void**)&d64, t64.size() * sizeof(double));
    rc |= case_alloc(s, (void**)&d32, t32.size() * sizeof(float));
    if (rc) {
      impact_b200_case_destroy(c);
      return -1;
    }
    cudaMemcpy(d64, t64.data(), t64.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d32, t32.data(), t32.size() * sizeof(float), cudaMemcpyHostToDevice);
    s.mg64.n = s.mg32.n = s.mg_levels;
    for (int g = 0; g < s.mg_levels; ++g) {
      const Geom gg = make_geom(lv[g].M[0], lv[g].M[1], lv[g].M[2]);
      MGLevel<double>& a = s.mg64.lv[g];
      MGLevel<float>& b = s.mg32.lv[g];
      a.g = b.g = gg;
      for (int m = 0; m < 3; ++m) {
        a.cdg[m] = d64 + o_cdg[g * 3 + m];
        a.cI[m] = d64 + o_cI[g * 3 + m];
        b.cdg[m] = d32 + o_cdg[g * 3 + m];
        b.cI[m] = d32 + o_cI[g * 3 + m];
        a.ratio[m] = b.ratio[m] = lv[g].ratio[m];
      }
      a.zuni = b.zuni = rows_uniform(lv[g].cdg[2].data(), (size_t)(lv[g].M[2] - 1), 3);
      a.lmin = b.lmin = level_lmin(lv[g]);
      a.A = a.B = a.C = nullptr;
      b.A = b.B = b.C = nullptr;
      if (g == 0) continue;
      if (s.precision == 0) {
        for (double** q : {&a.A, &a.B, &a.C}) {
          rc |= case_alloc(s, (void**)q, (size_t)gg.nfield * sizeof(double));
          if (!rc) cudaMemsetAsync(*q, 0, (size_t)gg.nfield * sizeof(double), s.stream);
        }
      } else {
        for (float** q : {&b.A, &b.B, &b.C}) {
          rc |= case_alloc(s, (void**)q, (size_t)gg.nfield * sizeof(float));
          if (!rc) cudaMemsetAsync(*q, 0, (size_t)gg.nfield * sizeof(float), s.stream);
        }
      }
    }
    if (rc) {
      impact_b200_case_destroy(c);
      return -1;
    }
  }
  cudaError_t e = cudaMallocHost((void**)&s.hscal, 64 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&s.scal_host, sizeof(SolverScalars));
  if (e != cudaSuccess) {
    impact_b200_case_destroy(c);
    return impact_set_error(e, "cudaMallocHost", __FILE__, __LINE__);
  }
  s.kw64.scal_host = s.scal_host;
  s.mw.inner.scal_host = s.scal_host;
  // zero every field so that the ghost layers hold defined values
  for (void* p : s.allocs) (void)p;
  for (int q = 0; q < IMPACT_B200_NFIELDS; ++q) cudaMemsetAsync(s.f[q], 0, fb, s.stream);
  for (int q = 0; q < 3; ++q) cudaMemsetAsync(s.work[q], 0, fb, s.stream);
  if (s.precision == 1)
    for (int q = 0; q < 3; ++q) {
      cudaMemsetAsync(s.work32[q], 0, (size_t)g.nfield * sizeof(float), s.stream);
      cudaMemsetAsync(s.nl32[q], 0, (size_t)g.nfield * sizeof(float), s.stream);
    }
  cudaMemsetAsync(s.label, 1, (size_t)g.nfield, s.stream);
  if (s.precision == 0) {
    KrylovWork<double>& w = s.kw64;
    double* pf[8] = {w.rr, w.rh, w.pp, w.Ap, w.Ar, w.z1, w.z2, w.comp};
    for (double* q : pf) cudaMemsetAsync(q, 0, fb, s.stream);
  } else {
    MixedWork& w = s.mw;
    const size_t fb32 = (size_t)g.nfield * sizeof(float);
    cudaMemsetAsync(w.r64, 0, fb, s.stream);
    cudaMemsetAsync(w.r32, 0, fb32, s.stream);
    cudaMemsetAsync(w.e32, 0, fb32, s.stream);
    float* pf[8] = {w.inner.rr, w.inner.rh, w.inner.pp, w.inner.Ap, w.inner.Ar, w.inner.z1, w.inner.z2, w.inner.comp};
    for (float* q : pf) cudaMemsetAsync(q, 0, fb32, s.stream);
  }
  e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) {
    impact_b200_case_destroy(c);
    return impact_set_error(e, "case init", __FILE__, __LINE__);
  }
  *out = c;
  return 0;
}

extern "C" int impact_b200_case_upload(impact_b200_case* c, int field, const double* host) {
  if (!c || !host || field < 0 || field >= IMPACT_B200_NFIELDS)
    return impact_set_error_msg(-1, "impact_b200_case_upload: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.f[field], host, (size_t)s.g.nfield * sizeof(double), cudaMemcpyHostToDevice, s.stream));
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  return 0;
}
extern "C" int impact_b200_case_download(impact_b200_case* c, int field, double* host) {
  if (!c || !host || field < 0 || field >= IMPACT_B200_NFIELDS)
    return impact_set_error_msg(-1, "impact_b200_case_download: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  IMPACT_CUDA_CHECK(cudaMemcpyAsync(host, s.f[field], (size_t)s.g.nfield * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  return 0;
}
// the same copies enqueued on `stream` (the case stream when null) without waiting for them
// Element range [first, first + count) of a field; `host` is the base of the whole host field.
static int range_ok(const impact_b200_case* c, int field, const void* host, size_t first, size_t count) {
  return c && host && field >= 0 && field < IMPACT_B200_NFIELDS && first <= (size_t)c->s.g.nfield &&
         count <= (size_t)c->s.g.nfield - first;
}
extern "C" int impact_b200_case_upload_async(impact_b200_case* c, int field, const double* host, size_t first,
                                             size_t count, void* stream) {
  if (!range_ok(c, field, host, first, count))
    return impact_set_error_msg(-1, "impact_b200_case_upload_async: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s.stream;
  if (count)
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.f[field] + first, host + first, count * sizeof(double), cudaMemcpyHostToDevice, st));
  return 0;
}
extern "C" int impact_b200_case_download_async(impact_b200_case* c, int field, double* host, size_t first,
                                               size_t count, void* stream) {
  if (!range_ok(c, field, host, first, count))
    return impact_set_error_msg(-1, "impact_b200_case_download_async: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s.stream;
  if (count)
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(host + first, s.f[field] + first, count * sizeof(double), cudaMemcpyDeviceToHost, st));
  return 0;
}
extern "C" int impact_b200_case_set_inflow_waveform(impact_b200_case* c, int n, const double* time,
                                                     const double* velocity) {
  if (!c || n < 0 || n == 1 || (n > 0 && (!time || !velocity)))
    return impact_set_error_msg(-1, "impact_b200_case_set_inflow_waveform: bad arguments");
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(time[i]) || !std::isfinite(velocity[i]) || (i > 0 && time[i] < time[i - 1]))
      return impact_set_error_msg(-1, "impact_b200_case_set_inflow_waveform: times must be finite and non-decreasing");
  }
  if (n > 0 && !(time[n - 1] > 0.0))
    return impact_set_error_msg(-1, "impact_b200_case_set_inflow_waveform: the pulse length (last time) must be positive");
  c->s.inflow_t.assign(time, time + n);
  c->s.inflow_u.assign(velocity, velocity + n);
  return 0;
}
extern "C" int impact_b200_case_snapshot(impact_b200_case* c, int nfields, const int* fields, double* const* host,
                                         void* stream) {
  if (!c || nfields < 1 || nfields > IMPACT_B200_NFIELDS || !fields || !host)
    return impact_set_error_msg(-1, "impact_b200_case_snapshot: bad arguments");
  for (int q = 0; q < nfields; ++q) {
    if (fields[q] < 0 || fields[q] >= IMPACT_B200_NFIELDS || !host[q])
      return impact_set_error_msg(-1, "impact_b200_case_snapshot: bad field or host buffer");
    for (int r = 0; r < q; ++r)
      if (fields[r] == fields[q]) return impact_set_error_msg(-1, "impact_b200_case_snapshot: a field appears twice");
  }
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  const size_t fb = (size_t)s.g.nfield * sizeof(double);
  if (!s.snap_taken) {
    IMPACT_CUDA_CHECK(cudaEventCreateWithFlags(&s.snap_taken, cudaEventDisableTiming));
    IMPACT_CUDA_CHECK(cudaEventCreateWithFlags(&s.snap_read, cudaEventDisableTiming));
  }
  if (s.snap_pending) IMPACT_CUDA_CHECK(cudaStreamWaitEvent(s.stream, s.snap_read, 0));  // buffer free again
  if (nfields > s.snap_cap) {  // grow (the old buffer stays with the case until it is destroyed)
    double* p = nullptr;
    if (case_alloc(s, (void**)&p, (size_t)nfields * fb)) return -1;
    s.snap = p;
    s.snap_cap = nfields;
  }
  for (int q = 0; q < nfields; ++q)
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.snap + (size_t)q * s.g.nfield, s.f[fields[q]], fb, cudaMemcpyDeviceToDevice, s.stream));
  IMPACT_CUDA_CHECK(cudaEventRecord(s.snap_taken, s.stream));
  cudaStream_t cs = stream ? static_cast<cudaStream_t>(stream) : s.stream;
  IMPACT_CUDA_CHECK(cudaStreamWaitEvent(cs, s.snap_taken, 0));
  for (int q = 0; q < nfields; ++q)
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(host[q], s.snap + (size_t)q * s.g.nfield, fb, cudaMemcpyDeviceToHost, cs));
  IMPACT_CUDA_CHECK(cudaEventRecord(s.snap_read, cs));
  s.snap_pending = true;
  return 0;
}
extern "C" int impact_b200_case_synchronize(impact_b200_case* c) {
  if (!c) return impact_set_error_msg(-1, "impact_b200_case_synchronize: bad arguments");
  IMPACT_CUDA_CHECK(cudaSetDevice(c->s.device));
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(c->s.stream));
  return 0;
}
extern "C" int impact_b200_case_defer_pressure(impact_b200_case* c, void* event) {
  if (!c || !event) return impact_set_error_msg(-1, "impact_b200_case_defer_pressure: bad arguments");
  c->s.pre_wait = static_cast<cudaEvent_t>(event);
  return 0;
}
extern "C" int impact_b200_case_set_labels(impact_b200_case* c, const uint8_t* host) {
  if (!c || !host) return impact_set_error_msg(-1, "impact_b200_case_set_labels: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.label, host, (size_t)s.g.nfield, cudaMemcpyHostToDevice, s.stream));
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  return 0;
}
extern "C" double* impact_b200_case_field_ptr(impact_b200_case* c, int field) {
  if (!c || field < 0 || field >= IMPACT_B200_NFIELDS) return nullptr;
  return c->s.f[field];
}
extern "C" void* impact_b200_case_stream(impact_b200_case* c) { return c ? (void*)c->s.stream : nullptr; }

static EngineParams engine_params(const CaseState& s, const impact_b200_solver_params* p) {
  EngineParams ep;
  ep.precond = p->precond;
  ep.n_sweeps = p->n_sweeps;
  ep.mg_down = p->mg_down > 0 ? p->mg_down : 4;
  ep.mg_up = p->mg_up > 0 ? p->mg_up : 4;
  ep.mg_bottom = p->mg_bottom > 0 ? p->mg_bottom : 4;
  ep.omega = p->omega;
  ep.check_every = p->check_every > 0 ? p->check_every : 1;
  const char* kc = std::getenv("IMPACT_B200_KC");
  ep.kc = p->tile_kc > 0 ? p->tile_kc : (kc ? std::atoi(kc) : 32);
  ep.kc = ep.kc < 1 ? 1 : (ep.kc > KC_MAX ? KC_MAX : ep.kc);
  ep.use_graph = std::getenv("IMPACT_B200_NO_GRAPH") ? 0 : 1;
  ep.fuse = p->smooth_unfused ? 0 : 1;
  ep.bottom_cheb = p->bottom_cheb > 0 ? p->bottom_cheb : 0;
  (void)s;
  return ep;
}

// build (or rebuild) the case's own engine for these parameters and fields
static int ensure_engine(CaseState& s, const double* b, double* x, const EngineParams& ep) {
  if (s.precision == 0) {
    if (!s.e64) s.e64 = new Engine<double>();
    if (s.e64->built() && s.e64->params() == ep && s.eng_b == b && s.eng_x == x) return 0;
    EngineCase<double> ec{};
    ec.g = s.g;
    for (int m = 0; m < 3; ++m) {
      ec.W[m] = s.W64[m];
      ec.cdg[m] = s.c64.cdg[m];
    }
    ec.zuni = s.zuni;
    ec.xuni = s.xuni;
    ec.cdg_zuni = s.cdg_zuni;
    ec.mg = s.mg_levels ? &s.mg64 : nullptr;
    ec.bb = b;
    ec.phi = x;
    const KrylovWork<double>& w = s.kw64;
    ec.rr = w.rr;
    ec.rh = w.rh;
    ec.pp = w.pp;
    ec.Ap = w.Ap;
    ec.Ar = w.Ar;
    ec.z1 = w.z1;
    ec.z2 = w.z2;
    ec.comp = w.comp;
    int rc = s.e64->build({ec}, ep, s.stream);
    if (rc) return rc;
  } else {
    if (!s.emx) s.emx = new MixedEngine();
    if (s.emx->built() && s.emx->params() == ep && s.eng_b == b && s.eng_x == x) return 0;
    MixedEngine::Case mc{};
    mc.g = s.g;
    for (int m = 0; m < 3; ++m) mc.W64[m] = s.W64[m];
    mc.zuni = s.zuni;
    mc.xuni = s.xuni;
    mc.bb = b;
    mc.x = x;
    mc.r64 = s.mw.r64;
    mc.r32 = s.mw.r32;
    mc.e32 = s.mw.e32;
    EngineCase<float>& ec = mc.inner;
    ec.g = s.g;
    for (int m = 0; m < 3; ++m) {
      ec.W[m] = s.W32[m];
      ec.cdg[m] = s.c32.cdg[m];
    }
    ec.zuni = s.zuni;
    ec.xuni = s.xuni;
    ec.cdg_zuni = s.cdg_zuni;
    ec.mg = s.mg_levels ? &s.mg32 : nullptr;
    ec.bb = s.mw.r32;
    ec.phi = s.mw.e32;
    const KrylovWork<float>& w = s.mw.inner;
    ec.rr = w.rr;
    // the inner solve starts from e = 0, so its shadow residual is its right-hand side: the two
    // share the buffer (the outer loop rewrites it before every inner solve)
    ec.rh = s.mw.r32;
    ec.pp = w.pp;
    ec.Ap = w.Ap;
    ec.Ar = w.Ar;
    ec.z1 = w.z1;
    ec.z2 = w.z2;
    ec.comp = w.comp;
    int rc = s.emx->build({mc}, ep, s.stream);
    if (rc) return rc;
  }
  s.eng_b = b;
  s.eng_x = x;
  return 0;
}

static int run_poisson(CaseState& s, const double* b, double* x, const impact_b200_solver_params* p,
                       impact_b200_solver_result* r) {
  if (p->precond == 1 && s.mg_levels == 0)
    return impact_set_error_msg(-1, "multigrid preconditioner requested but the case was created without coordinates");
  const EngineParams ep = engine_params(s, p);
  int rc = ensure_engine(s, b, x, ep);
  if (rc) return rc;
  SolverResult res{};
  int inner = 0;
  if (s.precision == 0) {
    SolverScalars init{};
    init.tol_rel = p->tol_rel;
    init.tol_abs_inf = p->tol_abs_inf;
    init.max_it = p->max_it;
    std::vector<SolverResult> out;
    rc = s.e64->solve({init}, p->init_yes, out);
    if (rc) return rc;
    res = out[0];
  } else {
    SolverScalars outer{};
    outer.tol_rel = p->tol_rel;
    outer.tol_abs_inf = p->tol_abs_inf;
    outer.max_it = p->max_it;
    const double itol = p->inner_tol_rel > 0 ? p->inner_tol_rel : 1e-4;
    const int imax = p->inner_max_it > 0 ? p->inner_max_it : p->max_it * 4;
    std::vector<SolverResult> out;
    std::vector<int> its;
    rc = s.emx->solve({outer}, itol, imax, p->init_yes, out, its);
    if (rc) return rc;
    res = out[0];
    inner = its[0];
  }
  if (r) {
    r->iterations = res.iterations;
    r->inner_iterations = inner;
    r->status = res.status;
    r->res_inf = res.res_inf;
    r->res_two = res.res_two;
    r->b_two = res.b_two;
  }
  return 0;
}

// measurement entry: `iters` launches of one engine kernel kind on the case's resident fields in
// its solve precision (FP64, or FP32 for the inner solve of a mixed case); see Engine::bench
extern "C" int impact_b200_case_engine_bench(impact_b200_case* c, int kind, int iters,
                                             const impact_b200_solver_params* p, double* ms, double* bytes) {
  if (!c || !p || iters < 1 || !ms || !bytes) return impact_set_error_msg(-1, "impact_b200_case_engine_bench: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  if (p->precond == 1 && s.mg_levels == 0) return impact_set_error_msg(-1, "engine bench: no multigrid hierarchy");
  EngineParams ep = engine_params(s, p);
  int rc = ensure_engine(s, s.f[IMPACT_B200_RES], s.f[IMPACT_B200_PRE], ep);
  if (rc) return rc;
  rc = s.precision == 0 ? s.e64->bench(kind, iters, ms, bytes) : s.emx->inner().bench(kind, iters, ms, bytes);
  return rc;
}

extern "C" int impact_b200_case_poisson(impact_b200_case* c, int field_b, int field_x,
                                        const impact_b200_solver_params* p, impact_b200_solver_result* r) {
  if (!c || !p || field_b < 0 || field_x < 0 || field_b >= IMPACT_B200_NFIELDS || field_x >= IMPACT_B200_NFIELDS ||
      field_b == field_x)
    return impact_set_error_msg(-1, "impact_b200_case_poisson: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  int rc = run_poisson(s, s.f[field_b], s.f[field_x], p, r);
  if (rc) return rc;
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  IMPACT_CUDA_CHECK(cudaGetLastError());
  prof::flush();
  return 0;
}

extern "C" int impact_b200_case_mg_levels(impact_b200_case* c) { return c ? c->s.mg_levels : 0; }

extern "C" int impact_b200_case_precond(impact_b200_case* c, int field_in, int field_out,
                                        const impact_b200_solver_params* p) {
  if (!c || !p || field_in < 0 || field_out < 0 || field_in >= IMPACT_B200_NFIELDS || field_out >= IMPACT_B200_NFIELDS ||
      field_in == field_out)
    return impact_set_error_msg(-1, "impact_b200_case_precond: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  if (p->precond == 1 && s.mg_levels == 0)
    return impact_set_error_msg(-1, "impact_b200_case_precond: case has no multigrid hierarchy");
  if (p->precond != 1 && p->n_sweeps < 1)
    return impact_set_error_msg(-1, "impact_b200_case_precond: n_sweeps must be >= 1");
  // one application of the preconditioner: field_out = M field_in
  EngineParams ep = engine_params(s, p);
  ep.use_graph = 0;
  if (s.precision == 1) {  // the FP32 preconditioner of the mixed solve's inner iteration
    const long long nf = s.g.nfield;
    float* buf = nullptr;  // input, output
    IMPACT_CUDA_CHECK(cudaMalloc((void**)&buf, 2 * nf * sizeof(float)));
    const int nb = (int)std::min<long long>((nf + 255) / 256, 148LL * 32);
    k_narrow<<<nb, 256, 0, s.stream>>>(s.f[field_in], buf, nf);
    EngineCase<float> ef{};
    ef.g = s.g;
    for (int m = 0; m < 3; ++m) {
      ef.W[m] = s.W32[m];
      ef.cdg[m] = s.c32.cdg[m];
    }
    ef.zuni = s.zuni;
    ef.xuni = s.xuni;
    ef.cdg_zuni = s.cdg_zuni;
    ef.mg = s.mg_levels ? &s.mg32 : nullptr;
    const KrylovWork<float>& w = s.mw.inner;
    ef.bb = ef.pp = buf;
    ef.phi = ef.Ar = w.Ar;
    ef.rr = w.rr;
    ef.rh = w.rh;
    ef.Ap = w.Ap;
    ef.z1 = buf + nf;
    ef.z2 = w.z2;
    ef.comp = w.comp;
    int rc = 0;
    {
      Engine<float> e;
      rc = e.build({ef}, ep, s.stream);
      if (!rc) rc = e.apply_precond();
    }
    if (!rc) {
      k_widen<<<nb, 256, 0, s.stream>>>(buf + nf, s.f[field_out], nf);
      prof::count(2);
      cudaError_t ce = cudaStreamSynchronize(s.stream);
      if (ce != cudaSuccess) rc = impact_set_error(ce, "impact_b200_case_precond", __FILE__, __LINE__);
    }
    cudaFree(buf);
    return rc;
  }
  EngineCase<double> ec{};
  ec.g = s.g;
  for (int m = 0; m < 3; ++m) {
    ec.W[m] = s.W64[m];
    ec.cdg[m] = s.c64.cdg[m];
  }
  ec.zuni = s.zuni;
  ec.xuni = s.xuni;
  ec.cdg_zuni = s.cdg_zuni;
  ec.mg = s.mg_levels ? &s.mg64 : nullptr;
  const KrylovWork<double>& w = s.kw64;
  ec.bb = s.f[field_in];
  ec.phi = w.Ar;
  ec.rr = w.rr;
  ec.rh = w.rh;
  ec.pp = s.f[field_in];
  ec.Ap = w.Ap;
  ec.Ar = w.Ar;
  ec.z1 = s.f[field_out];
  ec.z2 = w.z2;
  ec.comp = w.comp;
  Engine<double> e;
  int rc = e.build({ec}, ep, s.stream);
  if (!rc) rc = e.apply_precond();
  if (rc) return rc;
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  IMPACT_CUDA_CHECK(cudaGetLastError());
  return 0;
}

extern "C" int impact_b200_case_apply(impact_b200_case* c, int op, int field_in, int field_out) {
  if (!c || field_in < 0 || field_out < 0 || field_in >= IMPACT_B200_NFIELDS || field_out >= IMPACT_B200_NFIELDS ||
      field_in == field_out || op < 0 || op > 2)
    return impact_set_error_msg(-1, "impact_b200_case_apply: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  if (op == 1) {  // field_out = divergence2 of the velocity (field_in unused)
    if (field_out <= IMPACT_B200_VEL3) return impact_set_error_msg(-1, "impact_b200_case_apply: output overlaps the velocity");
    launch_divergence2<double>(s.g, s.c64.cD[0], s.c64.cD[1], s.c64.cD[2], s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2],
                               s.f[IMPACT_B200_VEL3], s.f[field_out], s.stream);
    prof::count(1);
    IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
    IMPACT_CUDA_CHECK(cudaGetLastError());
    return 0;
  }
  impact_b200_solver_params p{};
  p.precond = 0;
  p.omega = 0.8;
  EngineParams ep = engine_params(s, &p);
  ep.use_graph = 0;
  if (op == 2) {  // field_out = A field_in in FP32 (the operator of the mixed solve's inner solve)
    const long long nf = s.g.nfield;
    float* buf = nullptr;  // input, output, unused Krylov slots
    IMPACT_CUDA_CHECK(cudaMalloc((void**)&buf, 3 * nf * sizeof(float)));
    const int nb = (int)std::min<long long>((nf + 255) / 256, 148LL * 32);
    k_narrow<<<nb, 256, 0, s.stream>>>(s.f[field_in], buf, nf);
    EngineCase<float> ef{};
    ef.g = s.g;
    for (int m = 0; m < 3; ++m) {
      ef.W[m] = s.W32[m];
      ef.cdg[m] = s.c32.cdg[m];
    }
    ef.zuni = s.zuni;
    ef.xuni = s.xuni;
    ef.cdg_zuni = s.cdg_zuni;
    ef.mg = nullptr;
    ef.bb = ef.phi = buf;
    ef.rr = buf + nf;
    ef.rh = ef.pp = ef.Ap = ef.Ar = ef.z1 = ef.z2 = ef.comp = buf + 2 * nf;
    int rc = 0;
    {
      Engine<float> e;
      rc = e.build({ef}, ep, s.stream);
      if (!rc) rc = e.apply_operator();
    }
    if (!rc) {
      k_widen<<<nb, 256, 0, s.stream>>>(buf + nf, s.f[field_out], nf);
      prof::count(2);
      cudaError_t ce = cudaStreamSynchronize(s.stream);
      if (ce != cudaSuccess) rc = impact_set_error(ce, "impact_b200_case_apply", __FILE__, __LINE__);
    }
    cudaFree(buf);
    return rc;
  }
  EngineCase<double> ec{};
  ec.g = s.g;
  for (int m = 0; m < 3; ++m) {
    ec.W[m] = s.W64[m];
    ec.cdg[m] = s.c64.cdg[m];
  }
  ec.zuni = s.zuni;
  ec.xuni = s.xuni;
  ec.cdg_zuni = s.cdg_zuni;
  ec.mg = nullptr;
  // field_out = A field_in (product_div_grad); the Krylov work fields of an FP64 case or the
  // library's own fields serve as unused slots
  double* spare = s.work[0];
  ec.bb = s.f[field_in];
  ec.phi = s.f[field_in];
  ec.rr = s.f[field_out];
  ec.rh = ec.pp = ec.Ap = ec.Ar = ec.z1 = ec.z2 = ec.comp = spare;
  Engine<double> e;
  int rc = e.build({ec}, ep, s.stream);
  if (!rc) rc = e.apply_operator();
  if (rc) return rc;
  IMPACT_CUDA_CHECK(cudaGetLastError());
  return 0;
}

static double stab_host[41];
static bool stab_ready = false;

static void stability_limits(double* lim) {
  // first r > 0 with |1 + z + z^2/2 + z^3/6| = 1 on the ray z = r(-sin t + i cos t), t = n pi / 80
  for (int n = 0; n <= 40; ++n) {
    const double t = n * 3.14159265358979323846 / 80.0;
    auto g = [t](double r) {
      const double zr = -r * std::sin(t), zi = r * std::cos(t);
      const double z2r = zr * zr - zi * zi, z2i = 2.0 * zr * zi;
      const double z3r = z2r * zr - z2i * zi, z3i = z2r * zi + z2i * zr;
      const double re = 1.0 + zr + 0.5 * z2r + z3r / 6.0, im = zi + 0.5 * z2i + z3i / 6.0;
      return re * re + im * im - 1.0;
    };
    double lo = 1e-3, hi = lo;
    while (g(hi) < 0.0 && hi < 10.0) {
      lo = hi;
      hi += 1e-3;
    }
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      (g(mid) < 0.0 ? lo : hi) = mid;
    }
    lim[n] = 0.5 * (lo + hi);
  }
}

// ---- phases of one time step of one case, on stream st (shared by single cases and batches) ----
static int upload_stab(cudaStream_t st) {
  if (!stab_ready) {
    stability_limits(stab_host);
    stab_ready = true;
  }
  IMPACT_CUDA_CHECK(cudaMemcpyToSymbolAsync(c_stab, stab_host, sizeof(stab_host), 0, cudaMemcpyHostToDevice, st));
  return 0;
}

// get_dtime: the CFL bound beta of the case lands in s.dscal[0]
static void step_beta(CaseState& s, const impact_b200_step_params* p, cudaStream_t st) {
  const Geom& g = s.g;
  k_dtime<<<grid3(g), dim3(BX, BY), 0, st>>>(g, s.c64, s.dt, p->Re, s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2],
                                             s.f[IMPACT_B200_VEL3], s.partial);
  k_reduce_partials<<<1, 1024, 0, st>>>(s.partial, nblocks(g), 1, s.dscal);
  prof::count(2);
}

static double dt_from_beta(double beta1, const impact_b200_step_params* p, const impact_b200_step_state* stt) {
  double dt;
  const double dinv = beta1 / p->CFL;
  if (std::fabs(dinv) < 1.0 / p->dtime_max)
    dt = p->dtime_max;
  else
    dt = 1.0 / dinv;
  if (stt->timestep == 0 && dt > p->dtime0) dt = p->dtime0;
  return dt;
}

// rhs_vel and the right-hand side of the pressure equation of substep sub
static void substep_rhs(CaseState& s, const impact_b200_step_params* p, double dt, int sub, cudaStream_t st) {
  const Geom& g = s.g;
  const dim3 gr = grid3(g), bl(BX, BY);
  const double cells = (double)g.n1 * g.n2 * g.n3;
  double* vel[3] = {s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2], s.f[IMPACT_B200_VEL3]};
  double* nl[3] = {s.f[IMPACT_B200_NL1], s.f[IMPACT_B200_NL2], s.f[IMPACT_B200_NL3]};
  double* rhs[3] = {s.f[IMPACT_B200_RHS1], s.f[IMPACT_B200_RHS2], s.f[IMPACT_B200_RHS3]};
  const double multL = 1.0 / p->Re;
  const double mb = dt * bRK[sub], ma = dt * aRK[sub];
  const int use_old = sub != 0;
  if (s.precision == 1 && p->explicit_fp32) {  // FP32 rhs_vel pass: FP32 work fields and nonlinear term
    k_interp_vel3_32<<<gr, bl, 0, st>>>(g, s.c64, vel[0], vel[1], vel[2], s.work32[0], s.work32[1], s.work32[2]);
    prof::count(1);
    // bytes: vel 8 (the staged tile and the point), work 3 x 4, nl 4 (+4 old), rhs 8
    const double nlb = (use_old ? 36.0 : 32.0) * cells;
    for (int m = 0; m < 3; ++m)
      IMPACT_PROF(prof::K_NL_RHS, nlb, st,
                  launch_rhs_march32(m, g, s.c32, multL, mb, ma, use_old, vel[m], s.work32, s.nl32[m], rhs[m], st));
  } else {
    k_interp_vel3<<<gr, bl, 0, st>>>(g, s.c64, vel[0], vel[1], vel[2], s.work[0], s.work[1], s.work[2]);
    prof::count(1);
    const double nlb = (use_old ? 7.0 : 6.0) * 8.0 * cells;
    for (int m = 0; m < 3; ++m)
      IMPACT_PROF(prof::K_NL_RHS, nlb, st,
                  launch_rhs_march(m, g, s.c64, multL, mb, ma, use_old, vel[m], s.work, nl[m], rhs[m], st));
  }
  // divergence2 reads no pressure: it runs before the pressure's first read, so that a deferred
  // pressure upload overlaps it too
  IMPACT_PROF(prof::K_DIV2, 4.0 * 8.0 * cells, st,
              (k_div2<<<gr, bl, 0, st>>>(g, s.c64, rhs[0], rhs[1], rhs[2], s.f[IMPACT_B200_RES])));
  const double ab = aRK[sub] + bRK[sub];
  if (s.pre_wait) {  // a deferred pressure upload: wait for it here, at the step's first read
    cudaStreamWaitEvent(st, s.pre_wait, 0);
    s.pre_wait = nullptr;
  }
  k_scale_pre<<<gr, bl, 0, st>>>(g, ab, dt, 0, s.f[IMPACT_B200_PRE]);
  prof::count(1);
}

// projection vel = rhs - G pre and the pressure scaling back (mod_timeint.f90:372)
static void substep_project(CaseState& s, double dt, int sub, cudaStream_t st) {
  const Geom& g = s.g;
  const dim3 gr = grid3(g), bl(BX, BY);
  const double cells = (double)g.n1 * g.n2 * g.n3;
  double* pre = s.f[IMPACT_B200_PRE];
  IMPACT_PROF(prof::K_PROJECT, 7.0 * 8.0 * cells, st,
              k_project<<<gr, bl, 0, st>>>(g, s.c64, pre, s.f[IMPACT_B200_RHS1], s.f[IMPACT_B200_RHS2],
                                           s.f[IMPACT_B200_RHS3], s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2],
                                           s.f[IMPACT_B200_VEL3]));
  k_scale_pre<<<gr, bl, 0, st>>>(g, aRK[sub] + bRK[sub], dt, 1, pre);
  prof::count(1);
}

// Inflow velocity of the label-5 voxels at nondimensional time t.  With a measured waveform
// (apply_CT_forcing, usr_func.f90:923-945): t is shifted into the current pulse (pulse length =
// the last table time, get_pulse_number_and_length :753-760, get_shifted_time_in_pulse
// :899-906) and the velocity is the value at the start of the last table interval [t_i, t_i+1]
// that holds it (no such interval: *on = 0, the voxels keep their velocity; the reference's
// loop also visits a last interval past the table, which is left out here).  Without one:
// U0 (1 + sin(2 pi t / T) / 2).
static double inflow_velocity(const CaseState& s, const impact_b200_step_params* p, double t, int* on) {
  *on = 1;
  const size_t n = s.inflow_t.size();
  if (n < 2) return p->U0 * (1.0 + 0.5 * std::sin(2.0 * 3.14159265358979323846 * t / p->T_pulse));
  const double len = s.inflow_t[n - 1];
  const double pulse = std::floor(t / len) + 1.0;
  const double ts = t - (pulse - 1.0) * len;
  double u = 0.0;
  *on = 0;
  for (size_t i = 0; i + 1 < n; ++i)
    if (ts >= s.inflow_t[i] && ts <= s.inflow_t[i + 1]) {
      u = s.inflow_u[i];
      *on = 1;
    }
  return u;
}

// end of the step: mask forcing at the new time, level_pressure
static void step_finish(CaseState& s, const impact_b200_step_params* p, impact_b200_step_state* stt, double dt,
                        cudaStream_t st) {
  const Geom& g = s.g;
  const dim3 gr = grid3(g), bl(BX, BY);
  stt->timestep += 1;
  stt->time += dt;
  int on = 1;
  const double u_in = inflow_velocity(s, p, stt->time, &on);
  k_mask<<<gr, bl, 0, st>>>(g, s.label, u_in, on, s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2], s.f[IMPACT_B200_VEL3]);
  prof::count(1);
  if (p->level_pressure) {
    k_sum<<<gr, bl, 0, st>>>(g, s.f[IMPACT_B200_PRE], s.partial);
    k_reduce_partials<<<1, 1024, 0, st>>>(s.partial, nblocks(g), 0, s.dscal + 1);
    k_sub_mean<<<gr, bl, 0, st>>>(g, s.dscal + 1, s.f[IMPACT_B200_PRE]);
    prof::count(3);
  }
}

static void record_solve(impact_b200_step_state* stt, int sub, const impact_b200_solver_result& r) {
  stt->poisson_iterations[sub] = r.iterations;
  stt->inner_iterations[sub] = r.inner_iterations;
  stt->poisson_status[sub] = r.status;
  stt->poisson_res_rel[sub] = r.b_two > 0.0 ? r.res_two / r.b_two : 0.0;
}

extern "C" int impact_b200_case_step(impact_b200_case* c, const impact_b200_step_params* p,
                                     impact_b200_step_state* st, int nsteps) {
  if (!c || !p || !st || nsteps < 0) return impact_set_error_msg(-1, "impact_b200_case_step: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  if (upload_stab(s.stream)) return -1;
  for (int step = 0; step < nsteps; ++step) {
    step_beta(s, p, s.stream);
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.hscal, s.dscal, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
    const double dt = dt_from_beta(s.hscal[0], p, st);
    st->dtime = dt;
    for (int sub = 0; sub < 3; ++sub) {
      substep_rhs(s, p, dt, sub, s.stream);
      impact_b200_solver_result r{};
      int rc = run_poisson(s, s.f[IMPACT_B200_RES], s.f[IMPACT_B200_PRE], &p->poisson, &r);
      if (rc) return rc;
      record_solve(st, sub, r);
      substep_project(s, dt, sub, s.stream);
    }
    step_finish(s, p, st, dt, s.stream);
  }
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  IMPACT_CUDA_CHECK(cudaGetLastError());
  prof::flush();
  return 0;
}

// =========================================================================================
// batches: several cases of one device and precision advanced together; every kernel of the
// pressure solve is one launch over all cases, the explicit parts run per case on the batch
// stream
// =========================================================================================
struct impact_b200_batch {
  std::vector<impact_b200_case*> cases;
  int device = 0, precision = 0;
  cudaStream_t stream = nullptr;
  Engine<double> e64;
  MixedEngine emx;
  double* hbeta = nullptr;  // pinned, one per case
  // the explicit part's job lists (built on the first step) and per-step scalars
  ExJob* d_ex = nullptr;
  RhsJob* d_rhs = nullptr;
  StepScal* d_sc = nullptr;
  StepScal* h_sc = nullptr;  // pinned
  double* d_beta = nullptr;
  int ex_blocks = 0, ex_pblocks = 0, rhs_blocks = 0;  // grid3 blocks, XPL-plane blocks, rhs_vel blocks
};

extern "C" int impact_b200_batch_destroy(impact_b200_batch* b) {
  if (!b) return 0;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  b->e64.release();
  b->emx.release();
  if (b->hbeta) cudaFreeHost(b->hbeta);
  if (b->h_sc) cudaFreeHost(b->h_sc);
  cudaFree(b->d_ex);
  cudaFree(b->d_rhs);
  cudaFree(b->d_sc);
  cudaFree(b->d_beta);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return 0;
}

extern "C" int impact_b200_batch_create(impact_b200_case* const* cases, int ncases, impact_b200_batch** out) {
  if (!cases || ncases < 1 || !out) return impact_set_error_msg(-1, "impact_b200_batch_create: bad arguments");
  *out = nullptr;
  for (int c = 0; c < ncases; ++c) {
    if (!cases[c]) return impact_set_error_msg(-1, "impact_b200_batch_create: null case");
    if (cases[c]->s.device != cases[0]->s.device || cases[c]->s.precision != cases[0]->s.precision)
      return impact_set_error_msg(-1, "impact_b200_batch_create: cases differ in device or precision");
    for (int d = 0; d < c; ++d)
      if (cases[d] == cases[c]) return impact_set_error_msg(-1, "impact_b200_batch_create: a case appears twice");
  }
  IMPACT_CUDA_CHECK(cudaSetDevice(cases[0]->s.device));
  impact_b200_batch* b = new impact_b200_batch();
  b->cases.assign(cases, cases + ncases);
  b->device = cases[0]->s.device;
  b->precision = cases[0]->s.precision;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->hbeta, ncases * sizeof(double));
  if (e != cudaSuccess) {
    impact_b200_batch_destroy(b);
    return impact_set_error(e, "impact_b200_batch_create", __FILE__, __LINE__);
  }
  *out = b;
  return 0;
}

// the explicit part's job lists of a batch (the cases' fields do not move while they exist)
static int batch_jobs(impact_b200_batch* b) {
  if (b->d_ex) return 0;
  const int n = (int)b->cases.size();
  std::vector<ExJob> ex(n);
  std::vector<RhsJob> rj(n);
  int eb = 0, rb = 0;
  cudaError_t e = cudaMalloc((void**)&b->d_sc, n * sizeof(StepScal));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_sc, n * sizeof(StepScal));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_beta, n * sizeof(double));
  // the rhs_vel blocks of all cases run in one launch: their depth follows the batch's total
  // (small cases alone would get shallow blocks that read their 6 halo planes again and again)
  long long colpl = 0;
  for (int c = 0; c < n; ++c) colpl += rhs_march_column_planes(b->cases[c]->s.g);
  const int kz_batch = rhs_march_kz_for(colpl);
  int pb = 0;
  for (int c = 0; c < n && e == cudaSuccess; ++c) {
    CaseState& s = b->cases[c]->s;
    ExJob& J = ex[c];
    J = ExJob{};
    J.g = s.g;
    J.c = s.c64;
    J.dr = s.dt;
    for (int m = 0; m < 3; ++m) {
      J.vel[m] = s.f[IMPACT_B200_VEL1 + m];
      J.nl[m] = s.f[IMPACT_B200_NL1 + m];
      J.rhs[m] = s.f[IMPACT_B200_RHS1 + m];
      J.work[m] = s.work[m];
      J.work32[m] = s.work32[m];
    }
    J.pre = s.f[IMPACT_B200_PRE];
    J.res = s.f[IMPACT_B200_RES];
    J.label = s.label;
    J.partial = s.partial;
    J.dscal = s.dscal;
    J.sc = b->d_sc + c;
    const dim3 d = grid3(s.g);
    J.gx = d.x;
    J.gy = d.y;
    J.gz = d.z;
    J.b0 = eb;
    eb += J.gx * J.gy * J.gz;
    J.pb0 = pb;
    pb += J.gx * J.gy * ((J.gz + XPL - 1) / XPL);
    RhsJob& R = rj[c];
    R = RhsJob{};
    R.g = s.g;
    R.c = s.c64;
    R.c32 = s.c32;
    R.Re = &b->d_sc[c].Re;
    R.dt = &b->d_sc[c].dt;
    for (int m = 0; m < 3; ++m) {
      R.vel[m] = J.vel[m];
      R.work[m] = J.work[m];
      R.nl[m] = J.nl[m];
      R.work32[m] = s.work32[m];
      R.nl32[m] = s.nl32[m];
      R.rhs[m] = J.rhs[m];
    }
    rhs_march_job_grid(s.g, R, kz_batch);
    R.b0 = rb;
    rb += R.gx * R.gy * R.gz;
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_ex, n * sizeof(ExJob));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_rhs, n * sizeof(RhsJob));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_ex, ex.data(), n * sizeof(ExJob), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_rhs, rj.data(), n * sizeof(RhsJob), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(b->d_ex);
    b->d_ex = nullptr;
    return impact_set_error(e, "batch job lists", __FILE__, __LINE__);
  }
  b->ex_blocks = eb;
  b->ex_pblocks = pb;
  b->rhs_blocks = rb;
  return 0;
}

// (re)build the batch engine when the solver parameters change
static int batch_engine(impact_b200_batch* b, const impact_b200_solver_params* p) {
  const int n = (int)b->cases.size();
  const EngineParams ep = engine_params(b->cases[0]->s, p);
  if (p->precond == 1)
    for (auto* c : b->cases)
      if (c->s.mg_levels == 0)
        return impact_set_error_msg(-1, "batch: multigrid requested but a case was created without coordinates");
  if (b->precision == 0) {
    if (b->e64.built() && b->e64.params() == ep) return 0;
    std::vector<EngineCase<double>> ec(n);
    for (int c = 0; c < n; ++c) {
      CaseState& s = b->cases[c]->s;
      EngineCase<double>& E = ec[c];
      E = EngineCase<double>{};
      E.g = s.g;
      for (int m = 0; m < 3; ++m) {
        E.W[m] = s.W64[m];
        E.cdg[m] = s.c64.cdg[m];
      }
      E.zuni = s.zuni;
      E.xuni = s.xuni;
      E.cdg_zuni = s.cdg_zuni;
      E.mg = s.mg_levels ? &s.mg64 : nullptr;
      E.bb = s.f[IMPACT_B200_RES];
      E.phi = s.f[IMPACT_B200_PRE];
      const KrylovWork<double>& w = s.kw64;
      E.rr = w.rr;
      E.rh = w.rh;
      E.pp = w.pp;
      E.Ap = w.Ap;
      E.Ar = w.Ar;
      E.z1 = w.z1;
      E.z2 = w.z2;
      E.comp = w.comp;
    }
    return b->e64.build(ec, ep, b->stream);
  }
  if (b->emx.built() && b->emx.params() == ep) return 0;
  std::vector<MixedEngine::Case> mc(n);
  for (int c = 0; c < n; ++c) {
    CaseState& s = b->cases[c]->s;
    MixedEngine::Case& M = mc[c];
    M = MixedEngine::Case{};
    M.g = s.g;
    for (int m = 0; m < 3; ++m) M.W64[m] = s.W64[m];
    M.zuni = s.zuni;
    M.xuni = s.xuni;
    M.bb = s.f[IMPACT_B200_RES];
    M.x = s.f[IMPACT_B200_PRE];
    M.r64 = s.mw.r64;
    M.r32 = s.mw.r32;
    M.e32 = s.mw.e32;
    EngineCase<float>& E = M.inner;
    E.g = s.g;
    for (int m = 0; m < 3; ++m) {
      E.W[m] = s.W32[m];
      E.cdg[m] = s.c32.cdg[m];
    }
    E.zuni = s.zuni;
    E.xuni = s.xuni;
    E.cdg_zuni = s.cdg_zuni;
    E.mg = s.mg_levels ? &s.mg32 : nullptr;
    E.bb = s.mw.r32;
    E.phi = s.mw.e32;
    const KrylovWork<float>& w = s.mw.inner;
    E.rr = w.rr;
    E.rh = s.mw.r32;  // shadow residual = right-hand side (e = 0 at the start), one buffer
    E.pp = w.pp;
    E.Ap = w.Ap;
    E.Ar = w.Ar;
    E.z1 = w.z1;
    E.z2 = w.z2;
    E.comp = w.comp;
  }
  return b->emx.build(mc, ep, b->stream);
}

extern "C" int impact_b200_batch_step(impact_b200_batch* b, const impact_b200_step_params* p,
                                      impact_b200_step_state* st, int nsteps) {
  if (!b || !p || !st || nsteps < 0) return impact_set_error_msg(-1, "impact_b200_batch_step: bad arguments");
  const int n = (int)b->cases.size();
  IMPACT_CUDA_CHECK(cudaSetDevice(b->device));
  cudaStream_t bs = b->stream;
  for (auto* c : b->cases) IMPACT_CUDA_CHECK(cudaStreamSynchronize(c->s.stream));
  int rc = batch_engine(b, &p[0].poisson);
  if (rc) return rc;
  if (upload_stab(bs)) return -1;
  std::vector<double> dt(n);
  std::vector<SolverScalars> init(n);
  std::vector<SolverResult> res;
  std::vector<int> its;
  if (batch_jobs(b)) return -1;
  const ExJob* EJ = b->d_ex;
  double cells = 0.0;
  for (auto* c : b->cases) cells += (double)c->s.g.n1 * c->s.g.n2 * c->s.g.n3;
  const dim3 bl(BX, BY);
  for (int step = 0; step < nsteps; ++step) {
    // get_dtime of every case in one launch, the CFL bounds back in one copy
    for (int c = 0; c < n; ++c) {
      b->h_sc[c] = StepScal{0.0, p[c].Re, 0.0, 1, p[c].level_pressure};
    }
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(b->d_sc, b->h_sc, n * sizeof(StepScal), cudaMemcpyHostToDevice, bs));
    k_b_dtime<<<b->ex_blocks, bl, 0, bs>>>(EJ, n);
    k_b_reduce<<<n, 1024, 0, bs>>>(EJ, 1, 0, 0, b->d_beta);
    prof::count(2);
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(b->hbeta, b->d_beta, n * sizeof(double), cudaMemcpyDeviceToHost, bs));
    IMPACT_CUDA_CHECK(cudaStreamSynchronize(bs));
    for (int c = 0; c < n; ++c) {
      dt[c] = dt_from_beta(b->hbeta[c], &p[c], &st[c]);
      st[c].dtime = dt[c];
      int on = 1;
      const double u_in = inflow_velocity(b->cases[c]->s, &p[c], st[c].time + dt[c], &on);
      b->h_sc[c] = StepScal{dt[c], p[c].Re, u_in, on, p[c].level_pressure};
    }
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(b->d_sc, b->h_sc, n * sizeof(StepScal), cudaMemcpyHostToDevice, bs));
    for (int sub = 0; sub < 3; ++sub) {
      // rhs_vel and the pressure equation's right-hand side of every case, one launch per kernel
      const int f32 = b->precision == 1 && p[0].explicit_fp32;
      k_b_interp<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n, f32);
      prof::count(1);
      for (int m = 0; m < 3; ++m)
        IMPACT_PROF(prof::K_NL_RHS, (f32 ? (sub != 0 ? 36.0 : 32.0) : (sub != 0 ? 56.0 : 48.0)) * cells, bs,
                    launch_rhs_march_batch(m, b->d_rhs, n, b->rhs_blocks, sub, f32, bs));
      IMPACT_PROF(prof::K_DIV2, 4.0 * 8.0 * cells, bs, (k_b_div2<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n)));
      for (auto* c : b->cases)
        if (c->s.pre_wait) {  // a deferred pressure upload: wait for it at the first read
          IMPACT_CUDA_CHECK(cudaStreamWaitEvent(bs, c->s.pre_wait, 0));
          c->s.pre_wait = nullptr;
        }
      k_b_scale_pre<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n, sub, 0);
      prof::count(1);
      for (int c = 0; c < n; ++c) {
        init[c] = SolverScalars{};
        init[c].tol_rel = p[c].poisson.tol_rel;
        init[c].tol_abs_inf = p[c].poisson.tol_abs_inf;
        init[c].max_it = p[c].poisson.max_it;
      }
      if (b->precision == 0) {
        rc = b->e64.solve(init, p[0].poisson.init_yes, res);
        its.assign(n, 0);
      } else {
        const double itol = p[0].poisson.inner_tol_rel > 0 ? p[0].poisson.inner_tol_rel : 1e-4;
        const int imax = p[0].poisson.inner_max_it > 0 ? p[0].poisson.inner_max_it : p[0].poisson.max_it * 4;
        rc = b->emx.solve(init, itol, imax, p[0].poisson.init_yes, res, its);
      }
      if (rc) return rc;
      for (int c = 0; c < n; ++c) {
        impact_b200_solver_result r{};
        r.iterations = res[c].iterations;
        r.inner_iterations = its[c];
        r.status = res[c].status;
        r.res_inf = res[c].res_inf;
        r.res_two = res[c].res_two;
        r.b_two = res[c].b_two;
        record_solve(&st[c], sub, r);
      }
      IMPACT_PROF(prof::K_PROJECT, 7.0 * 8.0 * cells, bs, (k_b_project<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n)));
      k_b_scale_pre<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n, sub, 1);
      prof::count(1);
    }
    // mask forcing at the new time and level_pressure of every case
    bool lp = false;
    for (int c = 0; c < n; ++c) {
      st[c].timestep += 1;
      st[c].time += dt[c];
      lp = lp || p[c].level_pressure;
    }
    k_b_mask<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n);
    prof::count(1);
    if (lp) {
      k_b_sum<<<b->ex_blocks, bl, 0, bs>>>(EJ, n);
      k_b_reduce<<<n, 1024, 0, bs>>>(EJ, 0, 1, 1, nullptr);
      k_b_sub_mean<<<b->ex_pblocks, bl, 0, bs>>>(EJ, n);
      prof::count(3);
    }
  }
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(bs));
  IMPACT_CUDA_CHECK(cudaGetLastError());
  prof::flush();
  return 0;
}

extern "C" int impact_b200_batch_size(impact_b200_batch* b) { return b ? (int)b->cases.size() : 0; }
extern "C" void* impact_b200_batch_stream(impact_b200_batch* b) { return b ? (void*)b->stream : nullptr; }

// ---------------------------------------------------------------------------------------
// measurement entry: launch one hot kernel `iters` times on the case's resident fields
// (kid 0 Jacobi sweep, 1 fused init+sweep, 2 A x with one inner product, 3 A x alone,
//  4 the reference-style one-thread-per-point Jacobi sweep) in the case's precision;
// returns the average milliseconds per launch (CUDA events on the case stream).
// ---------------------------------------------------------------------------------------
#include "stencil25d.cuh"
extern "C" int impact_b200_case_kernel_bench(impact_b200_case* c, int kid, int iters, double* ms_per_launch) {
  if (!c || iters < 1 || !ms_per_launch) return impact_set_error_msg(-1, "impact_b200_case_kernel_bench: bad arguments");
  CaseState& s = c->s;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  const Geom& g = s.g;
  cudaEvent_t a, b;
  IMPACT_CUDA_CHECK(cudaEventCreate(&a));
  IMPACT_CUDA_CHECK(cudaEventCreate(&b));
  auto launch = [&]() -> int {
    if (kid >= 10) {  // FP64 passes of the time step on the resident velocity, work and nl fields
      double* vel[3] = {s.f[IMPACT_B200_VEL1], s.f[IMPACT_B200_VEL2], s.f[IMPACT_B200_VEL3]};
      double* nl[3] = {s.f[IMPACT_B200_NL1], s.f[IMPACT_B200_NL2], s.f[IMPACT_B200_NL3]};
      double* rhs[3] = {s.f[IMPACT_B200_RHS1], s.f[IMPACT_B200_RHS2], s.f[IMPACT_B200_RHS3]};
      const dim3 gr = grid3(g), bl(BX, BY);
      switch (kid) {
        case 10: case 11: case 12: {
          const int m = kid - 10;
          launch_rhs_march(m, g, s.c64, 2e-3, -0.01, 0.02, 1, vel[m], s.work, nl[m], rhs[m], s.stream);
          break;
        }
        case 13: k_interp_vel3<<<gr, bl, 0, s.stream>>>(g, s.c64, vel[0], vel[1], vel[2], s.work[0], s.work[1], s.work[2]); break;
        case 14: k_project<<<gr, bl, 0, s.stream>>>(g, s.c64, s.f[IMPACT_B200_PRE], rhs[0], rhs[1], rhs[2], vel[0], vel[1], vel[2]); break;
        case 15: k_div2<<<gr, bl, 0, s.stream>>>(g, s.c64, rhs[0], rhs[1], rhs[2], s.f[IMPACT_B200_RES]); break;
        default: return -1;
      }
      return 0;
    }
    if (s.precision == 0) {
      double* x = s.f[IMPACT_B200_PRE];
      double* bb = s.f[IMPACT_B200_RES];
      double* o = s.f[IMPACT_B200_RHS1];
      switch (kid) {
        case 0: launch_jacobi25<double, 0>(g, s.c64, nullptr, 0.8, bb, x, o, s.stream); break;
        case 1: launch_jacobi25<double, 1>(g, s.c64, nullptr, 0.8, bb, nullptr, o, s.stream); break;
        case 2: launch_divgrad25<double, 1>(g, s.c64, nullptr, x, o, bb, s.partial, s.stream); break;
        case 3: launch_divgrad25<double, 0>(g, s.c64, nullptr, x, o, nullptr, nullptr, s.stream); break;
        case 4: launch_jacobi<double>(g, s.c64.cdg[0], s.c64.cdg[1], s.c64.cdg[2], 0.8, bb, x, o, s.stream); break;
        default: return -1;
      }
    } else {
      float* x = s.mw.inner.z1;
      float* bb = s.mw.inner.rr;
      float* o = s.mw.inner.z2;
      switch (kid) {
        case 0: launch_jacobi25<float, 0>(g, s.c32, nullptr, 0.8f, bb, x, o, s.stream); break;
        case 1: launch_jacobi25<float, 1>(g, s.c32, nullptr, 0.8f, bb, nullptr, o, s.stream); break;
        case 2: launch_divgrad25<float, 1>(g, s.c32, nullptr, x, o, bb, s.partial, s.stream); break;
        case 3: launch_divgrad25<float, 0>(g, s.c32, nullptr, x, o, nullptr, nullptr, s.stream); break;
        case 4: launch_jacobi<float>(g, s.c32.cdg[0], s.c32.cdg[1], s.c32.cdg[2], 0.8f, bb, x, o, s.stream); break;
        default: return -1;
      }
    }
    return 0;
  };
  if (launch()) return impact_set_error_msg(-1, "impact_b200_case_kernel_bench: unknown kernel id");
  cudaEventRecord(a, s.stream);
  for (int t = 0; t < iters; ++t) launch();
  cudaEventRecord(b, s.stream);
  IMPACT_CUDA_CHECK(cudaEventSynchronize(b));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  *ms_per_launch = ms / iters;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  IMPACT_CUDA_CHECK(cudaGetLastError());
  return 0;
}
