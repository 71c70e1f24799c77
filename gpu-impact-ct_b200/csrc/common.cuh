// common.cuh -- shared device-side definitions of the IMPACT B200 hot path.
//
// Field layout (identical to the reference device buffers, mod_mem_GPU.f90:27-31 and
// every *_kernel.cu): a field of a grid with N1 x N2 x N3 points is a column-major array
// phi(-3:N1+3, -3:N2+3, -3:N3+3); Fortran index i sits at C offset i+3, nx = N1+7.
// Boundaries are periodic in all three directions (the only configuration the reference
// kernels support, jor_kernel_launcher.cu:18-33): the unique points are 1..n with
// n = N-1, and stencils wrap their neighbour indices into 1..n instead of reading ghost
// planes, so no ghost exchange is ever needed between kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace impact {

// Stencil widths of IMPACT (mod_vars.f90:157-214).
constexpr int B_LO = -3, B_HI = 3, NB = 7;  // central / upwind tables (b, n)
constexpr int D_LO = -3, D_HI = 2, ND = 6;  // divergence, velocity->pressure interpolation
constexpr int G_LO = -2, G_HI = 3, NG = 6;  // gradient, pressure->velocity interpolation

struct Geom {
  int n1, n2, n3;     // unique periodic points per axis (N - 1)
  int nx, ny;         // padded extents N1+7, N2+7
  long long nxy;      // nx*ny
  long long nfield;   // nx*ny*(N3+7)
};

__host__ __device__ inline Geom make_geom(int N1, int N2, int N3) {
  Geom g;
  g.n1 = N1 - 1;
  g.n2 = N2 - 1;
  g.n3 = N3 - 1;
  g.nx = N1 + 7;
  g.ny = N2 + 7;
  g.nxy = (long long)g.nx * g.ny;
  g.nfield = g.nxy * (long long)(N3 + 7);
  return g;
}

// offset of Fortran point (i,j,k), 1 <= i <= n1 etc.
__host__ __device__ __forceinline__ long long off(const Geom& g, int i, int j, int k) {
  return (long long)(i + 3) + (long long)g.nx * (j + 3) + g.nxy * (long long)(k + 3);
}
// periodic wrap of an index that is at most one period outside 1..n
__device__ __forceinline__ int wrapi(int i, int n) {
  return i < 1 ? i + n : (i > n ? i - n : i);
}

// All coefficient tables of one grid, already on the device.  Each table row i (Fortran
// point index 0..N) holds the stencil weights c(lo:hi, i) contiguously, exactly as the
// reference uploads them (mod_mem_GPU.f90:348-434).  The compact Laplacian cdg(-1:1, 1:N)
// is stored with row i-1.
template <typename T>
struct Coeffs {
  const T* cG[3];    // cGp1..3     (g-range)
  const T* cD[3];    // cDu1,cDv2,cDw3 (d-range)
  const T* cIpu[3];  // cIpu,cIpv,cIpw (g-range)
  const T* cIup[3];  // cIup,cIvp,cIwp (d-range)
  const T* cNpU[3];  // cNp1U..3 (b-range)
  const T* cNpD[3];
  const T* cNuU[3];  // cNu1U,cNv2U,cNw3U
  const T* cNuD[3];
  const T* cp1[3];   // cp1..3 first derivative, pressure grid
  const T* cpp[3];   // cp11,cp22,cp33
  const T* cuu[3];   // cu11,cv22,cw33
  const T* cdg[3];   // cdg1..3
};

// Per-case device scalars of the Krylov solver; kept in device memory so that no host
// round trip is needed inside an iteration.
struct SolverScalars {
  double rhr, rhr_prev, rhr_next, alpha, omega, beta, rhAp, rAr, ArAr;
  double norm_inf, norm_two_sq, b_two_sq;
  double tol_rel, tol_abs_inf;
  int it;         // iterations started
  int max_it;
  int done;       // 1 once converged or out of iterations: every later kernel is a no-op
  int status;     // 0 ok, 1 max iterations, 2 breakdown, 3 non-finite, 4 shadow residual lost
  int phi_zero;   // 1 until the first x update: phi holds no value yet and that update starts from 0
  int rr_in_rh;   // 1: the caller wrote r0 to rh and pp, not to rr: the first iteration reads it there
};

}  // namespace impact

#define IMPACT_CUDA_CHECK(expr)                                    \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) return impact_set_error(_e, #expr, __FILE__, __LINE__); \
  } while (0)

int impact_set_error(cudaError_t e, const char* what, const char* file, int line);
int impact_set_error_msg(int code, const char* msg);
