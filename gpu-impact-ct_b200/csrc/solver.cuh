// solver.cuh -- device-resident pressure Poisson solvers (internal interface).
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "mg.cuh"

namespace impact {

struct SolverOpts {
  double tol_rel;      // ||r||_2 <= tol_rel * ||b||_2   (0 = off)
  double tol_abs_inf;  // ||r||_inf < tol_abs_inf        (0 = off; the reference's epsU)
  int max_it;
  int n_sweeps;        // Jacobi sweeps per preconditioner application (0 = no preconditioner)
  double omega;        // relaxation of the preconditioner sweeps
  int init_yes;        // start from phi = 0
  int check_every;     // read the residual norm back to the host every this many iterations
  int precond;         // 0: n_sweeps Jacobi sweeps (none if 0); 1: multigrid V-cycle (mg)
  const void* mg;      // MGData<T>* of the field type when precond == 1
};

struct SolverResult {
  int iterations;
  int status;  // 0 converged, 1 max iterations, 2 breakdown, 3 non-finite
  double res_inf, res_two, b_two;
};

// Work fields of one BiCGstab instance (field type T) plus its reduction scratch.
template <typename T>
struct KrylovWork {
  T *rr, *rh, *pp, *Ap, *Ar, *z1, *z2, *comp;
  double* partial;       // >= partial_capacity doubles
  long long partial_capacity;
  SolverScalars* scal;   // device
  SolverScalars* scal_host;  // pinned host mirror
};

template <typename T>
long long krylov_partial_doubles(const Geom& g);

// BiCGstab_orig (mod_solvers.f90:1509-1935), problem_type 2: A = product_div_grad,
// preconditioner = n_sweeps damped-Jacobi sweeps of the compact Laplacian from zero
// (the single-level multigridV, mod_solvers.f90:456-585 with n_grids = 1).
template <typename T>
int bicgstab(const Geom& g, const Coeffs<T>& c, const SolverOpts& o, const T* bb, T* phi, KrylovWork<T>& w,
             cudaStream_t s, SolverResult* res);

// Mixed precision: FP64 outer residual and correction, FP32 inner BiCGstab (fields, stencils,
// Jacobi sweeps in FP32; inner products and norms accumulated in FP64).
struct MixedWork {
  double* r64;     // outer residual
  float* r32;      // inner right-hand side
  float* e32;      // inner correction
  KrylovWork<float> inner;
  double* partial64;
  SolverScalars* scal64;
  SolverScalars* scal64_host;
};
int mixed_solve(const Geom& g, const Coeffs<double>& c64, const Coeffs<float>& c32, const SolverOpts& outer,
                const SolverOpts& inner, const double* bb, double* phi, MixedWork& w, cudaStream_t s,
                SolverResult* res, int* inner_iterations);

// helpers used by the step driver
template <typename T>
void reduce_dot(const Geom& g, const T* a, const T* b, double* partial, double* out_dev, cudaStream_t s);
template <typename T>
void reduce_norms(const Geom& g, const T* a, double* partial, double* out_dev /*[inf, two_sq]*/, cudaStream_t s);
long long reduce_partial_doubles(const Geom& g, int nq);

}  // namespace impact
