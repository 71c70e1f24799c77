// solver.cuh -- work-field sets of the Poisson solves and the library's stand-alone reduction
// (internal interface).
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "mg.cuh"

namespace impact {

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

// Work fields of a mixed-precision solve: FP64 outer residual and correction around the FP32
// inner Krylov set.
struct MixedWork {
  double* r64;     // outer residual
  float* r32;      // inner right-hand side
  float* e32;      // inner correction
  KrylovWork<float> inner;
  double* partial64;
  SolverScalars* scal64;
  SolverScalars* scal64_host;
};
// deterministic inner product sum a.b over the unique points into *out_dev (solver.cu); partial
// holds reduce_partial_doubles(g, 1) doubles
template <typename T>
void reduce_dot(const Geom& g, const T* a, const T* b, double* partial, double* out_dev, cudaStream_t s);
long long reduce_partial_doubles(const Geom& g, int nq);

}  // namespace impact
