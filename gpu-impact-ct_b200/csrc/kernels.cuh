// kernels.cuh -- host-side launch wrappers of the IMPACT B200 kernels (internal).
#pragma once
#include "common.cuh"

namespace impact {

// ---- one-axis stencils as streaming passes (march.cu): out (=, += for OP 1) the CNT-point
// stencil from LO along axis a (0 x, 1 y, 2 z) of f; OP 2 the upwind term (cA where pp >= 0,
// else cB; overwrite when first).  Returns false (nothing launched) when n1 is not divisible by
// the 16-byte vector width or a field is not 16-byte aligned.
template <typename T, int LO, int CNT, int OP>
bool launch_march1(int a, const Geom& g, const T* cA, const T* cB, const T* f, const T* pp, T* out, int first,
                   cudaStream_t s);

// Helmholtz_explicit and the Jacobi / JOR sweep as z-marching passes (march.cu); false when
// not applicable (as launch_march1)
template <typename T>
bool launch_helm_march(const Geom& g, const T* cx, const T* cy, const T* cz, T multL, const T* vel, T* nl,
                       cudaStream_t s);
template <typename T>
bool launch_jacobi_march(const Geom& g, const T* c1, const T* c2, const T* c3, T omega, const T* bb, const T* rel,
                         T* out, cudaStream_t s);

// ---- staggered-grid operators (mod_diff.f90) ----
template <typename T>
void launch_gradient(int m, const Geom& g, const T* cG, const T* phi, T* grad, cudaStream_t s);
template <typename T>
void launch_divergence(int m, const Geom& g, const T* cD, const T* phi, T* div, cudaStream_t s);
template <typename T>
void launch_divergence2(const Geom& g, const T* cD1, const T* cD2, const T* cD3, const T* u,
                        const T* v, const T* w, T* div, cudaStream_t s);
template <typename T>
void launch_helmholtz(int m, const Geom& g, const T* cx, const T* cy, const T* cz, T multL,
                      const T* vel, T* nl, cudaStream_t s);
template <typename T>
void launch_interp_pre_vel(int m, const Geom& g, const T* cI, const T* phi, T* out, cudaStream_t s);
template <typename T>
void launch_interp_vel_pre(int m, const Geom& g, const T* cI, const T* phi, T* out, cudaStream_t s);
template <typename T>
void launch_nonlinear_upwind(int cid, const Geom& g, const T* cU, const T* cDn, const T* pp,
                             const T* vel, T* nl, cudaStream_t s);
template <typename T>
void launch_axpby(const Geom& g, T a, T b, const T* x, const T* y, T* z, cudaStream_t s);

// ---- Laplacians and relaxation (mod_laplace.f90) ----
template <typename T>
void launch_dg_relax(const Geom& g, const T* c1, const T* c2, const T* c3, const T* x, T* lap,
                     cudaStream_t s);
// out = omega*(bb - offdiag(rel))/diag + (1-omega)*rel  (out-of-place)
template <typename T>
void launch_jacobi(const Geom& g, const T* c1, const T* c2, const T* c3, T omega, const T* bb,
                   const T* rel, T* out, cudaStream_t s);
// out = one Jacobi sweep applied to the implicit start rel = omega*bb/diag
// (the init sweep of relaxation_div_grad fused with the sweep after it)
template <typename T>
void launch_jacobi_init2(const Geom& g, const T* c1, const T* c2, const T* c3, T omega,
                         const T* bb, T* out, cudaStream_t s);
template <typename T>
void launch_jacobi_init1(const Geom& g, const T* c1, const T* c2, const T* c3, T omega,
                         const T* bb, T* out, cudaStream_t s);
// JOR sweep reading boundary neighbours from the six ghost-face arrays of the reference
// interface (jor_kernel_v2.cu), out-of-place.
void launch_jor_faces(const Geom& g, int ny_cdg1, int ny_cdg2, int ny_cdg3, int grid_id,
                      double omega, const double* c1, const double* c2, const double* c3,
                      const double* rel, const double* bb, const double* rear, const double* front,
                      const double* upper, const double* lower, const double* west,
                      const double* east, double* out, cudaStream_t s);
void launch_get_ghost(const Geom& g, const double* rel, double* rear, double* front, double* upper,
                      double* lower, double* west, double* east, cudaStream_t s);
void launch_copy_interior(const Geom& g, const double* src, double* dst, cudaStream_t s);
void launch_fill_ghosts(const Geom& g, double* phi, cudaStream_t s);

// ---- high-order Laplacian A = sum_m D_m G_m (product_div_grad) ----
// lap = A x; if dot_with != nullptr also accumulates per-block partial sums of lap*dot_with
template <typename T>
void launch_div_grad(const Geom& g, const Coeffs<T>& c, const T* x, T* lap, cudaStream_t s);

// ---- pressure BC (set_pressure_BC_kernel.cu / apply_pressure_BC_CT) ----
void launch_pressure_bc(const Geom& g, int t1, int t2, int t3, int k_start_index, double p_in,
                        double p_out, double p_out2, const uint8_t* label, double* rel,
                        cudaStream_t s);
void launch_pressure_bc_f64label(const Geom& g, int t1, int t2, int t3, int k_start_index,
                                 double p_in, double p_out, double p_out2, const double* label,
                                 double* rel, cudaStream_t s);

// ---- deterministic FP64 reductions ----
constexpr int RED_BLOCKS = 592;   // 4 x 148 SMs
constexpr int RED_THREADS = 256;
// partial[b*nq + q] for q < nq quantities; finalize sums them in block order.
template <typename T>
void launch_dot_partials(const Geom& g, const T* a, const T* b, double* partial, cudaStream_t s);
template <typename T>
void launch_norm_partials(const Geom& g, const T* a, double* partial, cudaStream_t s);
// sum nq quantities over RED_BLOCKS partials in a fixed order into out[0..nq); kinds: 0 sum, 1 max
void launch_finalize(const double* partial, int nq, const int* kinds_host, double* out,
                     cudaStream_t s);

}  // namespace impact
