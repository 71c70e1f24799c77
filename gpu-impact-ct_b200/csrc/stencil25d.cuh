// stencil25d.cuh -- 2.5D streaming stencil kernels of the Poisson solve (internal).
//
// A block owns a TX x TY column tile and marches along z over KC planes.  Values along z live in
// a per-thread register queue; each plane's x/y neighbourhood is staged once in shared memory
// (periodic wrap applied when the halo is loaded), so every field element is read from DRAM
// about once per pass.  Reductions fused into a pass produce one partial per block.
#pragma once
#include "common.cuh"

namespace impact {

constexpr int S25_TX = 32, S25_TY = 16, S25_KC = 32;

inline dim3 s25_grid(const Geom& g) {
  return dim3((g.n1 + S25_TX - 1) / S25_TX, (g.n2 + S25_TY - 1) / S25_TY, (g.n3 + S25_KC - 1) / S25_KC);
}
inline long long s25_blocks(const Geom& g) {
  const dim3 d = s25_grid(g);
  return (long long)d.x * d.y * d.z;
}

// A x (high-order div(grad), product_div_grad) with fused inner products.
// MODE 0: none; 1: partial[b] = sum out*d1; 2: partial[2b] = sum d1*out, partial[2b+1] = sum out*out
template <typename T, int MODE>
void launch_divgrad25(const Geom& g, const Coeffs<T>& c, const SolverScalars* sc, const T* x, T* out, const T* d1,
                      double* partial, cudaStream_t s);

// damped-Jacobi sweep of the compact Laplacian cdg: out = omega (bb - offdiag rel)/diag + (1-omega) rel.
// INIT = 1: rel is the implicit start omega*bb/diag (init sweep fused with the first sweep).
template <typename T, int INIT>
void launch_jacobi25(const Geom& g, const Coeffs<T>& c, const SolverScalars* sc, T omega, const T* bb, const T* rel,
                     T* out, cudaStream_t s);

}  // namespace impact
