// solver.cu -- deterministic device reductions for the library entry points outside the Poisson
// engine (impact_b200_product_scalar: product_scalar, mod_solvers.f90:2319-2360).
//
// A reduction is three fixed-order stages: every block of a 32 x 8 x n3 grid writes its partial
// (warp shuffles, then one warp over the block's warps), FIN1_BLOCKS blocks each sum a contiguous
// chunk of the block partials, and one block sums those; the result lands in device memory.  The
// order depends only on the grid, so a result is the same run to run.  (The Poisson solves run in
// the engine, engine.cu, with their own per-tile partials and finalisation.)
#include <cmath>
#include <cstdio>

#include "prof.cuh"
#include "solver.cuh"

namespace impact {

constexpr int BX = 32, BY = 8, NT = BX * BY;
constexpr int FIN1_BLOCKS = 256;

static inline dim3 grid3(const Geom& g) { return dim3((g.n1 + BX - 1) / BX, (g.n2 + BY - 1) / BY, g.n3); }
static inline long long nblocks3(const Geom& g) {
  const dim3 d = grid3(g);
  return (long long)d.x * d.y * d.z;
}

// layout of a partial buffer: [nb x 4 block partials][FIN1_BLOCKS x 4 stage-1 sums][64 results]
long long reduce_partial_doubles(const Geom& g, int nq) {
  (void)nq;
  return nblocks3(g) * 4 + FIN1_BLOCKS * 4 + 64;
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block partial of one sum over the block's 32 x 8 threads
__device__ __forceinline__ void block_sum(double v, double* __restrict__ partial) {
  __shared__ double sh[NT / 32];
  const int tid = threadIdx.x + BX * threadIdx.y;
  const int lane = tid & 31, w = tid >> 5;
  v = wsum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    double x = lane < NT / 32 ? sh[lane] : 0.0;
    x = wsum(x);
    if (lane == 0) partial[bid] = x;
  }
}

// stage 1: block b sums its contiguous chunk of the nb block partials
__global__ void __launch_bounds__(256) k_fin1(const double* __restrict__ partial, long long nb,
                                              double* __restrict__ out) {
  const long long chunk = (nb + gridDim.x - 1) / gridDim.x;
  const long long b0 = blockIdx.x * chunk, b1 = min(nb, b0 + chunk);
  __shared__ double sh[8];
  double v = 0.0;
  for (long long b = b0 + threadIdx.x; b < b1; b += blockDim.x) v += partial[b];
  v = wsum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < 8 ? sh[threadIdx.x] : 0.0;
    x = wsum(x);
    if (threadIdx.x == 0) out[blockIdx.x] = x;
  }
}

// stage 2: one block sums the stage-1 results into *out
__global__ void __launch_bounds__(256) k_fin2(const double* __restrict__ p1, int nb, double* __restrict__ out) {
  __shared__ double sh[8];
  double v = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) v += p1[b];
  v = wsum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < 8 ? sh[threadIdx.x] : 0.0;
    x = wsum(x);
    if (threadIdx.x == 0) *out = x;
  }
}

template <typename T>
__global__ void __launch_bounds__(NT) k_dot(Geom g, const T* __restrict__ a, const T* __restrict__ b,
                                            double* __restrict__ partial) {
  const int i = blockIdx.x * BX + threadIdx.x + 1;
  const int j = blockIdx.y * BY + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const bool in = (i <= g.n1) && (j <= g.n2);
  const long long p = in ? off(g, i, j, k) : 0;
  block_sum(in ? (double)a[p] * (double)b[p] : 0.0, partial);
}

template <typename T>
void reduce_dot(const Geom& g, const T* a, const T* b, double* partial, double* out_dev, cudaStream_t s) {
  const long long nb = nblocks3(g);
  double* p1 = partial + nb * 4;
  k_dot<T><<<grid3(g), dim3(BX, BY), 0, s>>>(g, a, b, partial);
  k_fin1<<<FIN1_BLOCKS, 256, 0, s>>>(partial, nb, p1);
  k_fin2<<<1, 256, 0, s>>>(p1, FIN1_BLOCKS, out_dev);
  prof::count(3);
}
template void reduce_dot<double>(const Geom&, const double*, const double*, double*, double*, cudaStream_t);
template void reduce_dot<float>(const Geom&, const float*, const float*, double*, double*, cudaStream_t);

}  // namespace impact
