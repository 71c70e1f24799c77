// noalloc.cu -- an inner product entry point that allocates no device memory.
//
// impact_b200_product_scalar keeps its per-block partial sums in a library scratch buffer that
// it allocates with cudaMalloc on first use (and reallocates when a larger grid arrives).  Some
// callers cannot allow that: a host code whose device memory is entirely claimed up front by its
// own allocator (cudaMalloc would fail), or a latency-bound loop that must not pay for
// cudaMalloc/cudaFree, which can synchronise the whole device.  This variant keeps its scratch in
// a fixed file-scope __device__ array instead; the caller still passes the two input fields and
// a host pointer for the result.
//
// Contract:
//  * scratch: one partial per z-plane plus the final sum, at most NOALLOC_MAX_PLANES planes
//    (N3 - 1 <= 16384, 128 KiB); larger grids are rejected with an error message.
//  * every GPU that loads the library holds this array until the process exits.
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//    that device current; make that first call before any stream capture on the device.
//  * all calls share the one array: two calls whose kernels overlap on the GPU race on it and
//    must be serialised by the caller (e.g. by issuing them on one stream, one after the other).
//    Nothing carries over between calls: every slot a call reads is written earlier in that call.
//  * runs on the library's current stream (impact_b200_set_stream; the legacy default stream
//    unless set), like impact_b200_product_scalar and the Part 1 launchers, so it is ordered
//    after the launchers queued on that stream; it returns once the result is on the host.
//  * its sum runs per z-plane, then over the planes: deterministic, and equal to
//    impact_b200_product_scalar's result up to rounding (that one sums per-tile partials).
//  * no cudaMalloc, cudaFree or allocating library routine is called.
#include <cstdio>
#include <mutex>

#include "../../include/impact_b200.h"
#include "common.cuh"

cudaStream_t impact_launcher_stream();  // capi.cu

namespace {

constexpr int NOALLOC_MAX_PLANES = 16384;
constexpr int NOALLOC_THREADS = 256;

// partial sums of every z-plane followed by the final sum
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_PLANES + 32];

std::mutex g_mu;
void* g_addr[256] = {};  // device address of g_noalloc_scratch per device ordinal

__device__ __forceinline__ double noalloc_wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// one block per unique z-plane: partial[k-1] = sum over the plane of a*b, fixed order
__global__ void __launch_bounds__(NOALLOC_THREADS) k_plane_dot(impact::Geom g, const double* __restrict__ a,
                                                               const double* __restrict__ b, double* __restrict__ partial) {
  const int k = blockIdx.x + 1;
  const long long npl = (long long)g.n1 * g.n2;
  double v = 0.0;
  for (long long t = threadIdx.x; t < npl; t += NOALLOC_THREADS) {
    const int i = (int)(t % g.n1) + 1, j = (int)(t / g.n1) + 1;
    const long long p = impact::off(g, i, j, k);
    v += a[p] * b[p];
  }
  __shared__ double sh[NOALLOC_THREADS / 32];
  v = noalloc_wsum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < NOALLOC_THREADS / 32 ? sh[threadIdx.x] : 0.0;
    x = noalloc_wsum(x);
    if (threadIdx.x == 0) partial[blockIdx.x] = x;
  }
}

// sums the n plane partials in plane order into out
__global__ void __launch_bounds__(NOALLOC_THREADS) k_plane_sum(const double* __restrict__ partial, int n,
                                                               double* __restrict__ out) {
  __shared__ double sh[NOALLOC_THREADS / 32];
  double v = 0.0;
  for (int t = threadIdx.x; t < n; t += NOALLOC_THREADS) v += partial[t];
  v = noalloc_wsum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < NOALLOC_THREADS / 32 ? sh[threadIdx.x] : 0.0;
    x = noalloc_wsum(x);
    if (threadIdx.x == 0) *out = x;
  }
}

}  // namespace

extern "C" int impact_b200_product_scalar_noalloc(int N1, int N2, int N3, const double* a_dev, const double* b_dev,
                                                  double* result) {
  if (N1 < 9 || N2 < 9 || N3 < 9 || !a_dev || !b_dev || !result)
    return impact_set_error_msg(-1, "impact_b200_product_scalar_noalloc: bad arguments");
  if (N3 - 1 > NOALLOC_MAX_PLANES)
    return impact_set_error_msg(-1, "impact_b200_product_scalar_noalloc: at most 16384 unique z-planes (N3 <= 16385); "
                                    "use impact_b200_product_scalar for larger grids");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return impact_set_error(e, "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= 256) return impact_set_error_msg(-1, "impact_b200_product_scalar_noalloc: device ordinal >= 256");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return impact_set_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      g_addr[dev] = p;
    }
    scratch = static_cast<double*>(g_addr[dev]);
  }
  const impact::Geom g = impact::make_geom(N1, N2, N3);
  const int planes = N3 - 1;
  double* out = scratch + NOALLOC_MAX_PLANES;
  // runs on the launchers' stream and returns after the result has reached the host
  cudaStream_t s = impact_launcher_stream();
  k_plane_dot<<<planes, NOALLOC_THREADS, 0, s>>>(g, a_dev, b_dev, scratch);
  k_plane_sum<<<1, NOALLOC_THREADS, 0, s>>>(scratch, planes, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return impact_set_error(e, "impact_b200_product_scalar_noalloc launch", __FILE__, __LINE__);
  e = cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return impact_set_error(e, "impact_b200_product_scalar_noalloc", __FILE__, __LINE__);
  return 0;
}
