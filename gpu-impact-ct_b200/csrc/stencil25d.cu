// stencil25d.cu -- 2.5D streaming kernels of the Poisson solve (see stencil25d.cuh).
//
//   k_divgrad25  A x = sum_m D_m (G_m x)   product_div_grad, mod_laplace.f90:38-197
//   k_jacobi25   damped Jacobi / JOR sweep  relaxation_div_grad, mod_laplace.f90:339-613
//
// Both keep the reference's per-point order of floating-point operations: the gradient at each
// velocity point is formed as c(-2) x(-2) + ... + c(3) x(3), then the divergence weights are
// applied (x axis first, then y and z accumulated), exactly as gradient() followed by
// divergence() would; the Jacobi update subtracts the six neighbours in the order
// x-, x+, y-, y+, z-, z+.
#include "prof.cuh"
#include "stencil25d.cuh"

namespace impact {

namespace {
constexpr int TX = S25_TX, TY = S25_TY, KC = S25_KC, NT = TX * TY;

__device__ __forceinline__ bool halted25(const SolverScalars* sc) { return sc != nullptr && (sc->done | sc->status); }
// periodic image in 1..n of any integer index
__device__ __forceinline__ int wrapm(int i, int n) {
  int r = (i - 1) % n;
  return (r < 0 ? r + n : r) + 1;
}
// asynchronous global -> shared copies of single elements (cp.async, kept in L1 for the halo reuse)
template <typename T>
__device__ __forceinline__ void cp_async_el(T* smem, const T* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ double wsum25(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int NQ>
__device__ __forceinline__ void block_sum_store(double (&v)[NQ], double* __restrict__ partial) {
  __shared__ double sh[NQ][NT / 32];
  const int tid = threadIdx.x + TX * threadIdx.y;
  const int lane = tid & 31, w = tid >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = wsum25(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[q][w] = v[q];
  }
  __syncthreads();
  if (w == 0) {
    const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < NT / 32 ? sh[q][lane] : 0.0;
      x = wsum25(x);
      if (lane == 0) partial[bid * NQ + q] = x;
    }
  }
}
}  // namespace

// ------------------------------------------------------------------------------------------
// A x, fused inner products
// ------------------------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(NT, 2) k_divgrad25(Geom g, Coeffs<T> c, const SolverScalars* __restrict__ sc,
                                                  const T* __restrict__ x, T* __restrict__ out,
                                                  const T* __restrict__ d1, double* __restrict__ partial) {
  if (halted25(sc)) return;
  constexpr int RX = TX + 10, RY = TY + 10, TILE = RX * RY;
  constexpr int D = 4;   // planes of the tile ring (3 in flight while one is consumed)
  constexpr int P = 3;   // register prefetch depth of the z column
  constexpr int PER = (TILE + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*ring)[RY][RX] = reinterpret_cast<T(*)[RY][RX]>(smem_raw);
  __shared__ T sgx[TY][TX + 5];  // x-gradient at velocity points i0-2 .. i0+TX+2
  __shared__ T sgy[TY + 5][TX];  // y-gradient at velocity points j0-2 .. j0+TY+2
  __shared__ T cgx[TX + 5][6], cdx[TX][6], cgy[TY + 5][6], cdy[TY][6], cgz[KC + 5][6], cdz[KC][6];

  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int n1 = g.n1, n2 = g.n2, n3 = g.n3;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * KC;
  const int i = i0 + tx + 1, j = j0 + ty + 1;
  const bool in = (i <= n1) && (j <= n2);
  const int iw = wrapm(i, n1), jw = wrapm(j, n2);
  const int nk = min(KC, n3 - k0);

  for (int e = tid; e < (TX + 5) * 6; e += NT) cgx[e / 6][e % 6] = c.cG[0][(long long)wrapm(i0 - 2 + e / 6, n1) * NG + e % 6];
  for (int e = tid; e < TX * 6; e += NT) cdx[e / 6][e % 6] = c.cD[0][(long long)wrapm(i0 + 1 + e / 6, n1) * ND + e % 6];
  for (int e = tid; e < (TY + 5) * 6; e += NT) cgy[e / 6][e % 6] = c.cG[1][(long long)wrapm(j0 - 2 + e / 6, n2) * NG + e % 6];
  for (int e = tid; e < TY * 6; e += NT) cdy[e / 6][e % 6] = c.cD[1][(long long)wrapm(j0 + 1 + e / 6, n2) * ND + e % 6];
  for (int e = tid; e < (KC + 5) * 6; e += NT) cgz[e / 6][e % 6] = c.cG[2][(long long)wrapm(k0 - 2 + e / 6, n3) * NG + e % 6];
  for (int e = tid; e < KC * 6; e += NT) cdz[e / 6][e % 6] = c.cD[2][(long long)wrapm(k0 + 1 + e / 6, n3) * ND + e % 6];

  // tile elements this thread copies (row-major over RY x RX; smem (r, q) <-> Fortran (i0-4+q, j0-4+r))
  long long toff[PER];
  int tsm[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * NT;
    const int r = e / RX, q = e % RX;
    tsm[u] = e < TILE ? e : -1;
    toff[u] = (long long)(wrapm(i0 - 4 + q, n1) + 3) + (long long)g.nx * (wrapm(j0 - 4 + r, n2) + 3);
  }
  auto issue_tile = [&](int z) {  // z: 1-based plane of this block (Fortran k0 + z)
    const long long zo = g.nxy * (long long)(wrapm(k0 + z, n3) + 3);
    T* base = &ring[z % D][0][0];
#pragma unroll
    for (int u = 0; u < PER; ++u)
      if (tsm[u] >= 0) cp_async_el(base + tsm[u], x + toff[u] + zo);
  };
  const long long col = (long long)(iw + 3) + (long long)g.nx * (jw + 3);
  auto zat = [&](int k) { return x[col + g.nxy * (long long)(wrapm(k, n3) + 3)]; };

  // prologue: tiles of planes 1 .. D-1 in flight; z queues of the first plane
#pragma unroll
  for (int z = 1; z <= D - 1; ++z) {
    if (z <= nk) issue_tile(z);
    cp_commit();
  }
  T xq[6], gzq[6], zf[P];
  {
    T xs[11];
#pragma unroll
    for (int l = 0; l < 11; ++l) xs[l] = zat(k0 - 4 + l);
#pragma unroll
    for (int l = 0; l < P; ++l) zf[l] = zat(k0 + 7 + l);
    __syncthreads();  // coefficient rows ready
#pragma unroll
    for (int l = 0; l < 6; ++l) {
      T v = cgz[l][0] * xs[l];
#pragma unroll
      for (int r = 1; r < 6; ++r) v = v + cgz[l][r] * xs[l + r];
      gzq[l] = v;
      xq[l] = xs[5 + l];
    }
  }
  double acc[MODE > 0 ? MODE : 1] = {};
  for (int kk = 0; kk < nk; ++kk) {
    const int z = kk + 1;
    if (z + D - 1 <= nk) issue_tile(z + D - 1);
    cp_commit();
    const T xfar = zat(k0 + z + 6 + P);  // z column, P planes ahead of its use
    cp_wait<D - 1>();
    __syncthreads();
    T(*sx)[RX] = ring[z % D];
    {
      T v = cgx[tx][0] * sx[ty + 5][tx];
#pragma unroll
      for (int r = 1; r < 6; ++r) v = v + cgx[tx][r] * sx[ty + 5][tx + r];
      sgx[ty][tx] = v;
      if (tx < 5) {
        T w = cgx[TX + tx][0] * sx[ty + 5][TX + tx];
#pragma unroll
        for (int r = 1; r < 6; ++r) w = w + cgx[TX + tx][r] * sx[ty + 5][TX + tx + r];
        sgx[ty][TX + tx] = w;
      }
      T u = cgy[ty][0] * sx[ty][tx + 5];
#pragma unroll
      for (int r = 1; r < 6; ++r) u = u + cgy[ty][r] * sx[ty + r][tx + 5];
      sgy[ty][tx] = u;
      if (ty < 5) {
        T w = cgy[TY + ty][0] * sx[TY + ty][tx + 5];
#pragma unroll
        for (int r = 1; r < 6; ++r) w = w + cgy[TY + ty][r] * sx[TY + ty + r][tx + 5];
        sgy[TY + ty][tx] = w;
      }
    }
    __syncthreads();
    T s = cdx[tx][0] * sgx[ty][tx];
#pragma unroll
    for (int l = 1; l < 6; ++l) s = s + cdx[tx][l] * sgx[ty][tx + l];
#pragma unroll
    for (int l = 0; l < 6; ++l) s = s + cdy[ty][l] * sgy[ty + l][tx];
#pragma unroll
    for (int l = 0; l < 6; ++l) s = s + cdz[kk][l] * gzq[l];
    if (in) {
      const long long p = col + g.nxy * (long long)(wrapm(k0 + z, n3) + 3);
      out[p] = s;
      if (MODE == 1) acc[0] += (double)s * (double)d1[p];
      if (MODE == 2) {
        acc[0] += (double)d1[p] * (double)s;
        acc[1] += (double)s * (double)s;
      }
    }
    // advance the z queues to plane k+1
#pragma unroll
    for (int l = 0; l < 5; ++l) xq[l] = xq[l + 1];
    xq[5] = zf[0];
#pragma unroll
    for (int l = 0; l < P - 1; ++l) zf[l] = zf[l + 1];
    zf[P - 1] = xfar;
    if (kk + 1 < nk) {
      T v = cgz[kk + 6][0] * xq[0];
#pragma unroll
      for (int r = 1; r < 6; ++r) v = v + cgz[kk + 6][r] * xq[r];
#pragma unroll
      for (int l = 0; l < 5; ++l) gzq[l] = gzq[l + 1];
      gzq[5] = v;
    }
  }
  cp_wait<0>();
  if constexpr (MODE > 0) block_sum_store<MODE>(acc, partial);
}

template <typename T>
constexpr size_t divgrad25_smem() {
  return (size_t)4 * (TY + 10) * (TX + 10) * sizeof(T);
}

template <typename T, int MODE>
void launch_divgrad25(const Geom& g, const Coeffs<T>& c, const SolverScalars* sc, const T* x, T* out, const T* d1,
                      double* partial, cudaStream_t s) {
  constexpr size_t sm = divgrad25_smem<T>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_divgrad25<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  k_divgrad25<T, MODE><<<s25_grid(g), dim3(TX, TY), sm, s>>>(g, c, sc, x, out, d1, partial);
}

// ------------------------------------------------------------------------------------------
// damped-Jacobi sweep (INIT: start values omega*bb/diag formed on the fly)
// ------------------------------------------------------------------------------------------
template <typename T, int INIT>
__global__ void __launch_bounds__(NT, 3) k_jacobi25(Geom g, Coeffs<T> c, const SolverScalars* __restrict__ sc, T omega,
                                                 const T* __restrict__ bb, const T* __restrict__ rel,
                                                 T* __restrict__ out) {
  if (halted25(sc)) return;
  constexpr int RX = TX + 2, RY = TY + 2, TILE = RX * RY;
  constexpr int D = 6;  // planes in the ring: k-1, k, k+1 consumed, 3 more in flight
  constexpr int PER = (TILE + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*ring)[RY][RX] = reinterpret_cast<T(*)[RY][RX]>(smem_raw);                        // rel (or bb) tiles
  T(*bring)[TY][TX] = reinterpret_cast<T(*)[TY][TX]>(smem_raw + (size_t)D * TILE * sizeof(T));  // bb centres
  __shared__ T c1[TX + 2][3], c2[TY + 2][3], c3[KC + 2][3];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int n1 = g.n1, n2 = g.n2, n3 = g.n3;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * KC;
  const int i = i0 + tx + 1, j = j0 + ty + 1;
  const bool in = (i <= n1) && (j <= n2);
  const int iw = wrapm(i, n1), jw = wrapm(j, n2);
  const int nk = min(KC, n3 - k0);
  // cdg rows: c1[r] = cdg1(:, i0 + r), r = 0..TX+1 (Fortran rows i0 .. i0+TX+1), likewise y and z
  for (int e = tid; e < (TX + 2) * 3; e += NT) c1[e / 3][e % 3] = c.cdg[0][(long long)(wrapm(i0 + e / 3, n1) - 1) * 3 + e % 3];
  for (int e = tid; e < (TY + 2) * 3; e += NT) c2[e / 3][e % 3] = c.cdg[1][(long long)(wrapm(j0 + e / 3, n2) - 1) * 3 + e % 3];
  for (int e = tid; e < (KC + 2) * 3; e += NT) c3[e / 3][e % 3] = c.cdg[2][(long long)(wrapm(k0 + e / 3, n3) - 1) * 3 + e % 3];

  const T* src = INIT ? bb : rel;
  long long toff[PER];
  int tsm[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * NT;
    const int r = e / RX, q = e % RX;  // smem (r, q) <-> Fortran (i0 + q, j0 + r)
    tsm[u] = e < TILE ? e : -1;
    toff[u] = (long long)(wrapm(i0 + q, n1) + 3) + (long long)g.nx * (wrapm(j0 + r, n2) + 3);
  }
  const long long colc = (long long)(iw + 3) + (long long)g.nx * (jw + 3);
  // plane z of this block: Fortran k0 + z, z = 0 .. nk + 1
  auto issue = [&](int z) {
    const long long zo = g.nxy * (long long)(wrapm(k0 + z, n3) + 3);
    T* base = &ring[z % D][0][0];
#pragma unroll
    for (int u = 0; u < PER; ++u)
      if (tsm[u] >= 0) cp_async_el(base + tsm[u], src + toff[u] + zo);
    if (!INIT && z >= 1 && z <= nk) cp_async_el(&bring[z % D][ty][tx], bb + colc + zo);
  };
#pragma unroll
  for (int z = 0; z <= D - 2; ++z) {
    if (z <= nk + 1) issue(z);
    cp_commit();
  }
  __syncthreads();  // coefficient rows ready
  auto start = [&](T b, int ri, int rj, int rk) { return omega * b / (c1[ri][1] + c2[rj][1] + c3[rk][1]); };
  for (int kk = 0; kk < nk; ++kk) {
    const int z = kk + 1;  // output plane
    if (z + D - 2 <= nk + 1) issue(z + D - 2);
    cp_commit();
    cp_wait<D - 3>();  // planes z-1, z, z+1 have landed
    __syncthreads();
    if (in) {
      T(*pm)[RX] = ring[(z - 1) % D];
      T(*pc)[RX] = ring[z % D];
      T(*pp)[RX] = ring[(z + 1) % D];
      const T* a = c1[tx + 1];
      const T* b = c2[ty + 1];
      const T* cz = c3[kk + 1];
      T xc, xw, xe, xs, xn, xm, xp, bcen;
      if (INIT) {
        bcen = pc[ty + 1][tx + 1];
        xc = start(bcen, tx + 1, ty + 1, kk + 1);
        xw = start(pc[ty + 1][tx], tx, ty + 1, kk + 1);
        xe = start(pc[ty + 1][tx + 2], tx + 2, ty + 1, kk + 1);
        xs = start(pc[ty][tx + 1], tx + 1, ty, kk + 1);
        xn = start(pc[ty + 2][tx + 1], tx + 1, ty + 2, kk + 1);
        xm = start(pm[ty + 1][tx + 1], tx + 1, ty + 1, kk);
        xp = start(pp[ty + 1][tx + 1], tx + 1, ty + 1, kk + 2);
      } else {
        bcen = bring[z % D][ty][tx];
        xc = pc[ty + 1][tx + 1];
        xw = pc[ty + 1][tx];
        xe = pc[ty + 1][tx + 2];
        xs = pc[ty][tx + 1];
        xn = pc[ty + 2][tx + 1];
        xm = pm[ty + 1][tx + 1];
        xp = pp[ty + 1][tx + 1];
      }
      const T r = omega * (bcen - a[0] * xw - a[2] * xe - b[0] * xs - b[2] * xn - cz[0] * xm - cz[2] * xp) /
                      (a[1] + b[1] + cz[1]) +
                  (T(1) - omega) * xc;
      out[colc + g.nxy * (long long)(wrapm(k0 + z, n3) + 3)] = r;
    }
    __syncthreads();  // the slot of plane z-1 is refilled by the next iteration
  }
  cp_wait<0>();
}

template <typename T>
constexpr size_t jacobi25_smem() {
  return (size_t)6 * ((TY + 2) * (TX + 2) + TY * TX) * sizeof(T);
}

template <typename T, int INIT>
void launch_jacobi25(const Geom& g, const Coeffs<T>& c, const SolverScalars* sc, T omega, const T* bb, const T* rel,
                     T* out, cudaStream_t s) {
  constexpr size_t sm = jacobi25_smem<T>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_jacobi25<T, INIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  k_jacobi25<T, INIT><<<s25_grid(g), dim3(TX, TY), sm, s>>>(g, c, sc, omega, bb, rel, out);
}

#define INST25(T)                                                                                                    \
  template void launch_divgrad25<T, 0>(const Geom&, const Coeffs<T>&, const SolverScalars*, const T*, T*, const T*,  \
                                       double*, cudaStream_t);                                                       \
  template void launch_divgrad25<T, 1>(const Geom&, const Coeffs<T>&, const SolverScalars*, const T*, T*, const T*,  \
                                       double*, cudaStream_t);                                                       \
  template void launch_divgrad25<T, 2>(const Geom&, const Coeffs<T>&, const SolverScalars*, const T*, T*, const T*,  \
                                       double*, cudaStream_t);                                                       \
  template void launch_jacobi25<T, 0>(const Geom&, const Coeffs<T>&, const SolverScalars*, T, const T*, const T*, T*, \
                                      cudaStream_t);                                                                 \
  template void launch_jacobi25<T, 1>(const Geom&, const Coeffs<T>&, const SolverScalars*, T, const T*, const T*, T*, \
                                      cudaStream_t);
INST25(double)
INST25(float)
#undef INST25

}  // namespace impact
