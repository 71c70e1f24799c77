// engine.cu -- batched pressure Poisson engine: BiCGstab_orig with the multigrid V-cycle (or
// damped-Jacobi sweeps) as preconditioner, every kernel over a job list of cases / levels.
//
//   BiCGstab_orig           mod_solvers.f90:1509-1935   k_kr_* and the scalar finalisation
//   product_div_grad        mod_laplace.f90:38-197      k_kr_ax / k_kr_ax32 (collapsed 11-point form, z-march)
//   multigridV              mod_solvers.f90:456-585     schedule built in Engine::build
//   relaxation_div_grad     mod_laplace.f90:339-613     k_lv_smooth
//   product_div_grad_relax  mod_laplace.f90:216-327     k_lv_resid (fused with the subtraction)
//   restrict                mod_solvers.f90:588-808     k_lv_restrict
//   interpolate             mod_solvers.f90:955-1141    k_lv_prolong
//   product_scalar/get_norms mod_solvers.f90:2319-2470  per-tile partials + fixed-order k_efin
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>

#include "engine.cuh"
#include "prof.cuh"

namespace impact {

namespace {

enum EFin { EFIN_RAW = 0, EFIN_INIT, EFIN_ALPHA, EFIN_OMEGA, EFIN_NORMS, EFIN_RESET, EFIN_INIT_EXT };

__device__ __forceinline__ bool e_halted(const SolverScalars* sc) { return sc->done | sc->status; }

// job owning tile b: the largest q with ts[q] <= b (jobs without tiles are skipped over)
__device__ __forceinline__ int find_job(const int* __restrict__ ts, int nj, int b) {
  int lo = 0, hi = nj - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(ts + mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// tile t of grid g: this thread's column (i, j) (the first of vw consecutive columns) and the
// plane range k0..k1
__device__ __forceinline__ void tile_at(const Geom& g, int kc, int t, int& i, int& j, int& k0, int& k1, int vw = 1) {
  const int tx = (g.n1 + ETX * vw - 1) / (ETX * vw), ty = (g.n2 + ETY - 1) / ETY;
  const int a = t % tx;
  const int r = t / tx;
  const int c = r / ty;
  i = (a * ETX + threadIdx.x) * vw + 1;
  j = (r - c * ty) * ETY + threadIdx.y + 1;
  k0 = c * kc + 1;
  k1 = min(g.n3, k0 + kc - 1);
}

__device__ __forceinline__ double e_wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double e_wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// elements per block of loads: 4 planes in FP32, 2 in FP64
template <typename T>
struct Ublk {
  static constexpr int U = sizeof(T) == 4 ? 4 : 2;
};

// 16-byte vectors: 4 floats or 2 doubles per thread in the vectorised level kernels
template <typename T>
struct VecT;
template <>
struct VecT<float> {
  static constexpr int W = 4;
};
template <>
struct VecT<double> {
  static constexpr int W = 2;
};
template <typename T>
__device__ __forceinline__ void vload(const T* p, T (&o)[VecT<T>::W]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  } else {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = v.x;
    o[1] = v.y;
  }
}
template <typename T>
__device__ __forceinline__ void vstore(T* p, const T (&o)[VecT<T>::W]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  }
}

// NQ block-wide partials of one tile into out[0..NQ-1]; bit q of MAXMASK: max instead of sum
template <int NQ, int MAXMASK, int NTH = ENT>
__device__ __forceinline__ void tile_partials(double (&v)[NQ], double* __restrict__ out) {
  __shared__ double sh[NQ][NTH / 32];
  const int tid = threadIdx.x + ETX * threadIdx.y;
  const int lane = tid & 31, w = tid >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = ((MAXMASK >> q) & 1) ? e_wmax(v[q]) : e_wsum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[q][w] = v[q];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < NTH / 32 ? sh[q][lane] : 0.0;
      x = ((MAXMASK >> q) & 1) ? e_wmax(x) : e_wsum(x);
      if (lane == 0) out[q] = x;
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------------
// scalar finalisation: one block per job, the job's tile partials in tile order
// ------------------------------------------------------------------------------------------
__device__ void e_scalar_update(int mode, const double* q, SolverScalars* sc) {
  switch (mode) {
    case EFIN_INIT:      // q = [max|r|, sum r^2, r.rh, sum b^2]
    case EFIN_INIT_EXT:  // r = rh = b (from 0): q = [max|r|, -, -, sum r^2] of the caller's kernel
      sc->norm_inf = q[0];
      sc->norm_two_sq = mode == EFIN_INIT ? q[1] : q[3];
      sc->rhr_next = mode == EFIN_INIT ? q[2] : q[3];
      sc->b_two_sq = q[3];
      sc->rhr = 0.0;
      sc->alpha = sc->omega = sc->beta = 0.0;
      sc->it = 0;
      sc->status = 0;
      sc->done = (q[0] == 0.0) ? 1 : 0;  // the reference iterates at least once unless r == 0
      if (sc->max_it <= 0) sc->done = 1;
      if (!isfinite(q[0]) || !isfinite(sc->norm_two_sq)) sc->status = 3;
      break;
    case EFIN_ALPHA:
      sc->rhAp = q[0];
      if (q[0] == 0.0)
        sc->status = 2;
      else
        sc->alpha = sc->rhr / q[0];
      break;
    case EFIN_OMEGA:
      sc->rAr = q[0];
      sc->ArAr = q[1];
      if (q[1] == 0.0)
        sc->status = 2;
      else
        sc->omega = q[0] / q[1];
      break;
    case EFIN_NORMS: {  // after an x update
      sc->phi_zero = 0;
      sc->norm_inf = q[0];
      sc->norm_two_sq = q[1];
      sc->rhr_next = q[2];
      if (!isfinite(q[0]) || !isfinite(q[1])) {
        sc->status = 3;
        break;
      }
      const bool conv = (sc->tol_abs_inf > 0.0 && q[0] < sc->tol_abs_inf) ||
                        (sc->tol_rel > 0.0 && sqrt(q[1]) <= sc->tol_rel * sqrt(sc->b_two_sq));
      if (conv) {
        sc->done = 1;
      } else if (sc->it >= sc->max_it) {
        sc->done = 1;
        sc->status = 1;
      }
      break;
    }
    case EFIN_RESET:  // new shadow residual rh = rr: rhr = rr.rr, redo the iteration start
      sc->rhr_next = q[0];
      sc->status = 0;
      sc->it -= 1;
      sc->rhr = sc->rhr_prev;
      break;
    default:
      break;
  }
}

__global__ void __launch_bounds__(256) k_efin(const int* __restrict__ ts, const double* __restrict__ partial, int nq,
                                              int maxmask, int mode, SolverScalars* __restrict__ scal,
                                              double* __restrict__ raw) {
  const int q = blockIdx.x;
  SolverScalars* sc = scal ? scal + q : nullptr;
  if (sc) {
    if (mode == EFIN_RESET) {
      if (sc->status != 4) return;
    } else if (mode == EFIN_INIT || mode == EFIN_INIT_EXT) {
      if (sc->done) return;
    } else if (mode != EFIN_RAW) {
      if (e_halted(sc)) return;
    }
  }
  const int t0 = ts[q], t1 = ts[q + 1];
  __shared__ double sh[4][8];
  __shared__ double tot[4];
  for (int c = 0; c < nq; ++c) {
    const bool mx = (maxmask >> c) & 1;
    double v = 0.0;
    for (int t = t0 + threadIdx.x; t < t1; t += 256) {
      const double x = partial[(long long)t * 4 + c];
      v = mx ? fmax(v, x) : v + x;
    }
    v = mx ? e_wmax(v) : e_wsum(v);
    if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int c = 0; c < nq; ++c) {
      const bool mx = (maxmask >> c) & 1;
      double x = threadIdx.x < 8 ? sh[c][threadIdx.x] : 0.0;
      x = mx ? e_wmax(x) : e_wsum(x);
      if (threadIdx.x == 0) tot[c] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < nq; ++c) r[c] = tot[c];
    if (mode == EFIN_RAW) {
      for (int c = 0; c < 4; ++c) raw[q * 4 + c] = r[c];
    } else {
      e_scalar_update(mode, r, sc);
    }
  }
}

// start of an iteration (mod_solvers.f90:~1600-1680): rhr, breakdown tests, beta, omega
__global__ void k_ebegin(SolverScalars* __restrict__ scal, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  SolverScalars* sc = scal + q;
  if (e_halted(sc)) return;
  sc->it += 1;
  sc->rhr_prev = sc->rhr;
  sc->rhr = sc->rhr_next;
  if (sc->rhr == 0.0) {  // shadow residual orthogonal to r: the host resets rh = rr
    sc->status = 4;
    return;
  }
  if (sc->it >= 2) {
    if (sc->omega == 0.0 || sc->rhr_prev == 0.0) {
      sc->status = 2;
      return;
    }
    sc->beta = (sc->alpha / sc->omega) * (sc->rhr / sc->rhr_prev);
    sc->omega = -sc->beta * sc->omega;
  }
}

// ------------------------------------------------------------------------------------------
// BiCGstab vector kernels over the Krylov job list
// ------------------------------------------------------------------------------------------
// initial residual: rr = bb - rr (rr = A phi), or rr = bb from phi = 0 (zero_phi 1: phi = 0
// written; 2: not written, the first x update starts from 0, SolverScalars::phi_zero); rh = rr
// partials [max|rr|, sum rr^2, rr.rh, sum bb^2]
template <typename T>
__global__ void __launch_bounds__(ENT) k_kr_init(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                 int nj, int ntiles, int zero_phi, double* __restrict__ partial) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    if (J.sc->done) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (i <= g.n1 && j <= g.n2) {
      const T* bb = J.bb;  // rh may share bb's buffer: neither is restrict-qualified
      T* __restrict__ phi = J.phi;
      T* __restrict__ rr = J.rr;
      T* rh = J.rh;
      const long long nxy = g.nxy;
      long long p = off(g, i, j, k0);
      // from phi = 0 with rh sharing bb's buffer (the mixed solve's inner solve) rh already holds r
      const bool write_rh = !(zero_phi && rh == bb);
      auto point = [&](long long q, T bv, T a) {
        T r;
        if (zero_phi) {
          if (zero_phi == 1) phi[q] = T(0);
          r = bv;
        } else {
          r = bv - a;
        }
        rr[q] = r;
        if (write_rh) rh[q] = r;
        const double rd = (double)r, bd = (double)bv;
        v[0] = fmax(v[0], fabs(rd));
        v[1] += rd * rd;
        v[2] += rd * rd;
        v[3] += bd * bd;
      };
      // blocks of U planes: all loads of a block are issued before its stores
      constexpr int U = 2 * Ublk<T>::U;
      int k = k0;
      for (; k + U - 1 <= k1; k += U, p += U * nxy) {
        T bv[U], a[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          bv[u] = bb[p + u * nxy];
          a[u] = zero_phi ? T(0) : rr[p + u * nxy];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) point(p + u * nxy, bv[u], a[u]);
      }
      for (; k <= k1; ++k, p += nxy) point(p, bb[p], zero_phi ? T(0) : rr[p]);
    }
    tile_partials<4, 1>(v, partial + (long long)b * 4);
  }
}

// pp = rr (first iteration; nothing when the caller wrote pp = r0, SolverScalars::rr_in_rh) or
// pp = rr + beta pp + omega Ap (omega already holds -beta omega)
template <typename T>
__global__ void __launch_bounds__(ENT) k_kr_p(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts, int nj,
                                              int ntiles) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (e_halted(sc) || (sc->it == 1 && sc->rr_in_rh)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    if (i > g.n1 || j > g.n2) continue;
    const T* __restrict__ rr = J.rr;
    const T* __restrict__ Ap = J.Ap;
    T* __restrict__ pp = J.pp;
    constexpr int U = 2 * Ublk<T>::U;
    const long long nxy = g.nxy;
    long long p = off(g, i, j, k0);
    int k = k0;
    if (sc->it == 1) {
      for (; k + U - 1 <= k1; k += U, p += U * nxy) {
        T r[U];
#pragma unroll
        for (int u = 0; u < U; ++u) r[u] = rr[p + u * nxy];
#pragma unroll
        for (int u = 0; u < U; ++u) pp[p + u * nxy] = r[u];
      }
      for (; k <= k1; ++k, p += nxy) pp[p] = rr[p];
    } else {
      const T be = (T)sc->beta, om = (T)sc->omega;
      for (; k + U - 1 <= k1; k += U, p += U * nxy) {
        T r[U], q0[U], a[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          r[u] = rr[p + u * nxy];
          q0[u] = pp[p + u * nxy];
          a[u] = Ap[p + u * nxy];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) pp[p + u * nxy] = r[u] + be * q0[u] + om * a[u];
      }
      for (; k <= k1; ++k, p += nxy) pp[p] = rr[p] + be * pp[p] + om * Ap[p];
    }
  }
}

// rr = rr - alpha Ap (in the first iteration of a solve whose caller left rr unwritten:
// rr = rh - alpha Ap)
template <typename T>
__global__ void __launch_bounds__(ENT) k_kr_r(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts, int nj,
                                              int ntiles) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (e_halted(sc)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    if (i > g.n1 || j > g.n2) continue;
    const T* __restrict__ Ap = J.Ap;
    const T* rs = (sc->it == 1 && sc->rr_in_rh) ? J.rh : J.rr;  // rr itself, or rh (see above)
    T* rr = J.rr;
    const T al = (T)sc->alpha;
    constexpr int U = 2 * Ublk<T>::U;
    const long long nxy = g.nxy;
    long long p = off(g, i, j, k0);
    int k = k0;
    for (; k + U - 1 <= k1; k += U, p += U * nxy) {
      T r[U], a[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        r[u] = rs[p + u * nxy];
        a[u] = Ap[p + u * nxy];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) rr[p + u * nxy] = r[u] - al * a[u];
    }
    for (; k <= k1; ++k, p += nxy) rr[p] = rs[p] - al * Ap[p];
  }
}

// phi += omega z2 + alpha z1 ; rr -= omega Ar ; partials [max|rr|, sum rr^2, rr.rh]
template <typename T>
__global__ void __launch_bounds__(ENT) k_kr_x(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts, int nj,
                                              int ntiles, double* __restrict__ partial) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (e_halted(sc)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    double v[3] = {0.0, 0.0, 0.0};
    if (i <= g.n1 && j <= g.n2) {
      const T* __restrict__ z1 = J.z1;
      const T* __restrict__ z2 = J.z2;
      const T* __restrict__ Ar = J.Ar;
      const T* __restrict__ rh = J.rh;
      T* __restrict__ phi = J.phi;
      T* __restrict__ rr = J.rr;
      const T om = (T)sc->omega, al = (T)sc->alpha;
      const bool pz = sc->phi_zero != 0;  // the first update of a solve started from 0 without phi = 0
      constexpr int U = Ublk<T>::U;
      const long long nxy = g.nxy;
      long long p = off(g, i, j, k0);
      auto point = [&](long long q, T ph, T a2, T a1, T r0, T ar, T h) {
        // without a preconditioner z2 aliases rr: it was read before rr is overwritten
        phi[q] = ph + om * a2 + al * a1;
        const T r = r0 - om * ar;
        rr[q] = r;
        const double rd = (double)r;
        v[0] = fmax(v[0], fabs(rd));
        v[1] += rd * rd;
        v[2] += rd * (double)h;
      };
      int k = k0;
      for (; k + U - 1 <= k1; k += U, p += U * nxy) {
        T ph[U], a2[U], a1[U], r0[U], ar[U], h[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const long long q = p + u * nxy;
          ph[u] = pz ? T(0) : phi[q];
          a2[u] = z2[q];
          a1[u] = z1[q];
          r0[u] = rr[q];
          ar[u] = Ar[q];
          h[u] = rh[q];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) point(p + u * nxy, ph[u], a2[u], a1[u], r0[u], ar[u], h[u]);
      }
      for (; k <= k1; ++k, p += nxy) point(p, pz ? T(0) : phi[p], z2[p], z1[p], rr[p], Ar[p], rh[p]);
    }
    tile_partials<3, 1>(v, partial + (long long)b * 4);
  }
}

// rh = rr for the cases whose shadow residual was lost (status 4); partial sum rr.rr
template <typename T>
__global__ void __launch_bounds__(ENT) k_kr_reset(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                  int nj, int ntiles, double* __restrict__ partial) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    if (J.sc->status != 4) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    double v[1] = {0.0};
    if (i <= g.n1 && j <= g.n2) {
      // in the first iteration of a solve whose caller left rr unwritten, rh already is rr
      const bool keep = J.sc->it == 1 && J.sc->rr_in_rh;
      long long p = off(g, i, j, k0);
      for (int k = k0; k <= k1; ++k, p += g.nxy) {
        const T r = keep ? J.rh[p] : J.rr[p];
        if (!keep) J.rh[p] = r;
        v[0] += (double)r * (double)r;
      }
    }
    tile_partials<1, 0>(v, partial + (long long)b * 4);
  }
}

// asynchronous global -> shared copy of one element (kept in L1 as well), and its group control
template <typename T>
__device__ __forceinline__ void cp_async1(T* smem, const T* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// 16 bytes (both addresses 16-byte aligned), L2 only
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A x = sum_m D_m G_m x with the two 6-point stencils of each axis collapsed into one 11-point
// stencil W_m (weights formed once on the host in FP64).  A block of 32 x 4 threads owns one
// 32 x 8-column tile over kc planes; each thread computes the two adjacent rows ya = 2 ty and
// ya + 1 of its column, so that the 12 staged rows ya-5 .. ya+6 serve both y stencils.  Each
// plane of the tile with its 5-wide x/y halo (42 x 18 elements, periodic images), and the
// inner-product partner of the plane, are staged by cp.async into a ring of R shared-memory slots
// R-1 planes ahead of their use.  x and y neighbours come from the ring; the z values k-5 .. k+5
// of the two points stay in register windows, each step adding plane k+5 from the ring.  The y
// weights of the two rows and, on uniform z, the z weights are registers in FP32 and
// warp-broadcast shared-memory reads in FP64.
//   MODE 0: rr = A phi                 (initial residual)
//   MODE 1: Ap = A z1, partial rh.Ap   (alpha)
//   MODE 2: Ar = A z2, partials Ar.rr, Ar.Ar (omega)
//   MODE 3: FP64 only: r32 = (float)(bb - A phi), partials max|r|, sum r^2, sum bb^2 (the outer
//           residual of the mixed-precision solve and the right-hand side of its inner solve)
// The FP32 lists run k_kr_ax32 below (same operator and operation order per point).
constexpr int AXTY = ETY / 2, AXNT = ETX * AXTY;  // 32 x 4 threads, two rows each
constexpr int AX_TW = ETX + 10, AX_TH = ETY + 10, AX_TE = AX_TW * AX_TH;
constexpr int AX_PER = (AX_TE + AXNT - 1) / AXNT;  // staged elements per thread and plane
// ring depth: planes k .. k+5 are read at plane k, the rest of the ring is in flight
template <typename T>
struct AxRing {
  static constexpr int R = sizeof(T) == 4 ? 16 : 8;  // a power of two: slots by masking
};
template <typename T>
constexpr size_t ax_smem_bytes() {
  constexpr int R = AxRing<T>::R;
  return sizeof(T) * ((size_t)R * AX_TE + (size_t)R * ENT + (size_t)KC_MAX * AXW + ETY * AXW + AXW * ETX);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(AXNT, 2) k_kr_ax(const KrylovJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                   int nj, int ntiles, double* __restrict__ partial) {
  constexpr int AX_R = AxRing<T>::R;
  constexpr bool REG = sizeof(T) == 4;  // y and z weights in registers
  extern __shared__ __align__(16) unsigned char ax_smem[];
  T(*ring)[AX_TH][AX_TW] = reinterpret_cast<T(*)[AX_TH][AX_TW]>(ax_smem);
  T(*dring)[ENT] = reinterpret_cast<T(*)[ENT]>(ax_smem + sizeof(T) * AX_R * AX_TE);
  T(*wzs)[AXW] = reinterpret_cast<T(*)[AXW]>(ax_smem + sizeof(T) * (AX_R * AX_TE + AX_R * ENT));
  T(*wys)[AXW] = reinterpret_cast<T(*)[AXW]>(ax_smem + sizeof(T) * (AX_R * AX_TE + AX_R * ENT + KC_MAX * AXW));
  T(*wxs)[ETX] =
      reinterpret_cast<T(*)[ETX]>(ax_smem + sizeof(T) * (AX_R * AX_TE + AX_R * ENT + KC_MAX * AXW + ETY * AXW));
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + ETX * ty;
  const int ya = 2 * ty;  // tile rows ya and ya + 1 of this thread
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<T>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (J.vec || (MODE == 0 ? (sc->done != 0) : e_halted(sc))) continue;  // vector jobs: k_kr_ax64v
    const Geom g = J.g;
    const int ntx = (g.n1 + ETX - 1) / ETX, nty = (g.n2 + ETY - 1) / ETY;
    const int t0 = b - ts[q];
    const int ta = t0 % ntx, tr = t0 / ntx, tc = tr / nty;
    const int i0 = ta * ETX + 1, j0 = (tr - tc * nty) * ETY + 1;
    const int k0 = tc * J.kc + 1, k1 = min(g.n3, k0 + J.kc - 1);
    const int i = i0 + tx;
    const bool in0 = i <= g.n1 && j0 + ya <= g.n2, in1 = i <= g.n1 && j0 + ya + 1 <= g.n2;
    const T* __restrict__ x = (MODE == 0 || MODE == 3) ? J.phi : (MODE == 1 ? J.z1 : J.z2);
    T* __restrict__ out = MODE == 0 ? J.rr : (MODE == 1 ? J.Ap : J.Ar);
    const T* __restrict__ d1 = MODE == 1 ? J.rh : (MODE == 3 ? J.bb : J.rr);
    const long long nxy = g.nxy;
    // weights of the tile: z rows of its planes, y rows of its 8 rows, x rows of its 32 columns
    const int nzw = (k1 - k0 + 1) * AXW;
    for (int t = tid; t < nzw; t += AXNT) wzs[t / AXW][t % AXW] = J.W[2][(k0 - 1) * AXW + t];
    for (int t = tid; t < ETY * AXW; t += AXNT) {
      const int jj = j0 + t / AXW;
      wys[t / AXW][t % AXW] = jj <= g.n2 ? J.W[1][(jj - 1) * AXW + t % AXW] : T(0);
    }
    for (int t = tid; t < ETX * AXW; t += AXNT) {
      const int ii = i0 + t / AXW;
      wxs[t % AXW][t / AXW] = ii <= g.n1 ? J.W[0][(ii - 1) * AXW + t % AXW] : T(0);
    }
    // in-plane offsets of this thread's staged elements (periodic images of the halo)
    int eo[AX_PER];
#pragma unroll
    for (int e = 0; e < AX_PER; ++e) {
      const int t = tid + e * AXNT;
      const int r = t / AX_TW, c = t % AX_TW;
      const int gi = wrapi(i0 - 5 + c, g.n1), gj = wrapi(j0 - 5 + r, g.n2);
      eo[e] = t < AX_TE ? (gi + 3) + g.nx * (gj + 3) : -1;
    }
    // the two points' in-plane offsets (an idle point reads a valid column and stores nothing)
    const int own0 = (in0 ? i + 3 : 4) + g.nx * ((in0 ? j0 + ya : 1) + 3);
    const int own1 = (in1 ? i + 3 : 4) + g.nx * ((in1 ? j0 + ya + 1 : 1) + 3);
    const int pa = ya * ETX + tx, pb = pa + ETX;  // the points' slots in the partner ring
    auto zoff = [&](int k) -> long long {  // plane k (periodic) + 3 ghost planes
      return (long long)((k < 1 ? k + g.n3 : (k > g.n3 ? k - g.n3 : k)) + 3) * nxy;
    };
    // plane kk (k0-5 <= kk <= k1+5) into its ring slot; the partner only for kk in k0..k1
    auto stage = [&](int kk) {
      if (kk <= k1 + 5) {
        const int sl = (kk - k0) & (AX_R - 1);
        T* slot = &ring[sl][0][0];
        const T* src = x + zoff(kk);
#pragma unroll
        for (int e = 0; e < AX_PER; ++e)
          if (eo[e] >= 0) cp_async1(slot + tid + e * AXNT, src + eo[e]);
        if (MODE != 0 && kk >= k0 && kk <= k1) {
          if (in0) cp_async1(&dring[sl][pa], d1 + zoff(kk) + own0);
          if (in1) cp_async1(&dring[sl][pb], d1 + zoff(kk) + own1);
        }
      }
      cp_commit();
    };
    __syncthreads();  // weights visible
    const bool zu = J.zuni != 0;
    T wx[AXW], wya[AXW], wyb[AXW], wzr[AXW];
#pragma unroll
    for (int l = 0; l < AXW; ++l) {
      wx[l] = wxs[l][tx];
      wya[l] = REG ? wys[ya][l] : T(0);
      wyb[l] = REG ? wys[ya + 1][l] : T(0);
      wzr[l] = REG ? wzs[0][l] : T(0);
    }
    // z windows: planes k-5 .. k+5 of the two points; the past ones now, the rest from the ring
    T za[AXW], zb[AXW];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      za[l] = x[zoff(k0 - 5 + l) + own0];
      zb[l] = x[zoff(k0 - 5 + l) + own1];
    }
#pragma unroll
    for (int l = 5; l < AXW; ++l) za[l] = zb[l] = T(0);
#pragma unroll
    for (int l = 0; l < AX_R - 1; ++l) stage(k0 + l);
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    const long long ob0 = (long long)(k0 + 3) * nxy + own0, ob1 = (long long)(k0 + 3) * nxy + own1;
    auto walk = [&](auto zreg) {
      constexpr bool ZR = decltype(zreg)::value;
      for (int k = k0; k <= k1; ++k) {
        cp_wait<AX_R - 7>();  // this thread's copies of planes k .. k+5 have landed
        __syncthreads();      // everybody's have; the slot of plane k-1 is free again
        stage(k + AX_R - 1);
        const int sl = (k - k0) & (AX_R - 1);
        const T (*sp)[AX_TW] = ring[sl];
        if (k == k0) {  // the windows' planes k0 .. k0+5
#pragma unroll
          for (int l = 0; l < 6; ++l) {
            za[5 + l] = ring[(sl + l) & (AX_R - 1)][ya + 5][tx + 5];
            zb[5 + l] = ring[(sl + l) & (AX_R - 1)][ya + 6][tx + 5];
          }
        } else {
#pragma unroll
          for (int l = 0; l < AXW - 1; ++l) {
            za[l] = za[l + 1];
            zb[l] = zb[l + 1];
          }
          za[AXW - 1] = ring[(sl + 5) & (AX_R - 1)][ya + 5][tx + 5];
          zb[AXW - 1] = ring[(sl + 5) & (AX_R - 1)][ya + 6][tx + 5];
        }
        const T ca = za[5], cb = zb[5];
        // x stencils of both rows
        T axa = wx[0] * sp[ya + 5][tx], axb = wx[0] * sp[ya + 6][tx];
#pragma unroll
        for (int l = 1; l < AXW; ++l) {
          axa += wx[l] * (l == 5 ? ca : sp[ya + 5][tx + l]);
          axb += wx[l] * (l == 5 ? cb : sp[ya + 6][tx + l]);
        }
        // y stencils: staged rows ya .. ya+11 (ya+5, ya+6 are the centres) serve both points
        T yv[AXW + 1];
#pragma unroll
        for (int r = 0; r < AXW + 1; ++r) yv[r] = r == 5 ? ca : (r == 6 ? cb : sp[ya + r][tx + 5]);
        T aya = (REG ? wya[0] : wys[ya][0]) * yv[0], ayb = (REG ? wyb[0] : wys[ya + 1][0]) * yv[1];
#pragma unroll
        for (int l = 1; l < AXW; ++l) {
          aya += (REG ? wya[l] : wys[ya][l]) * yv[l];
          ayb += (REG ? wyb[l] : wys[ya + 1][l]) * yv[l + 1];
        }
        // z stencils from the windows
        const T* wz = wzs[k - k0];
        T aza = (ZR ? wzr[0] : wz[0]) * za[0], azb = (ZR ? wzr[0] : wz[0]) * zb[0];
#pragma unroll
        for (int l = 1; l < AXW; ++l) {
          aza += (ZR ? wzr[l] : wz[l]) * za[l];
          azb += (ZR ? wzr[l] : wz[l]) * zb[l];
        }
        const T ra = axa + aya + aza, rb = axb + ayb + azb;
        const long long dz = (long long)(k - k0) * nxy;
        if (MODE == 3) {
          if (in0) {
            const double bv = (double)dring[sl][pa];
            const double res = bv - (double)ra;
            const float rf = (float)res;
            J.r32[ob0 + dz] = rf;
            if (J.r32p) J.r32p[ob0 + dz] = rf;
            v0 = fmax(v0, fabs(res));
            v1 += res * res;
            v2 += bv * bv;
            v3 += (double)rf * (double)rf;
          }
          if (in1) {
            const double bv = (double)dring[sl][pb];
            const double res = bv - (double)rb;
            const float rf = (float)res;
            J.r32[ob1 + dz] = rf;
            if (J.r32p) J.r32p[ob1 + dz] = rf;
            v3 += (double)rf * (double)rf;
            v0 = fmax(v0, fabs(res));
            v1 += res * res;
            v2 += bv * bv;
          }
        } else {
          if (in0) out[ob0 + dz] = ra;
          if (in1) out[ob1 + dz] = rb;
          if (MODE == 1) {
            if (in0) v0 += (double)ra * (double)dring[sl][pa];
            if (in1) v0 += (double)rb * (double)dring[sl][pb];
          }
          if (MODE == 2) {
            if (in0) {
              v0 += (double)ra * (double)dring[sl][pa];
              v1 += (double)ra * (double)ra;
            }
            if (in1) {
              v0 += (double)rb * (double)dring[sl][pb];
              v1 += (double)rb * (double)rb;
            }
          }
        }
      }
    };
    if (REG && zu)
      walk(std::true_type{});
    else
      walk(std::false_type{});
    cp_wait<0>();
    if (MODE == 1) {
      double v[1] = {v0};
      tile_partials<1, 0, AXNT>(v, partial + (long long)b * 4);
    } else if (MODE == 2) {
      double v[2] = {v0, v1};
      tile_partials<2, 0, AXNT>(v, partial + (long long)b * 4);
    } else if (MODE == 3) {
      double v[4] = {v0, v1, v2, v3};
      tile_partials<4, 1, AXNT>(v, partial + (long long)b * 4);
    } else {
      __syncthreads();  // the ring and the weights are rewritten by the next tile
    }
  }
}

// ------------------------------------------------------------------------------------------
// multigrid kernels over level job lists
// ------------------------------------------------------------------------------------------
// The point operations of the damped-Jacobi sweep, the init sweep and the residual of the
// compact operator, with every rounding spelled out (fused multiply-adds and products by
// intrinsic, so the compiler contracts nothing on its own), so that the one-sweep kernels and
// the fused smoothing kernels produce the same bits.
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mulT(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulT(double a, double b) { return __dmul_rn(a, b); }
// ------------------------------------------------------------------------------------------
// The FP32 operator of the Krylov list (the inner solve of the mixed-precision Poisson solve):
// the same collapsed 11-point product_div_grad and the same operation order per point as
// k_kr_ax, with the plane ring staged in 16-byte chunks and the z march taken AXB planes at a
// time.
//
// Staged plane: AXA_H = 18 rows (y halo 5) of AXA_W = 48 columns whose first column is the
// 16-byte aligned element 8 left of the tile (the 5-wide x halo rounded out to whole chunks).
// Each thread stages up to AXA_PER chunks of a plane; a chunk is one 16-byte cp.async when its
// needed elements are interior points of the row and the field's rows are 16-byte aligned
// (nx a multiple of 4), else its needed elements one by one from their periodic images.
// Chunks no point of the tile reads are not staged.
//
// z march: the ring holds AXA_R = AXB * AXA_G planes in AXA_G groups of AXB planes, one
// cp.async group each.  A step outputs planes t .. t+AXB-1 of the tile; it needs planes up to
// t+AXB+4 in the ring, waits for them with one barrier, refills the group freed by the previous
// step, adds planes t+5 .. t+AXB+4 to the register windows (z values k-5 .. k+AXB+4 of the two
// points of the thread) and moves the windows on by AXB after the step, so a window value is
// moved once per AXB planes.  The inner-product partner of the step's points is loaded from
// global memory one step ahead.
constexpr int AXB = 4;                                     // planes per step
constexpr int AXA_G = 5;                                   // groups of AXB planes in the ring
constexpr int AXA_R = AXB * AXA_G;                         // ring slots
constexpr int AXA_V = 4;                                   // floats per 16-byte chunk
constexpr int AXA_HX = 8;                                  // staged columns left of the tile
constexpr int AXA_W = 48;                                  // staged row: 8 + 32 + 5, whole chunks
constexpr int AXA_H = ETY + 10;                            // staged rows
constexpr int AXA_CR = AXA_W / AXA_V;                      // chunks per row
constexpr int AXA_NCH = AXA_CR * AXA_H;                    // chunks per plane
constexpr int AXA_PER = (AXA_NCH + AXNT - 1) / AXNT;       // chunks per thread and plane
constexpr int AXA_PLANE = AXA_W * AXA_H;                   // floats per slot
constexpr int AXA_ZW = AXB + 10;                           // z window per point
static_assert((AXA_PLANE * 4) % 16 == 0, "slots must keep 16-byte alignment");
static_assert(AXB >= 1 && AXB <= 5, "group bookkeeping below assumes 4 / AXB <= 4");
constexpr int AXA_NEED = 1 + 4 / AXB;                      // groups beyond the step's own that it reads
constexpr int AXA_WAIT = AXA_G - 2 - AXA_NEED;             // groups left in flight at the wait
static_assert(AXA_WAIT >= 0, "ring too shallow for the step");

constexpr size_t axa_smem_bytes() {
  return sizeof(float) * ((size_t)AXA_R * AXA_PLANE + (size_t)KC_MAX * AXW + ETY * AXW + AXW * ETX);
}

template <int MODE>
__global__ void __launch_bounds__(AXNT, 3) k_kr_ax32(const KrylovJob<float>* __restrict__ jobs,
                                                     const int* __restrict__ ts, int nj, int ntiles,
                                                     double* __restrict__ partial) {
  static_assert(MODE >= 0 && MODE <= 2, "FP32 operator modes: 0 residual, 1 alpha, 2 omega");
  extern __shared__ __align__(16) unsigned char ax_smem[];
  float* ring = reinterpret_cast<float*>(ax_smem);
  float(*wzs)[AXW] = reinterpret_cast<float(*)[AXW]>(ax_smem + sizeof(float) * AXA_R * AXA_PLANE);
  float(*wys)[AXW] = reinterpret_cast<float(*)[AXW]>(ax_smem + sizeof(float) * (AXA_R * AXA_PLANE + KC_MAX * AXW));
  float(*wxs)[ETX] =
      reinterpret_cast<float(*)[ETX]>(ax_smem + sizeof(float) * (AXA_R * AXA_PLANE + KC_MAX * AXW + ETY * AXW));
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + ETX * ty;
  const int ya = 2 * ty;
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<float>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (J.vec || (MODE == 0 ? (sc->done != 0) : e_halted(sc))) continue;  // vector jobs: k_kr_ax32v
    const Geom g = J.g;
    const int ntx = (g.n1 + ETX - 1) / ETX, nty = (g.n2 + ETY - 1) / ETY;
    const int t0 = b - ts[q];
    const int ta = t0 % ntx, tr = t0 / ntx, tc = tr / nty;
    const int i0 = ta * ETX + 1, j0 = (tr - tc * nty) * ETY + 1;
    const int k0 = tc * J.kc + 1, k1 = min(g.n3, k0 + J.kc - 1);
    const int nk = k1 - k0 + 1;
    const int i = i0 + tx;
    const bool in0 = i <= g.n1 && j0 + ya <= g.n2, in1 = i <= g.n1 && j0 + ya + 1 <= g.n2;
    const float* __restrict__ x = MODE == 0 ? J.phi : (MODE == 1 ? J.z1 : J.z2);
    float* __restrict__ out = MODE == 0 ? J.rr : (MODE == 1 ? J.Ap : J.Ar);
    const float* __restrict__ d1 = MODE == 1 ? J.rh : J.rr;
    const long long nxy = g.nxy;
    const int nzw = nk * AXW;
    for (int t = tid; t < nzw; t += AXNT) wzs[t / AXW][t % AXW] = J.W[2][(k0 - 1) * AXW + t];
    for (int t = tid; t < ETY * AXW; t += AXNT) {
      const int jj = j0 + t / AXW;
      wys[t / AXW][t % AXW] = jj <= g.n2 ? J.W[1][(jj - 1) * AXW + t % AXW] : 0.f;
    }
    for (int t = tid; t < ETX * AXW; t += AXNT) {
      const int ii = i0 + t / AXW;
      wxs[t % AXW][t / AXW] = ii <= g.n1 ? J.W[0][(ii - 1) * AXW + t % AXW] : 0.f;
    }
    // this thread's chunks: in-plane source offsets (go[e][0] alone for a 16-byte chunk, one per
    // element otherwise, -1 where nothing is staged); columns and rows that a point of the tile
    // reads: i0-5 .. min(i0+31, n1)+5 and j0-5 .. min(j0+7, n2)+5
    const int ilast = min(i0 + ETX - 1, g.n1) + 5, jlast = min(j0 + ETY - 1, g.n2) + 5;
    const bool rows16 = (g.nx & (AXA_V - 1)) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
    int go[AXA_PER][AXA_V];
    unsigned vec = 0;
#pragma unroll
    for (int e = 0; e < AXA_PER; ++e) {
      const int cq = tid + e * AXNT;
      const int r = cq / AXA_CR, c0 = (cq % AXA_CR) * AXA_V;
      const int jj = j0 - 5 + r;
      const bool row_ok = cq < AXA_NCH && jj <= jlast;
      const int rowoff = g.nx * (wrapi(row_ok ? jj : 1, g.n2) + 3);
      bool v16 = row_ok && rows16, any = false;
#pragma unroll
      for (int v = 0; v < AXA_V; ++v) {
        const int ii = i0 - AXA_HX + c0 + v;
        const bool need = row_ok && ii >= i0 - 5 && ii <= ilast;
        any |= need;
        if (need && (ii < 1 || ii > g.n1)) v16 = false;
        if (ii < -3 || ii > g.n1 + 4) v16 = false;  // the chunk must lie inside the padded row
        go[e][v] = need ? (wrapi(ii, g.n1) + 3) + rowoff : -1;
      }
      if (v16 && any) {
        go[e][0] = (i0 - AXA_HX + c0 + 3) + rowoff;
        vec |= 1u << e;
      }
    }
    const int own0 = (in0 ? i + 3 : 4) + g.nx * ((in0 ? j0 + ya : 1) + 3);
    const int own1 = (in1 ? i + 3 : 4) + g.nx * ((in1 ? j0 + ya + 1 : 1) + 3);
    auto zoff = [&](int k) -> long long {
      return (long long)((k < 1 ? k + g.n3 : (k > g.n3 ? k - g.n3 : k)) + 3) * nxy;
    };
    // group gi: planes t = gi*AXB .. gi*AXB+AXB-1 of the tile (t < nk + 5) into their slots
    auto stage_group = [&](int gi) {
#pragma unroll
      for (int u = 0; u < AXB; ++u) {
        const int t = gi * AXB + u;
        if (t < nk + 5) {
          const float* src = x + zoff(k0 + t);
          float* dst = ring + (size_t)(t % AXA_R) * AXA_PLANE + tid * AXA_V;
#pragma unroll
          for (int e = 0; e < AXA_PER; ++e) {
            float* d = dst + e * AXNT * AXA_V;
            if ((vec >> e) & 1u) {
              cp_async16(d, src + go[e][0]);
            } else {
#pragma unroll
              for (int v = 0; v < AXA_V; ++v)
                if (go[e][v] >= 0) cp_async1(d + v, src + go[e][v]);
            }
          }
        }
      }
      cp_commit();
    };
    __syncthreads();  // weights visible; the ring is free
    const bool zu = J.zuni != 0;
    float wx[AXW], wya[AXW], wyb[AXW], wzr[AXW];
#pragma unroll
    for (int l = 0; l < AXW; ++l) {
      wx[l] = wxs[l][tx];
      wya[l] = wys[ya][l];
      wyb[l] = wys[ya + 1][l];
      wzr[l] = wzs[0][l];
    }
    float za[AXA_ZW], zb[AXA_ZW];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      za[l] = x[zoff(k0 - 5 + l) + own0];
      zb[l] = x[zoff(k0 - 5 + l) + own1];
    }
#pragma unroll
    for (int l = 5; l < AXA_ZW; ++l) za[l] = zb[l] = 0.f;
#pragma unroll
    for (int gi = 0; gi < AXA_G - 1; ++gi) stage_group(gi);
    // partners of the first step
    float pa[AXB], pb[AXB];
#pragma unroll
    for (int u = 0; u < AXB; ++u) {
      pa[u] = pb[u] = 0.f;
      if (MODE != 0 && u < nk) {
        if (in0) pa[u] = d1[zoff(k0 + u) + own0];
        if (in1) pb[u] = d1[zoff(k0 + u) + own1];
      }
    }
    double v0 = 0.0, v1 = 0.0;
    float* o0 = out + (long long)(k0 + 3) * nxy + own0;
    float* o1 = out + (long long)(k0 + 3) * nxy + own1;
    const int cx = tx + AXA_HX;  // the thread's column in the staged plane
    auto walk = [&](auto zreg) {
      constexpr bool ZR = decltype(zreg)::value;
      const int nsteps = (nk + AXB - 1) / AXB;
      for (int s = 0; s < nsteps; ++s) {
        const int tb = s * AXB;
        cp_wait<AXA_WAIT>();  // this thread's copies of planes up to tb+AXB+4 have landed
        __syncthreads();      // everybody's have; the previous step's group is free
        stage_group(s + AXA_G - 1);
        // partners of the next step
        float na[AXB], nb[AXB];
#pragma unroll
        for (int u = 0; u < AXB; ++u) {
          na[u] = nb[u] = 0.f;
          if (MODE != 0 && tb + AXB + u < nk) {
            const long long zo = zoff(k0 + tb + AXB + u);
            if (in0) na[u] = d1[zo + own0];
            if (in1) nb[u] = d1[zo + own1];
          }
        }
        if (s == 0) {  // window planes 0 .. 4 of the tile
#pragma unroll
          for (int l = 0; l < 5; ++l) {
            za[5 + l] = ring[(size_t)l * AXA_PLANE + (ya + 5) * AXA_W + cx];
            zb[5 + l] = ring[(size_t)l * AXA_PLANE + (ya + 6) * AXA_W + cx];
          }
        }
#pragma unroll
        for (int u = 0; u < AXB; ++u) {  // window planes tb+5 .. tb+AXB+4
          const float* sp = ring + (size_t)((tb + 5 + u) % AXA_R) * AXA_PLANE;
          za[10 + u] = sp[(ya + 5) * AXA_W + cx];
          zb[10 + u] = sp[(ya + 6) * AXA_W + cx];
        }
#pragma unroll
        for (int u = 0; u < AXB; ++u) {
          const int t = tb + u;
          if (t < nk) {
            const float(*sp)[AXA_W] = reinterpret_cast<const float(*)[AXA_W]>(ring + (size_t)(t % AXA_R) * AXA_PLANE);
            const float ca = za[5 + u], cb = zb[5 + u];
            float axa = mulT(wx[0], sp[ya + 5][cx - 5]), axb = mulT(wx[0], sp[ya + 6][cx - 5]);
#pragma unroll
            for (int l = 1; l < AXW; ++l) {
              axa = fmaT(wx[l], l == 5 ? ca : sp[ya + 5][cx - 5 + l], axa);
              axb = fmaT(wx[l], l == 5 ? cb : sp[ya + 6][cx - 5 + l], axb);
            }
            float yv[AXW + 1];
#pragma unroll
            for (int r = 0; r < AXW + 1; ++r) yv[r] = r == 5 ? ca : (r == 6 ? cb : sp[ya + r][cx]);
            float aya = mulT(wya[0], yv[0]), ayb = mulT(wyb[0], yv[1]);
#pragma unroll
            for (int l = 1; l < AXW; ++l) {
              aya = fmaT(wya[l], yv[l], aya);
              ayb = fmaT(wyb[l], yv[l + 1], ayb);
            }
            const float* wz = wzs[t];
            float aza = mulT(ZR ? wzr[0] : wz[0], za[u]), azb = mulT(ZR ? wzr[0] : wz[0], zb[u]);
#pragma unroll
            for (int l = 1; l < AXW; ++l) {
              aza = fmaT(ZR ? wzr[l] : wz[l], za[u + l], aza);
              azb = fmaT(ZR ? wzr[l] : wz[l], zb[u + l], azb);
            }
            const float ra = __fadd_rn(__fadd_rn(axa, aya), aza), rb = __fadd_rn(__fadd_rn(axb, ayb), azb);
            if (in0) *o0 = ra;
            if (in1) *o1 = rb;
            if (MODE == 1) {
              if (in0) v0 += (double)ra * (double)pa[u];
              if (in1) v0 += (double)rb * (double)pb[u];
            }
            if (MODE == 2) {
              if (in0) {
                v0 += (double)ra * (double)pa[u];
                v1 += (double)ra * (double)ra;
              }
              if (in1) {
                v0 += (double)rb * (double)pb[u];
                v1 += (double)rb * (double)rb;
              }
            }
            o0 += nxy;
            o1 += nxy;
          }
        }
#pragma unroll
        for (int l = 0; l < 10; ++l) {
          za[l] = za[l + AXB];
          zb[l] = zb[l + AXB];
        }
#pragma unroll
        for (int u = 0; u < AXB; ++u) {
          pa[u] = na[u];
          pb[u] = nb[u];
        }
      }
    };
    if (zu)
      walk(std::true_type{});
    else
      walk(std::false_type{});
    cp_wait<0>();
    if (MODE == 1) {
      double v[1] = {v0};
      tile_partials<1, 0, AXNT>(v, partial + (long long)b * 4);
    } else if (MODE == 2) {
      double v[2] = {v0, v1};
      tile_partials<2, 0, AXNT>(v, partial + (long long)b * 4);
    } else {
      __syncthreads();  // the ring and the weights are rewritten by the next tile
    }
  }
}

// ------------------------------------------------------------------------------------------
// The FP32 operator on lists whose grids have n1 divisible by 4 and uniform x and z spacing
// (every row of W[0] and of W[2] the same): the same collapsed 11-point product_div_grad as
// k_kr_ax32, with the center weights of the three axes combined into one and every thread
// owning one 16-byte vector of 4 consecutive x points of one row.
//
// A block of 8 x 8 threads owns one 32 x 8-column tile over kc planes.  Each plane of the tile
// with its 5-wide halo is staged by 16-byte cp.async into a ring of AXV_R slots (48 x 18 floats:
// columns i0-8 .. i0+39, rows j0-5 .. j0+12; at the box ends each chunk from its periodic image),
// together with the plane's inner-product partners (the tile's 32 x 8 points).  x neighbours come
// from the thread's row of the slot (5 vectors), y neighbours from the 10 other rows (one vector
// each).  The z values k-5 .. k+AXV_B+4 of the 4 points stay in a register window of vectors
// moved on by AXV_B planes per step; the window's new planes are 16-byte loads from global
// memory issued one step ahead.  The arithmetic runs on packed FP32 pairs (fma.rn.f32x2: two
// IEEE fmas per instruction), the per-plane inner-product terms are summed in FP32 and added
// in FP64.  The ring holds two groups of AXV_B planes: a step computes on one while the
// next is in flight (35.8 KB of shared memory and 166 registers: 6 blocks per SM).
constexpr int AXV_TX = ETX / 4, AXV_NT = AXV_TX * ETY;   // 8 x 8 threads, 4 columns each
constexpr int AXV_HX = 8;                                // staged columns left of the tile
constexpr int AXV_W = ETX + 16;                          // staged row: 8 + 32 + 8 (5 needed each side)
constexpr int AXV_H = ETY + 10;                          // staged rows
constexpr int AXV_CR = AXV_W / 4;                        // 16-byte chunks per row
constexpr int AXV_NCH = AXV_CR * AXV_H;                  // chunks per plane
constexpr int AXV_PER = (AXV_NCH + AXV_NT - 1) / AXV_NT; // chunks per thread and plane
constexpr int AXV_PLANE = AXV_W * AXV_H;                 // floats per slot
constexpr int AXV_PP = ETX * ETY;                        // partner floats per slot
constexpr int AXV_B = 4;                                 // planes per step
constexpr int AXV_G = 2;                                 // groups of AXV_B planes in the ring
constexpr int AXV_R = AXV_B * AXV_G;                     // ring slots
constexpr int AXV_ZW = AXV_B + 10;                       // z window (planes t-5 .. t+AXV_B+4)
static_assert((AXV_PLANE * 4) % 16 == 0 && (AXV_PP * 4) % 16 == 0, "slots must keep 16-byte alignment");
constexpr size_t axv_smem_bytes() { return sizeof(float) * (size_t)AXV_R * (AXV_PLANE + AXV_PP); }

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

template <int MODE>
__global__ void __launch_bounds__(AXV_NT, 5) k_kr_ax32v(const KrylovJob<float>* __restrict__ jobs,
                                                        const int* __restrict__ ts, int nj, int ntiles,
                                                        double* __restrict__ partial) {
  static_assert(MODE >= 0 && MODE <= 2, "FP32 operator modes: 0 residual, 1 alpha, 2 omega");
  extern __shared__ __align__(16) unsigned char axv_smem[];
  float* ring = reinterpret_cast<float*>(axv_smem);
  float* pring = ring + (size_t)AXV_R * AXV_PLANE;
  __shared__ double red[2][AXV_NT / 32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + AXV_TX * ty;
  const int cx = AXV_HX + 4 * tx;   // the thread's first column in a staged row
  const int pq = ty * ETX + 4 * tx;  // the thread's vector in a partner slot
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<float>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (!J.vec || (MODE == 0 ? (sc->done != 0) : e_halted(sc))) continue;  // the others: k_kr_ax32
    const Geom g = J.g;
    const int ntx = (g.n1 + ETX - 1) / ETX, nty = (g.n2 + ETY - 1) / ETY;
    const int t0 = b - ts[q];
    const int ta = t0 % ntx, tr = t0 / ntx, tc = tr / nty;
    const int i0 = ta * ETX + 1, j0 = (tr - tc * nty) * ETY + 1;
    const int k0 = tc * J.kc + 1, k1 = min(g.n3, k0 + J.kc - 1);
    const int nk = k1 - k0 + 1;
    const int i = i0 + 4 * tx, j = j0 + ty;
    const bool act = i <= g.n1 && j <= g.n2;  // n1 % 4 == 0: the 4 columns are valid together
    const float* __restrict__ x = MODE == 0 ? J.phi : (MODE == 1 ? J.z1 : J.z2);
    float* __restrict__ out = MODE == 0 ? J.rr : (MODE == 1 ? J.Ap : J.Ar);
    const float* __restrict__ d1 = MODE == 1 ? J.rh : J.rr;
    const long long nxy = g.nxy;
    // weights: x and z uniform (first rows), y of this thread's row; the three center weights
    // combined
    float wx[AXW], wy[AXW], wz[AXW];
    const int jr = j <= g.n2 ? j : 1;
#pragma unroll
    for (int l = 0; l < AXW; ++l) {
      wx[l] = __ldg(J.W[0] + l);
      wy[l] = __ldg(J.W[1] + (size_t)(jr - 1) * AXW + l);
      wz[l] = __ldg(J.W[2] + l);
    }
    const float wc = __fadd_rn(__fadd_rn(wx[5], wy[5]), wz[5]);
    // this thread's chunks of a staged plane: chunk cq = tid + e*AXV_NT holds columns
    // i0-8+4(cq%12) .. +3 of row j0-5+cq/12.  The points of the tile read columns
    // i0-5 .. min(i0+31, n1)+5 and rows j0-5 .. min(j0+7, n2)+5; cb[e] is the chunk's in-plane
    // offset, -1 for a chunk nothing needs.  A chunk starts at a column = 1 (mod 4) and n1 % 4 == 0,
    // so a chunk outside 1..n1 lies whole in one periodic image (n1 >= 8): every chunk, at the box
    // ends too, is one 16-byte copy from its image.
    const int ilast = min(i0 + ETX - 1, g.n1) + 5, jlast = min(j0 + ETY - 1, g.n2) + 5;
    int cb[AXV_PER];
#pragma unroll
    for (int e = 0; e < AXV_PER; ++e) {
      const int cq = tid + e * AXV_NT;
      const int r = cq / AXV_CR, c0 = (cq % AXV_CR) * 4;
      const int jj = j0 - 5 + r, ii = i0 - AXV_HX + c0;
      const bool need = cq < AXV_NCH && jj <= jlast && ii + 3 >= i0 - 5 && ii <= ilast;
      cb[e] = need ? (wrapi(ii, g.n1) + 3) + g.nx * (wrapi(jj, g.n2) + 3) : -1;
    }
    const int own = (act ? i + 3 : 4) + g.nx * (jr + 3);  // in-plane offset of the thread's vector
    auto zoff = [&](int k) -> long long {  // plane k (periodic) + 3 ghost planes
      return (long long)((k < 1 ? k + g.n3 : (k > g.n3 ? k - g.n3 : k)) + 3) * nxy;
    };
    // group gi: planes t = gi*AXV_B .. +AXV_B-1 of the tile (t < nk) and their partners into
    // their slots
    auto stage_group = [&](int gi) {
#pragma unroll
      for (int u = 0; u < AXV_B; ++u) {
        const int t = gi * AXV_B + u;
        if (t < nk) {
          const long long zo = zoff(k0 + t);
          const float* src = x + zo;
          float* dst = ring + (size_t)(t % AXV_R) * AXV_PLANE + tid * 4;
#pragma unroll
          for (int e = 0; e < AXV_PER; ++e)
            if (cb[e] >= 0) cp_async16(dst + e * AXV_NT * 4, src + cb[e]);
          if (MODE != 0 && act) cp_async16(pring + (size_t)(t % AXV_R) * AXV_PP + pq, d1 + zo + own);
        }
      }
      cp_commit();
    };
    __syncthreads();  // the ring is free (previous tile done)
#pragma unroll
    for (int gi = 0; gi < AXV_G - 1; ++gi) stage_group(gi);
    // z window: planes k0-5 .. k0+AXV_B+4
    float4 win[AXV_ZW];
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int l = 0; l < AXV_ZW; ++l) win[l] = act ? ldg4(x + zoff(k0 - 5 + l) + own) : zero4;
    double v0 = 0.0, v1 = 0.0;
    float* o = out + (long long)(k0 + 3) * nxy + own;
    const int nsteps = (nk + AXV_B - 1) / AXV_B;
    for (int s = 0; s < nsteps; ++s) {
      const int tb = s * AXV_B;
      cp_wait<AXV_G - 2>();  // this thread's copies of the step's group have landed
      __syncthreads();       // everybody's have; the previous step's group is free
      stage_group(s + AXV_G - 1);
      // the next step's window planes
      float4 nw[AXV_B];
      const bool more = act && tb + AXV_B < nk;
#pragma unroll
      for (int u = 0; u < AXV_B; ++u) nw[u] = more ? ldg4(x + zoff(k0 + tb + AXV_B + 5 + u) + own) : zero4;
#pragma unroll
      for (int u = 0; u < AXV_B; ++u) {
        const int t = tb + u;
        if (t < nk) {
          const float* sp = ring + (size_t)(t % AXV_R) * AXV_PLANE;
          // x: the thread's row, columns cx-8 .. cx+11 (own vector at 8..11)
          float xv[20];
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            const float4 v = lds4(sp + (ty + 5) * AXV_W + cx - 8 + 4 * m);
            xv[4 * m] = v.x;
            xv[4 * m + 1] = v.y;
            xv[4 * m + 2] = v.z;
            xv[4 * m + 3] = v.w;
          }
          // packed FP32 pairs (points 0,1 and 2,3; each lane one IEEE fma, the order of the
          // scalar chains): center, x (odd offsets from the aligned pairs of the row, even ones
          // per lane), y and z, then (x + y) + z
          const float4 cc = win[u + 5];
          float2 a01 = __fmul2_rn(make_float2(wc, wc), make_float2(cc.x, cc.y));
          float2 a23 = __fmul2_rn(make_float2(wc, wc), make_float2(cc.z, cc.w));
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            if (l & 1) {
              const float2 w2 = make_float2(wx[l], wx[l]);
              a01 = __ffma2_rn(w2, make_float2(xv[3 + l], xv[4 + l]), a01);
              a23 = __ffma2_rn(w2, make_float2(xv[5 + l], xv[6 + l]), a23);
            } else {
              a01.x = fmaT(wx[l], xv[3 + l], a01.x);
              a01.y = fmaT(wx[l], xv[4 + l], a01.y);
              a23.x = fmaT(wx[l], xv[5 + l], a23.x);
              a23.y = fmaT(wx[l], xv[6 + l], a23.y);
            }
          }
          float2 y01 = make_float2(0.f, 0.f), y23 = make_float2(0.f, 0.f);
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            const float4 v = lds4(sp + (ty + l) * AXV_W + cx);
            const float2 w2 = make_float2(wy[l], wy[l]);
            y01 = __ffma2_rn(w2, make_float2(v.x, v.y), y01);
            y23 = __ffma2_rn(w2, make_float2(v.z, v.w), y23);
          }
          float2 z01 = make_float2(0.f, 0.f), z23 = make_float2(0.f, 0.f);
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            const float2 w2 = make_float2(wz[l], wz[l]);
            z01 = __ffma2_rn(w2, make_float2(win[u + l].x, win[u + l].y), z01);
            z23 = __ffma2_rn(w2, make_float2(win[u + l].z, win[u + l].w), z23);
          }
          a01 = __fadd2_rn(__fadd2_rn(a01, y01), z01);
          a23 = __fadd2_rn(__fadd2_rn(a23, y23), z23);
          if (act) {
            *reinterpret_cast<float4*>(o) = make_float4(a01.x, a01.y, a23.x, a23.y);
            // the plane's 4 products summed in FP32, the sum added in FP64
            if (MODE != 0) {
              const float4 pv = lds4(pring + (size_t)(t % AXV_R) * AXV_PP + pq);
              const float2 d = __ffma2_rn(a23, make_float2(pv.z, pv.w), __fmul2_rn(a01, make_float2(pv.x, pv.y)));
              v0 += (double)__fadd_rn(d.x, d.y);
            }
            if (MODE == 2) {
              const float2 d = __ffma2_rn(a23, a23, __fmul2_rn(a01, a01));
              v1 += (double)__fadd_rn(d.x, d.y);
            }
          }
          o += nxy;
        }
      }
#pragma unroll
      for (int l = 0; l < AXV_ZW - AXV_B; ++l) win[l] = win[l + AXV_B];
#pragma unroll
      for (int u = 0; u < AXV_B; ++u) win[AXV_ZW - AXV_B + u] = nw[u];
    }
    cp_wait<0>();
    if (MODE != 0) {
      v0 = e_wsum(v0);
      v1 = e_wsum(v1);
      if ((tid & 31) == 0) {
        red[0][tid >> 5] = v0;
        red[1][tid >> 5] = v1;
      }
      __syncthreads();
      if (tid == 0) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int w = 0; w < AXV_NT / 32; ++w) {
          s0 += red[0][w];
          s1 += red[1][w];
        }
        partial[(long long)b * 4] = s0;
        if (MODE == 2) partial[(long long)b * 4 + 1] = s1;
      }
    }
    // the ring and red are rewritten by the next tile only after its first barrier
  }
}

// ------------------------------------------------------------------------------------------
// The FP64 operator (the Krylov list of an FP64 solve, and the outer residual of the mixed
// solve) on grids with n1 divisible by 2: the collapsed 11-point product_div_grad with every
// thread owning one 16-byte vector of 2 consecutive x points of one row.  The staging and z
// window of k_kr_ax32v (16 x 8 threads per 32 x 8-column tile, 48 x 18 staged doubles per plane,
// a ring of 2 groups of 4 planes, the window k-5 .. k+8 in registers); the weights are the per-row
// weights of every axis (the FP64 operator defines the residual): x rows of the thread's two
// columns and the y row of its row in registers, the z rows of the tile's planes in shared memory.
//   MODE 0: rr = A phi;  1: Ap = A z1, partial rh.Ap;  2: Ar = A z2, partials Ar.rr, Ar.Ar;
//   3: r32 = (float)(bb - A phi), partials max|r|, sum r^2, sum bb^2
constexpr int AXD_TX = ETX / 2, AXD_NT = AXD_TX * ETY;   // 16 x 8 threads, 2 columns each
constexpr int AXD_W = ETX + 16, AXD_H = ETY + 10;        // staged plane, doubles
constexpr int AXD_CR = AXD_W / 2;                        // 16-byte chunks per row
constexpr int AXD_NCH = AXD_CR * AXD_H;
constexpr int AXD_PER = (AXD_NCH + AXD_NT - 1) / AXD_NT;
constexpr int AXD_PLANE = AXD_W * AXD_H;
constexpr int AXD_PP = ETX * ETY;
constexpr int AXD_B = 4, AXD_G = 2, AXD_R = AXD_B * AXD_G, AXD_ZW = AXD_B + 10;
constexpr size_t axd_smem_bytes() {
  return sizeof(double) * ((size_t)AXD_R * (AXD_PLANE + AXD_PP) + (size_t)KC_MAX * AXW);
}
__device__ __forceinline__ double2 ldg2d(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ double2 lds2d(const double* p) { return *reinterpret_cast<const double2*>(p); }

template <int MODE>
__global__ void __launch_bounds__(AXD_NT, 2) k_kr_ax64v(const KrylovJob<double>* __restrict__ jobs,
                                                        const int* __restrict__ ts, int nj, int ntiles,
                                                        double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char axd_smem[];
  double* ring = reinterpret_cast<double*>(axd_smem);
  double* pring = ring + (size_t)AXD_R * AXD_PLANE;
  double(*wzs)[AXW] = reinterpret_cast<double(*)[AXW]>(pring + (size_t)AXD_R * AXD_PP);
  __shared__ double red[4][AXD_NT / 32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + AXD_TX * ty;
  const int cx = 8 + 2 * tx;          // the thread's first column in a staged row
  const int pq = ty * ETX + 2 * tx;   // the thread's vector in a partner slot
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const KrylovJob<double>& J = jobs[q];
    const SolverScalars* sc = J.sc;
    if (!J.vec || (MODE == 0 ? (sc->done != 0) : e_halted(sc))) continue;  // the others: k_kr_ax
    const Geom g = J.g;
    const int ntx = (g.n1 + ETX - 1) / ETX, nty = (g.n2 + ETY - 1) / ETY;
    const int t0 = b - ts[q];
    const int ta = t0 % ntx, tr = t0 / ntx, tc = tr / nty;
    const int i0 = ta * ETX + 1, j0 = (tr - tc * nty) * ETY + 1;
    const int k0 = tc * J.kc + 1, k1 = min(g.n3, k0 + J.kc - 1);
    const int nk = k1 - k0 + 1;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const bool act = i <= g.n1 && j <= g.n2;  // n1 % 2 == 0: both columns valid together
    const double* __restrict__ x = (MODE == 0 || MODE == 3) ? J.phi : (MODE == 1 ? J.z1 : J.z2);
    const double* __restrict__ d1 = MODE == 1 ? J.rh : (MODE == 3 ? J.bb : J.rr);
    const long long nxy = g.nxy;
    const int ir = act ? i : 1, jr = j <= g.n2 ? j : 1;
    double wx0[AXW], wx1[AXW], wy[AXW];
#pragma unroll
    for (int l = 0; l < AXW; ++l) {
      wx0[l] = __ldg(J.W[0] + (size_t)(ir - 1) * AXW + l);
      wx1[l] = __ldg(J.W[0] + (size_t)ir * AXW + l);
      wy[l] = __ldg(J.W[1] + (size_t)(jr - 1) * AXW + l);
    }
    for (int t = tid; t < nk * AXW; t += AXD_NT) wzs[t / AXW][t % AXW] = __ldg(J.W[2] + (size_t)(k0 - 1) * AXW + t);
    const int ilast = min(i0 + ETX - 1, g.n1) + 5, jlast = min(j0 + ETY - 1, g.n2) + 5;
    // a chunk starts at an odd column and n1 is even, so a chunk outside 1..n1 lies whole in one
    // periodic image (n1 >= 8): every chunk is one 16-byte copy from its image
    int cb[AXD_PER];
#pragma unroll
    for (int e = 0; e < AXD_PER; ++e) {
      const int cq = tid + e * AXD_NT;
      const int r = cq / AXD_CR, c0 = (cq % AXD_CR) * 2;
      const int jj = j0 - 5 + r, ii = i0 - 8 + c0;
      const bool need = cq < AXD_NCH && jj <= jlast && ii + 1 >= i0 - 5 && ii <= ilast;
      cb[e] = need ? (wrapi(ii, g.n1) + 3) + g.nx * (wrapi(jj, g.n2) + 3) : -1;
    }
    const int own = (act ? i + 3 : 4) + g.nx * (jr + 3);
    auto zoff = [&](int k) -> long long {
      return (long long)((k < 1 ? k + g.n3 : (k > g.n3 ? k - g.n3 : k)) + 3) * nxy;
    };
    auto stage_group = [&](int gi) {
#pragma unroll
      for (int u = 0; u < AXD_B; ++u) {
        const int t = gi * AXD_B + u;
        if (t < nk) {
          const long long zo = zoff(k0 + t);
          const double* src = x + zo;
          double* dst = ring + (size_t)(t % AXD_R) * AXD_PLANE + tid * 2;
#pragma unroll
          for (int e = 0; e < AXD_PER; ++e)
            if (cb[e] >= 0) cp_async16(dst + e * AXD_NT * 2, src + cb[e]);
          if (MODE != 0 && act) cp_async16(pring + (size_t)(t % AXD_R) * AXD_PP + pq, d1 + zo + own);
        }
      }
      cp_commit();
    };
    __syncthreads();  // the ring and the z weights of the previous tile are no longer read
#pragma unroll
    for (int gi = 0; gi < AXD_G - 1; ++gi) stage_group(gi);
    double2 win[AXD_ZW];
    const double2 zero2 = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < AXD_ZW; ++l) win[l] = act ? ldg2d(x + zoff(k0 - 5 + l) + own) : zero2;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    const long long obase = (long long)(k0 + 3) * nxy + own;
    const int nsteps = (nk + AXD_B - 1) / AXD_B;
    for (int s = 0; s < nsteps; ++s) {
      const int tb = s * AXD_B;
      cp_wait<AXD_G - 2>();
      __syncthreads();  // everybody's copies of the step's group (and the z weights) are visible
      stage_group(s + AXD_G - 1);
      double2 nw[AXD_B];
      const bool more = act && tb + AXD_B < nk;
#pragma unroll
      for (int u = 0; u < AXD_B; ++u) nw[u] = more ? ldg2d(x + zoff(k0 + tb + AXD_B + 5 + u) + own) : zero2;
#pragma unroll
      for (int u = 0; u < AXD_B; ++u) {
        const int t = tb + u;
        if (t < nk) {
          const double* sp = ring + (size_t)(t % AXD_R) * AXD_PLANE;
          const double* wz = wzs[t];
          double xv[14];  // the thread's row, columns cx-6 .. cx+7 (own at 6, 7)
#pragma unroll
          for (int m = 0; m < 7; ++m) {
            const double2 v = lds2d(sp + (ty + 5) * AXD_W + cx - 6 + 2 * m);
            xv[2 * m] = v.x;
            xv[2 * m + 1] = v.y;
          }
          const double wyz = __dadd_rn(wy[5], wz[5]);
          const double2 cc = win[u + 5];
          double r0 = mulT(__dadd_rn(wx0[5], wyz), cc.x), r1 = mulT(__dadd_rn(wx1[5], wyz), cc.y);
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            r0 = fmaT(wx0[l], xv[1 + l], r0);
            r1 = fmaT(wx1[l], xv[2 + l], r1);
          }
          double y0 = 0.0, y1 = 0.0;
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            const double2 v = lds2d(sp + (ty + l) * AXD_W + cx);
            y0 = fmaT(wy[l], v.x, y0);
            y1 = fmaT(wy[l], v.y, y1);
          }
          double z0 = 0.0, z1 = 0.0;
#pragma unroll
          for (int l = 0; l < AXW; ++l) {
            if (l == 5) continue;
            const double w = wz[l];
            z0 = fmaT(w, win[u + l].x, z0);
            z1 = fmaT(w, win[u + l].y, z1);
          }
          r0 = __dadd_rn(__dadd_rn(r0, y0), z0);
          r1 = __dadd_rn(__dadd_rn(r1, y1), z1);
          if (act) {
            const long long o = obase + (long long)t * nxy;
            if (MODE == 3) {
              const double2 bv = lds2d(pring + (size_t)(t % AXD_R) * AXD_PP + pq);
              const double e0 = bv.x - r0, e1 = bv.y - r1;
              const float2 ef = make_float2((float)e0, (float)e1);
              *reinterpret_cast<float2*>(J.r32 + o) = ef;
              if (J.r32p) *reinterpret_cast<float2*>(J.r32p + o) = ef;
              v3 += (double)ef.x * (double)ef.x;
              v3 += (double)ef.y * (double)ef.y;
              v0 = fmax(v0, fmax(fabs(e0), fabs(e1)));
              v1 += e0 * e0;
              v1 += e1 * e1;
              v2 += bv.x * bv.x;
              v2 += bv.y * bv.y;
            } else {
              double* out = MODE == 0 ? J.rr : (MODE == 1 ? J.Ap : J.Ar);
              *reinterpret_cast<double2*>(out + o) = make_double2(r0, r1);
              if (MODE != 0) {
                const double2 pv = lds2d(pring + (size_t)(t % AXD_R) * AXD_PP + pq);
                v0 += r0 * pv.x;
                v0 += r1 * pv.y;
              }
              if (MODE == 2) {
                v1 += r0 * r0;
                v1 += r1 * r1;
              }
            }
          }
        }
      }
#pragma unroll
      for (int l = 0; l < AXD_ZW - AXD_B; ++l) win[l] = win[l + AXD_B];
#pragma unroll
      for (int u = 0; u < AXD_B; ++u) win[AXD_ZW - AXD_B + u] = nw[u];
    }
    cp_wait<0>();
    if (MODE != 0) {
      v0 = MODE == 3 ? e_wmax(v0) : e_wsum(v0);
      v1 = e_wsum(v1);
      v2 = e_wsum(v2);
      v3 = e_wsum(v3);
      if ((tid & 31) == 0) {
        red[0][tid >> 5] = v0;
        red[1][tid >> 5] = v1;
        red[2][tid >> 5] = v2;
        red[3][tid >> 5] = v3;
      }
      __syncthreads();
      if (tid == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
        for (int w = 0; w < AXD_NT / 32; ++w) {
          s0 = MODE == 3 ? fmax(s0, red[0][w]) : s0 + red[0][w];
          s1 += red[1][w];
          s2 += red[2][w];
          s3 += red[3][w];
        }
        partial[(long long)b * 4] = s0;
        if (MODE >= 2) partial[(long long)b * 4 + 1] = s1;
        if (MODE == 3) {
          partial[(long long)b * 4 + 2] = s2;
          partial[(long long)b * 4 + 3] = s3;
        }
      }
    }
  }
}

// bv - a0 w - a2 e - b0 s - b2 n - cm zm - cp zp
template <typename T>
__device__ __forceinline__ T jres(T bv, T a0, T w, T a2, T e, T b0, T s, T b2, T n, T cm, T zm, T cp, T zp) {
  T r = fmaT(-a0, w, bv);
  r = fmaT(-a2, e, r);
  r = fmaT(-b0, s, r);
  r = fmaT(-b2, n, r);
  r = fmaT(-cm, zm, r);
  return fmaT(-cp, zp, r);
}
// damped-Jacobi update of centre value zc from r: omega r / diag + (1 - omega) zc; on uniform z
// r (omega / diag) with inv = omega / diag formed once per column
template <typename T>
__device__ __forceinline__ T jsweep(T r, T zc, T omega, bool zu, T inv, T diag) {
  const T q = zu ? mulT(r, inv) : mulT(omega, r) / diag;
  return fmaT(T(1) - omega, zc, q);
}
// init sweep omega v / diag (uniform z: v inv)
template <typename T>
__device__ __forceinline__ T jinit(T v, T omega, bool zu, T inv, T diag) {
  return zu ? mulT(v, inv) : mulT(omega, v) / diag;
}
// residual bv - (a0 w + a2 e + b0 s + b2 n + cm zm + cp zp + diag zc)
template <typename T>
__device__ __forceinline__ T jresid(T bv, T a0, T w, T a2, T e, T b0, T s, T b2, T n, T cm, T zm, T cp, T zp, T diag,
                                    T zc) {
  T l = mulT(a0, w);
  l = fmaT(a2, e, l);
  l = fmaT(b0, s, l);
  l = fmaT(b2, n, l);
  l = fmaT(cm, zm, l);
  l = fmaT(cp, zp, l);
  l = fmaT(diag, zc, l);
  return bv - l;
}

// One column (i, j), planes k0..k1, of the compact 7-point operator cdg.  The column is walked
// in blocks of U planes: all loads of a block (the next planes' centres, the right-hand side
// and the four lateral neighbours) are issued before its stores, so that every thread keeps
// several DRAM requests in flight; the z-neighbours stay in registers.
//   OP 0: damped-Jacobi sweep  out = omega (bb - offdiag x) / diag + (1 - omega) x
//   OP 1: residual             out = bb - (offdiag x + diag x)
template <typename T, int OP, int U, bool ZU>
__device__ __forceinline__ void march7(const Geom& g, int i, int j, int k0, int k1, const T* __restrict__ cx,
                                       const T* __restrict__ cy, const T* __restrict__ cz, T omega,
                                       const T* __restrict__ bb, const T* __restrict__ x, T* __restrict__ out) {
  const T a0 = cx[3 * (i - 1)], a1 = cx[3 * (i - 1) + 1], a2 = cx[3 * (i - 1) + 2];
  const T b0 = cy[3 * (j - 1)], b1 = cy[3 * (j - 1) + 1], b2 = cy[3 * (j - 1) + 2];
  // uniform z: one z row for the whole column, and omega / diag formed once (the per-point
  // division omega r / diag becomes r (omega / diag))
  const T zcm = ZU ? cz[0] : T(0), zcc = ZU ? cz[1] : T(0), zcp = ZU ? cz[2] : T(0);
  const T inv = ZU ? omega / (a1 + b1 + zcc) : T(0);
  const T dg = ZU ? a1 + b1 + zcc : T(0);
  const long long nxy = g.nxy;
  const int dW = (i == 1) ? g.n1 - 1 : -1;
  const int dE = (i == g.n1) ? 1 - g.n1 : 1;
  const int dS = (j == 1) ? (g.n2 - 1) * g.nx : -g.nx;
  const int dN = (j == g.n2) ? -(g.n2 - 1) * g.nx : g.nx;
  const long long wz = (long long)(g.n3 - 1) * nxy;
  long long p = off(g, i, j, k0);
  T xm = x[k0 == 1 ? p + wz : p - nxy];
  T xc = x[p];
  auto point = [&](int k, long long q, T bv, T w, T e, T s, T n, T zm, T zc, T zp) {
    const T cm = ZU ? zcm : cz[3 * (k - 1)];
    const T cc = ZU ? zcc : cz[3 * (k - 1) + 1];
    const T cp = ZU ? zcp : cz[3 * (k - 1) + 2];
    if (OP == 0) {
      const T r = jres(bv, a0, w, a2, e, b0, s, b2, n, cm, zm, cp, zp);
      out[q] = jsweep(r, zc, omega, ZU, inv, ZU ? dg : a1 + b1 + cc);
    } else {
      out[q] = jresid(bv, a0, w, a2, e, b0, s, b2, n, cm, zm, cp, zp, ZU ? dg : a1 + b1 + cc, zc);
    }
  };
  int k = k0;
  for (; k + U - 1 <= k1; k += U) {
    T xn[U], bv[U], w[U], e[U], s[U], n[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long q = p + u * nxy;
      xn[u] = x[(k + u == g.n3) ? q - wz : q + nxy];
      bv[u] = bb[q];
      w[u] = x[q + dW];
      e[u] = x[q + dE];
      s[u] = x[q + dS];
      n[u] = x[q + dN];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const T zc = u == 0 ? xc : xn[u - 1];
      const T zm = u == 0 ? xm : (u == 1 ? xc : xn[u - 2]);
      point(k + u, p + u * nxy, bv[u], w[u], e[u], s[u], n[u], zm, zc, xn[u]);
    }
    xm = U >= 2 ? xn[U - 2] : xc;
    xc = xn[U - 1];
    p += U * nxy;
  }
  for (; k <= k1; ++k, p += nxy) {
    const T xp = x[k == g.n3 ? p - wz : p + nxy];
    point(k, p, bb[p], x[p + dW], x[p + dE], x[p + dS], x[p + dN], xm, xc, xp);
    xm = xc;
    xc = xp;
  }
}

// The same column walk for W = 16 / sizeof(T) consecutive columns i .. i+W-1 per thread, with
// 16-byte loads and stores (requires n1 % W == 0).  The x-neighbours inside the vector are
// registers, the ones across vectors come from the adjacent lanes by shuffles (a scalar load at
// the warp edges and at the periodic boundary).  Every lane of the warp runs the walk (inactive
// lanes only take part in the shuffles).
template <typename T, int OP, int U, bool ZU>
__device__ __forceinline__ void march7v(const Geom& g, int i, int j, int k0, int k1, bool act,
                                        const T* __restrict__ cx, const T* __restrict__ cy,
                                        const T* __restrict__ cz, T omega, const T* __restrict__ bb,
                                        const T* __restrict__ x, T* __restrict__ out) {
  constexpr int V = VecT<T>::W;
  const int lane = threadIdx.x & 31;
  const int ic = act ? i : 1, jc = act ? j : 1;
  T a0[V], a1[V], a2[V], inv[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    a0[v] = cx[3 * (ic - 1 + v)];
    a1[v] = cx[3 * (ic - 1 + v) + 1];
    a2[v] = cx[3 * (ic - 1 + v) + 2];
  }
  const T b0 = cy[3 * (jc - 1)], b1 = cy[3 * (jc - 1) + 1], b2 = cy[3 * (jc - 1) + 2];
  const T zcm = ZU ? cz[0] : T(0), zcc = ZU ? cz[1] : T(0), zcp = ZU ? cz[2] : T(0);
#pragma unroll
  for (int v = 0; v < V; ++v) inv[v] = ZU ? omega / (a1[v] + b1 + zcc) : T(0);
  const long long nxy = g.nxy;
  const int dS = (jc == 1) ? (g.n2 - 1) * g.nx : -g.nx;
  const int dN = (jc == g.n2) ? -(g.n2 - 1) * g.nx : g.nx;
  const int wOff = (ic == 1) ? g.n1 - 1 : -1;            // west of the first column
  const int eOff = (ic + V - 1 == g.n1) ? 1 - ic : V;    // east of the last column
  const bool lw = lane == 0 || ic == 1;
  const bool le = lane == 31 || ic + V - 1 == g.n1;
  const long long wzf = (long long)(g.n3 - 1) * nxy;
  long long p = off(g, ic, jc, k0);
  T xm[V], xc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) xm[v] = xc[v] = T(0);
  if (act) {
    vload(x + (k0 == 1 ? p + wzf : p - nxy), xm);
    vload(x + p, xc);
  }
  for (int k = k0; k <= k1; k += U) {
    const int nk = min(U, k1 - k + 1);
    T xn[U][V], bv[U][V], sv[U][V], nv[U][V], ws[U], es[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      ws[u] = es[u] = T(0);
#pragma unroll
      for (int v = 0; v < V; ++v) xn[u][v] = bv[u][v] = sv[u][v] = nv[u][v] = T(0);
      if (act && u < nk) {
        const long long q = p + u * nxy;
        vload(x + ((k + u == g.n3) ? q - wzf : q + nxy), xn[u]);
        vload(bb + q, bv[u]);
        vload(x + q + dS, sv[u]);
        vload(x + q + dN, nv[u]);
        if (lw) ws[u] = x[q + wOff];
        if (le) es[u] = x[q + eOff];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u < nk) {
        T zc[V], zm[V], ov[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
          zc[v] = u == 0 ? xc[v] : xn[u - 1][v];
          zm[v] = u == 0 ? xm[v] : (u == 1 ? xc[v] : xn[u - 2][v]);
        }
        const T wsh = __shfl_up_sync(0xffffffffu, zc[V - 1], 1);
        const T esh = __shfl_down_sync(0xffffffffu, zc[0], 1);
        const int kk = k + u;
        const T cm = ZU ? zcm : cz[3 * (kk - 1)];
        const T cc = ZU ? zcc : cz[3 * (kk - 1) + 1];
        const T cp = ZU ? zcp : cz[3 * (kk - 1) + 2];
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const T w = v == 0 ? (lw ? ws[u] : wsh) : zc[v - 1];
          const T e = v == V - 1 ? (le ? es[u] : esh) : zc[v + 1];
          if (OP == 0) {
            const T r = jres(bv[u][v], a0[v], w, a2[v], e, b0, sv[u][v], b2, nv[u][v], cm, zm[v], cp, xn[u][v]);
            ov[v] = jsweep(r, zc[v], omega, ZU, inv[v], a1[v] + b1 + cc);
          } else {
            ov[v] = jresid(bv[u][v], a0[v], w, a2[v], e, b0, sv[u][v], b2, nv[u][v], cm, zm[v], cp, xn[u][v],
                           a1[v] + b1 + cc, zc[v]);
          }
        }
        if (act) vstore(out + p + u * nxy, ov);
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      xm[v] = U >= 2 ? xn[U - 2][v] : xc[v];
      xc[v] = xn[U - 1][v];
    }
    p += U * nxy;
  }
}

// MODE 0: one damped-Jacobi sweep  dst = omega (A - offdiag src) / diag + (1 - omega) src
// MODE 1: the init sweep           dst = omega A / diag
// MODE 2: copy                     C = B
// flip selects the buffers: sweep 0: B -> C, 1: C -> B; init: destination 0 = B, 1 = C
template <typename T, int MODE>
__global__ void __launch_bounds__(ENT) k_lv_smooth(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                   int nj, int ntiles, T omega, int flip) {
  constexpr int U = Ublk<T>::U;
  constexpr int V = VecT<T>::W;
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    const int vw = J.vw;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1, vw);
    const bool act = i <= g.n1 && j <= g.n2;
    if (MODE == 0) {
      const T* src = flip ? J.C : J.B;
      T* dst = flip ? J.B : J.C;
      if (vw > 1) {  // every lane walks (shuffles); inactive lanes load and store nothing
        if (J.zuni)
          march7v<T, 0, 2, true>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], omega, J.A, src, dst);
        else
          march7v<T, 0, 2, false>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], omega, J.A, src, dst);
      } else if (act) {
        if (J.zuni)
          march7<T, 0, U, true>(g, i, j, k0, k1, J.cdg[0], J.cdg[1], J.cdg[2], omega, J.A, src, dst);
        else
          march7<T, 0, U, false>(g, i, j, k0, k1, J.cdg[0], J.cdg[1], J.cdg[2], omega, J.A, src, dst);
      }
      continue;
    }
    if (!act) continue;
    long long p = off(g, i, j, k0);
    const long long nxy = g.nxy;
    if (MODE == 2) {
      const T* __restrict__ src = J.B;
      T* __restrict__ dst = J.C;
      if (vw > 1) {
        int k = k0;
        for (; k + 3 <= k1; k += 4, p += 4 * nxy) {
          T v[4][V];
#pragma unroll
          for (int u = 0; u < 4; ++u) vload(src + p + u * nxy, v[u]);
#pragma unroll
          for (int u = 0; u < 4; ++u) vstore(dst + p + u * nxy, v[u]);
        }
        for (; k <= k1; ++k, p += nxy) {
          T v[V];
          vload(src + p, v);
          vstore(dst + p, v);
        }
      } else {
        int k = k0;
        for (; k + 2 * U - 1 <= k1; k += 2 * U, p += 2 * U * nxy) {
          T v[2 * U];
#pragma unroll
          for (int u = 0; u < 2 * U; ++u) v[u] = src[p + u * nxy];
#pragma unroll
          for (int u = 0; u < 2 * U; ++u) dst[p + u * nxy] = v[u];
        }
        for (; k <= k1; ++k, p += nxy) dst[p] = src[p];
      }
      continue;
    }
    const T b1 = J.cdg[1][3 * (j - 1) + 1];
    const T* __restrict__ c3 = J.cdg[2];
    const T* __restrict__ bb = J.A;
    T* __restrict__ dst = flip ? J.C : J.B;
    const bool zu = J.zuni != 0;
    if (vw > 1) {
      T a1[V], inv[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        a1[v] = J.cdg[0][3 * (i - 1 + v) + 1];
        inv[v] = omega / (a1[v] + b1 + c3[1]);  // uniform z: omega / diag of the whole column
      }
      int k = k0;
      for (; k + 3 <= k1; k += 4, p += 4 * nxy) {
        T v[4][V];
#pragma unroll
        for (int u = 0; u < 4; ++u) vload(bb + p + u * nxy, v[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int c = 0; c < V; ++c)
            v[u][c] = jinit(v[u][c], omega, zu, inv[c], a1[c] + b1 + c3[3 * (k + u - 1) + 1]);
          vstore(dst + p + u * nxy, v[u]);
        }
      }
      for (; k <= k1; ++k, p += nxy) {
        T v[V];
        vload(bb + p, v);
#pragma unroll
        for (int c = 0; c < V; ++c) v[c] = jinit(v[c], omega, zu, inv[c], a1[c] + b1 + c3[3 * (k - 1) + 1]);
        vstore(dst + p, v);
      }
      continue;
    }
    const T a1 = J.cdg[0][3 * (i - 1) + 1];
    const T inv = omega / (a1 + b1 + c3[1]);
    int k = k0;
    for (; k + 2 * U - 1 <= k1; k += 2 * U, p += 2 * U * nxy) {
      T v[2 * U];
#pragma unroll
      for (int u = 0; u < 2 * U; ++u) v[u] = bb[p + u * nxy];
#pragma unroll
      for (int u = 0; u < 2 * U; ++u)
        dst[p + u * nxy] = jinit(v[u], omega, zu, inv, a1 + b1 + c3[3 * (k + u - 1) + 1]);
    }
    for (; k <= k1; ++k, p += nxy) dst[p] = jinit(bb[p], omega, zu, inv, a1 + b1 + c3[3 * (k - 1) + 1]);
  }
}

// The common case as its own kernel, for lists whose every job has several columns per thread
// and uniform z: only the vectorised walk is compiled, which keeps the register count (and so
// the occupancy) of the streaming loop low.  OP 0: sweep (flip as in k_lv_smooth), 1: residual.
template <typename T, int OP, int U, int MINB>
__global__ void __launch_bounds__(ENT, MINB) k_lv_fast(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                       int nj, int ntiles, T omega, int flip) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1, VecT<T>::W);
    const bool act = i <= g.n1 && j <= g.n2;
    if (OP == 0)
      march7v<T, 0, U, true>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], omega, J.A, flip ? J.C : J.B,
                             flip ? J.B : J.C);
    else
      march7v<T, 1, U, true>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], T(0), J.A, J.B, J.C);
  }
}

// C = A - cdg(B): the residual that restrict forms as fine1 - fine2 (fine2 = product_div_grad_relax)
template <typename T>
__global__ void __launch_bounds__(ENT) k_lv_resid(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                  int nj, int ntiles) {
  constexpr int U = Ublk<T>::U;
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1, J.vw);
    const bool act = i <= g.n1 && j <= g.n2;
    if (J.vw > 1) {
      if (J.zuni)
        march7v<T, 1, 2, true>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], T(0), J.A, J.B, J.C);
      else
        march7v<T, 1, 2, false>(g, i, j, k0, k1, act, J.cdg[0], J.cdg[1], J.cdg[2], T(0), J.A, J.B, J.C);
      continue;
    }
    if (!act) continue;
    if (J.zuni)
      march7<T, 1, U, true>(g, i, j, k0, k1, J.cdg[0], J.cdg[1], J.cdg[2], T(0), J.A, J.B, J.C);
    else
      march7<T, 1, U, false>(g, i, j, k0, k1, J.cdg[0], J.cdg[1], J.cdg[2], T(0), J.A, J.B, J.C);
  }
}

// this (coarse) level: A(ii,jj,kk) = (1.5 d(c) + sum over the six fine neighbours of 1/4 d) / 3
// the restriction of the fine residual to one coarse point (restrict, mod_solvers.f90:588-808):
// weights 1/4, 2/4, 1/4 per axis, the centre's three halves summed first, every rounding spelled
// out (the same bits in every restriction kernel)
template <typename T>
__device__ __forceinline__ T restrict7(T dc, T xm, T xp, T ym, T yp, T zm, T zp) {
  const T cm = T(1) / T(4), c0 = T(2) / T(4), cp = T(1) / T(4);
  T v = mulT(c0 + c0 + c0, dc);
  v = fmaT(cm, xm, v);
  v = fmaT(cp, xp, v);
  v = fmaT(cm, ym, v);
  v = fmaT(cp, yp, v);
  v = fmaT(cm, zm, v);
  v = fmaT(cp, zp, v);
  return v / T(3);
}

template <typename T>
__global__ void __launch_bounds__(ENT) k_lv_restrict(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                     int nj, int ntiles) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    int i0, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i0, j, k0, k1, J.vw);
    for (int i = i0; i < i0 + J.vw; ++i) {
    if (i > g.n1 || j > g.n2) continue;
    const Geom gf = J.gf;
    const T* __restrict__ d = J.Cf;
    T* __restrict__ coarse = const_cast<T*>(J.A);
    const int fi = J.rf[0] * (i - 1) + 1, fj = J.rf[1] * (j - 1) + 1;
    const int fim = wrapi(fi - 1, gf.n1), fip = wrapi(fi + 1, gf.n1);
    const int fjm = wrapi(fj - 1, gf.n2), fjp = wrapi(fj + 1, gf.n2);
    for (int k = k0; k <= k1; ++k) {
      const int fk = J.rf[2] * (k - 1) + 1;
      coarse[off(g, i, j, k)] = restrict7(d[off(gf, fi, fj, fk)], d[off(gf, fim, fj, fk)], d[off(gf, fip, fj, fk)],
                                          d[off(gf, fi, fjm, fk)], d[off(gf, fi, fjp, fk)],
                                          d[off(gf, fi, fj, wrapi(fk - 1, gf.n3))], d[off(gf, fi, fj, wrapi(fk + 1, gf.n3))]);
    }
    }
  }
}

// one linear-interpolation pass of the prolongation: m ? w0 a + w1 b : a, with every rounding
// spelled out (the same bits in every prolongation kernel)
template <typename T>
__device__ __forceinline__ T pmix(bool m, T w0, T a, T w1, T b) {
  return m ? fmaT(w1, b, mulT(w0, a)) : a;
}

// coarse indices bracketing fine index q (lo == hi for coincident points)
__device__ __forceinline__ void bracket(int q, int r, int nc, int& lo, int& hi, bool& mid) {
  if (r == 1) {
    lo = hi = q;
    mid = false;
  } else if (q & 1) {
    lo = hi = (q - 1) / 2 + 1;
    mid = false;
  } else {
    lo = q / 2;
    hi = q / 2 + 1 > nc ? 1 : q / 2 + 1;
    mid = true;
  }
}

// V consecutive fine columns i .. i+V-1 of B += P Bc, per fine point exactly as the sequential
// z, y, x passes would (z weights first, then y, then x).  Every column keeps the four (x, y)
// corner values of the two most recent coarse planes in registers, so consecutive fine planes
// reuse them; with V > 1 the fine values move as 16-byte vectors.
template <typename T, int V>
__device__ __forceinline__ void prolong_cols(const LevelJob<T>& J, const Geom& g, int i, int j, int k0, int k1,
                                             T* __restrict__ dst) {
  const Geom gc = J.gc;
  const T* __restrict__ coarse = J.Bc;
  const T* __restrict__ cI3 = J.cI[2];
  const T* __restrict__ fine = J.B;
  int yl, yh;
  bool my;
  bracket(j, J.rc[1], gc.n2, yl, yh, my);
  const T wy0 = J.cI[1][2 * j], wy1 = J.cI[1][2 * j + 1];
  bool mx[V];
  T wx0[V], wx1[V];
  int o[V][4];  // corners (xl,yl), (xl,yh), (xh,yl), (xh,yh) of each column in coarse plane 0
  const T* __restrict__ c0 = coarse + off(gc, 0, 0, 0);
#pragma unroll
  for (int v = 0; v < V; ++v) {
    int xl, xh;
    bracket(i + v, J.rc[0], gc.n1, xl, xh, mx[v]);
    wx0[v] = J.cI[0][2 * (i + v)];
    wx1[v] = J.cI[0][2 * (i + v) + 1];
    o[v][0] = xl + gc.nx * yl;
    o[v][1] = xl + gc.nx * yh;
    o[v][2] = xh + gc.nx * yl;
    o[v][3] = xh + gc.nx * yh;
  }
  // coarse planes zl (P0) and zl + 1 (P1) of the current fine plane, kept while k advances
  int zcur = -1;
  bool have1 = false;
  T P0[V][4], P1[V][4];
  auto load = [&](int z, T (&w)[V][4]) {
    const T* __restrict__ cz = c0 + (long long)z * gc.nxy;
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int c = 0; c < 4; ++c) w[v][c] = cz[o[v][c]];
  };
  long long p = off(g, i, j, k0);
  for (int k = k0; k <= k1; ++k, p += g.nxy) {
    int zl, zh;
    bool mz;
    bracket(k, J.rc[2], gc.n3, zl, zh, mz);
    if (zl != zcur) {
      const int nxt = zcur + 1 > gc.n3 ? 1 : zcur + 1;
      if (zcur >= 0 && have1 && zl == nxt) {
#pragma unroll
        for (int v = 0; v < V; ++v)
#pragma unroll
          for (int c = 0; c < 4; ++c) P0[v][c] = P1[v][c];
      } else {
        load(zl, P0);
      }
      zcur = zl;
      have1 = false;
    }
    if (mz && !have1) {
      load(zh, P1);
      have1 = true;
    }
    const T wz0 = cI3[2 * k], wz1 = cI3[2 * k + 1];
    T f[V];
    if constexpr (V > 1)
      vload(fine + p, f);
    else
      f[0] = fine[p];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      T Z[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) Z[c] = pmix(mz, wz0, P0[v][c], wz1, P1[v][c]);
      const T Yl = pmix(my, wy0, Z[0], wy1, Z[1]);  // x = xl
      const T Yh = pmix(my, wy0, Z[2], wy1, Z[3]);  // x = xh
      f[v] = f[v] + pmix(mx[v], wx0[v], Yl, wx1[v], Yh);
    }
    if constexpr (V > 1)
      vstore(dst + p, f);
    else
      dst[p] = f[0];
  }
}

// The same for V > 1 fine columns i .. i+V-1 (i odd) when x is coarsened by 2: they span only
// V/2 + 1 coarse columns, so each coarse plane costs (V/2 + 1) x 2 loads instead of 4 V; every
// fine point sees the same operations in the same order as in prolong_cols.
template <typename T, int V>
__device__ __forceinline__ void prolong_cols_x2(const LevelJob<T>& J, const Geom& g, int i, int j, int k0, int k1,
                                                T* __restrict__ dst) {
  constexpr int NC = V / 2 + 1;
  const Geom gc = J.gc;
  const T* __restrict__ cI3 = J.cI[2];
  const T* __restrict__ fine = J.B;
  int yl, yh;
  bool my;
  bracket(j, J.rc[1], gc.n2, yl, yh, my);
  const T wy0 = J.cI[1][2 * j], wy1 = J.cI[1][2 * j + 1];
  T wx0[V], wx1[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    wx0[v] = J.cI[0][2 * (i + v)];
    wx1[v] = J.cI[0][2 * (i + v) + 1];
  }
  const int a = (i + 1) / 2;  // coarse column of fine column i
  int oc[NC][2];
#pragma unroll
  for (int m = 0; m < NC; ++m) {
    const int cx = a + m > gc.n1 ? a + m - gc.n1 : a + m;
    oc[m][0] = cx + gc.nx * yl;
    oc[m][1] = cx + gc.nx * yh;
  }
  const T* __restrict__ c0 = J.Bc + off(gc, 0, 0, 0);
  int zcur = -1;
  bool have1 = false;
  T P0[NC][2], P1[NC][2];
  auto load = [&](int z, T (&w)[NC][2]) {
    const T* __restrict__ cz = c0 + (long long)z * gc.nxy;
#pragma unroll
    for (int m = 0; m < NC; ++m) {
      w[m][0] = cz[oc[m][0]];
      w[m][1] = cz[oc[m][1]];
    }
  };
  // blocks of U planes: the fine vectors of the block are loaded before any store, so that each
  // thread keeps several DRAM requests in flight
  constexpr int U = 8;
  long long p = off(g, i, j, k0);
  for (int kb = k0; kb <= k1; kb += U, p += U * g.nxy) {
    const int nk = min(U, k1 - kb + 1);
    if (sizeof(T) == 4 && nk == U && J.rc[2] == 2 && (kb & 1)) {
      // FP32, a full block starting on a coincident plane: fine planes kb .. kb+U-1 lie on coarse
      // planes c .. c+U/2 (c = (kb+1)/2, periodic); all of them are loaded with the fine vectors
      // before any use, so the coarse loads no longer wait on one another (in FP64 the extra
      // registers cost more than the overlap gains)
      T f[U][V], Q[U / 2 + 1][NC][2];
#pragma unroll
      for (int u = 0; u < U; ++u) vload(fine + p + u * g.nxy, f[u]);
      const int c = (kb + 1) / 2;
#pragma unroll
      for (int m = 0; m <= U / 2; ++m) load(c + m > gc.n3 ? c + m - gc.n3 : c + m, Q[m]);
      zcur = -1;  // the plane-by-plane path below reloads what it needs
      have1 = false;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = kb + u;
        const bool mz = (u & 1) != 0;  // even fine plane: between coarse planes lo and lo + 1
        const int lo = u / 2;
        const T wz0 = cI3[2 * k], wz1 = cI3[2 * k + 1];
        T Y[NC];
#pragma unroll
        for (int m = 0; m < NC; ++m) {
          const T Zl = pmix(mz, wz0, Q[lo][m][0], wz1, Q[lo + 1 <= U / 2 ? lo + 1 : lo][m][0]);
          const T Zh = pmix(mz, wz0, Q[lo][m][1], wz1, Q[lo + 1 <= U / 2 ? lo + 1 : lo][m][1]);
          Y[m] = pmix(my, wy0, Zl, wy1, Zh);
        }
#pragma unroll
        for (int v = 0; v < V; ++v)
          f[u][v] = f[u][v] + ((v & 1) ? pmix(true, wx0[v], Y[(v - 1) / 2], wx1[v], Y[(v + 1) / 2]) : Y[v / 2]);
        vstore(dst + p + u * g.nxy, f[u]);
      }
      continue;
    }
    T f[U][V];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (u < nk) vload(fine + p + u * g.nxy, f[u]);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u >= nk) continue;
      const int k = kb + u;
      int zl, zh;
      bool mz;
      bracket(k, J.rc[2], gc.n3, zl, zh, mz);
      if (zl != zcur) {
        const int nxt = zcur + 1 > gc.n3 ? 1 : zcur + 1;
        if (zcur >= 0 && have1 && zl == nxt) {
#pragma unroll
          for (int m = 0; m < NC; ++m) {
            P0[m][0] = P1[m][0];
            P0[m][1] = P1[m][1];
          }
        } else {
          load(zl, P0);
        }
        zcur = zl;
        have1 = false;
      }
      if (mz && !have1) {
        load(zh, P1);
        have1 = true;
      }
      const T wz0 = cI3[2 * k], wz1 = cI3[2 * k + 1];
      T Y[NC];
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        const T Zl = pmix(mz, wz0, P0[m][0], wz1, P1[m][0]);
        const T Zh = pmix(mz, wz0, P0[m][1], wz1, P1[m][1]);
        Y[m] = pmix(my, wy0, Zl, wy1, Zh);
      }
#pragma unroll
      for (int v = 0; v < V; ++v)  // even v: coincident with coarse column v/2; odd v: between two
        f[u][v] = f[u][v] + ((v & 1) ? pmix(true, wx0[v], Y[(v - 1) / 2], wx1[v], Y[(v + 1) / 2]) : Y[v / 2]);
      vstore(dst + p + u * g.nxy, f[u]);
    }
  }
}

// this (fine) level: B += P Bc (interpolate, mod_solvers.f90:955-1141); with flip, C = B + P Bc
// (B unchanged) for the fused smoothing that follows.  Latency-bound: FP32 runs at 3 blocks per
// SM (80 registers, a few spilled: 0.22 against 0.24 ms at 384 x 384 x 768), FP64 at 2 (its
// spills at 3 cost more than the warps gain)
template <typename T>
__global__ void __launch_bounds__(ENT, sizeof(T) == 4 ? 3 : 2) k_lv_prolong(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                    int nj, int ntiles, int flip) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1, J.vw);
    if (i > g.n1 || j > g.n2) continue;
    T* dst = flip ? J.C : J.B;
    if (J.vw > 1 && J.rc[0] == 2) {
      prolong_cols_x2<T, VecT<T>::W>(J, g, i, j, k0, k1, dst);
    } else {
      for (int v = 0; v < J.vw; ++v) prolong_cols<T, 1>(J, g, i + v, j, k0, k1, dst);
    }
  }
}

// ------------------------------------------------------------------------------------------
// fused V-cycle smoothing: the sweeps of one smoothing phase (and the residual after them) in
// one z-march
// ------------------------------------------------------------------------------------------
// Stage 0 is the start iterate x0 (INIT: the init sweep omega A / diag, computed from A; else
// read from C), stages 1..NSW are damped-Jacobi sweeps and, with RES, stage NSW + 1 is the
// residual A - cdg(x_NSW).  A block covers an input region of W0 x H0 = 16 V x 32 columns
// (V = 16 bytes / element size): each half-warp is one row, thread (l, ty) owning the V
// consecutive columns x = V (l mod 16) .. + V-1 of row y = 2 ty + l / 16 for the whole march
// (MNT = 512 threads: 32 rows).
// With S stencil stages the outputs are the X x Y = (W0 - 2S) x (H0 - 2S) interior columns
// (stage s is valid on the region shrunk by s on every side).  At each step the block takes one
// new plane of A (and of C) -- staged by cp.async MPF planes ahead, each thread its own columns
// -- and advances every stage by one plane, stage s lagging s planes behind the newest: stage s
// at plane k needs stage s-1 at k-1..k+1 of its own columns (register windows), at k of the x
// neighbours (its own registers, or the next lane's by a shuffle) and of the y neighbours
// (16-byte rows published in shared memory one step earlier), so one barrier per step suffices.
// Every point is evaluated with the operations of the one-sweep kernels (jres / jsweep / jinit
// / jresid), so the fused phase gives the same iterate bit for bit.
// Outputs: PRE (INIT, RES): B = x_NSW and C = residual; POST: B = x_NSW.
constexpr int MPF = 2;  // planes staged ahead of the newest one in use
const dim3 kMBlock(32, MNT / 32);
static_assert(MNT / 32 <= 16, "one named barrier per pair of neighbouring warps (ids 1..15)");
// named barrier `id` (1..15) of two warps, every thread of both warps arriving
__device__ __forceinline__ void bar_pair(int id) { asm volatile("bar.sync %0, 64;\n" ::"r"(id) : "memory"); }

template <typename T, int S, bool INIT>
struct MLayout {
  static constexpr int V = VecT<T>::W;
  static constexpr int W0 = 16 * V, H0 = 2 * MNT / 32, R0 = W0 * H0;
  static constexpr int NBR = S + 1 + MPF;  // A ring: planes t-S .. t+MPF
  static constexpr int NCR = MPF + 1;      // C ring (POST): planes t .. t+MPF
  static constexpr int pub() { return 0; }                   // 2 slots x S stages x R0
  static constexpr int rhs() { return 2 * S * R0; }         // NBR x R0
  static constexpr int cin() { return rhs() + NBR * R0; }   // NCR x R0 (POST only)
  static constexpr int total() { return cin() + (INIT ? 0 : NCR * R0); }
};
template <typename T, int NSW, bool INIT, bool RES>
constexpr size_t multi_smem_bytes() {
  return sizeof(T) * (size_t)MLayout<T, NSW + (RES ? 1 : 0), INIT>::total();
}

// periodic image of index i in 1..n, for any integer i
__device__ __forceinline__ int wrapn(int i, int n) {
  int r = (i - 1) % n;
  if (r < 0) r += n;
  return r + 1;
}
// 16-byte shared-memory vectors
template <typename T>
__device__ __forceinline__ void sload(const T* p, T (&o)[VecT<T>::W]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  } else {
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x;
    o[1] = v.y;
  }
}

// FAST: every job of the list has n1 divisible by V and uniform z.  The region then starts HX =
// S rounded up to V columns left of the tile, so that every thread's V columns are one aligned
// 16-byte vector of the field (a periodic wrap never splits it): one 16-byte cp.async per plane
// and vector stores of the outputs; the z coefficients are constants.  Otherwise HX = S and
// every column moves on its own.
template <typename T, int NSW, bool INIT, bool RES, bool FAST>
__global__ void __launch_bounds__(MNT, 1) k_lv_multi(const LevelJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                     int nj, int ntiles, T omega) {
  constexpr int S = NSW + (RES ? 1 : 0);
  using LY = MLayout<T, S, INIT>;
  constexpr int V = LY::V;
  constexpr int W0 = LY::W0, H0 = LY::H0, R0 = LY::R0, NBR = LY::NBR, NCR = LY::NCR;
  constexpr int HX = FAST ? (S + V - 1) / V * V : S;  // x halo of the region
  constexpr int X = W0 - 2 * HX, Y = H0 - 2 * S;
  extern __shared__ __align__(16) unsigned char lm_raw[];
  T* const sm = reinterpret_cast<T*>(lm_raw);
  T* const pub = sm + LY::pub();  // pub[(slot * S + s) * R0 + y * W0 + x]
  T* const br = sm + LY::rhs();
  T* const cr = sm + LY::cin();
  const int x0 = V * (threadIdx.x & 15);               // this thread's first column in the region
  const int y = 2 * threadIdx.y + (threadIdx.x >> 4);  // and its row
  const int e0 = y * W0 + x0;
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    const LevelJob<T>& J = jobs[q];
    if (e_halted(J.sc)) continue;
    const Geom g = J.g;
    const int kc = J.kc;
    const int ntx = (g.n1 + X - 1) / X, nty = (g.n2 + Y - 1) / Y;
    const int t0 = b - ts[q];
    const int ta = t0 % ntx, tr = t0 / ntx, tc = tr / nty;
    const int i0 = ta * X + 1, j0 = (tr - tc * nty) * Y + 1;  // first output column of the tile
    const int k0 = tc * kc + 1, k1 = min(g.n3, k0 + kc - 1);
    const int nq = (k1 - k0 + 1) + 2 * S;  // planes k0-S .. k1+S
    const T* __restrict__ cz = J.cdg[2];
    const bool zu = FAST || J.zuni != 0;
    T a0[V], a1[V], a2[V], inv[V];
    int xo[V];
#pragma unroll
    for (int c = 0; c < V; ++c) {
      const int gi = wrapn(i0 - HX + x0 + c, g.n1);
      a0[c] = J.cdg[0][3 * (gi - 1)];
      a1[c] = J.cdg[0][3 * (gi - 1) + 1];
      a2[c] = J.cdg[0][3 * (gi - 1) + 2];
      xo[c] = gi + 3;
    }
    const int gj = wrapn(j0 - S + y, g.n2);
    const T b0 = J.cdg[1][3 * (gj - 1)], b1 = J.cdg[1][3 * (gj - 1) + 1], b2 = J.cdg[1][3 * (gj - 1) + 2];
    const int yo = g.nx * (gj + 3);
    const T zcm = cz[0], zcc = cz[1], zcp = cz[2];  // the z row of a uniform z axis
#pragma unroll
    for (int c = 0; c < V; ++c) inv[c] = zu ? omega / (a1[c] + b1 + zcc) : T(0);
    // FP32 fast path: the point operations on packed pairs (columns 0,1 and 2,3; fma.rn.f32x2
    // and mul.rn.f32x2 lanes are the scalar operations, so the iterate is the same bit for bit)
    constexpr bool PAIRS = FAST && sizeof(T) == 4;
    float2 pna0[2], pna2[2], pa0[2], pa2[2], pinv[2], pdg[2];
    if constexpr (PAIRS) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        pa0[h] = make_float2(a0[2 * h], a0[2 * h + 1]);
        pa2[h] = make_float2(a2[2 * h], a2[2 * h + 1]);
        pna0[h] = make_float2(-a0[2 * h], -a0[2 * h + 1]);
        pna2[h] = make_float2(-a2[2 * h], -a2[2 * h + 1]);
        pinv[h] = make_float2(inv[2 * h], inv[2 * h + 1]);
        pdg[h] = make_float2(a1[2 * h] + b1 + zcc, a1[2 * h + 1] + b1 + zcc);
      }
    }
    // outputs of this thread: columns i = io + c of row jo, when its vector lies in the tile interior
    const int io = i0 + x0 - HX, jo = j0 + y - S;
    const bool rowout = y >= S && y < H0 - S && jo <= g.n2;
    const long long obase = (long long)(io + 3) + (long long)g.nx * (jo + 3);
    const T* __restrict__ Ab = J.A + yo + (FAST ? xo[0] : 0);
    const T* __restrict__ Cb = J.C + yo + (FAST ? xo[0] : 0);
    int kin = wrapn(k0 - S, g.n3);  // wrapped plane of the next stage_in
    auto stage_in = [&](int qq) {  // plane qq of A (and of C) at this thread's columns
      if (qq < nq) {
        const long long zo = (long long)(kin + 3) * g.nxy;
        kin = kin == g.n3 ? 1 : kin + 1;
        T* bd = br + (qq % NBR) * R0 + e0;
        T* cd = cr + (qq % NCR) * R0 + e0;
        if constexpr (FAST) {
          cp_async16(bd, Ab + zo);
          if (!INIT) cp_async16(cd, Cb + zo);
        } else {
#pragma unroll
          for (int c = 0; c < V; ++c) {
            cp_async1(bd + c, Ab + zo + xo[c]);
            if (!INIT) cp_async1(cd + c, Cb + zo + xo[c]);
          }
        }
      }
      cp_commit();
    };
#pragma unroll
    for (int qq = 0; qq < MPF; ++qq) stage_in(qq);
    // register windows: stage s at plane p of column x0 + c lives in Qz[s][c][p % 3]
    T Qz[S][V][3];
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
      for (int c = 0; c < V; ++c) Qz[s][c][0] = Qz[s][c][1] = Qz[s][c][2] = T(0);
    // A warp (rows 2w, 2w+1) reads, of the rows other warps publish, only rows 2w-1 and 2w+2, and
    // its own rows are read only by warps w-1 and w+1: a step need not wait for the whole block,
    // only for those two warps.  Warps w, w+1 meet on named barrier w+1 (64 threads, ids 1..15;
    // 0 is __syncthreads); even warps meet their upper neighbour first, odd warps their lower one,
    // so every pair completes in one of two rounds and no cycle of waits can form.  Neighbouring
    // warps are never more than one step apart, so the two publication slots suffice.
    const int wid = threadIdx.y;  // warp-uniform
    auto sync_rows = [&]() {
      const bool lo = wid > 0, hi = wid + 1 < MNT / 32;
      if (wid & 1) {
        if (lo) bar_pair(wid);
        if (hi) bar_pair(wid + 1);
      } else {
        if (hi) bar_pair(wid + 1);
        if (lo) bar_pair(wid);
      }
    };
    // one step; R = t % 3 at compile time, so that every window slot is a fixed register
    auto step = [&](int t, auto rt) {
      constexpr int R = decltype(rt)::value;
      cp_wait<MPF - 1>();  // this thread's copies of plane t have landed (only it reads them)
      sync_rows();         // the rows published at step t-1 are visible; slot t%2 is free again
      stage_in(t + MPF);
      const int wslot = t & 1, rslot = wslot ^ 1;
      {  // stage 0 at plane t
        const T cc = zu ? zcc : cz[3 * (wrapn(k0 - S + t, g.n3) - 1) + 1];
        T v[V];
        sload(INIT ? br + (t % NBR) * R0 + e0 : cr + (t % NCR) * R0 + e0, v);
#pragma unroll
        for (int c = 0; c < V; ++c) {
          if (INIT) v[c] = jinit(v[c], omega, zu, inv[c], a1[c] + b1 + cc);
          Qz[0][c][R] = v[c];
        }
        vstore(pub + (wslot * S + 0) * R0 + e0, v);
      }
#pragma unroll
      for (int s = 1; s <= S; ++s) {
        const int qs = t - s;  // plane of stage s at this step (block-uniform)
        // window slots of stage s-1 at planes qs-1, qs, qs+1 and of stage s at qs
        const int sm1 = ((R - s - 1) % 3 + 3) % 3, s0 = ((R - s) % 3 + 3) % 3, sp1 = ((R - s + 1) % 3 + 3) % 3;
        if (qs >= s) {
          const bool rowin = y >= s && y < H0 - s;  // the row lies inside stage s's region
          const T* pr = pub + (rslot * S + (s - 1)) * R0;  // stage s-1 at plane qs (published at t-1)
          const int kk = k0 - S + qs;  // unwrapped; the outputs (s == S) lie in k0..k1
          T cm = zcm, cc = zcc, cp = zcp;
          if (!zu) {
            const int k3 = 3 * (wrapn(kk, g.n3) - 1);
            cm = cz[k3];
            cc = cz[k3 + 1];
            cp = cz[k3 + 2];
          }
          // x neighbours across vectors: every lane takes part in the shuffles
          const T wl = __shfl_up_sync(0xffffffffu, Qz[s - 1][V - 1][s0], 1, 16);  // column x0 - 1
          const T er = __shfl_down_sync(0xffffffffu, Qz[s - 1][0][s0], 1, 16);    // column x0 + V
          T ov[V];
#pragma unroll
          for (int c = 0; c < V; ++c) ov[c] = T(0);
          if (rowin) {
            T so[V], no[V], bv[V];
            sload(pr + e0 - W0, so);
            sload(pr + e0 + W0, no);
            sload(br + (qs % NBR) * R0 + e0, bv);
            T rv[V];
            if constexpr (PAIRS) {
              // jres / jsweep / jresid of columns 2h, 2h+1 (fast path: z uniform, cc = zcc)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int c = 2 * h;
                const float2 zm = make_float2(Qz[s - 1][c][sm1], Qz[s - 1][c + 1][sm1]);
                const float2 zc = make_float2(Qz[s - 1][c][s0], Qz[s - 1][c + 1][s0]);
                const float2 zp = make_float2(Qz[s - 1][c][sp1], Qz[s - 1][c + 1][sp1]);
                const float2 w = make_float2(c == 0 ? wl : Qz[s - 1][c - 1][s0], Qz[s - 1][c][s0]);
                const float2 ea = make_float2(Qz[s - 1][c + 1][s0], c + 1 == V - 1 ? er : Qz[s - 1][c + 2][s0]);
                const float2 bb2 = make_float2(bv[c], bv[c + 1]);
                const float2 so2 = make_float2(so[c], so[c + 1]), no2 = make_float2(no[c], no[c + 1]);
                if (RES && s == S) {
                  float2 l = __fmul2_rn(pa0[h], w);
                  l = __ffma2_rn(pa2[h], ea, l);
                  l = __ffma2_rn(make_float2(b0, b0), so2, l);
                  l = __ffma2_rn(make_float2(b2, b2), no2, l);
                  l = __ffma2_rn(make_float2(cm, cm), zm, l);
                  l = __ffma2_rn(make_float2(cp, cp), zp, l);
                  l = __ffma2_rn(pdg[h], zc, l);
                  const float2 r = __ffma2_rn(make_float2(-1.f, -1.f), l, bb2);  // bv - l
                  rv[c] = r.x;
                  rv[c + 1] = r.y;
                  ov[c] = zc.x;
                  ov[c + 1] = zc.y;
                } else {
                  float2 r = __ffma2_rn(pna0[h], w, bb2);
                  r = __ffma2_rn(pna2[h], ea, r);
                  r = __ffma2_rn(make_float2(-b0, -b0), so2, r);
                  r = __ffma2_rn(make_float2(-b2, -b2), no2, r);
                  r = __ffma2_rn(make_float2(-cm, -cm), zm, r);
                  r = __ffma2_rn(make_float2(-cp, -cp), zp, r);
                  const float2 o = __ffma2_rn(make_float2(1.f - omega, 1.f - omega), zc, __fmul2_rn(r, pinv[h]));
                  ov[c] = o.x;
                  ov[c + 1] = o.y;
                }
              }
            } else {
#pragma unroll
              for (int c = 0; c < V; ++c) {
                const T zm = Qz[s - 1][c][sm1], zc = Qz[s - 1][c][s0], zp = Qz[s - 1][c][sp1];
                const T w = c == 0 ? wl : Qz[s - 1][c - 1][s0];
                const T ea = c == V - 1 ? er : Qz[s - 1][c + 1][s0];
                if (RES && s == S) {
                  rv[c] = jresid(bv[c], a0[c], w, a2[c], ea, b0, so[c], b2, no[c], cm, zm, cp, zp, a1[c] + b1 + cc, zc);
                  ov[c] = zc;
                } else {
                  const T rr = jres(bv[c], a0[c], w, a2[c], ea, b0, so[c], b2, no[c], cm, zm, cp, zp);
                  ov[c] = jsweep(rr, zc, omega, zu, inv[c], a1[c] + b1 + cc);
                }
              }
            }
            if (s == S && rowout) {  // the outputs: B = the last sweep (or x_NSW), C = the residual
              const long long ob = obase + (long long)g.nxy * (kk + 3);
              if constexpr (FAST) {
                if (x0 >= HX && x0 < W0 - HX && io <= g.n1) {
                  vstore(J.B + ob, ov);
                  if (RES) vstore(J.C + ob, rv);
                }
              } else {
#pragma unroll
                for (int c = 0; c < V; ++c)
                  if (x0 + c >= HX && x0 + c < W0 - HX && io + c <= g.n1) {
                    J.B[ob + c] = ov[c];
                    if (RES) J.C[ob + c] = rv[c];
                  }
              }
            }
          }
          if (s < S) {
#pragma unroll
            for (int c = 0; c < V; ++c) Qz[s][c][s0] = ov[c];
            vstore(pub + (wslot * S + s) * R0 + e0, ov);
          }
        }
      }
    };
    int t = 0;
    for (; t + 2 < nq; t += 3) {
      step(t, std::integral_constant<int, 0>{});
      step(t + 1, std::integral_constant<int, 1>{});
      step(t + 2, std::integral_constant<int, 2>{});
    }
    if (t < nq) step(t, std::integral_constant<int, 0>{});
    if (t + 1 < nq) step(t + 1, std::integral_constant<int, 1>{});
    cp_wait<0>();
    __syncthreads();  // the rings are rewritten by the next tile
  }
}

// ------------------------------------------------------------------------------------------
// coarse tail of the V-cycle in one block per case
// ------------------------------------------------------------------------------------------
// The coarsest levels of a case (lt .. lt + nl - 1, every field of them together within
// TAIL_BYTES of shared memory) run their whole part of the V-cycle in one block: the
// right-hand side of level lt comes from global memory (the restriction into it), every later
// phase -- init sweep, sweeps and residual of each level, the restriction to the next, the
// bottom sweeps, the prolongation back and the sweeps after it -- works on shared-memory copies,
// one barrier per phase, and the final iterate of level lt goes back to global memory for the
// prolongation into level lt - 1.  On a 384 x 384 x 768 case these levels are 12 x 12 x 24 and
// smaller, whose one-launch-per-phase schedule is some 25 launches of a few microseconds each.
// Every point sees the operations of the per-level kernels (jinit / jres / jsweep / jresid,
// restrict7, pmix), so the V-cycle is the same bit for bit.
// With cheb > 0 the coarsest level gets cheb steps of the Chebyshev semi-iteration of the
// Jacobi-scaled operator D^-1 A (D = diag A) from x = 0 instead of its Jacobi sweeps, for the
// eigenvalue interval [lmin, 2] (Gershgorin bounds D^-1 A by 2; lmin from the level's geometry):
//   x_1 = x_0 + g z_0,  x_{k+1} = w_{k+1} (x_k + g z_k - x_{k-1}) + x_{k-1},  z_k = D^-1 (b - A x_k),
//   g = 2 / (lmin + 2), s = (2 - lmin) / (2 + lmin), w_2 = 2 / (2 - s^2), w_{k+1} = 1 / (1 - s^2 w_k / 4)
// (the Chebyshev semi-iterative method, Golub and Varga 1961): the error polynomial is the scaled
// Chebyshev polynomial of degree cheb on the interval, bounded by 1 on [0, 2], so the smooth
// modes that damped Jacobi removes in O(n^2) sweeps fall in O(n) steps, and the preconditioner
// stays a fixed linear operator.  Such a tail may be the coarsest level alone.
constexpr int TNT = 512;
constexpr size_t TAIL_BYTES = 200 * 1024;
template <typename T>
struct TailJob {
  int nl;                          // levels in the tail (>= 2; >= 1 with cheb)
  int cheb;                        // Chebyshev steps on the coarsest level (0: Jacobi sweeps)
  T cgam, csig2;                   // their g and s^2
  LevelJob<T> lv[MG_MAX_LEVELS];   // their level jobs; lv[0].A / lv[0].B are the global fields
};

// the cells idx = tid, tid + TNT, ... of an n1 x n2 x n3 level with their 1-based (i, j, k),
// advanced by carries instead of one division per cell
template <typename F>
__device__ __forceinline__ void tail_cells(const Geom& g, F&& f) {
  const int m = g.n1 * g.n2 * g.n3;
  int idx = threadIdx.x;
  int i = idx % g.n1, r = idx / g.n1, j = r % g.n2, k = r / g.n2;
  const int di = TNT % g.n1, r2 = TNT / g.n1, dj = r2 % g.n2, dk = r2 / g.n2;
  for (; idx < m; idx += TNT) {
    f(idx, i + 1, j + 1, k + 1);
    i += di;
    const int ci = i >= g.n1;
    if (ci) i -= g.n1;
    j += dj + ci;
    const int cj = j >= g.n2;
    if (cj) j -= g.n2;
    k += dk + cj;
  }
}

template <typename T>
__global__ void __launch_bounds__(TNT, 1) k_lv_tail(const TailJob<T>* __restrict__ jobs, const int* __restrict__ ts,
                                                    int nj, int ntiles, T omega, int n_down, int n_up, int n_bottom) {
  extern __shared__ __align__(16) unsigned char tl_raw[];
  T* const sm = reinterpret_cast<T*>(tl_raw);
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q0 = find_job(ts, nj, b);
    const TailJob<T>& TJ = jobs[q0];
    if (e_halted(TJ.lv[0].sc)) continue;
    const int nl = TJ.nl;
    // shared-memory arrays of level q: A, X0, X1 (compact, i fastest)
    T* Aq[MG_MAX_LEVELS];
    T* X0[MG_MAX_LEVELS];
    T* X1[MG_MAX_LEVELS];
    int cur[MG_MAX_LEVELS];  // which of X0 / X1 holds the level's iterate
    {
      size_t o = 0;
      for (int q = 0; q < nl; ++q) {
        const Geom& g = TJ.lv[q].g;
        const size_t m = (size_t)g.n1 * g.n2 * g.n3;
        Aq[q] = sm + o;
        X0[q] = sm + o + m;
        X1[q] = sm + o + 2 * m;
        o += 3 * m;
        cur[q] = 0;
      }
    }
    auto X = [&](int q, int which) { return which ? X1[q] : X0[q]; };
    // right-hand side of the first level from global memory
    {
      const Geom& g = TJ.lv[0].g;
      T* a0 = Aq[0];
      const T* src = TJ.lv[0].A;
      tail_cells(g, [&](int idx, int i, int j, int k) { a0[idx] = src[off(g, i, j, k)]; });
    }
    __syncthreads();
    // OP 0: dst = init(A); 1: dst = sweep(A, src); 2: dst = A - cdg(src)
    auto relax = [&](int q, int op, const T* src, T* dst) {
      const LevelJob<T>& J = TJ.lv[q];
      const Geom& g = J.g;
      const bool zu = J.zuni != 0;
      const T* __restrict__ cz = J.cdg[2];
      const T* a = Aq[q];
      tail_cells(g, [&](int idx, int i, int j, int k) {
        const T a0 = J.cdg[0][3 * (i - 1)], a1 = J.cdg[0][3 * (i - 1) + 1], a2 = J.cdg[0][3 * (i - 1) + 2];
        const T b0 = J.cdg[1][3 * (j - 1)], b1 = J.cdg[1][3 * (j - 1) + 1], b2 = J.cdg[1][3 * (j - 1) + 2];
        const T cm = zu ? cz[0] : cz[3 * (k - 1)], cc = zu ? cz[1] : cz[3 * (k - 1) + 1],
                cp = zu ? cz[2] : cz[3 * (k - 1) + 2];
        const T inv = zu ? omega / (a1 + b1 + cz[1]) : T(0);
        const T diag = a1 + b1 + cc;
        if (op == 0) {
          dst[idx] = jinit(a[idx], omega, zu, inv, diag);
          return;
        }
        const int im = i == 1 ? idx + g.n1 - 1 : idx - 1, ip = i == g.n1 ? idx - g.n1 + 1 : idx + 1;
        const int sy = g.n1, sz = g.n1 * g.n2;
        const int jm = j == 1 ? idx + (g.n2 - 1) * sy : idx - sy, jp = j == g.n2 ? idx - (g.n2 - 1) * sy : idx + sy;
        const int km = k == 1 ? idx + (g.n3 - 1) * sz : idx - sz, kp = k == g.n3 ? idx - (g.n3 - 1) * sz : idx + sz;
        const T zc = src[idx];
        if (op == 1) {
          const T rr = jres(a[idx], a0, src[im], a2, src[ip], b0, src[jm], b2, src[jp], cm, src[km], cp, src[kp]);
          dst[idx] = jsweep(rr, zc, omega, zu, inv, diag);
        } else {
          dst[idx] = jresid(a[idx], a0, src[im], a2, src[ip], b0, src[jm], b2, src[jp], cm, src[km], cp, src[kp], diag, zc);
        }
      });
      __syncthreads();
    };
    // n sweeps of level q (after an init sweep when init): the iterate moves between X0 and X1
    auto smooth = [&](int q, int init, int n) {
      for (int w = 0; w < n; ++w) {
        if (init && w == 0) {
          relax(q, 0, nullptr, X(q, cur[q]));
        } else {
          relax(q, 1, X(q, cur[q]), X(q, cur[q] ^ 1));
          cur[q] ^= 1;
        }
      }
    };
    // the residual of level q (in its spare buffer) restricted into the right-hand side of q + 1
    auto restrict_down = [&](int q) {
      const LevelJob<T>& C = TJ.lv[q + 1];
      const Geom& gf = TJ.lv[q].g;
      const Geom& g = C.g;
      const T* d = X(q, cur[q] ^ 1);
      T* aq = Aq[q + 1];
      tail_cells(g, [&](int idx, int i, int j, int k) {
        const int fi = C.rf[0] * (i - 1) + 1, fj = C.rf[1] * (j - 1) + 1, fk = C.rf[2] * (k - 1) + 1;
        auto at = [&](int a, int bq, int c) { return d[(a - 1) + gf.n1 * ((bq - 1) + gf.n2 * (c - 1))]; };
        aq[idx] = restrict7(at(fi, fj, fk), at(wrapi(fi - 1, gf.n1), fj, fk), at(wrapi(fi + 1, gf.n1), fj, fk),
                            at(fi, wrapi(fj - 1, gf.n2), fk), at(fi, wrapi(fj + 1, gf.n2), fk),
                            at(fi, fj, wrapi(fk - 1, gf.n3)), at(fi, fj, wrapi(fk + 1, gf.n3)));
      });
      __syncthreads();
    };
    // spare buffer of level q = its iterate + P (iterate of q + 1); then it holds the iterate
    auto prolong_up = [&](int q) {
      const LevelJob<T>& J = TJ.lv[q];
      const Geom& g = J.g;
      const Geom& gc = TJ.lv[q + 1].g;
      const T* xf = X(q, cur[q]);
      const T* xc = X(q + 1, cur[q + 1]);
      T* out = X(q, cur[q] ^ 1);
      tail_cells(g, [&](int idx, int i, int j, int k) {
        int xl, xh, yl, yh, zl, zh;
        bool mx, my, mz;
        bracket(i, J.rc[0], gc.n1, xl, xh, mx);
        bracket(j, J.rc[1], gc.n2, yl, yh, my);
        bracket(k, J.rc[2], gc.n3, zl, zh, mz);
        auto P = [&](int a, int bq, int c) { return xc[(a - 1) + gc.n1 * ((bq - 1) + gc.n2 * (c - 1))]; };
        const T wz0 = J.cI[2][2 * k], wz1 = J.cI[2][2 * k + 1];
        const T wy0 = J.cI[1][2 * j], wy1 = J.cI[1][2 * j + 1];
        const T wx0 = J.cI[0][2 * i], wx1 = J.cI[0][2 * i + 1];
        const T Z0 = pmix(mz, wz0, P(xl, yl, zl), wz1, P(xl, yl, zh));
        const T Z1 = pmix(mz, wz0, P(xl, yh, zl), wz1, P(xl, yh, zh));
        const T Z2 = pmix(mz, wz0, P(xh, yl, zl), wz1, P(xh, yl, zh));
        const T Z3 = pmix(mz, wz0, P(xh, yh, zl), wz1, P(xh, yh, zh));
        const T Yl = pmix(my, wy0, Z0, wy1, Z1);
        const T Yh = pmix(my, wy0, Z2, wy1, Z3);
        out[idx] = xf[idx] + pmix(mx, wx0, Yl, wx1, Yh);
      });
      cur[q] ^= 1;
      __syncthreads();
    };
    for (int q = 0; q + 1 < nl; ++q) {  // relax_restrict
      smooth(q, 1, n_down);
      relax(q, 2, X(q, cur[q]), X(q, cur[q] ^ 1));
      restrict_down(q);
    }
    if (TJ.cheb > 0) {  // Chebyshev semi-iteration on the coarsest level, from x = 0
      const int q = nl - 1;
      const LevelJob<T>& J = TJ.lv[q];
      const Geom& g = J.g;
      const bool zu = J.zuni != 0;
      const T* __restrict__ cz = J.cdg[2];
      const T* a = Aq[q];
      T* x0 = X0[q];
      T* x1 = X1[q];
      tail_cells(g, [&](int idx, int, int, int) { x0[idx] = T(0); x1[idx] = T(0); });
      __syncthreads();
      const T gam = TJ.cgam, s2 = TJ.csig2;
      T w = T(1);
      for (int it = 0; it < TJ.cheb; ++it) {
        w = it == 0 ? T(1) : (it == 1 ? T(2) / (T(2) - s2) : T(1) / (T(1) - s2 * w / T(4)));
        const T* src = X(q, cur[q]);
        T* dst = X(q, cur[q] ^ 1);  // holds x_{k-1} (x_0 = 0 on the first step)
        tail_cells(g, [&](int idx, int i, int j, int k) {
          const T a0 = J.cdg[0][3 * (i - 1)], a1 = J.cdg[0][3 * (i - 1) + 1], a2 = J.cdg[0][3 * (i - 1) + 2];
          const T b0 = J.cdg[1][3 * (j - 1)], b1 = J.cdg[1][3 * (j - 1) + 1], b2 = J.cdg[1][3 * (j - 1) + 2];
          const T cm = zu ? cz[0] : cz[3 * (k - 1)], cc = zu ? cz[1] : cz[3 * (k - 1) + 1],
                  cp = zu ? cz[2] : cz[3 * (k - 1) + 2];
          const T diag = a1 + b1 + cc;
          const int im = i == 1 ? idx + g.n1 - 1 : idx - 1, ip = i == g.n1 ? idx - g.n1 + 1 : idx + 1;
          const int sy = g.n1, sz = g.n1 * g.n2;
          const int jm = j == 1 ? idx + (g.n2 - 1) * sy : idx - sy, jp = j == g.n2 ? idx - (g.n2 - 1) * sy : idx + sy;
          const int km = k == 1 ? idx + (g.n3 - 1) * sz : idx - sz, kp = k == g.n3 ? idx - (g.n3 - 1) * sz : idx + sz;
          const T xk = src[idx];
          const T r = jresid(a[idx], a0, src[im], a2, src[ip], b0, src[jm], b2, src[jp], cm, src[km], cp, src[kp], diag, xk);
          const T xm = it == 0 ? xk : dst[idx];
          dst[idx] = xm + w * (xk + gam * r / diag - xm);
        });
        cur[q] ^= 1;
        __syncthreads();
      }
    } else {
      smooth(nl - 1, 1, n_bottom);  // relax_bottom
      smooth(nl - 1, 0, n_bottom);
    }
    for (int q = nl - 2; q >= 0; --q) {  // interpolate_relax
      prolong_up(q);
      smooth(q, 0, n_up);
    }
    {
      const Geom& g = TJ.lv[0].g;
      const T* x0 = X(0, cur[0]);
      T* dst = TJ.lv[0].B;
      tail_cells(g, [&](int idx, int i, int j, int k) { dst[off(g, i, j, k)] = x0[idx]; });
    }
    __syncthreads();  // shared memory is rewritten by the next case
  }
}

// ------------------------------------------------------------------------------------------
// mixed precision: FP64 residual / conversion / correction over the MixJob list
// ------------------------------------------------------------------------------------------
// x += e for the cases whose inner solve ended with status 0 or 1
__global__ void __launch_bounds__(ENT) k_mx_apply(const MixJob* __restrict__ jobs, const int* __restrict__ ts, int nj,
                                                  int ntiles, const SolverScalars* __restrict__ osc) {
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int q = find_job(ts, nj, b);
    if (osc[q].done) continue;
    const MixJob& J = jobs[q];
    const int st = J.isc->status;
    if ((st != 0 && st != 1) || J.isc->phi_zero) continue;  // no correction (or none written)
    const Geom g = J.g;
    int i, j, k0, k1;
    tile_at(g, J.kc, b - ts[q], i, j, k0, k1);
    if (i > g.n1 || j > g.n2) continue;
    const float* __restrict__ e = J.e32;
    double* __restrict__ x = J.x;
    long long p = off(g, i, j, k0);
#pragma unroll 4
    for (int k = k0; k <= k1; ++k, p += g.nxy) x[p] = x[p] + (double)e[p];
  }
}

// grids of the vector operator kernels: the blocks resident at once on the device (a grid-stride
// kernel given more would leave its last blocks to run after the others, one tile step behind)
int g_axv_grid = 0, g_axd_grid = 0;
// the operator kernels use more than 48 KB of dynamic shared memory: opt in once per process
// and device
void ax_attributes() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaFuncSetAttribute(k_kr_ax<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ax_smem_bytes<double>());
  cudaFuncSetAttribute(k_kr_ax<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ax_smem_bytes<double>());
  cudaFuncSetAttribute(k_kr_ax<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ax_smem_bytes<double>());
  cudaFuncSetAttribute(k_kr_ax<double, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ax_smem_bytes<double>());
  cudaFuncSetAttribute(k_kr_ax32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axa_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axa_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axa_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax64v<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axd_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax64v<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axd_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax64v<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axd_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax64v<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axd_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax32v<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axv_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax32v<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axv_smem_bytes());
  cudaFuncSetAttribute(k_kr_ax32v<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axv_smem_bytes());
  auto occ = [](auto kernel, int threads, size_t smem) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess || nb < 1) nb = 1;
    return nb;
  };
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (nsm <= 0) nsm = 148;
  g_axv_grid = nsm * std::min({occ(k_kr_ax32v<0>, AXV_NT, axv_smem_bytes()), occ(k_kr_ax32v<1>, AXV_NT, axv_smem_bytes()),
                               occ(k_kr_ax32v<2>, AXV_NT, axv_smem_bytes())});
  g_axd_grid = nsm * std::min({occ(k_kr_ax64v<0>, AXD_NT, axd_smem_bytes()), occ(k_kr_ax64v<1>, AXD_NT, axd_smem_bytes()),
                               occ(k_kr_ax64v<2>, AXD_NT, axd_smem_bytes()), occ(k_kr_ax64v<3>, AXD_NT, axd_smem_bytes())});
  cudaFuncSetAttribute(k_lv_tail<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_BYTES);
  cudaFuncSetAttribute(k_lv_tail<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_BYTES);
#define IMPACT_MULTI_ATTR(T, N, I, R)                                                                           \
  cudaFuncSetAttribute(k_lv_multi<T, N, I, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,               \
                       (int)multi_smem_bytes<T, N, I, R>());                                                    \
  cudaFuncSetAttribute(k_lv_multi<T, N, I, R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                       (int)multi_smem_bytes<T, N, I, R>())
  IMPACT_MULTI_ATTR(float, 1, true, true);
  IMPACT_MULTI_ATTR(float, 2, true, true);
  IMPACT_MULTI_ATTR(float, 2, false, false);
  IMPACT_MULTI_ATTR(float, 3, false, false);
  IMPACT_MULTI_ATTR(double, 1, true, true);
  IMPACT_MULTI_ATTR(double, 2, true, true);
  IMPACT_MULTI_ATTR(double, 2, false, false);
  IMPACT_MULTI_ATTR(double, 3, false, false);
#undef IMPACT_MULTI_ATTR
  done[dev] = true;
}

int g_sms = 0;
inline int grid_for(int ntiles) {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  const int cap = g_sms * 8;
  return ntiles < cap ? ntiles : cap;
}
const dim3 kBlock(ETX, ETY);
const dim3 kAxBlock(ETX, AXTY);  // k_kr_ax: two rows per thread
// the operator over a Krylov list: FP32 by the vector kernel for the jobs that qualify (vec:
// 1 all, 2 some), by the 16-byte staged, stepped kernel for the others; FP64 alike
template <typename T, int MODE>
void launch_ax(int grid, const KrylovJob<T>* J, const int* ts, int n, int ntiles, double* partial, cudaStream_t s,
               int vec) {
  if constexpr (std::is_same<T, float>::value && MODE <= 2) {
    const int gv = g_axv_grid > 0 ? std::min(g_axv_grid, ntiles) : grid;
    if (vec != 0) k_kr_ax32v<MODE><<<gv, dim3(AXV_TX, ETY), axv_smem_bytes(), s>>>(J, ts, n, ntiles, partial);
    if (vec != 1) k_kr_ax32<MODE><<<grid, kAxBlock, axa_smem_bytes(), s>>>(J, ts, n, ntiles, partial);
    if (vec == 2) prof::count(1);  // two launches where the callers count one
  } else {
    const int gv = g_axd_grid > 0 ? std::min(g_axd_grid, ntiles) : grid;
    if (vec != 0) k_kr_ax64v<MODE><<<gv, dim3(AXD_TX, ETY), axd_smem_bytes(), s>>>(J, ts, n, ntiles, partial);
    if (vec != 1) k_kr_ax<T, MODE><<<grid, kAxBlock, ax_smem_bytes<T>(), s>>>(J, ts, n, ntiles, partial);
    if (vec == 2) prof::count(1);
  }
}
// the fused smoothing kernel runs one block per tile (one block per SM at a time)
inline int grid_multi(int ntiles) { return ntiles; }

}  // namespace

// =========================================================================================
// host side
// =========================================================================================
void collapse_divgrad(int M, const double* cG, const double* cD, std::vector<double>& W) {
  const int n = M - 1;
  W.assign((size_t)n * AXW, 0.0);
  auto wrap = [n](int q) { return q < 1 ? q + n : (q > n ? q - n : q); };
  for (int i = 1; i <= n; ++i)
    for (int o = -5; o <= 5; ++o) {
      double s = 0.0;
      for (int a = -3; a <= 2; ++a) {
        const int bq = o - a;
        if (bq < -2 || bq > 3) continue;
        s += cD[(size_t)i * 6 + (a + 3)] * cG[(size_t)wrap(i + a) * 6 + (bq + 2)];
      }
      W[(size_t)(i - 1) * AXW + (o + 5)] = s;
    }
}

template <typename J>
int ListArena::add(const std::vector<J>& jobs, const std::vector<int>& tiles) {
  auto align = [this](size_t a) {
    while (host.size() % a) host.push_back(0);
  };
  DevList L;
  L.njobs = (int)jobs.size();
  align(16);
  ts_off.push_back(host.size());
  int acc = 0;
  std::vector<int> ts(jobs.size() + 1);
  for (size_t q = 0; q < jobs.size(); ++q) {
    ts[q] = acc;
    acc += tiles[q];
  }
  ts[jobs.size()] = acc;
  L.ntiles = acc;
  const unsigned char* tb = reinterpret_cast<const unsigned char*>(ts.data());
  host.insert(host.end(), tb, tb + ts.size() * sizeof(int));
  align(16);
  job_off.push_back(host.size());
  const unsigned char* jb = reinterpret_cast<const unsigned char*>(jobs.data());
  host.insert(host.end(), jb, jb + jobs.size() * sizeof(J));
  lists.push_back(L);
  return (int)lists.size() - 1;
}

int ListArena::upload(cudaStream_t s) {
  if (dev) {
    cudaFree(dev);
    dev = nullptr;
  }
  if (host.empty()) return 0;
  cudaError_t e = cudaMalloc((void**)&dev, host.size());
  if (e != cudaSuccess) return impact_set_error(e, "cudaMalloc (job lists)", __FILE__, __LINE__);
  e = cudaMemcpyAsync(dev, host.data(), host.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return impact_set_error(e, "job list upload", __FILE__, __LINE__);
  for (size_t q = 0; q < lists.size(); ++q) {
    lists[q].ts = reinterpret_cast<const int*>(dev + ts_off[q]);
    lists[q].jobs = dev + job_off[q];
  }
  return 0;
}

void ListArena::release() {
  if (dev) cudaFree(dev);
  dev = nullptr;
  host.clear();
  lists.clear();
  ts_off.clear();
  job_off.clear();
}

template <typename T>
void Engine<T>::release() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  prof::graph_release(gpairs_);
  arena_.release();
  if (partial_) cudaFree(partial_);
  if (scal_) cudaFree(scal_);
  if (scal_host_) cudaFreeHost(scal_host_);
  partial_ = nullptr;
  scal_ = nullptr;
  scal_host_ = nullptr;
  vc_[0].clear();
  vc_[1].clear();
  pre0_ = post0_ = -1;
  cells_.clear();
  cells_f_.clear();
  cells_c_.clear();
  fast_.clear();
  cs_.clear();
  built_ = false;
}

template <typename T>
void Engine<T>::smooth(std::vector<Phase>& out, int list, int init, int sweeps) {
  if (sweeps <= 0) return;
  // targets alternate so that the last write lands in B; the first write may not read its target
  int tgt = (sweeps % 2 == 1) ? 0 : 1;
  int src = 0;
  int w = 0;
  if (init) {
    out.push_back({PH_INIT, list, tgt});
    src = tgt;
    tgt ^= 1;
    ++w;
  } else if (tgt == 0) {  // odd number of plain sweeps: stage the start in C first
    out.push_back({PH_COPY, list, 0});
    src = 1;
  }
  for (; w < sweeps; ++w) {
    out.push_back({PH_SWEEP, list, src});
    src = tgt;
    tgt ^= 1;
  }
}

template <typename T>
int Engine<T>::build(const std::vector<EngineCase<T>>& cs, const EngineParams& p, cudaStream_t s) {
  release();
  ax_attributes();
  cs_ = cs;
  p_ = p;
  p_.kc = std::max(1, std::min(KC_MAX, p.kc));
  s_ = s;
  const int n = (int)cs.size();
  if (n == 0) return impact_set_error_msg(-1, "engine: no cases");
  const bool use_mg = p_.precond == 1;
  if (use_mg)
    for (const auto& c : cs)
      if (!c.mg || c.mg->n < 1) return impact_set_error_msg(-1, "engine: multigrid requested for a case without hierarchy");
  const bool pre_on = use_mg || p_.n_sweeps > 0;
  const int kc = p_.kc;
  cudaError_t e = cudaMalloc((void**)&scal_, n * sizeof(SolverScalars));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&scal_host_, n * sizeof(SolverScalars));
  long long tiles_fine = 0;
  for (const auto& c : cs) tiles_fine += tiles_of(c.g, kc);
  if (e == cudaSuccess) e = cudaMalloc((void**)&partial_, (size_t)(tiles_fine * 4 + 64) * sizeof(double));
  if (e != cudaSuccess) {
    release();
    return impact_set_error(e, "engine allocation", __FILE__, __LINE__);
  }
  cudaMemsetAsync(scal_, 0, n * sizeof(SolverScalars), s);
  // ---- Krylov list ----
  {
    std::vector<KrylovJob<T>> kj(n);
    std::vector<int> kt(n);
    for (int c = 0; c < n; ++c) {
      KrylovJob<T>& J = kj[c];
      const EngineCase<T>& C = cs[c];
      J = KrylovJob<T>{};
      J.g = C.g;
      J.kc = kc;
      for (int m = 0; m < 3; ++m) J.W[m] = C.W[m];
      J.zuni = C.zuni;
      J.xuni = C.xuni;
      J.bb = C.bb;
      J.phi = C.phi;
      J.rr = C.rr;
      J.rh = C.rh;
      J.pp = C.pp;
      J.Ap = C.Ap;
      J.Ar = C.Ar;
      J.z1 = pre_on ? C.z1 : C.pp;
      J.z2 = pre_on ? C.z2 : C.rr;
      J.sc = scal_ + c;
      kt[c] = tiles_of(C.g, kc);
    }
    // the vector kernels take the jobs whose rows hold whole 16-byte vectors and whose fields are
    // 16-byte aligned: FP32 (k_kr_ax32v) n1 % 4 == 0, n1 >= 8, with uniform x and z weights (it
    // keeps one row of each), FP64 (k_kr_ax64v, per-row weights) n1 % 2 == 0, n1 >= 8; the others
    // stay with the staged kernels.  The choice is per job, so a case's result does not depend on
    // the other cases of its batch.
    int nv = 0;
    for (auto& J : kj) {
      const void* f[] = {J.phi, J.z1, J.z2, J.rr, J.Ap, J.Ar, J.rh};
      bool al = true;
      for (const void* q : f) al = al && (reinterpret_cast<uintptr_t>(q) & 15) == 0;
      J.vec = std::is_same<T, float>::value ? (J.g.n1 % 4 == 0 && J.g.n1 >= 8 && J.xuni && J.zuni && al)
                                             : (J.g.n1 % 2 == 0 && J.g.n1 >= 8 && al);
      nv += J.vec;
    }
    kr_vec_ = nv == 0 ? 0 : (nv == n ? 1 : 2);
    kr_list_ = arena_.add(kj, kt);
  }
  // ---- preconditioner schedules ----
  auto lvjob = [&](int c, int g, int variant) {
    const EngineCase<T>& C = cs[c];
    LevelJob<T> J{};
    const MGData<T>* mg = (C.mg && C.mg->n > 0) ? C.mg : nullptr;
    if (mg) {
      const MGLevel<T>& L = mg->lv[g];
      J.g = L.g;
      J.zuni = L.zuni;
      for (int m = 0; m < 3; ++m) J.cdg[m] = L.cdg[m];
    } else {
      J.g = C.g;
      J.zuni = C.cdg_zuni;
      for (int m = 0; m < 3; ++m) J.cdg[m] = C.cdg[m];
    }
    J.kc = kc;
    J.vw = (J.g.n1 % VecT<T>::W == 0) ? VecT<T>::W : 1;
    if (g == 0) {
      J.A = variant ? C.rr : C.pp;
      J.B = variant ? C.z2 : C.z1;
      J.C = C.comp;
    } else {
      J.A = mg->lv[g].A;
      J.B = mg->lv[g].B;
      J.C = mg->lv[g].C;
      const MGLevel<T>& F = mg->lv[g - 1];
      J.gf = F.g;
      for (int m = 0; m < 3; ++m) J.rf[m] = F.ratio[m];
      J.Cf = (g - 1 == 0) ? C.comp : F.C;
    }
    if (mg && g + 1 < mg->n) {
      const MGLevel<T>& L = mg->lv[g];
      const MGLevel<T>& Cc = mg->lv[g + 1];
      J.gc = Cc.g;
      for (int m = 0; m < 3; ++m) {
        J.rc[m] = L.ratio[m];
        J.cI[m] = L.cI[m];
      }
      J.Bc = Cc.B;
    }
    J.sc = scal_ + c;
    return J;
  };
  auto vol = [](const Geom& g) { return (double)g.n1 * g.n2 * g.n3; };
  auto note = [&](int list, double c, double f, double cc, bool fast = false) {
    cells_.resize(list + 1, 0.0);
    cells_f_.resize(list + 1, 0.0);
    cells_c_.resize(list + 1, 0.0);
    fast_.resize(list + 1, 0);
    cells_[list] = c;
    cells_f_[list] = f;
    cells_c_[list] = cc;
    fast_[list] = fast ? 1 : 0;
  };
  {
    double c = 0.0;
    for (const auto& C : cs) c += vol(C.g);
    note(kr_list_, c, 0.0, 0.0);
  }
  // vec: allow several columns per thread (lists walked by the smoothing and residual kernels);
  // the restriction lists keep one column per thread.  fusedS > 0: a list of the fused smoothing
  // kernel with S stencil stages (its own tile shape; tile depth per job, deep enough to stream,
  // shallow enough to give every SM a few tiles)
  auto add_list = [&](const std::vector<std::pair<int, int>>& members, int variant, bool vec = true, int fusedS = 0) {
    std::vector<LevelJob<T>> jobs;
    std::vector<int> tiles;
    double c = 0.0, f = 0.0, cc = 0.0;
    bool fast = !members.empty();
    bool mfast = true;  // fused lists: every job vectorisable with uniform z (the kernel's FAST path)
    for (auto& m : members) {
      const LevelJob<T> Jt = lvjob(m.first, m.second, variant);
      mfast = mfast && Jt.vw == VecT<T>::W && Jt.zuni;
    }
    for (auto& m : members) {
      jobs.push_back(lvjob(m.first, m.second, variant));
      if (!vec) jobs.back().vw = 1;
    }
    auto tiles_at_kc = [&](const LevelJob<T>& J, int kcj) {
      return fusedS > 0 ? tiles_multi(J.g, kcj, (int)sizeof(T), fusedS, mfast) : tiles_of(J.g, kcj, J.vw);
    };
    // tile depth of the list: the engine's (the deepest for the fused kernels), halved while the
    // list has fewer than two tiles per SM, so that the small coarse levels march short columns
    // on many SMs instead of long ones on a few
    int kcl = fusedS > 0 ? KC_MAX : kc;
    auto total_at = [&](int kcj) {
      long long tot = 0;
      for (const auto& J : jobs) tot += tiles_at_kc(J, kcj);
      return tot;
    };
    if (fusedS > 0) {
      // the fused kernel runs one block per SM and marches kc + 2S planes per tile (plus a few
      // planes' worth of set-up): pick the depth with the fewest waves x planes per tile
      int nsm = 0, dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (nsm <= 0) nsm = 148;
      double best = 0.0;
      for (int kcj = KC_MAX; kcj >= 1; --kcj) {
        const double cost = (double)((total_at(kcj) + nsm - 1) / nsm) * (kcj + 2 * fusedS + 4);
        if (kcj == KC_MAX || cost < best) {
          best = cost;
          kcl = kcj;
        }
      }
    } else {
      while (total_at(kcl) < 2 * 148 && kcl > 1) kcl /= 2;
    }
    for (auto& J : jobs) {
      J.kc = kcl;
      tiles.push_back(tiles_at_kc(J, kcl));
      c += vol(J.g);
      if (J.Cf) f += vol(J.gf);
      if (J.Bc) cc += vol(J.gc);
      fast = fast && J.vw == VecT<T>::W && J.zuni;
    }
    const int id = arena_.add(jobs, tiles);
    note(id, c, f, cc, fast);
    return id;
  };
  std::vector<int> nlev(n, 1);
  int gmax = 1;
  for (int c = 0; c < n; ++c) {
    nlev[c] = (use_mg && cs[c].mg) ? cs[c].mg->n : 1;
    gmax = std::max(gmax, nlev[c]);
  }
  // lt[c]: the first level of case c's coarse tail (k_lv_tail), the coarsest level from which
  // all levels' three fields fit in TAIL_BYTES; -1 without one (one-sweep schedule, no hierarchy,
  // or fewer than two levels that fit -- one suffices with the Chebyshev bottom).  Levels from
  // lt[c] on leave the per-level lists.
  std::vector<int> lt(n, -1);
  if (use_mg && p_.fuse && p_.mg_down >= 1 && p_.mg_bottom >= 1 && p_.mg_up >= 0) {
    for (int c = 0; c < n; ++c) {
      if (nlev[c] < 2) continue;
      double bytes = 0.0;
      int first = -1;
      for (int g = nlev[c] - 1; g >= 0; --g) {
        const Geom& gg = cs[c].mg->lv[g].g;
        bytes += 3.0 * sizeof(T) * gg.n1 * gg.n2 * gg.n3;
        if (bytes > (double)TAIL_BYTES) break;
        first = g;
      }
      if (first >= 0 && (nlev[c] - first >= 2 || p_.bottom_cheb > 0)) lt[c] = first;
    }
  }
  auto in_lists = [&](int c, int g) { return lt[c] < 0 || g < lt[c]; };
  if (use_mg) {
    // fused smoothing phases for the sweep counts that have kernels
    const int spre = (p_.fuse && p_.mg_down >= 2 && p_.mg_down <= 3) ? p_.mg_down : 0;
    const int spost = (p_.fuse && p_.mg_up >= 2 && p_.mg_up <= 3) ? p_.mg_up : 0;
    // level >= 1 lists are shared by both schedules
    std::vector<int> down(gmax, -1), rs(gmax, -1), dpre(gmax, -1), dpost(gmax, -1);
    for (int g = 1; g + 1 < gmax; ++g) {
      std::vector<std::pair<int, int>> m;
      for (int c = 0; c < n; ++c)
        if (nlev[c] >= g + 2 && in_lists(c, g)) m.push_back({c, g});
      down[g] = add_list(m, 0);
      if (spre) dpre[g] = add_list(m, 0, true, spre);
      if (spost) dpost[g] = add_list(m, 0, true, spost);
    }
    for (int g = 1; g < gmax; ++g) {  // restriction into level g (into a tail's first level too)
      std::vector<std::pair<int, int>> m;
      for (int c = 0; c < n; ++c)
        if (nlev[c] >= g + 1 && (lt[c] < 0 || g <= lt[c])) m.push_back({c, g});
      rs[g] = add_list(m, 0, false);
    }
    for (int v = 0; v < 2; ++v) {
      std::vector<std::pair<int, int>> m0, bot;
      std::vector<TailJob<T>> tj;
      std::vector<int> tt;
      for (int c = 0; c < n; ++c) {
        if (nlev[c] >= 2 && in_lists(c, 0)) m0.push_back({c, 0});
        if (lt[c] < 0) {
          bot.push_back({c, nlev[c] - 1});
        } else {
          TailJob<T> job{};
          job.nl = nlev[c] - lt[c];
          for (int q = 0; q < job.nl; ++q) job.lv[q] = lvjob(c, lt[c] + q, v);
          if (p_.bottom_cheb > 0) {
            const double lo = std::max(1e-6, std::min(1.0, cs[c].mg->lv[nlev[c] - 1].lmin));
            const double sg = (2.0 - lo) / (2.0 + lo);
            job.cheb = p_.bottom_cheb;
            job.cgam = (T)(2.0 / (2.0 + lo));
            job.csig2 = (T)(sg * sg);
          }
          tj.push_back(job);
          tt.push_back(1);
        }
      }
      const int down0 = add_list(m0, v);
      const int botl = add_list(bot, v);
      const int taill = tj.empty() ? -1 : arena_.add(tj, tt);
      if (taill >= 0) {
        double tc = 0.0;
        for (int c = 0; c < n; ++c)
          if (lt[c] >= 0) tc += vol(cs[c].mg->lv[lt[c]].g);
        note(taill, tc, 0.0, 0.0);
      }
      if (spre) dpre[0] = add_list(m0, v, true, spre);
      if (spost) dpost[0] = add_list(m0, v, true, spost);
      if (v == 0) {
        down0_ = down0;
        rs1_ = gmax > 1 ? rs[1] : -1;
        pre0_ = dpre[0];
        post0_ = dpost[0];
      }
      std::vector<Phase>& sch = vc_[v];
      for (int g = 0; g + 1 < gmax; ++g) {  // relax_restrict
        const int D = g == 0 ? down0 : down[g];
        if (spre) {
          sch.push_back({PH_PRE, dpre[g], 0});
        } else {
          smooth(sch, D, 1, p_.mg_down);
          sch.push_back({PH_RESID, D, 0});
        }
        sch.push_back({PH_RESTRICT, rs[g + 1], 0});
      }
      smooth(sch, botl, 1, p_.mg_bottom);  // relax_bottom
      smooth(sch, botl, 0, p_.mg_bottom);
      if (taill >= 0) sch.push_back({PH_TAIL, taill, 0});  // the cases' coarse tails
      for (int g = gmax - 2; g >= 0; --g) {  // interpolate_relax
        const int D = g == 0 ? down0 : down[g];
        if (spost) {
          sch.push_back({PH_PROLONG, D, 1});
          sch.push_back({PH_POST, dpost[g], 0});
        } else {
          sch.push_back({PH_PROLONG, D, 0});
          smooth(sch, D, 0, p_.mg_up);
        }
      }
    }
  } else if (p_.n_sweeps > 0) {
    for (int v = 0; v < 2; ++v) {
      std::vector<std::pair<int, int>> m0;
      for (int c = 0; c < n; ++c) m0.push_back({c, 0});
      const int l0 = add_list(m0, v);
      if (v == 0) down0_ = l0;
      smooth(vc_[v], l0, 1, p_.n_sweeps);
    }
  }
  int rc = arena_.upload(s);
  if (rc) {
    release();
    return rc;
  }
  // launches per iteration (for the launch counter under graph replay)
  long long l = 9;
  for (int v = 0; v < 2; ++v)
    for (const Phase& ph : vc_[v])
      if (arena_.lists[ph.list].ntiles > 0) ++l;
  launches_iter_ = l;
  built_ = true;
  return 0;
}

// fused smoothing launches: pre-smoothing with mg_down sweeps, post-smoothing with mg_up sweeps
template <typename T, int NSW, bool INIT, bool RES>
void launch_multi(bool fast, const LevelJob<T>* J, const DevList& L, T om, cudaStream_t s) {
  if (fast)
    k_lv_multi<T, NSW, INIT, RES, true><<<grid_multi(L.ntiles), kMBlock, multi_smem_bytes<T, NSW, INIT, RES>(), s>>>(
        J, L.ts, L.njobs, L.ntiles, om);
  else
    k_lv_multi<T, NSW, INIT, RES, false><<<grid_multi(L.ntiles), kMBlock, multi_smem_bytes<T, NSW, INIT, RES>(), s>>>(
        J, L.ts, L.njobs, L.ntiles, om);
}
template <typename T>
void launch_multi_pre(int sweeps, bool fast, const LevelJob<T>* J, const DevList& L, T om, cudaStream_t s) {
  if (sweeps == 2)
    launch_multi<T, 1, true, true>(fast, J, L, om, s);
  else
    launch_multi<T, 2, true, true>(fast, J, L, om, s);
}
template <typename T>
void launch_multi_post(int sweeps, bool fast, const LevelJob<T>* J, const DevList& L, T om, cudaStream_t s) {
  if (sweeps == 2)
    launch_multi<T, 2, false, false>(fast, J, L, om, s);
  else
    launch_multi<T, 3, false, false>(fast, J, L, om, s);
}

template <typename T>
void Engine<T>::enqueue_phase(const Phase& ph) {
  const DevList& L = arena_.lists[ph.list];
  if (L.ntiles == 0) return;
  const LevelJob<T>* J = static_cast<const LevelJob<T>*>(L.jobs);
  const int grid = grid_for(L.ntiles);
  const T om = (T)p_.omega;
  cudaStream_t s = s_;
  const double sz = sizeof(T), c = cells_[ph.list], cf = cells_f_[ph.list], cc = cells_c_[ph.list];
  switch (ph.kind) {
    case PH_INIT:
      IMPACT_PROF(prof::K_MG_INIT, 2 * sz * c, s, (k_lv_smooth<T, 1><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, om, ph.flip)));
      break;
    case PH_SWEEP:
      if (fast_[ph.list])
        IMPACT_PROF(prof::K_MG_SWEEP, 3 * sz * c, s, (k_lv_fast<T, 0, 2, 1><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, om, ph.flip)));
      else
        IMPACT_PROF(prof::K_MG_SWEEP, 3 * sz * c, s, (k_lv_smooth<T, 0><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, om, ph.flip)));
      break;
    case PH_COPY:
      IMPACT_PROF(prof::K_MG_OTHER, 2 * sz * c, s, (k_lv_smooth<T, 2><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, om, 0)));
      break;
    case PH_RESID:
      if (fast_[ph.list])
        IMPACT_PROF(prof::K_MG_RESID, 3 * sz * c, s, (k_lv_fast<T, 1, 2, 1><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, om, 0)));
      else
        IMPACT_PROF(prof::K_MG_RESID, 3 * sz * c, s, (k_lv_resid<T><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles)));
      break;
    case PH_RESTRICT:
      IMPACT_PROF(prof::K_MG_OTHER, sz * (c + cf), s, (k_lv_restrict<T><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles)));
      break;
    case PH_PROLONG:
      IMPACT_PROF(prof::K_MG_OTHER, sz * (2 * c + cc), s, (k_lv_prolong<T><<<grid, kBlock, 0, s>>>(J, L.ts, L.njobs, L.ntiles, ph.flip)));
      break;
    case PH_PRE:  // mg_down 2 or 3
      IMPACT_PROF(prof::K_MG_PRE, 3 * sz * c, s, launch_multi_pre<T>(p_.mg_down, fast_[ph.list] != 0, J, L, om, s));
      break;
    case PH_POST:  // mg_up 2 or 3
      IMPACT_PROF(prof::K_MG_POST, 3 * sz * c, s, launch_multi_post<T>(p_.mg_up, fast_[ph.list] != 0, J, L, om, s));
      break;
    case PH_TAIL:  // one block per case; bytes: read the first level's right-hand side, write its iterate
      IMPACT_PROF(prof::K_MG_TAIL, 2 * sz * c, s,
                  (k_lv_tail<T><<<L.ntiles, TNT, TAIL_BYTES, s>>>(static_cast<const TailJob<T>*>(L.jobs), L.ts, L.njobs,
                                                                  L.ntiles, om, p_.mg_down, p_.mg_up, p_.mg_bottom)));
      break;
    default:
      break;
  }
}

template <typename T>
void Engine<T>::enqueue_precond(int variant) {
  for (const Phase& ph : vc_[variant]) enqueue_phase(ph);
}

template <typename T>
void Engine<T>::enqueue_iteration() {
  const DevList& K = arena_.lists[kr_list_];
  const KrylovJob<T>* J = static_cast<const KrylovJob<T>*>(K.jobs);
  const int n = K.njobs;
  const int grid = grid_for(K.ntiles);
  cudaStream_t s = s_;
  const double fb = sizeof(T) * cells_[kr_list_];
  k_ebegin<<<(n + 31) / 32, 32, 0, s>>>(scal_, n);
  prof::count(1);
  IMPACT_PROF(prof::K_P_UPDATE, 4 * fb, s, (k_kr_p<T><<<grid, kBlock, 0, s>>>(J, K.ts, n, K.ntiles)));
  enqueue_precond(0);
  IMPACT_PROF(prof::K_DIVGRAD, 3 * fb, s, (launch_ax<T, 1>(grid, J, K.ts, n, K.ntiles, partial_, s, kr_vec_)));
  k_efin<<<n, 256, 0, s>>>(K.ts, partial_, 1, 0, EFIN_ALPHA, scal_, nullptr);
  IMPACT_PROF(prof::K_R_UPDATE, 3 * fb, s, (k_kr_r<T><<<grid, kBlock, 0, s>>>(J, K.ts, n, K.ntiles)));
  enqueue_precond(1);
  IMPACT_PROF(prof::K_DIVGRAD, 3 * fb, s, (launch_ax<T, 2>(grid, J, K.ts, n, K.ntiles, partial_, s, kr_vec_)));
  k_efin<<<n, 256, 0, s>>>(K.ts, partial_, 2, 0, EFIN_OMEGA, scal_, nullptr);
  IMPACT_PROF(prof::K_X_UPDATE, 8 * fb, s, (k_kr_x<T><<<grid, kBlock, 0, s>>>(J, K.ts, n, K.ntiles, partial_)));
  k_efin<<<n, 256, 0, s>>>(K.ts, partial_, 3, 1, EFIN_NORMS, scal_, nullptr);
  prof::count(3);
}

template <typename T>
int Engine<T>::poll(bool& all_done) {
  const int n = (int)cs_.size();
  cudaError_t e = cudaMemcpyAsync(scal_host_, scal_, n * sizeof(SolverScalars), cudaMemcpyDeviceToHost, s_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine poll", __FILE__, __LINE__);
  prof::flush();
  all_done = true;
  for (int c = 0; c < n; ++c) {
    const SolverScalars& h = scal_host_[c];
    if (!(h.done || (h.status != 0 && h.status != 4))) all_done = false;
  }
  return 0;
}

template <typename T>
int Engine<T>::solve(const std::vector<SolverScalars>& init, int zero_phi, std::vector<SolverResult>& res,
                     const int* ext_ts, const double* ext_partial) {
  if (!built_) return impact_set_error_msg(-1, "engine: not built");
  const int n = (int)cs_.size();
  if ((int)init.size() != n) return impact_set_error_msg(-1, "engine: wrong number of initial scalars");
  int max_it = 0;
  for (int c = 0; c < n; ++c) {
    scal_host_[c] = init[c];
    scal_host_[c].it = 0;
    scal_host_[c].status = 0;
    scal_host_[c].phi_zero = zero_phi == 2 ? 1 : 0;
    scal_host_[c].rr_in_rh = zero_phi && ext_partial ? 1 : 0;
    if (!init[c].done) max_it = std::max(max_it, init[c].max_it);
  }
  cudaError_t e = cudaMemcpyAsync(scal_, scal_host_, n * sizeof(SolverScalars), cudaMemcpyHostToDevice, s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine scalars", __FILE__, __LINE__);
  const DevList& K = arena_.lists[kr_list_];
  const KrylovJob<T>* J = static_cast<const KrylovJob<T>*>(K.jobs);
  const int grid = grid_for(K.ntiles);
  if (zero_phi && ext_partial) {  // rh = bb = pp = r0 and its norms come from the caller's kernel
    k_efin<<<n, 256, 0, s_>>>(ext_ts, ext_partial, 4, 1, EFIN_INIT_EXT, scal_, nullptr);
    prof::count(1);
  } else {
    if (!zero_phi) {
      launch_ax<T, 0>(grid, J, K.ts, n, K.ntiles, partial_, s_, kr_vec_);
      prof::count(1);
    }
    IMPACT_PROF(prof::K_KR_INIT, 4.0 * sizeof(T) * cells_[kr_list_], s_,
                (k_kr_init<T><<<grid, kBlock, 0, s_>>>(J, K.ts, n, K.ntiles, zero_phi, partial_)));
    k_efin<<<n, 256, 0, s_>>>(K.ts, partial_, 4, 1, EFIN_INIT, scal_, nullptr);
    prof::count(1);
  }
  const int chunk = p_.check_every > 0 ? p_.check_every : 1;
  const bool profiling = prof::enabled();
  if (graph_ && graph_prof_ != profiling) {  // the profiler was switched: capture again
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    prof::graph_release(gpairs_);
  }
  if (p_.use_graph && !graph_) {
    cudaGraph_t gr = nullptr;
    e = cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      if (profiling) prof::capture_begin();
      for (int t = 0; t < chunk; ++t) enqueue_iteration();
      if (profiling) gpairs_ = prof::capture_end();
      e = cudaStreamEndCapture(s_, &gr);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&graph_, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (e != cudaSuccess) {  // capture unavailable on this stream: launch directly from now on
      cudaGetLastError();
      graph_ = nullptr;
      prof::graph_release(gpairs_);
      p_.use_graph = 0;
    }
    graph_prof_ = profiling;
    prof::count(-(long long)chunk * launches_iter_);  // the capture counted launches that did not run
  }
  int launched = 0;
  for (;;) {
    if (graph_) {
      e = cudaGraphLaunch(graph_, s_);
      if (e != cudaSuccess) return impact_set_error(e, "engine graph launch", __FILE__, __LINE__);
      prof::count((long long)chunk * launches_iter_);
    } else {
      for (int t = 0; t < chunk; ++t) enqueue_iteration();
    }
    launched += chunk;
    bool all_done = false;
    int rc = poll(all_done);
    if (rc) return rc;
    if (graph_ && graph_prof_) prof::graph_account(gpairs_);  // the replay has completed
    bool reset = false;
    for (int c = 0; c < n; ++c)
      if (scal_host_[c].status == 4) reset = true;
    if (reset) {
      // rhr == 0: new shadow residual rh = rr, as the reference does, then redo the iteration start
      k_kr_reset<T><<<grid, kBlock, 0, s_>>>(J, K.ts, n, K.ntiles, partial_);
      k_efin<<<n, 256, 0, s_>>>(K.ts, partial_, 1, 0, EFIN_RESET, scal_, nullptr);
      prof::count(2);
      continue;
    }
    if (all_done) break;
    if (launched > max_it + 8) break;  // safety net: the device flags should have stopped it
  }
  res.resize(n);
  for (int c = 0; c < n; ++c) {
    const SolverScalars& h = scal_host_[c];
    res[c].iterations = h.it;
    res[c].status = h.status;
    res[c].res_inf = h.norm_inf;
    res[c].res_two = std::sqrt(h.norm_two_sq);
    res[c].b_two = std::sqrt(h.b_two_sq);
  }
  return 0;
}

template <typename T>
int Engine<T>::apply_precond() {
  if (!built_) return impact_set_error_msg(-1, "engine: not built");
  const int n = (int)cs_.size();
  for (int c = 0; c < n; ++c) scal_host_[c] = SolverScalars{};
  cudaError_t e = cudaMemcpyAsync(scal_, scal_host_, n * sizeof(SolverScalars), cudaMemcpyHostToDevice, s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine scalars", __FILE__, __LINE__);
  enqueue_precond(0);
  e = cudaStreamSynchronize(s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine precond", __FILE__, __LINE__);
  return 0;
}

template <typename T>
int Engine<T>::apply_operator() {
  if (!built_) return impact_set_error_msg(-1, "engine: not built");
  const int n = (int)cs_.size();
  for (int c = 0; c < n; ++c) scal_host_[c] = SolverScalars{};
  cudaError_t e = cudaMemcpyAsync(scal_, scal_host_, n * sizeof(SolverScalars), cudaMemcpyHostToDevice, s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine scalars", __FILE__, __LINE__);
  const DevList& K = arena_.lists[kr_list_];
  const KrylovJob<T>* J = static_cast<const KrylovJob<T>*>(K.jobs);
  launch_ax<T, 0>(grid_for(K.ntiles), J, K.ts, n, K.ntiles, partial_, s_, kr_vec_);
  prof::count(1);
  e = cudaStreamSynchronize(s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine operator", __FILE__, __LINE__);
  return 0;
}

template <typename T>
int Engine<T>::bench(int kind, int iters, double* ms, double* bytes) {
  if (!built_) return impact_set_error_msg(-1, "engine: not built");
  const int n = (int)cs_.size();
  for (int c = 0; c < n; ++c) {
    scal_host_[c] = SolverScalars{};
    scal_host_[c].it = 2;
    scal_host_[c].max_it = 1 << 30;
  }
  cudaError_t e = cudaMemcpyAsync(scal_, scal_host_, n * sizeof(SolverScalars), cudaMemcpyHostToDevice, s_);
  if (e != cudaSuccess) return impact_set_error(e, "engine scalars", __FILE__, __LINE__);
  const DevList& K = arena_.lists[kr_list_];
  const KrylovJob<T>* J = static_cast<const KrylovJob<T>*>(K.jobs);
  const int grid = grid_for(K.ntiles);
  const double sz = sizeof(T), fc = cells_[kr_list_];
  double by = 0.0;
  std::function<void()> f;
  auto need = [&](int l) { return l >= 0 && arena_.lists[l].ntiles > 0; };
  switch (kind) {
    case 0:
    case 1:
    case 2:
    case 3: {
      if (!need(down0_)) return impact_set_error_msg(-1, "engine bench: no finest-level list");
      if (kind == 3 && rs1_ < 0) return impact_set_error_msg(-1, "engine bench: no coarse level");
      const int kinds[4] = {PH_SWEEP, PH_INIT, PH_RESID, PH_PROLONG};
      const Phase ph{kinds[kind], down0_, 0};
      const double c = cells_[down0_];
      by = kind == 0 || kind == 2 ? 3 * sz * c : (kind == 1 ? 2 * sz * c : sz * (2 * c + cells_c_[down0_]));
      f = [this, ph]() { enqueue_phase(ph); };
      break;
    }
    case 4: {
      if (!need(rs1_)) return impact_set_error_msg(-1, "engine bench: no coarse level");
      const Phase ph{PH_RESTRICT, rs1_, 0};
      by = sz * (cells_[rs1_] + cells_f_[rs1_]);
      f = [this, ph]() { enqueue_phase(ph); };
      break;
    }
    case 5:
      by = 3 * sz * fc;
      f = [&]() { launch_ax<T, 1>(grid, J, K.ts, n, K.ntiles, partial_, s_, kr_vec_); };
      break;
    case 6:
      by = 3 * sz * fc;
      f = [&]() { launch_ax<T, 2>(grid, J, K.ts, n, K.ntiles, partial_, s_, kr_vec_); };
      break;
    case 7:
      by = 8 * sz * fc;
      f = [&]() { k_kr_x<T><<<grid, kBlock, 0, s_>>>(J, K.ts, n, K.ntiles, partial_); };
      break;
    case 8:
      by = 4 * sz * fc;
      f = [&]() { k_kr_p<T><<<grid, kBlock, 0, s_>>>(J, K.ts, n, K.ntiles); };
      break;
    case 9:
      by = 3 * sz * fc;
      f = [&]() { k_kr_r<T><<<grid, kBlock, 0, s_>>>(J, K.ts, n, K.ntiles); };
      break;
    case 10:
      f = [this]() { enqueue_precond(0); };
      break;
    case 12:
    case 13: {
      const int l = kind == 12 ? pre0_ : post0_;
      if (!need(l)) return impact_set_error_msg(-1, "engine bench: no fused smoothing list (sweep count 2..4, fusion on)");
      const Phase ph{kind == 12 ? PH_PRE : PH_POST, l, 0};
      by = 3 * sz * cells_[l];
      f = [this, ph]() { enqueue_phase(ph); };
      break;
    }
    case 11:
      f = [this]() { enqueue_iteration(); };
      break;
    default:
      return impact_set_error_msg(-1, "engine bench: unknown kernel kind");
  }
  f();  // warm-up
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s_);
  for (int t = 0; t < iters; ++t) f();
  cudaEventRecord(b, s_);
  e = cudaEventSynchronize(b);
  float t_ms = 0.f;
  cudaEventElapsedTime(&t_ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return impact_set_error(e, "engine bench", __FILE__, __LINE__);
  *ms = t_ms / iters;
  *bytes = by;
  return 0;
}

template class Engine<double>;
template class Engine<float>;

// =========================================================================================
// mixed precision
// =========================================================================================
void MixedEngine::release() {
  inner_.release();
  arena_.release();
  if (partial_) cudaFree(partial_);
  if (q_) cudaFree(q_);
  if (q_host_) cudaFreeHost(q_host_);
  if (oscal_) cudaFree(oscal_);
  partial_ = nullptr;
  q_ = nullptr;
  q_host_ = nullptr;
  oscal_ = nullptr;
  cs_.clear();
  built_ = false;
}

int MixedEngine::build(const std::vector<Case>& cs, const EngineParams& p, cudaStream_t s) {
  release();
  cs_ = cs;
  s_ = s;
  const int n = (int)cs.size();
  std::vector<EngineCase<float>> ic;
  for (const Case& c : cs) {
    // the outer residual writes r0 once, into the inner solve's right-hand side, which must also
    // be its shadow residual (the inner solve starts from e = 0)
    if (c.inner.bb != c.r32 || c.inner.rh != c.r32)
      return impact_set_error_msg(-1, "mixed engine: the inner bb and rh must be the FP32 residual buffer");
    ic.push_back(c.inner);
  }
  int rc = inner_.build(ic, p, s);
  if (rc) return rc;
  const int kc = inner_.params().kc;
  long long tiles = 0;
  for (const Case& c : cs) tiles += tiles_of(c.g, kc);
  cudaError_t e = cudaMalloc((void**)&partial_, (size_t)(tiles * 4 + 64) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&q_, (size_t)n * 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&q_host_, (size_t)n * 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&oscal_, (size_t)n * sizeof(SolverScalars));
  if (e != cudaSuccess) {
    release();
    return impact_set_error(e, "mixed engine allocation", __FILE__, __LINE__);
  }
  cudaMemsetAsync(oscal_, 0, (size_t)n * sizeof(SolverScalars), s);
  std::vector<KrylovJob<double>> aj(n);
  std::vector<MixJob> mj(n);
  std::vector<int> t(n);
  for (int c = 0; c < n; ++c) {
    const Case& C = cs[c];
    KrylovJob<double>& A = aj[c];
    A = KrylovJob<double>{};
    A.g = C.g;
    A.kc = kc;
    for (int m = 0; m < 3; ++m) A.W[m] = C.W64[m];
    A.zuni = C.zuni;
    A.xuni = C.xuni;
    A.phi = C.x;
    A.bb = C.bb;
    A.rr = C.r64;
    A.r32 = C.r32;
    A.r32p = C.inner.pp;  // the inner solve's first search direction, written with r32
    A.sc = oscal_ + c;
    A.vec = C.g.n1 % 2 == 0 && C.g.n1 >= 8 && (reinterpret_cast<uintptr_t>(C.x) & 15) == 0 &&
            (reinterpret_cast<uintptr_t>(C.bb) & 15) == 0 && (reinterpret_cast<uintptr_t>(C.r32) & 7) == 0 &&
            (reinterpret_cast<uintptr_t>(C.inner.pp) & 7) == 0;
    MixJob& M = mj[c];
    M = MixJob{};
    M.g = C.g;
    M.kc = kc;
    M.bb = C.bb;
    M.x = C.x;
    M.r64 = C.r64;
    M.r32 = C.r32;
    M.e32 = C.e32;
    M.q = q_ + 4 * c;
    M.isc = inner_.scal_dev() + c;
    t[c] = tiles_of(C.g, kc);
  }
  {
    int nv = 0;
    for (const auto& A : aj) nv += A.vec;
    ax_vec_ = nv == 0 ? 0 : (nv == n ? 1 : 2);
  }
  ax_list_ = arena_.add(aj, t);
  mix_list_ = arena_.add(mj, t);
  rc = arena_.upload(s);
  if (rc) {
    release();
    return rc;
  }
  built_ = true;
  return 0;
}

// Iterative refinement (no counterpart in mod_solvers.f90; the FP64 outer loop wraps the
// reference's BiCGstab run in FP32): r = b - A x in FP64, e ~ A^-1 r by the FP32 engine on the
// FP32 image of r, x += e.  A case whose inner solve breaks down or turns non-finite has
// its correction discarded and is retried with a looser tolerance (twice at most).
int MixedEngine::solve(const std::vector<SolverScalars>& outer, double inner_tol, int inner_max_it, int zero_x,
                       std::vector<SolverResult>& res, std::vector<int>& inner_its) {
  if (!built_) return impact_set_error_msg(-1, "mixed engine: not built");
  const int n = (int)cs_.size();
  const bool dbg = std::getenv("IMPACT_B200_DEBUG") != nullptr;
  res.assign(n, SolverResult{});
  inner_its.assign(n, 0);
  std::vector<int> done(n, 0), outer_it(n, 0), retries(n, 0);
  std::vector<SolverScalars> osc(n);
  for (int c = 0; c < n; ++c) {
    done[c] = outer[c].done;
    res[c].status = 1;
    if (zero_x && !done[c]) cudaMemsetAsync(cs_[c].x, 0, (size_t)cs_[c].g.nfield * sizeof(double), s_);
  }
  const DevList& AL = arena_.lists[ax_list_];
  const DevList& ML = arena_.lists[mix_list_];
  double cells = 0.0;  // algorithmic bytes of both kernels: 20 per cell (x, b or e, r32 or x)
  for (const auto& c : cs_) cells += (double)c.g.n1 * c.g.n2 * c.g.n3;
  const KrylovJob<double>* AJ = static_cast<const KrylovJob<double>*>(AL.jobs);
  const MixJob* MJ = static_cast<const MixJob*>(ML.jobs);
  const int grid = grid_for(ML.ntiles);
  auto push_flags = [&]() -> int {
    for (int c = 0; c < n; ++c) {
      osc[c] = SolverScalars{};
      osc[c].done = done[c];
    }
    cudaError_t e = cudaMemcpyAsync(oscal_, osc.data(), n * sizeof(SolverScalars), cudaMemcpyHostToDevice, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);  // osc is pageable and reused
    if (e != cudaSuccess) return impact_set_error(e, "mixed engine flags", __FILE__, __LINE__);
    return 0;
  };
  std::vector<SolverScalars> init(n);
  std::vector<SolverResult> ir;
  for (;;) {
    int rc = push_flags();
    if (rc) return rc;
    // r = b - A x in FP64 (the reference operator), stored as the FP32 right-hand side of the
    // inner solve, with its norms
    IMPACT_PROF(prof::K_MX_RESID, 20.0 * cells, s_, (launch_ax<double, 3>(grid, AJ, AL.ts, n, AL.ntiles, partial_, s_, ax_vec_)));
    k_efin<<<n, 256, 0, s_>>>(AL.ts, partial_, 3, 1, EFIN_RAW, nullptr, q_);
    prof::count(1);
    cudaError_t e = cudaMemcpyAsync(q_host_, q_, (size_t)n * 4 * sizeof(double), cudaMemcpyDeviceToHost, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    if (e != cudaSuccess) return impact_set_error(e, "mixed engine residual", __FILE__, __LINE__);
    bool any = false;
    for (int c = 0; c < n; ++c) {
      init[c] = SolverScalars{};
      init[c].done = 1;
      if (done[c]) continue;
      const double rinf = q_host_[4 * c], r2 = std::sqrt(q_host_[4 * c + 1]), b2 = std::sqrt(q_host_[4 * c + 2]);
      if (dbg)
        std::fprintf(stderr, "[impact_b200] case %d outer %d: |r|inf %.3e |r|2 %.3e |b|2 %.3e inner so far %d\n", c,
                     outer_it[c], rinf, r2, b2, inner_its[c]);
      res[c].res_inf = rinf;
      res[c].res_two = r2;
      res[c].b_two = b2;
      if (!std::isfinite(rinf) || !std::isfinite(r2)) {
        res[c].status = 3;
        done[c] = 1;
        continue;
      }
      const SolverScalars& o = outer[c];
      const bool conv = (o.tol_abs_inf > 0.0 && rinf < o.tol_abs_inf) || (o.tol_rel > 0.0 && r2 <= o.tol_rel * b2) ||
                        rinf == 0.0;
      if (conv) {
        res[c].status = 0;
        done[c] = 1;
        continue;
      }
      if (outer_it[c] >= o.max_it) {
        res[c].status = 1;
        done[c] = 1;
        continue;
      }
      // inner FP32 solve A e = r from e = 0
      double tol = inner_tol;
      int mit = inner_max_it;
      if (retries[c] > 0) {
        tol = std::fmax(tol, 0.1);
        mit = std::min(mit, 200);
      }
      if (o.tol_rel > 0.0 && r2 > 0.0) {
        const double need = o.tol_rel * b2 / r2;  // reduction still required
        if (need > tol) tol = std::fmin(0.5, need * 0.5);
      }
      init[c].done = 0;
      init[c].tol_rel = tol;
      init[c].tol_abs_inf = 0.0;
      init[c].max_it = mit;
      any = true;
    }
    if (!any) break;
    rc = push_flags();
    if (rc) return rc;
    // e from 0, not written before the first x update; rr and the norms from the residual kernel
    rc = inner_.solve(init, 2, ir, AL.ts, partial_);
    if (rc) return rc;
    for (int c = 0; c < n; ++c) {
      if (init[c].done) continue;
      if (dbg)
        std::fprintf(stderr, "[impact_b200] case %d   inner: it %d status %d |r|2/|b|2 %.3e tol %.1e\n", c,
                     ir[c].iterations, ir[c].status, ir[c].b_two > 0 ? ir[c].res_two / ir[c].b_two : 0.0,
                     init[c].tol_rel);
      inner_its[c] += ir[c].iterations;
      if (ir[c].status == 2 || ir[c].status == 3) {
        if (++retries[c] > 2) {
          res[c].status = ir[c].status;
          done[c] = 1;
        }
      } else {
        ++outer_it[c];
      }
    }
    rc = push_flags();
    if (rc) return rc;
    IMPACT_PROF(prof::K_MX_APPLY, 20.0 * cells, s_, (k_mx_apply<<<grid, kBlock, 0, s_>>>(MJ, ML.ts, n, ML.ntiles, oscal_)));
  }
  for (int c = 0; c < n; ++c) res[c].iterations = outer_it[c];
  return 0;
}

}  // namespace impact
