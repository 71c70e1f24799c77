// solver.cu -- device-resident pressure Poisson solve of the IMPACT fractional step.
//
// BiCGstab_orig (mod_solvers.f90:1509-1935) with every scalar kept on the device: the
// reductions finish in a fixed order (deterministic), single-thread "scalar" kernels form
// alpha, beta, omega and the convergence flag, and every vector kernel becomes a no-op once
// the flag is set.  The host only polls the flag every `check_every` iterations, so a chunk
// of iterations runs without any host round trip.
#include <cmath>
#include <cstdio>

#include "prof.cuh"
#include "solver.cuh"
#include "stencil25d.cuh"
#include <cstdlib>

namespace impact {

constexpr int BX = 32, BY = 8, NT = BX * BY;
constexpr int FIN1_BLOCKS = 256;

static inline dim3 grid3(const Geom& g) { return dim3((g.n1 + BX - 1) / BX, (g.n2 + BY - 1) / BY, g.n3); }
static inline long long nblocks3(const Geom& g) {
  const dim3 d = grid3(g);
  return (long long)d.x * d.y * d.z;
}

// layout of a partial buffer: [nb x nq block partials][FIN1_BLOCKS x nq stage-1 sums][64 raw results]
long long reduce_partial_doubles(const Geom& g, int nq) {
  (void)nq;
  return nblocks3(g) * 4 + FIN1_BLOCKS * 4 + 64;
}
// stage-1 sums live at partial + nb*4 with nb the block count of the producing kernel; the raw
// results of callers sit past the largest such region
static inline double* raw_results(double* partial, const Geom& g) { return partial + nblocks3(g) * 4 + FIN1_BLOCKS * 4; }
template <typename T>
long long krylov_partial_doubles(const Geom& g) {
  return reduce_partial_doubles(g, 4);
}
template long long krylov_partial_doubles<double>(const Geom&);
template long long krylov_partial_doubles<float>(const Geom&);

__device__ __forceinline__ bool halted(const SolverScalars* sc) { return sc->done | sc->status; }

// ---------------------------------------------------------------------------------------
// block partials: NQ quantities, bit q of MAXMASK set = max-reduction, else sum
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <int NQ, int MAXMASK>
__device__ __forceinline__ void block_partials(double (&v)[NQ], double* __restrict__ partial) {
  __shared__ double sh[NQ][NT / 32];
  const int tid = threadIdx.x + BX * threadIdx.y;
  const int lane = tid & 31, w = tid >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = ((MAXMASK >> q) & 1) ? wmax(v[q]) : wsum(v[q]);
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
      x = ((MAXMASK >> q) & 1) ? wmax(x) : wsum(x);
      if (lane == 0) partial[bid * NQ + q] = x;
    }
  }
}

// stage 1: block b reduces its contiguous chunk of the nb block partials (fixed order)
__global__ void __launch_bounds__(256) k_fin1(const double* __restrict__ partial, long long nb, int nq, int maxmask,
                                              double* __restrict__ out, const SolverScalars* sc) {
  if (sc && halted(sc)) return;
  const long long chunk = (nb + gridDim.x - 1) / gridDim.x;
  const long long b0 = blockIdx.x * chunk, b1 = min(nb, b0 + chunk);
  __shared__ double sh[4][8];
  for (int q = 0; q < nq; ++q) {
    const bool mx = (maxmask >> q) & 1;
    double v = 0.0;
    for (long long b = b0 + threadIdx.x; b < b1; b += blockDim.x) {
      const double x = partial[b * nq + q];
      v = mx ? fmax(v, x) : v + x;
    }
    v = mx ? wmax(v) : wsum(v);
    if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int q = 0; q < nq; ++q) {
      const bool mx = (maxmask >> q) & 1;
      double x = threadIdx.x < 8 ? sh[q][threadIdx.x] : 0.0;
      x = mx ? wmax(x) : wsum(x);
      if (threadIdx.x == 0) out[(long long)blockIdx.x * nq + q] = x;
    }
  }
}

// stage 2 + scalar update
enum FinMode { FIN_RAW = 0, FIN_INIT = 1, FIN_BEGIN = 2, FIN_ALPHA = 3, FIN_OMEGA = 4, FIN_NORMS = 5 };

__device__ void scalar_update(int mode, int nq, const double* q, SolverScalars* sc, double* raw_out) {
  switch (mode) {
    case FIN_RAW:
      for (int i = 0; i < nq; ++i) raw_out[i] = q[i];
      break;
    case FIN_INIT: {  // q = [max|r|, sum r^2, r.rh, sum b^2]
      sc->norm_inf = q[0];
      sc->norm_two_sq = q[1];
      sc->rhr_next = q[2];
      sc->b_two_sq = q[3];
      sc->rhr = 0.0;
      sc->alpha = sc->omega = sc->beta = 0.0;
      sc->it = 0;
      sc->status = 0;
      sc->done = (q[0] == 0.0) ? 1 : 0;  // the reference iterates at least once unless r == 0
      if (sc->max_it <= 0) sc->done = 1;
      if (!isfinite(q[0]) || !isfinite(q[1])) sc->status = 3;
      break;
    }
    case FIN_ALPHA:
      sc->rhAp = q[0];
      if (q[0] == 0.0) {
        sc->status = 2;
      } else {
        sc->alpha = sc->rhr / q[0];
      }
      break;
    case FIN_OMEGA:
      sc->rAr = q[0];
      sc->ArAr = q[1];
      if (q[1] == 0.0) {
        sc->status = 2;
      } else {
        sc->omega = q[0] / q[1];
      }
      break;
    case FIN_NORMS: {
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
    default:
      break;
  }
}

__global__ void __launch_bounds__(256) k_fin2(const double* __restrict__ p1, int nb, int nq, int maxmask, int mode,
                                              SolverScalars* sc, double* raw_out) {
  if (mode != FIN_RAW && mode != FIN_INIT && halted(sc)) return;
  __shared__ double sh[4][8];
  __shared__ double tot[4];
  for (int q = 0; q < nq; ++q) {
    const bool mx = (maxmask >> q) & 1;
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const double x = p1[(long long)b * nq + q];
      v = mx ? fmax(v, x) : v + x;
    }
    v = mx ? wmax(v) : wsum(v);
    if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int q = 0; q < nq; ++q) {
      const bool mx = (maxmask >> q) & 1;
      double x = threadIdx.x < 8 ? sh[q][threadIdx.x] : 0.0;
      x = mx ? wmax(x) : wsum(x);
      if (threadIdx.x == 0) tot[q] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double q4[4] = {0, 0, 0, 0};
    for (int q = 0; q < nq; ++q) q4[q] = tot[q];
    scalar_update(mode, nq, q4, sc, raw_out);
  }
}

// begin of an iteration (mod_solvers.f90:~1600-1680): rhr, breakdown tests, beta, omega
__global__ void k_begin(SolverScalars* sc) {
  if (halted(sc)) return;
  sc->it += 1;
  sc->rhr_prev = sc->rhr;
  sc->rhr = sc->rhr_next;
  if (sc->rhr == 0.0) {  // rh must be reset to rr (reference resets and continues); host handles it
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

static void finalize(const double* partial, long long nb, int nq, int maxmask, int mode, SolverScalars* sc,
                     double* raw_out, cudaStream_t s) {
  double* p1 = const_cast<double*>(partial) + nb * 4;
  k_fin1<<<FIN1_BLOCKS, 256, 0, s>>>(partial, nb, nq, maxmask, p1, (mode == FIN_RAW || mode == FIN_INIT) ? nullptr : sc);
  k_fin2<<<1, 256, 0, s>>>(p1, FIN1_BLOCKS, nq, maxmask, mode, sc, raw_out);
  prof::count(2);
}

// ---------------------------------------------------------------------------------------
// fused vector kernels of one BiCGstab iteration (scalars read from device memory)
// ---------------------------------------------------------------------------------------
#define PT_SETUP                                              \
  const int i = blockIdx.x * BX + threadIdx.x + 1;            \
  const int j = blockIdx.y * BY + threadIdx.y + 1;            \
  const int k = blockIdx.z + 1;                               \
  const bool in = (i <= g.n1) && (j <= g.n2);                 \
  const long long p = in ? off(g, i, j, k) : 0;

template <typename T>
__global__ void __launch_bounds__(NT) k_p_update(Geom g, const SolverScalars* __restrict__ sc, const T* __restrict__ rr,
                                                 const T* __restrict__ Ap, T* __restrict__ pp) {
  if (halted(sc)) return;
  PT_SETUP
  if (!in) return;
  if (sc->it == 1) {
    pp[p] = rr[p];
  } else {
    pp[p] = (T)((double)rr[p] + sc->beta * (double)pp[p] + sc->omega * (double)Ap[p]);
  }
}
template <typename T>
__global__ void __launch_bounds__(NT) k_r_update(Geom g, const SolverScalars* __restrict__ sc, const T* __restrict__ Ap,
                                                 T* __restrict__ rr) {
  if (halted(sc)) return;
  PT_SETUP
  if (!in) return;
  rr[p] = (T)((double)rr[p] - sc->alpha * (double)Ap[p]);
}
// phi += omega*z2 + alpha*z1 ; rr -= omega*Ar ; partials [max|rr|, sum rr^2, rr.rh]
template <typename T>
__global__ void __launch_bounds__(NT) k_x_update(Geom g, const SolverScalars* __restrict__ sc, const T* __restrict__ z1,
                                                 const T* __restrict__ z2, const T* __restrict__ Ar,
                                                 const T* __restrict__ rh, T* __restrict__ phi, T* __restrict__ rr,
                                                 double* __restrict__ partial) {
  if (halted(sc)) return;
  PT_SETUP
  double v[3] = {0.0, 0.0, 0.0};
  if (in) {
    const double om = sc->omega, al = sc->alpha;
    phi[p] = (T)((double)phi[p] + om * (double)z2[p] + al * (double)z1[p]);
    const T r = (T)((double)rr[p] - om * (double)Ar[p]);
    rr[p] = r;
    const double rd = (double)r;
    v[0] = fabs(rd);
    v[1] = rd * rd;
    v[2] = rd * (double)rh[p];
  }
  block_partials<3, 1>(v, partial);
}
// initial residual: rr = bb - rr(=A phi) ; rh = rr ; partials [max|rr|, sum rr^2, rr.rh, sum bb^2]
template <typename T>
__global__ void __launch_bounds__(NT) k_init_residual(Geom g, int zero_phi, const T* __restrict__ bb, T* __restrict__ phi,
                                                      T* __restrict__ rr, T* __restrict__ rh, double* __restrict__ partial) {
  PT_SETUP
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (in) {
    const T b = bb[p];
    T r;
    if (zero_phi) {
      phi[p] = T(0);
      r = b;
    } else {
      r = b - rr[p];
    }
    rr[p] = r;
    rh[p] = r;
    const double rd = (double)r, bd = (double)b;
    v[0] = fabs(rd);
    v[1] = rd * rd;
    v[2] = rd * rd;
    v[3] = bd * bd;
  }
  block_partials<4, 1>(v, partial);
}

// Jacobi preconditioner sweeps, halted-aware wrappers
template <typename T>
__device__ __forceinline__ T init_val(const T* c1, const T* c2, const T* c3, T omega, T bb, int i, int j, int k) {
  return omega * bb / (c1[3 * (i - 1) + 1] + c2[3 * (j - 1) + 1] + c3[3 * (k - 1) + 1]);
}
template <typename T>
__device__ __forceinline__ T jac(const T* a, const T* b, const T* c, T omega, T bb, T xc, T xm, T xp, T ym, T yp, T zm,
                                 T zp) {
  return omega * (bb - a[0] * xm - a[2] * xp - b[0] * ym - b[2] * yp - c[0] * zm - c[2] * zp) / (a[1] + b[1] + c[1]) +
         (T(1) - omega) * xc;
}
template <typename T>
__global__ void __launch_bounds__(NT) k_pc_init1(Geom g, Coeffs<T> c, T omega, const SolverScalars* __restrict__ sc,
                                                 const T* __restrict__ bb, T* __restrict__ out) {
  if (halted(sc)) return;
  PT_SETUP
  if (!in) return;
  out[p] = init_val(c.cdg[0], c.cdg[1], c.cdg[2], omega, bb[p], i, j, k);
}
template <typename T>
static void precond(const Geom& g, const Coeffs<T>& c, int n, T omega, const SolverScalars* sc, const T* v, T* z,
                    T* comp, cudaStream_t s) {
  const dim3 gr = grid3(g), bl(BX, BY);
  const double cells = (double)g.n1 * g.n2 * g.n3;
  if (n == 1) {
    IMPACT_PROF(prof::K_PC_INIT2, 2.0 * sizeof(T) * cells, s, k_pc_init1<T><<<gr, bl, 0, s>>>(g, c, omega, sc, v, z));
    return;
  }
  // writes w_1 .. w_{n-1}; the last one must land in z
  T* bufs[2] = {z, comp};
  int tgt = ((n - 1) % 2 == 1) ? 0 : 1;
  IMPACT_PROF(prof::K_PC_INIT2, 2.0 * sizeof(T) * cells, s,
              (launch_jacobi25<T, 1>(g, c, sc, omega, v, nullptr, bufs[tgt], s)));
  for (int w = 2; w <= n - 1; ++w) {
    const int nt = 1 - tgt;
    IMPACT_PROF(prof::K_PC_SWEEP, 3.0 * sizeof(T) * cells, s,
                (launch_jacobi25<T, 0>(g, c, sc, omega, v, bufs[tgt], bufs[nt], s)));
    tgt = nt;
  }
}

__global__ void k_resume(SolverScalars* sc) {
  sc->status = 0;
  sc->it -= 1;
  sc->rhr = sc->rhr_prev;
}

template <typename T>
__global__ void k_copy(Geom g, const T* __restrict__ a, T* __restrict__ b) {
  PT_SETUP
  if (!in) return;
  b[p] = a[p];
}

// ---------------------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------------------
template <typename T>
int bicgstab(const Geom& g, const Coeffs<T>& c, const SolverOpts& o, const T* bb, T* phi, KrylovWork<T>& w,
             cudaStream_t s, SolverResult* res) {
  const dim3 gr = grid3(g), bl(BX, BY);
  const long long nb = nblocks3(g);
  const long long nb25 = s25_blocks(g);
  const double cells = (double)g.n1 * g.n2 * g.n3;
  const bool use_mg = o.precond == 1 && o.mg != nullptr;
  const bool pre_on = use_mg || o.n_sweeps > 0;
  const T om = (T)o.omega;
  const MGData<T>* mg = static_cast<const MGData<T>*>(o.mg);
  SolverScalars init{};
  init.tol_rel = o.tol_rel;
  init.tol_abs_inf = o.tol_abs_inf;
  init.max_it = o.max_it;
  cudaMemcpyAsync(w.scal, &init, sizeof(SolverScalars), cudaMemcpyHostToDevice, s);
  // initial residual
  if (!o.init_yes) launch_divgrad25<T, 0>(g, c, w.scal, phi, w.rr, nullptr, nullptr, s);
  k_init_residual<T><<<gr, bl, 0, s>>>(g, o.init_yes, bb, phi, w.rr, w.rh, w.partial);
  prof::count(o.init_yes ? 1 : 2);
  finalize(w.partial, nb, 4, 1, FIN_INIT, w.scal, nullptr, s);

  const int chunk = o.check_every > 0 ? o.check_every : 1;
  int launched = 0;
  for (;;) {
    for (int t = 0; t < chunk; ++t) {
      k_begin<<<1, 1, 0, s>>>(w.scal);
      prof::count(1);
      IMPACT_PROF(prof::K_P_UPDATE, 4.0 * sizeof(T) * cells, s,
                  k_p_update<T><<<gr, bl, 0, s>>>(g, w.scal, w.rr, w.Ap, w.pp));
      T* z1 = w.pp;
      if (use_mg) {
        mg_vcycle<T>(*mg, w.scal, w.pp, w.z1, w.comp, s);
        z1 = w.z1;
      } else if (pre_on) {
        precond<T>(g, c, o.n_sweeps, om, w.scal, w.pp, w.z1, w.comp, s);
        z1 = w.z1;
      }
      IMPACT_PROF(prof::K_DIVGRAD, 3.0 * sizeof(T) * cells, s,
                  (launch_divgrad25<T, 1>(g, c, w.scal, z1, w.Ap, w.rh, w.partial, s)));
      finalize(w.partial, nb25, 1, 0, FIN_ALPHA, w.scal, nullptr, s);
      IMPACT_PROF(prof::K_R_UPDATE, 3.0 * sizeof(T) * cells, s,
                  k_r_update<T><<<gr, bl, 0, s>>>(g, w.scal, w.Ap, w.rr));
      T* z2 = w.rr;
      if (use_mg) {
        mg_vcycle<T>(*mg, w.scal, w.rr, w.z2, w.comp, s);
        z2 = w.z2;
      } else if (pre_on) {
        precond<T>(g, c, o.n_sweeps, om, w.scal, w.rr, w.z2, w.comp, s);
        z2 = w.z2;
      }
      IMPACT_PROF(prof::K_DIVGRAD, 3.0 * sizeof(T) * cells, s,
                  (launch_divgrad25<T, 2>(g, c, w.scal, z2, w.Ar, w.rr, w.partial, s)));
      finalize(w.partial, nb25, 2, 0, FIN_OMEGA, w.scal, nullptr, s);
      // without a preconditioner z2 aliases rr: the x update reads rr before overwriting it
      IMPACT_PROF(prof::K_X_UPDATE, 8.0 * sizeof(T) * cells, s,
                  k_x_update<T><<<gr, bl, 0, s>>>(g, w.scal, z1, z2, w.Ar, w.rh, phi, w.rr, w.partial));
      finalize(w.partial, nb, 3, 1, FIN_NORMS, w.scal, nullptr, s);
      ++launched;
    }
    cudaError_t e = cudaMemcpyAsync(w.scal_host, w.scal, sizeof(SolverScalars), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return impact_set_error(e, "bicgstab poll", __FILE__, __LINE__);
    prof::flush();
    const SolverScalars& h = *w.scal_host;
    if (h.status == 4) {
      // rhr == 0: new shadow residual rh = rr, as the reference does, then redo the iteration start
      k_copy<T><<<gr, bl, 0, s>>>(g, w.rr, w.rh);
      reduce_dot<T>(g, w.rr, w.rh, w.partial, &w.scal->rhr_next, s);
      k_resume<<<1, 1, 0, s>>>(w.scal);
      continue;
    }
    if (h.done || h.status) break;
    if (launched > o.max_it + 8) break;  // safety net: the device flag should have stopped it
  }
  const SolverScalars& h = *w.scal_host;
  res->iterations = h.it;
  res->status = h.status;
  res->res_inf = h.norm_inf;
  res->res_two = sqrt(h.norm_two_sq);
  res->b_two = sqrt(h.b_two_sq);
  return 0;
}
template int bicgstab<double>(const Geom&, const Coeffs<double>&, const SolverOpts&, const double*, double*,
                              KrylovWork<double>&, cudaStream_t, SolverResult*);
template int bicgstab<float>(const Geom&, const Coeffs<float>&, const SolverOpts&, const float*, float*,
                             KrylovWork<float>&, cudaStream_t, SolverResult*);

// ---------------------------------------------------------------------------------------
// reductions for callers outside the Krylov loop (results land in device memory)
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_dot(Geom g, const T* __restrict__ a, const T* __restrict__ b,
                                            double* __restrict__ partial) {
  PT_SETUP
  double v[1] = {in ? (double)a[p] * (double)b[p] : 0.0};
  block_partials<1, 0>(v, partial);
}
template <typename T>
__global__ void __launch_bounds__(NT) k_norms(Geom g, const T* __restrict__ a, double* __restrict__ partial) {
  PT_SETUP
  const double x = in ? (double)a[p] : 0.0;
  double v[2] = {fabs(x), x * x};
  block_partials<2, 1>(v, partial);
}
template <typename T>
void reduce_dot(const Geom& g, const T* a, const T* b, double* partial, double* out_dev, cudaStream_t s) {
  k_dot<T><<<grid3(g), dim3(BX, BY), 0, s>>>(g, a, b, partial);
  finalize(partial, nblocks3(g), 1, 0, FIN_RAW, nullptr, out_dev, s);
}
template <typename T>
void reduce_norms(const Geom& g, const T* a, double* partial, double* out_dev, cudaStream_t s) {
  k_norms<T><<<grid3(g), dim3(BX, BY), 0, s>>>(g, a, partial);
  finalize(partial, nblocks3(g), 2, 1, FIN_RAW, nullptr, out_dev, s);
}
template void reduce_dot<double>(const Geom&, const double*, const double*, double*, double*, cudaStream_t);
template void reduce_dot<float>(const Geom&, const float*, const float*, double*, double*, cudaStream_t);
template void reduce_norms<double>(const Geom&, const double*, double*, double*, cudaStream_t);
template void reduce_norms<float>(const Geom&, const float*, double*, double*, cudaStream_t);

// ---------------------------------------------------------------------------------------
// mixed precision: FP64 iterative refinement around an FP32 BiCGstab
// ---------------------------------------------------------------------------------------
// r64 = b - A64 x ; partials [max|r|, sum r^2, sum b^2]
__global__ void __launch_bounds__(NT) k_outer_residual(Geom g, const double* __restrict__ bb,
                                                       const double* __restrict__ ax, double* __restrict__ r64,
                                                       double* __restrict__ partial) {
  PT_SETUP
  double v[3] = {0.0, 0.0, 0.0};
  if (in) {
    const double b = bb[p];
    const double r = b - ax[p];
    r64[p] = r;
    v[0] = fabs(r);
    v[1] = r * r;
    v[2] = b * b;
  }
  block_partials<3, 1>(v, partial);
}
// r32 = (float)(r64 * scale): the inner right-hand side normalised to |r|_inf = 1
__global__ void __launch_bounds__(NT) k_to_f32(Geom g, const double* __restrict__ r64, double scale,
                                               float* __restrict__ r32) {
  PT_SETUP
  if (!in) return;
  r32[p] = (float)(r64[p] * scale);
}
// x += unscale * e
__global__ void __launch_bounds__(NT) k_apply_correction(Geom g, const float* __restrict__ e, double unscale,
                                                         double* __restrict__ x) {
  PT_SETUP
  if (!in) return;
  x[p] = x[p] + unscale * (double)e[p];
}

// Iterative refinement (mod_solvers.f90 has no counterpart; the FP64 outer loop wraps the
// reference's BiCGstab run in FP32): r = b - A x in FP64, e = A^-1 r approximately by an FP32
// BiCGstab on the normalised r, x += e.  An inner solve that breaks down or turns non-finite is
// discarded and retried once with a looser tolerance.
int mixed_solve(const Geom& g, const Coeffs<double>& c64, const Coeffs<float>& c32, const SolverOpts& outer,
                const SolverOpts& inner, const double* bb, double* phi, MixedWork& w, cudaStream_t s,
                SolverResult* res, int* inner_iterations) {
  const dim3 gr = grid3(g), bl(BX, BY);
  const long long nb = nblocks3(g);
  const bool dbg = std::getenv("IMPACT_B200_DEBUG") != nullptr;
  int total_inner = 0;
  int outer_it = 0;
  int retries = 0;
  double q[4];
  double* qd = raw_results(w.partial64, g);
  res->status = 1;
  for (;;) {
    // r = b - A x  (FP64, the reference operator)
    launch_div_grad<double>(g, c64, phi, w.r64, s);
    k_outer_residual<<<gr, bl, 0, s>>>(g, bb, w.r64, w.r64, w.partial64);
    prof::count(2);
    finalize(w.partial64, nb, 3, 1, FIN_RAW, nullptr, qd, s);
    cudaError_t e = cudaMemcpyAsync(q, qd, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return impact_set_error(e, "mixed_solve residual", __FILE__, __LINE__);
    const double rinf = q[0], r2 = sqrt(q[1]), b2 = sqrt(q[2]);
    if (dbg)
      std::fprintf(stderr, "[impact_b200] mixed outer %d: |r|inf %.3e |r|2 %.3e |b|2 %.3e inner so far %d\n", outer_it,
                   rinf, r2, b2, total_inner);
    res->res_inf = rinf;
    res->res_two = r2;
    res->b_two = b2;
    if (!std::isfinite(rinf) || !std::isfinite(r2)) {
      res->status = 3;
      break;
    }
    const bool conv = (outer.tol_abs_inf > 0.0 && rinf < outer.tol_abs_inf) ||
                      (outer.tol_rel > 0.0 && r2 <= outer.tol_rel * b2) || rinf == 0.0;
    if (conv) {
      res->status = 0;
      break;
    }
    if (outer_it >= outer.max_it) {
      res->status = 1;
      break;
    }
    // inner FP32 solve A e = r / |r|_inf from e = 0
    SolverOpts io = inner;
    io.init_yes = 1;
    if (retries > 0) {
      io.tol_rel = fmax(io.tol_rel, 0.1);
      io.max_it = io.max_it < 200 ? io.max_it : 200;
    }
    if (outer.tol_rel > 0.0 && r2 > 0.0) {
      const double need = outer.tol_rel * b2 / r2;  // reduction still required
      if (need > io.tol_rel) io.tol_rel = fmin(0.5, need * 0.5);
    }
    k_to_f32<<<gr, bl, 0, s>>>(g, w.r64, 1.0 / rinf, w.r32);
    prof::count(1);
    SolverResult ir{};
    int rc = bicgstab<float>(g, c32, io, w.r32, w.e32, w.inner, s, &ir);
    if (rc) return rc;
    if (dbg)
      std::fprintf(stderr, "[impact_b200]   inner: it %d status %d |r|2/|b|2 %.3e tol %.1e\n", ir.iterations, ir.status,
                   ir.b_two > 0 ? ir.res_two / ir.b_two : 0.0, io.tol_rel);
    total_inner += ir.iterations;
    if (ir.status == 2 || ir.status == 3) {
      if (++retries > 2) {
        res->status = ir.status;
        break;
      }
      continue;  // discard this correction, retry with a looser tolerance
    }
    k_apply_correction<<<gr, bl, 0, s>>>(g, w.e32, rinf, phi);
    prof::count(1);
    ++outer_it;
  }
  res->iterations = outer_it;
  if (inner_iterations) *inner_iterations = total_inner;
  return 0;
}

}  // namespace impact
