// rhs.cu -- rhs_vel of one velocity component as a z-marching shared-memory stencil pass.
//
// rhs_vel (mod_rhs.f90:35-140) for component m forms, at every u_m point,
//   pp_a  = interpolate2_pre_vel(m, work_a)            (6-point, along axis m; mod_diff.f90:1567-1648)
//   nl_m  = sum_a pp_a * D^{up/down}_a vel_m           (7-point upwind-biased set chosen by the sign
//                                                       of pp_a; mod_diff.f90:784-1424)
//         - (1/Re) sum_a D2_a vel_m                    (Helmholtz_explicit, mod_diff.f90:549-762)
//   rhs_m = vel_m - dt bRK nl_m(old) - dt aRK nl_m(new)
// with the reference's operation order per point (each stencil sums its terms in table order;
// the advective terms and the three second derivatives accumulate axis by axis).
//
// A block owns TX x TY = 32 x 8 columns and walks them along z over KZ planes.  Every plane of
// vel_m (with its 3-wide x/y halo, periodic images) and of the three work fields (with the
// halo of the interpolation along axis m) is staged into a ring of R shared-memory slots by
// cp.async, R-4 planes ahead of its use.  The x and y neighbours come from the ring, the z
// values of the column from register windows: vel_m at k-3..k+3 and, for m = 3, work_a at
// k-2..k+3.  x coefficient rows (one per thread column) are staged once per block, transposed,
// the y rows of the block's 8 rows once per block (warp-uniform reads), and the z rows of every
// staged plane into its ring slot with the plane (block-uniform reads).
#include <cuda_runtime.h>

#include "common.cuh"
#include "rhs.cuh"

namespace impact {
namespace {

constexpr int RTX = 32, RTY = 8, RNT = RTX * RTY;
// RK3 coefficients (mod_vars.f90:774-775) for the batched pass, which forms dt aRK / dt bRK itself
__constant__ double RK_A[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
__constant__ double RK_B[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
constexpr int RR = 7;                                 // ring slots: planes c .. c+3 resident, 3 in flight
constexpr int VW = RTX + 6, VH = RTY + 6, VE = VW * VH;  // vel tile with the 3-wide halo
constexpr int NXR = 27;                               // x coefficient rows: U 7, D 7, D2 7, I 6
// y / z coefficient row in shared memory: U at 0, D at 8, D2 at 16, I at 24 (7, 7, 7, 6 values),
// every group 16-byte aligned so that uniform reads take two values per load
constexpr int NCR = 32;
constexpr int CU = 0, CD = 8, CH = 16, CI = 24;

template <int M>
struct WTile {  // work tile of one field: halo -2..3 along axis M only
  static constexpr int W = M == 0 ? RTX + 5 : RTX;
  static constexpr int H = M == 1 ? RTY + 5 : RTY;
  static constexpr int E = W * H;
};
template <int M>
constexpr int slot_elems() { return VE + 3 * WTile<M>::E + NCR; }  // vel tile, work tiles, z row
static_assert(VE % 2 == 0 && (3 * WTile<0>::E) % 2 == 0 && (3 * WTile<1>::E) % 2 == 0 && (3 * WTile<2>::E) % 2 == 0 &&
                  (NXR * RTX) % 2 == 0,
              "z rows and y rows must stay 16-byte aligned");
template <int M, typename TW = double>
constexpr size_t rhs_smem_bytes() {
  return sizeof(TW) * ((size_t)RR * slot_elems<M>() + (size_t)NXR * RTX + (size_t)RTY * NCR);
}

// periodic image of index i in 1..n, for any integer i
__device__ __forceinline__ int wrapg(int i, int n) {
  int r = (i - 1) % n;
  if (r < 0) r += n;
  return r + 1;
}

// N consecutive values from shared memory aligned to two values, two per load
template <int N>
__device__ __forceinline__ void ld_row(const double* p, double (&o)[N]) {
#pragma unroll
  for (int l = 0; l + 1 < N; l += 2) {
    const double2 v = *reinterpret_cast<const double2*>(p + l);
    o[l] = v.x;
    o[l + 1] = v.y;
  }
  if (N & 1) o[N - 1] = p[N - 1];
}
template <int N>
__device__ __forceinline__ void ld_row(const float* p, float (&o)[N]) {
#pragma unroll
  for (int l = 0; l + 1 < N; l += 2) {
    const float2 v = *reinterpret_cast<const float2*>(p + l);
    o[l] = v.x;
    o[l + 1] = v.y;
  }
  if (N & 1) o[N - 1] = p[N - 1];
}

__device__ __forceinline__ void cpa8(double* smem, const double* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa4(float* smem, const float* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa(double* smem, const double* gmem) { cpa8(smem, gmem); }
__device__ __forceinline__ void cpa(float* smem, const float* gmem) { cpa4(smem, gmem); }
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// the pass of block (bx, by, bz) of a case's grid of blocks.  TW is the type of the work fields,
// the nonlinear term, the staged tiles, the coefficients and the arithmetic: double (FP64 cases)
// or float (mixed-precision cases: FP32 stencils with FP32 accumulation; the velocity and rhs_m
// stay FP64, the FP64 velocity staged into FP32 tiles by ordinary loads one plane ahead).
template <int M, typename TW>
__device__ __forceinline__ void rhs_march_block(const Geom& g, const Coeffs<TW>& c, double multL, double mult_b,
                                                double mult_a, int use_old, int kz, const double* __restrict__ vel,
                                                const TW* __restrict__ wk0, const TW* __restrict__ wk1,
                                                const TW* __restrict__ wk2, TW* __restrict__ nl,
                                                double* __restrict__ rhs, int bx, int by, int bz) {
  using WT = WTile<M>;
  constexpr bool F32 = sizeof(TW) == 4;
  constexpr int SE = slot_elems<M>();
  constexpr int VPER = (VE + RNT - 1) / RNT;
  constexpr int WPER = (3 * WT::E + RNT - 1) / RNT;
  extern __shared__ __align__(16) unsigned char rsm_raw[];
  TW* rsm = reinterpret_cast<TW*>(rsm_raw);
  TW* ring = rsm;                      // RR slots of SE values: vel tile, work tiles 0..2, z row
  TW* sx = rsm + (size_t)RR * SE;      // NXR x RTX transposed x rows
  TW* sy = sx + NXR * RTX;             // RTY x NCR y rows of the block's rows
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + RTX * ty;
  const int i0 = bx * RTX + 1, j0 = by * RTY + 1;
  const int k0 = bz * kz + 1;
  const int k1 = min(k0 + kz - 1, g.n3);
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i <= g.n1 && j <= g.n2;
  const TW* yU = M == 1 ? c.cNuU[1] : c.cNpU[1];
  const TW* yD = M == 1 ? c.cNuD[1] : c.cNpD[1];
  const TW* yH = M == 1 ? c.cuu[1] : c.cpp[1];
  const TW* zU = M == 2 ? c.cNuU[2] : c.cNpU[2];
  const TW* zD = M == 2 ? c.cNuD[2] : c.cNpD[2];
  const TW* zH = M == 2 ? c.cuu[2] : c.cpp[2];

  // x rows of this block's columns, transposed: sx[l][tx]
  {
    const TW* xU = M == 0 ? c.cNuU[0] : c.cNpU[0];
    const TW* xD = M == 0 ? c.cNuD[0] : c.cNpD[0];
    const TW* xH = M == 0 ? c.cuu[0] : c.cpp[0];
    for (int t = tid; t < NXR * RTX; t += RNT) {
      const int l = t / RTX, col = t % RTX;
      const int row = wrapg(i0 + col, g.n1);
      TW v;
      if (l < 7) v = xU[row * NB + l];
      else if (l < 14) v = xD[row * NB + (l - 7)];
      else if (l < 21) v = xH[row * NB + (l - 14)];
      else v = M == 0 ? c.cIpu[0][row * NG + (l - 21)] : TW(0);
      sx[t] = v;
    }
    // y rows of the block's rows
    for (int t = tid; t < RTY * NCR; t += RNT) {
      const int r = t / NCR, e = t % NCR, grp = e / 8, l = e % 8;
      const int row = wrapg(j0 + r, g.n2);
      TW v = TW(0);
      if (grp == 0 && l < 7) v = yU[row * NB + l];
      else if (grp == 1 && l < 7) v = yD[row * NB + l];
      else if (grp == 2 && l < 7) v = yH[row * NB + l];
      else if (grp == 3 && l < 6 && M == 1) v = c.cIpu[1][row * NG + l];
      sy[t] = v;
    }
  }
  // in-plane source offsets of this thread's staged elements (periodic images)
  int vo[VPER];
#pragma unroll
  for (int e = 0; e < VPER; ++e) {
    const int t = tid + e * RNT;
    const int r = t / VW, col = t % VW;
    vo[e] = t < VE ? (wrapg(i0 - 3 + col, g.n1) + 3) + g.nx * (wrapg(j0 - 3 + r, g.n2) + 3) : -1;
  }
  const TW* wsrc[WPER];
  int wdst[WPER];
#pragma unroll
  for (int e = 0; e < WPER; ++e) {
    const int t = tid + e * RNT;
    const int f = t / WT::E, u = t % WT::E;
    const int r = u / WT::W, col = u % WT::W;
    const int gi = wrapg(i0 + col - (M == 0 ? 2 : 0), g.n1), gj = wrapg(j0 + r - (M == 1 ? 2 : 0), g.n2);
    const TW* base = f == 0 ? wk0 : (f == 1 ? wk1 : wk2);
    wsrc[e] = t < 3 * WT::E ? base + (gi + 3) + (long long)g.nx * (gj + 3) : nullptr;
    wdst[e] = VE + t;
  }
  const int nq = (k1 - k0 + 1) + 6;  // planes k0-3 .. k1+3
  auto zwrap = [&](int q) { const int kk = k0 - 3 + q; return kk < 1 ? kk + g.n3 : (kk > g.n3 ? kk - g.n3 : kk); };
  auto zoff = [&](int q) -> long long { return (long long)(zwrap(q) + 3) * g.nxy; };
  // z row of a staged plane: thread e < NCR copies element e of the row layout
  const int zg = tid / 8, zl = tid % 8;
  const bool zcopy = tid < NCR && (zg < 3 ? zl < 7 : (zl < 6 && M == 2));
  const TW* zsrc = zg == 0 ? zU + zl : (zg == 1 ? zD + zl : (zg == 2 ? zH + zl : c.cIpu[2] + zl));
  const int zstride = zg < 3 ? NB : NG;
  double vpend[VPER];  // FP32: the velocity of the plane staged last, stored at the next stage()
  auto stage = [&](int q) {
    if (F32 && q >= 1 && q - 1 < nq) {
      TW* prev = ring + (size_t)((q - 1) % RR) * SE;
#pragma unroll
      for (int e = 0; e < VPER; ++e)
        if (vo[e] >= 0) prev[tid + e * RNT] = (TW)vpend[e];
    }
    if (q < nq) {
      TW* slot = ring + (size_t)(q % RR) * SE;
      const long long zo = zoff(q);
#pragma unroll
      for (int e = 0; e < VPER; ++e) {
        if (vo[e] < 0) continue;
        if constexpr (F32)
          vpend[e] = __ldg(vel + zo + vo[e]);
        else
          cpa8(reinterpret_cast<double*>(slot) + tid + e * RNT, vel + zo + vo[e]);
      }
#pragma unroll
      for (int e = 0; e < WPER; ++e)
        if (wsrc[e]) cpa(slot + wdst[e], wsrc[e] + zo);
      if (zcopy) cpa(slot + (SE - NCR) + tid, zsrc + zwrap(q) * zstride);
    }
    cpa_commit();
  };
#pragma unroll
  for (int q = 0; q < RR - 4; ++q) stage(q);

  TW vq[7];                                        // vel of the column, planes c-3 .. c+3
  TW wq[3][6];                                    // m = 3: work_a of the column, planes c-2 .. c+3
#pragma unroll
  for (int l = 0; l < 7; ++l) vq[l] = TW(0);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int l = 0; l < 6; ++l) wq[a][l] = TW(0);

  const int own = (tx + 3) + VW * (ty + 3);
  const TW* cy = sy + ty * NCR;  // this thread's y row (warp-uniform)
  long long p = off(g, i, j, k0);    // output point of plane k (advanced per plane)

  for (int t = 0; t < nq; ++t) {
    cpa_wait<RR - 5>();   // this thread's copies of plane t have landed
    __syncthreads();      // everybody's have; the slot of plane t-4 is free again
    stage(t + RR - 4);
    const TW* slot = ring + (size_t)(t % RR) * SE;
#pragma unroll
    for (int l = 0; l < 6; ++l) vq[l] = vq[l + 1];
    vq[6] = slot[own];
    if (M == 2) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int l = 0; l < 5; ++l) wq[a][l] = wq[a][l + 1];
        wq[a][5] = slot[VE + a * WT::E + tid];
      }
    }
    if (t < 6) continue;
    if (t > 6) p += g.nxy;
    if (!in) continue;
    const TW* cs = ring + (size_t)((t - 3) % RR) * SE;  // plane k = k0 + t - 6
    const TW* cz = cs + (SE - NCR);                     // its z row (block-uniform)
    const TW nlo = use_old ? nl[p] : TW(0);
    // vel_m neighbours along x and y (plane k), z (register window)
    TW xv[7], yv[7];
#pragma unroll
    for (int l = 0; l < 7; ++l) {
      xv[l] = cs[(ty + 3) * VW + tx + l];
      yv[l] = cs[(ty + l) * VW + tx + 3];
    }
    // interpolation weights along axis m, shared by the three work fields
    TW ci[6];
    if (M == 0) {
#pragma unroll
      for (int l = 0; l < 6; ++l) ci[l] = sx[(21 + l) * RTX + tx];
    } else {
      ld_row((M == 1 ? cy : cz) + CI, ci);
    }
    TW acc = TW(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // pp = interpolate2_pre_vel(m, work_a) along axis m
      TW pp;
      if (M == 0) {
        const TW* w = cs + VE + a * WT::E + ty * WT::W + tx;
        pp = ci[0] * w[0];
#pragma unroll
        for (int l = 1; l < 6; ++l) pp = pp + ci[l] * w[l];
      } else if (M == 1) {
        const TW* w = cs + VE + a * WT::E + ty * WT::W + tx;
        pp = ci[0] * w[0];
#pragma unroll
        for (int l = 1; l < 6; ++l) pp = pp + ci[l] * w[l * WT::W];
      } else {
        pp = ci[0] * wq[a][0];
#pragma unroll
        for (int l = 1; l < 6; ++l) pp = pp + ci[l] * wq[a][l];
      }
      TW dd;
      if (a == 0) {
        const TW* cr = sx + (pp >= TW(0) ? 0 : 7) * RTX + tx;
        dd = cr[0] * xv[0];
#pragma unroll
        for (int l = 1; l < 7; ++l) dd = dd + cr[l * RTX] * xv[l];
      } else if (a == 1) {
        TW cr[7];
        ld_row(cy + (pp >= TW(0) ? CU : CD), cr);
        dd = cr[0] * yv[0];
#pragma unroll
        for (int l = 1; l < 7; ++l) dd = dd + cr[l] * yv[l];
      } else {
        TW cr[7];
        ld_row(cz + (pp >= TW(0) ? CU : CD), cr);
        dd = cr[0] * vq[0];
#pragma unroll
        for (int l = 1; l < 7; ++l) dd = dd + cr[l] * vq[l];
      }
      acc = (a == 0) ? dd * pp : acc + dd * pp;
    }
    // Helmholtz_explicit: x, y, z second derivatives of vel_m
    TW lap = sx[14 * RTX + tx] * xv[0];
#pragma unroll
    for (int l = 1; l < 7; ++l) lap = lap + sx[(14 + l) * RTX + tx] * xv[l];
    {
      TW ch[7];
      ld_row(cy + CH, ch);
#pragma unroll
      for (int l = 0; l < 7; ++l) lap = lap + ch[l] * yv[l];
      ld_row(cz + CH, ch);
#pragma unroll
      for (int l = 0; l < 7; ++l) lap = lap + ch[l] * vq[l];
    }
    const TW nln = acc - (TW)multL * lap;
    double r = F32 ? vel[p] : (double)vq[3];  // FP32 tiles: the FP64 velocity of the point itself
    if (use_old) r = r - mult_b * (double)nlo;
    r = r - mult_a * (double)nln;
    nl[p] = nln;
    rhs[p] = r;
  }
  cpa_wait<0>();
}

template <int M, typename TW>
__global__ void __launch_bounds__(RNT, 2) k_rhs_march(Geom g, Coeffs<TW> c, double multL, double mult_b,
                                                      double mult_a, int use_old, int kz,
                                                      const double* __restrict__ vel, const TW* __restrict__ wk0,
                                                      const TW* __restrict__ wk1, const TW* __restrict__ wk2,
                                                      TW* __restrict__ nl, double* __restrict__ rhs) {
  rhs_march_block<M, TW>(g, c, multL, mult_b, mult_a, use_old, kz, vel, wk0, wk1, wk2, nl, rhs, blockIdx.x,
                         blockIdx.y, blockIdx.z);
}

// the pass over the cases of a batch: block b of the launch is block b - job.b0 of its case
template <int M, typename TW>
__global__ void __launch_bounds__(RNT, 2) k_rhs_march_batch(const RhsJob* __restrict__ jobs, int nj, int sub) {
  int lo = 0, hi = nj - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].b0 <= b) lo = mid; else hi = mid - 1;
  }
  const RhsJob& J = jobs[lo];
  const int lb = b - J.b0;
  const int bx = lb % J.gx, by = (lb / J.gx) % J.gy, bz = lb / (J.gx * J.gy);
  const double dt = *J.dt;
  const double multL = 1.0 / *J.Re;
  if constexpr (sizeof(TW) == 8)
    rhs_march_block<M, double>(J.g, J.c, multL, dt * RK_B[sub], dt * RK_A[sub], sub != 0, J.kz, J.vel[M], J.work[0],
                               J.work[1], J.work[2], J.nl[M], J.rhs[M], bx, by, bz);
  else
    rhs_march_block<M, float>(J.g, J.c32, multL, dt * RK_B[sub], dt * RK_A[sub], sub != 0, J.kz, J.vel[M],
                              J.work32[0], J.work32[1], J.work32[2], J.nl32[M], J.rhs[M], bx, by, bz);
}

template <int M, typename TW>
void launch_m(const Geom& g, const Coeffs<TW>& c, double multL, double mult_b, double mult_a, int use_old,
              const double* vel, const TW* const work[3], TW* nl, double* rhs, cudaStream_t s) {
  static unsigned long long attr_set = 0;  // devices on which the shared-memory limit was raised
  constexpr size_t bytes = rhs_smem_bytes<M, TW>();
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set >> dev & 1ULL)) {
    cudaFuncSetAttribute(k_rhs_march<M, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    attr_set |= 1ULL << dev;
  }
  const int kz = rhs_march_kz(g);
  const dim3 grid((g.n1 + RTX - 1) / RTX, (g.n2 + RTY - 1) / RTY, (g.n3 + kz - 1) / kz);
  k_rhs_march<M, TW><<<grid, dim3(RTX, RTY), bytes, s>>>(g, c, multL, mult_b, mult_a, use_old, kz, vel, work[0],
                                                         work[1], work[2], nl, rhs);
}

template <int M, typename TW>
void launch_batch_m(const RhsJob* jobs, int nj, int blocks, int sub, cudaStream_t s) {
  static unsigned long long attr_set = 0;
  constexpr size_t bytes = rhs_smem_bytes<M, TW>();
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set >> dev & 1ULL)) {
    cudaFuncSetAttribute(k_rhs_march_batch<M, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    attr_set |= 1ULL << dev;
  }
  k_rhs_march_batch<M, TW><<<blocks, dim3(RTX, RTY), bytes, s>>>(jobs, nj, sub);
}

}  // namespace

void rhs_march_job_grid(const Geom& g, RhsJob& J, int kz) {
  J.kz = kz > 0 ? kz : rhs_march_kz(g);
  J.gx = (g.n1 + RTX - 1) / RTX;
  J.gy = (g.n2 + RTY - 1) / RTY;
  J.gz = (g.n3 + J.kz - 1) / J.kz;
}

void launch_rhs_march_batch(int m, const RhsJob* jobs, int nj, int blocks, int sub, int f32, cudaStream_t s) {
  if (f32) {
    if (m == 0)
      launch_batch_m<0, float>(jobs, nj, blocks, sub, s);
    else if (m == 1)
      launch_batch_m<1, float>(jobs, nj, blocks, sub, s);
    else
      launch_batch_m<2, float>(jobs, nj, blocks, sub, s);
  } else {
    if (m == 0)
      launch_batch_m<0, double>(jobs, nj, blocks, sub, s);
    else if (m == 1)
      launch_batch_m<1, double>(jobs, nj, blocks, sub, s);
    else
      launch_batch_m<2, double>(jobs, nj, blocks, sub, s);
  }
}

// planes per block: enough blocks for several waves of two blocks per SM, at most 64 planes (a
// block reads 6 planes beyond its own, so deeper blocks read less twice); column_planes = block
// columns x planes of the grid, or of all grids of a batch, whose blocks run in one launch
int rhs_march_kz_for(long long column_planes) {
  long long kz = column_planes / (148LL * 2 * 8);
  kz = kz < 8 ? 8 : (kz > 64 ? 64 : kz);
  return (int)kz;
}
long long rhs_march_column_planes(const Geom& g) {
  return (long long)((g.n1 + RTX - 1) / RTX) * ((g.n2 + RTY - 1) / RTY) * g.n3;
}
int rhs_march_kz(const Geom& g) { return rhs_march_kz_for(rhs_march_column_planes(g)); }

void launch_rhs_march(int m, const Geom& g, const Coeffs<double>& c, double multL, double mult_b, double mult_a,
                      int use_old, const double* vel, const double* const work[3], double* nl, double* rhs,
                      cudaStream_t s) {
  if (m == 0)
    launch_m<0, double>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
  else if (m == 1)
    launch_m<1, double>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
  else
    launch_m<2, double>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
}

void launch_rhs_march32(int m, const Geom& g, const Coeffs<float>& c, double multL, double mult_b, double mult_a,
                        int use_old, const double* vel, const float* const work[3], float* nl, double* rhs,
                        cudaStream_t s) {
  if (m == 0)
    launch_m<0, float>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
  else if (m == 1)
    launch_m<1, float>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
  else
    launch_m<2, float>(g, c, multL, mult_b, mult_a, use_old, vel, work, nl, rhs, s);
}

}  // namespace impact
