// march.cu -- the one-axis stencil operators of the launcher FFI as streaming passes.
//
// gradient (mod_diff.f90:309-414), divergence per axis (:52-118), both interpolations
// (:1567-1648, :1740-1825) and the upwind advection term (:784-1424) are 6- or 7-point stencils
// along one axis a: out(q) = sum_{l} c(l, q) f(q + LO + l), q the coordinate along a, with the
// row of coefficients c(., q) of that coordinate.  Here every thread owns one 16-byte vector of
// x points (2 doubles or 4 floats; rows are 16-byte aligned when n1 is divisible by the vector
// width) and:
//   a = y or z: marches along a over a segment of the axis, keeping the CNT vectors of its
//               stencil in registers (one new 16-byte load and one 16-byte store per step), the
//               coefficient row of the step being the same for the whole block;
//   a = x:      marches z as well, with the coefficient rows of its points loaded once; each
//               plane takes the few aligned vectors of the row that its points' stencils span
//               (neighbouring vectors, periodic images at the row ends).
// Periodic wrapping is applied to the coordinate along a only.  Each point sums its terms in
// table order with the same fused multiply-adds as the one-point-per-thread kernels of
// kernels.cu, so both give the same bits.
#include "kernels.cuh"

namespace impact {
namespace {

template <typename T>
struct V16;
template <>
struct V16<double> {
  using t = double2;
  static constexpr int W = 2;
};
template <>
struct V16<float> {
  using t = float4;
  static constexpr int W = 4;
};
template <typename T>
__device__ __forceinline__ void vld(const T* p, T (&o)[V16<T>::W]) {
  const typename V16<T>::t v = __ldg(reinterpret_cast<const typename V16<T>::t*>(p));
  if constexpr (V16<T>::W == 2) {
    o[0] = v.x;
    o[1] = v.y;
  } else {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  }
}
template <typename T>
__device__ __forceinline__ void vld_plain(const T* p, T (&o)[V16<T>::W]) {  // may alias the output
  const typename V16<T>::t v = *reinterpret_cast<const typename V16<T>::t*>(p);
  if constexpr (V16<T>::W == 2) {
    o[0] = v.x;
    o[1] = v.y;
  } else {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  }
}
template <typename T>
__device__ __forceinline__ void vst(T* p, const T (&o)[V16<T>::W]) {
  if constexpr (V16<T>::W == 2)
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  else
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mulT(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulT(double a, double b) { return __dmul_rn(a, b); }

// OP 0: out = S f;  OP 1: out = out + S f (terms added to the old value in order);
// OP 2: upwind, out = S_sel f * pp (first axis) or out + S_sel f * pp, S_sel the cA row where
// pp >= 0 and the cB row elsewhere
template <typename T, int CNT, int OP>
__device__ __forceinline__ T point_value(const T* __restrict__ ca, const T* __restrict__ cb, const T (&win)[CNT],
                                         T old, T ppv, int first) {
  if (OP == 1) {
    T s = old;
#pragma unroll
    for (int l = 0; l < CNT; ++l) s = fmaT(ca[l], win[l], s);
    return s;
  }
  const T* c = (OP == 2 && !(ppv >= T(0))) ? cb : ca;
  T s = mulT(c[0], win[0]);
#pragma unroll
  for (int l = 1; l < CNT; ++l) s = fmaT(c[l], win[l], s);
  if (OP == 2) return first ? mulT(s, ppv) : fmaT(s, ppv, old);
  return s;
}

constexpr int MBX = 32, MBY = 8;

// a = 1 (y) or 2 (z): thread (vector vx, other in-plane coordinate o) marches q = q0 .. q1
template <typename T, int LO, int CNT, int OP>
__global__ void __launch_bounds__(MBX* MBY) k_march_yz(int a, Geom g, const T* __restrict__ cA, const T* __restrict__ cB,
                                                       const T* __restrict__ f, const T* __restrict__ pp,
                                                       T* __restrict__ out, int first, int seg) {
  constexpr int W = V16<T>::W;
  const int i = 1 + W * (blockIdx.x * MBX + threadIdx.x);
  const int o = blockIdx.y * MBY + threadIdx.y + 1;
  const int na = a == 2 ? g.n3 : g.n2, no = a == 2 ? g.n2 : g.n3;
  if (i > g.n1 || o > no) return;
  const long long sa = a == 2 ? g.nxy : (long long)g.nx;
  const long long so = a == 2 ? (long long)g.nx : g.nxy;
  const long long base = (i + 3) + so * (o + 3) + sa * 3;  // (i, o, q = 0)
  const int q0 = blockIdx.z * seg + 1, q1 = min(na, q0 + seg - 1);
  T win[CNT][W];
#pragma unroll
  for (int l = 0; l < CNT; ++l) vld(f + base + sa * wrapi(q0 + LO + l, na), win[l]);
  for (int q = q0; q <= q1; ++q) {
    const long long p = base + sa * q;
    T old[W], pv[W], r[W];
    if (OP != 0) vld_plain(out + p, old);
    if (OP == 2) vld(pp + p, pv);
    const T* ca = cA + (long long)q * CNT;
    const T* cb = OP == 2 ? cB + (long long)q * CNT : ca;
    T ca_r[CNT], cb_r[CNT];
#pragma unroll
    for (int l = 0; l < CNT; ++l) {
      ca_r[l] = __ldg(ca + l);
      cb_r[l] = OP == 2 ? __ldg(cb + l) : ca_r[l];
    }
#pragma unroll
    for (int v = 0; v < W; ++v) {
      T wv[CNT];
#pragma unroll
      for (int l = 0; l < CNT; ++l) wv[l] = win[l][v];
      r[v] = point_value<T, CNT, OP>(ca_r, cb_r, wv, OP != 0 ? old[v] : T(0), OP == 2 ? pv[v] : T(0), first);
    }
    vst(out + p, r);
#pragma unroll
    for (int l = 0; l + 1 < CNT; ++l)
#pragma unroll
      for (int v = 0; v < W; ++v) win[l][v] = win[l + 1][v];
    if (q < q1) vld(f + base + sa * wrapi(q + 1 + LO + CNT - 1, na), win[CNT - 1]);
  }
}

// a = 0 (x): thread (vector, row j) marches z over a segment; the coefficient rows of its W
// points are loaded once, and each plane takes the few aligned vectors of the row that the W
// points' stencils span (neighbouring vectors, periodic images at the row ends)
template <typename T, int LO, int CNT, int OP>
__global__ void __launch_bounds__(MBX* MBY) k_march_x(Geom g, const T* __restrict__ cA, const T* __restrict__ cB,
                                                      const T* __restrict__ f, const T* __restrict__ pp,
                                                      T* __restrict__ out, int first, int seg) {
  constexpr int W = V16<T>::W;
  constexpr int FV = (LO - (W - 1)) / W;          // floor(LO / W) for LO < 0
  constexpr int LV = (W - 1 + LO + CNT - 1) / W;  // floor of the last position / W (>= 0)
  constexpr int NV = LV - FV + 1;
  const int vx = blockIdx.x * MBX + threadIdx.x;
  const int nvx = g.n1 / W;
  const int j = blockIdx.y * MBY + threadIdx.y + 1;
  if (vx >= nvx || j > g.n2) return;
  const int i = 1 + W * vx;
  const int k0 = blockIdx.z * seg + 1, k1 = min(g.n3, k0 + seg - 1);
  T ca[W][CNT], cb[W][CNT];
#pragma unroll
  for (int v = 0; v < W; ++v)
#pragma unroll
    for (int l = 0; l < CNT; ++l) {
      ca[v][l] = __ldg(cA + (long long)(i + v) * CNT + l);
      cb[v][l] = OP == 2 ? __ldg(cB + (long long)(i + v) * CNT + l) : ca[v][l];
    }
  int us[NV];
#pragma unroll
  for (int n = 0; n < NV; ++n) {
    const int u = vx + FV + n;
    us[n] = W * (u < 0 ? u + nvx : (u >= nvx ? u - nvx : u));
  }
  const long long rowj = 4 + (long long)g.nx * (j + 3);  // offset of (1, j, k = -3)
  for (int k = k0; k <= k1; ++k) {
    const long long row = rowj + g.nxy * (k + 3);
    T val[NV * W];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      T tmp[W];
      vld(f + row + us[n], tmp);
#pragma unroll
      for (int v = 0; v < W; ++v) val[n * W + v] = tmp[v];
    }
    const long long p = row + (i - 1);
    T old[W], pv[W], r[W];
    if (OP != 0) vld_plain(out + p, old);
    if (OP == 2) vld(pp + p, pv);
#pragma unroll
    for (int v = 0; v < W; ++v) {
      T wv[CNT];
#pragma unroll
      for (int l = 0; l < CNT; ++l) wv[l] = val[v + LO + l - FV * W];
      r[v] = point_value<T, CNT, OP>(ca[v], cb[v], wv, OP != 0 ? old[v] : T(0), OP == 2 ? pv[v] : T(0), first);
    }
    vst(out + p, r);
  }
}

// Helmholtz_explicit (mod_diff.f90:549-762): nl = nl - multL (cx u_xx + cy u_yy + cz u_zz), the
// three 7-point second derivatives summed in one chain x, then y, then z (as lap7_point in
// kernels.cu).  Thread (vector, row j) marches z over a segment: the column's z values k-3..k+3
// in registers, x neighbours from the aligned vectors of the row, y neighbours from the vectors
// of rows j-3..j+3 (shared with the block's other rows through L1).
template <typename T>
__global__ void __launch_bounds__(MBX* MBY) k_helm_march(Geom g, const T* __restrict__ cx, const T* __restrict__ cy,
                                                         const T* __restrict__ cz, T multL, const T* __restrict__ vel,
                                                         T* __restrict__ nl, int seg) {
  constexpr int W = V16<T>::W;
  constexpr int FV = (B_LO - (W - 1)) / W, LV = (W - 1 + B_LO + NB - 1) / W, NV = LV - FV + 1;
  const int vx = blockIdx.x * MBX + threadIdx.x;
  const int nvx = g.n1 / W;
  const int j = blockIdx.y * MBY + threadIdx.y + 1;
  if (vx >= nvx || j > g.n2) return;
  const int i = 1 + W * vx;
  const int k0 = blockIdx.z * seg + 1, k1 = min(g.n3, k0 + seg - 1);
  const long long rowj = 4 + (long long)g.nx * (j + 3);  // (1, j, k = -3)
  long long rows[NB];                                     // (1, j-3+l, k = -3)
#pragma unroll
  for (int l = 0; l < NB; ++l) rows[l] = 4 + (long long)g.nx * (wrapi(j + B_LO + l, g.n2) + 3);
  int us[NV];
#pragma unroll
  for (int n = 0; n < NV; ++n) {
    const int u = vx + FV + n;
    us[n] = W * (u < 0 ? u + nvx : (u >= nvx ? u - nvx : u));
  }
  T zc[NB][W];  // z window of the column: k-3 .. k+3
#pragma unroll
  for (int l = 0; l < NB; ++l) vld(vel + rowj + (long long)g.nxy * (wrapi(k0 + B_LO + l, g.n3) + 3) + (i - 1), zc[l]);
  T ycr[NB];
#pragma unroll
  for (int l = 0; l < NB; ++l) ycr[l] = __ldg(cy + (long long)j * NB + l);
  for (int k = k0; k <= k1; ++k) {
    const long long pz = g.nxy * (k + 3);
    T xv[NV * W];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      T tmp[W];
      vld(vel + rowj + pz + us[n], tmp);
#pragma unroll
      for (int v = 0; v < W; ++v) xv[n * W + v] = tmp[v];
    }
    T yv[NB][W];
#pragma unroll
    for (int l = 0; l < NB; ++l) {
      if (l == -B_LO) {
#pragma unroll
        for (int v = 0; v < W; ++v) yv[l][v] = zc[-B_LO][v];
      } else {
        vld(vel + rows[l] + pz + (i - 1), yv[l]);
      }
    }
    T zcr[NB];
#pragma unroll
    for (int l = 0; l < NB; ++l) zcr[l] = __ldg(cz + (long long)k * NB + l);
    const long long p = rowj + pz + (i - 1);
    T old[W], r[W];
    vld_plain(nl + p, old);
#pragma unroll
    for (int v = 0; v < W; ++v) {
      const T* xr = cx + (long long)(i + v) * NB;
      T d = mulT(__ldg(xr), xv[v + B_LO - FV * W]);
#pragma unroll
      for (int l = 1; l < NB; ++l) d = fmaT(__ldg(xr + l), xv[v + B_LO + l - FV * W], d);
#pragma unroll
      for (int l = 0; l < NB; ++l) d = fmaT(ycr[l], yv[l][v], d);
#pragma unroll
      for (int l = 0; l < NB; ++l) d = fmaT(zcr[l], zc[l][v], d);
      r[v] = fmaT(-multL, d, old[v]);
    }
    vst(nl + p, r);
#pragma unroll
    for (int l = 0; l + 1 < NB; ++l)
#pragma unroll
      for (int v = 0; v < W; ++v) zc[l][v] = zc[l + 1][v];
    if (k < k1) vld(vel + rowj + (long long)g.nxy * (wrapi(k + 1 - B_LO, g.n3) + 3) + (i - 1), zc[NB - 1]);
  }
}

// relaxation_div_grad / the JOR sweep (mod_laplace.f90:339-613, jacobi_kernel.cu):
// out = omega (bb - sum of the six off-diagonal terms of cdg) / diag + (1 - omega) rel, as
// jacobi_point in kernels.cu.  Thread (vector, row j) marches z with the column's rel at k-1..k+1
// in registers.
template <typename T>
__global__ void __launch_bounds__(MBX* MBY) k_jacobi_march(Geom g, const T* __restrict__ c1, const T* __restrict__ c2,
                                                           const T* __restrict__ c3, T omega, const T* __restrict__ bb,
                                                           const T* __restrict__ rel, T* __restrict__ out, int seg) {
  constexpr int W = V16<T>::W;
  const int vx = blockIdx.x * MBX + threadIdx.x;
  const int nvx = g.n1 / W;
  const int j = blockIdx.y * MBY + threadIdx.y + 1;
  if (vx >= nvx || j > g.n2) return;
  const int i = 1 + W * vx;
  const int k0 = blockIdx.z * seg + 1, k1 = min(g.n3, k0 + seg - 1);
  const long long rowj = 4 + (long long)g.nx * (j + 3);
  const long long rowm = 4 + (long long)g.nx * (wrapi(j - 1, g.n2) + 3), rowp = 4 + (long long)g.nx * (wrapi(j + 1, g.n2) + 3);
  const int um = W * (vx == 0 ? nvx - 1 : vx - 1), up = W * (vx == nvx - 1 ? 0 : vx + 1);
  T zc[3][W];
#pragma unroll
  for (int l = 0; l < 3; ++l) vld(rel + rowj + (long long)g.nxy * (wrapi(k0 - 1 + l, g.n3) + 3) + (i - 1), zc[l]);
  const T b0 = __ldg(c2 + 3 * (j - 1)), b1 = __ldg(c2 + 3 * (j - 1) + 1), b2 = __ldg(c2 + 3 * (j - 1) + 2);
  for (int k = k0; k <= k1; ++k) {
    const long long pz = g.nxy * (k + 3);
    const long long p = rowj + pz + (i - 1);
    T lm[W], rp[W], ym[W], yp[W], bv[W], r[W];
    vld(rel + rowj + pz + um, lm);
    vld(rel + rowj + pz + up, rp);
    vld(rel + rowm + pz + (i - 1), ym);
    vld(rel + rowp + pz + (i - 1), yp);
    vld(bb + p, bv);
    const T e0 = __ldg(c3 + 3 * (k - 1)), e1 = __ldg(c3 + 3 * (k - 1) + 1), e2 = __ldg(c3 + 3 * (k - 1) + 2);
#pragma unroll
    for (int v = 0; v < W; ++v) {
      const T* a = c1 + 3 * (i + v - 1);
      const T a0 = __ldg(a), a1 = __ldg(a + 1), a2 = __ldg(a + 2);
      const T xm = v == 0 ? lm[W - 1] : zc[1][v - 1];
      const T xp = v == W - 1 ? rp[0] : zc[1][v + 1];
      r[v] = omega * (bv[v] - a0 * xm - a2 * xp - b0 * ym[v] - b2 * yp[v] - e0 * zc[0][v] - e2 * zc[2][v]) /
                 (a1 + b1 + e1) +
             (T(1) - omega) * zc[1][v];
    }
    vst(out + p, r);
#pragma unroll
    for (int v = 0; v < W; ++v) {
      zc[0][v] = zc[1][v];
      zc[1][v] = zc[2][v];
    }
    if (k < k1) vld(rel + rowj + (long long)g.nxy * (wrapi(k + 2, g.n3) + 3) + (i - 1), zc[2]);
  }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// planes per marching thread: enough blocks for several waves, 16 .. 64 points per thread
inline int march_seg(long long blocks_xy, int na) {
  long long seg = blocks_xy * na / (148LL * 8);
  seg = seg < 16 ? 16 : (seg > 64 ? 64 : seg);
  return (int)std::min<long long>(seg, na);
}

}  // namespace

template <typename T, int LO, int CNT, int OP>
bool launch_march1(int a, const Geom& g, const T* cA, const T* cB, const T* f, const T* pp, T* out, int first,
                   cudaStream_t s) {
  constexpr int W = V16<T>::W;
  if (g.n1 % W != 0 || !aligned16(f) || !aligned16(out) || (OP == 2 && !aligned16(pp))) return false;
  const int nvx = g.n1 / W;
  if (a == 0) {
    const long long bx = (nvx + MBX - 1) / MBX, by = (g.n2 + MBY - 1) / MBY;
    const int seg = march_seg(bx * by, g.n3);
    const dim3 grid((unsigned)bx, (unsigned)by, (g.n3 + seg - 1) / seg);
    k_march_x<T, LO, CNT, OP><<<grid, dim3(MBX, MBY), 0, s>>>(g, cA, cB, f, pp, out, first, seg);
  } else {
    const int na = a == 2 ? g.n3 : g.n2, no = a == 2 ? g.n2 : g.n3;
    const long long bx = (nvx + MBX - 1) / MBX, by = (no + MBY - 1) / MBY;
    const int seg = march_seg(bx * by, na);
    const dim3 grid((unsigned)bx, (unsigned)by, (na + seg - 1) / seg);
    k_march_yz<T, LO, CNT, OP><<<grid, dim3(MBX, MBY), 0, s>>>(a, g, cA, cB, f, pp, out, first, seg);
  }
  return true;
}

template <typename T>
bool launch_helm_march(const Geom& g, const T* cx, const T* cy, const T* cz, T multL, const T* vel, T* nl,
                       cudaStream_t s) {
  constexpr int W = V16<T>::W;
  if (g.n1 % W != 0 || !aligned16(vel) || !aligned16(nl)) return false;
  const long long bx = (g.n1 / W + MBX - 1) / MBX, by = (g.n2 + MBY - 1) / MBY;
  const int seg = march_seg(bx * by, g.n3);
  k_helm_march<T><<<dim3((unsigned)bx, (unsigned)by, (g.n3 + seg - 1) / seg), dim3(MBX, MBY), 0, s>>>(g, cx, cy, cz, multL,
                                                                                                    vel, nl, seg);
  return true;
}

template <typename T>
bool launch_jacobi_march(const Geom& g, const T* c1, const T* c2, const T* c3, T omega, const T* bb, const T* rel,
                         T* out, cudaStream_t s) {
  constexpr int W = V16<T>::W;
  if (g.n1 % W != 0 || !aligned16(bb) || !aligned16(rel) || !aligned16(out)) return false;
  const long long bx = (g.n1 / W + MBX - 1) / MBX, by = (g.n2 + MBY - 1) / MBY;
  const int seg = march_seg(bx * by, g.n3);
  k_jacobi_march<T><<<dim3((unsigned)bx, (unsigned)by, (g.n3 + seg - 1) / seg), dim3(MBX, MBY), 0, s>>>(
      g, c1, c2, c3, omega, bb, rel, out, seg);
  return true;
}
template bool launch_helm_march<double>(const Geom&, const double*, const double*, const double*, double,
                                        const double*, double*, cudaStream_t);
template bool launch_helm_march<float>(const Geom&, const float*, const float*, const float*, float, const float*,
                                       float*, cudaStream_t);
template bool launch_jacobi_march<double>(const Geom&, const double*, const double*, const double*, double,
                                          const double*, const double*, double*, cudaStream_t);
template bool launch_jacobi_march<float>(const Geom&, const float*, const float*, const float*, float, const float*,
                                         const float*, float*, cudaStream_t);

#define MARCH_INST(T)                                                                                             \
  template bool launch_march1<T, G_LO, NG, 0>(int, const Geom&, const T*, const T*, const T*, const T*, T*, int,  \
                                              cudaStream_t);                                                      \
  template bool launch_march1<T, D_LO, ND, 0>(int, const Geom&, const T*, const T*, const T*, const T*, T*, int,  \
                                              cudaStream_t);                                                      \
  template bool launch_march1<T, D_LO, ND, 1>(int, const Geom&, const T*, const T*, const T*, const T*, T*, int,  \
                                              cudaStream_t);                                                      \
  template bool launch_march1<T, B_LO, NB, 2>(int, const Geom&, const T*, const T*, const T*, const T*, T*, int,  \
                                              cudaStream_t);
MARCH_INST(double)
MARCH_INST(float)
#undef MARCH_INST

}  // namespace impact
