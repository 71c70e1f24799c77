// ibm.cuh -- diffuse-interface immersed-boundary transfers between Lagrangian markers and the
// staggered velocity grids (mod_ibm.f90): the discrete delta kernels (discrete_delta,
// mod_ibm.f90:2021-2075), the vicinity of a marker along one axis (find_vicinity_coordinates,
// :743-876), the velocity at a marker (interpolate_vel_to_ib, :589-737) and the weight of a
// marker force at one grid point (spread_force_dens_to_vel_grid, :428-583).
//
// Everything here is plain arithmetic shared by the device kernels (ibm.cu) and by host code
// built from the same source: every product, sum and quotient is rounded on its own (no
// contraction into fused multiply-adds) and evaluated in the reference's order, so a marker's
// velocity is the same bit for bit wherever it is computed.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#if defined(__CUDACC__)
#define IBM_HD __host__ __device__
#else
#define IBM_HD
#endif

namespace impact {
namespace ibm {

// Grid points per axis a marker's support may span; set_markers rejects a reach that could
// exceed it on the case's grid.
constexpr int MAXW = 16;

IBM_HD inline double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
IBM_HD inline double add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
IBM_HD inline double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
IBM_HD inline double quo(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
IBM_HD inline double root(double a) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}

// Discrete delta of the given type at a signed distance (0 beyond the reach):
// 1 cosine, 2 linear hat, 3 and 4 the piecewise kernels of half-width reach / 2.
IBM_HD inline double delta(int type, double reach, double d) {
  const double ad = std::fabs(d);
  if (!(ad <= reach)) return 0.0;
  if (type == 1) {
    const double pi = 2.0 * 1.5707963267948966;  // 2 |acos(0)|
    return quo(add(1.0, std::cos(quo(mul(pi, ad), reach))), mul(2.0, reach));
  }
  if (type == 2) return quo(sub(reach, ad), mul(reach, reach));
  const double h = quo(reach, 2.0);
  if (type == 3) {
    const double q = quo(d, h);
    if (ad <= h) return quo(sub(1.0, mul(q, q)), h);
    return quo(add(sub(2.0, std::fabs(quo(mul(3.0, d), h))), mul(q, q)), h);
  }
  if (type == 4) {
    const double t = quo(ad, h);
    const double two = quo(mul(2.0, ad), h);
    const double tt = mul(4.0, mul(t, t));
    if (ad <= h)
      return quo(add(sub(3.0, two), root(sub(add(1.0, quo(mul(4.0, ad), h)), tt))), mul(4.0, reach));
    return quo(sub(sub(5.0, two), root(sub(add(-7.0, quo(mul(12.0, ad), h)), tt))), mul(4.0, reach));
  }
  return 0.0;
}

// Vicinity of y among the points 1..n of an increasing coordinate array (x[i] is point i):
// [lo, hi] = the first point with |y - x| <= reach up to the last point before the first one
// with x - y > reach; lo = hi = -1 when no point is within reach.  Two binary searches on the
// reference's own predicates (fl(y - x) decreases and fl(x - y) increases along the axis, and
// |fl(y - x)| <= reach holds exactly when both fl(y - x) <= reach and fl(x - y) <= reach), so
// the range is the one the reference's linear scan finds.
IBM_HD inline void vicinity(const double* x, int n, double y, double reach, int& lo, int& hi) {
  int a = 1, b = n + 1;  // first i with y - x[i] <= reach
  while (a < b) {
    const int c = (a + b) >> 1;
    if (sub(y, x[c]) <= reach) b = c; else a = c + 1;
  }
  const int i0 = a;
  a = 1;
  b = n + 1;  // first i with x[i] - y > reach
  while (a < b) {
    const int c = (a + b) >> 1;
    if (sub(x[c], y) > reach) b = c; else a = c + 1;
  }
  const int i1 = a;
  if (i0 <= n && i0 < i1) {
    lo = i0;
    hi = i1 - 1;
  } else {
    lo = hi = -1;
  }
}

// One axis of the case's grid as the transfers see it: the coordinates and cell widths of the
// pressure points (x_p, dx_p) and of the velocity points of this axis (x_u, dx_u), each an
// array over the points 1..n (index 0 unused).
struct Axis {
  int n;  // unique periodic points N - 1
  const double* xp;
  const double* xu;
  const double* dxp;
  const double* dxu;
};

// The support of marker y for velocity component c: per axis the vicinity on the velocity
// grid along axis c and on the pressure grid along the others.  Returns 1, or 0 when an axis
// has no point within reach (every weight of the marker is then zero; the reference adds zero
// terms there), or -1 when the support is wider than MAXW points (a reach that set_markers
// rejects beforehand; the caller reports it).
struct Support {
  int lo[3], hi[3];
  const double* x[3];
  const double* dx[3];
};

IBM_HD inline int support(const Axis* ax, const double y[3], double reach, int c, Support& s) {
  int ok = 1;
  for (int a = 0; a < 3; ++a) {
    s.x[a] = a == c ? ax[a].xu : ax[a].xp;
    s.dx[a] = a == c ? ax[a].dxu : ax[a].dxp;
    vicinity(s.x[a], ax[a].n, y[a], reach, s.lo[a], s.hi[a]);
    if (s.lo[a] < 0) return 0;
    if (s.hi[a] - s.lo[a] + 1 > MAXW) ok = -1;
  }
  return ok;
}

// Velocity component c at marker y: the sum over l, k, j (j fastest) of
// delta_x * delta_y * delta_z * u(j, k, l) * dx(j) * dy(k) * dz(l), each product rounded in that
// order and added to a sum that starts at 0.  u(j, k, l) = f[j + sx * k + sy * l] with f based
// at point (0, 0, 0) of the padded field.  *wide is set when the support is too wide (the
// velocity is then 0).
IBM_HD inline double gather(const Axis* ax, const double y[3], int type, double reach, int c, const double* f,
                            long long sx, long long sy, int* wide) {
  Support s;
  const int ok = support(ax, y, reach, c, s);
  if (ok < 0) *wide = 1;
  if (ok <= 0) return 0.0;
  double w0[MAXW], w1[MAXW], w2[MAXW];
  for (int j = s.lo[0]; j <= s.hi[0]; ++j) w0[j - s.lo[0]] = delta(type, reach, sub(y[0], s.x[0][j]));
  for (int k = s.lo[1]; k <= s.hi[1]; ++k) w1[k - s.lo[1]] = delta(type, reach, sub(y[1], s.x[1][k]));
  for (int l = s.lo[2]; l <= s.hi[2]; ++l) w2[l - s.lo[2]] = delta(type, reach, sub(y[2], s.x[2][l]));
  double u = 0.0;
  for (int l = s.lo[2]; l <= s.hi[2]; ++l)
    for (int k = s.lo[1]; k <= s.hi[1]; ++k)
      for (int j = s.lo[0]; j <= s.hi[0]; ++j) {
        double t = mul(mul(w0[j - s.lo[0]], w1[k - s.lo[1]]), w2[l - s.lo[2]]);
        t = mul(mul(mul(mul(t, f[j + sx * k + sy * l]), s.dx[0][j]), s.dx[1][k]), s.dx[2][l]);
        u = add(u, t);
      }
  return u;
}

// The amount marker force fc (component c) with node volume vol adds at point (j, k, l) of the
// support: fc * delta_x * delta_y * delta_z * vol, rounded in that order.
IBM_HD inline double spread_term(const Support& s, const double y[3], int type, double reach, double fc,
                                 double vol, int j, int k, int l) {
  double t = mul(fc, delta(type, reach, sub(y[0], s.x[0][j])));
  t = mul(t, delta(type, reach, sub(y[1], s.x[1][k])));
  t = mul(t, delta(type, reach, sub(y[2], s.x[2][l])));
  return mul(t, vol);
}

// Host: appends the four arrays of one axis -- xp, xu, dxp, dxu over the points 0..N-1, entry 0
// unused -- built from the global coordinates over -3..N+3 (offset 3).  The cell widths follow
// mod_geometry.f90:193-204 on a periodic axis: dxp(i) = xu(i) - xu(i-1), dxu(i) = xp(i+1) - xp(i).
inline void axis_tables(const double* xp, const double* xu, int N, std::vector<double>& out) {
  const size_t b = out.size();
  out.resize(b + 4 * (size_t)N, 0.0);
  double* p = out.data() + b;
  for (int i = 1; i <= N - 1; ++i) {
    p[i] = xp[i + 3];
    p[N + i] = xu[i + 3];
    p[2 * N + i] = xu[i + 3] - xu[i + 2];
    p[3 * N + i] = xp[i + 4] - xp[i + 3];
  }
}

// Host: the most points of either grid of an axis (the four arrays of axis_tables) that a
// window of width 2 reach (widened by a relative 1e-9 for rounding) can hold -- a bound on the
// width of any vicinity along the axis.
inline int widest_support(const double* tables, int N, double reach) {
  const double width = 2.0 * reach * (1.0 + 1e-9);
  int best = 0;
  for (int g = 0; g < 2; ++g) {
    const double* x = tables + (size_t)g * N;
    for (int i = 1, j = 1; i <= N - 1; ++i) {
      if (j < i) j = i;
      while (j + 1 <= N - 1 && x[j + 1] - x[i] <= width) ++j;
      best = std::max(best, j - i + 1);
    }
  }
  return best;
}

}  // namespace ibm
}  // namespace impact
