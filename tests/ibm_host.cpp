// Test harness: the immersed-boundary arithmetic of gpu-impact-ct_b200/csrc/ibm.cuh compiled for
// the host (g++ -ffp-contract=off), so that the CPU tests check the very functions the device
// kernels call -- vicinity search, delta kernels, marker velocity, spreading terms -- against the
// oracle's literal restatement of mod_ibm.f90.  Built by tests/test_ibm.py into a temporary
// directory; nothing in the product loads it.
#include <cstdint>
#include <vector>

#include "ibm.cuh"

using namespace impact::ibm;

namespace {

struct Grid {
  std::vector<double> tables;
  Axis ax[3];
};

void make_grid(const int* N, const double* const* xp, const double* const* xu, Grid& g) {
  for (int a = 0; a < 3; ++a) axis_tables(xp[a], xu[a], N[a], g.tables);
  const double* p = g.tables.data();
  for (int a = 0; a < 3; ++a) {
    g.ax[a] = Axis{N[a] - 1, p, p + N[a], p + 2 * N[a], p + 3 * N[a]};
    p += 4 * N[a];
  }
}

}  // namespace

extern "C" double host_ibm_delta(int type, double reach, double d) { return delta(type, reach, d); }

extern "C" void host_ibm_vicinity(const double* x, int n, double y, double reach, int* lo, int* hi) {
  vicinity(x, n, y, reach, *lo, *hi);
}

extern "C" int host_ibm_widest(int N, const double* xp, const double* xu, double reach) {
  std::vector<double> t;
  axis_tables(xp, xu, N, t);
  return widest_support(t.data(), N, reach);
}

// Velocity at every marker, column-major (n, 3); vel is three padded fields.
extern "C" int host_ibm_interpolate(int N1, int N2, int N3, const double* const* xp, const double* const* xu,
                                    int type, double reach, int n, const double* yb, const uint8_t* skip,
                                    const double* vel, double* ub) {
  const int N[3] = {N1, N2, N3};
  Grid g;
  make_grid(N, xp, xu, g);
  const long long sx = N1 + 7, sy = sx * (N2 + 7), fs = sy * (N3 + 7);
  const long long origin = 3 + 3 * sx + 3 * sy;
  int wide = 0;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < n; ++m) {
      double r = 0.0;
      if (!(skip && skip[m])) {
        const double y[3] = {yb[m], yb[n + m], yb[2 * n + m]};
        r = gather(g.ax, y, type, reach, c, vel + c * fs + origin, sx, sy, &wide);
      }
      ub[(long long)c * n + m] = r;
    }
  return wide;
}

// Force density of the marker forces, markers in order (the sequential sum of the reference).
extern "C" int host_ibm_spread(int N1, int N2, int N3, const double* const* xp, const double* const* xu, int type,
                               double reach, int n, const double* yb, const uint8_t* skip, const double* fb,
                               const double* vol, double* fd) {
  const int N[3] = {N1, N2, N3};
  Grid g;
  make_grid(N, xp, xu, g);
  const long long sx = N1 + 7, sy = sx * (N2 + 7), fs = sy * (N3 + 7);
  const long long origin = 3 + 3 * sx + 3 * sy;
  for (long long q = 0; q < 3 * fs; ++q) fd[q] = 0.0;
  int wide = 0;
  for (int m = 0; m < n; ++m) {
    if (skip && skip[m]) continue;
    const double y[3] = {yb[m], yb[n + m], yb[2 * n + m]};
    for (int c = 0; c < 3; ++c) {
      Support s;
      const int ok = support(g.ax, y, reach, c, s);
      if (ok < 0) wide = 1;
      if (ok <= 0) continue;
      double* f = fd + c * fs + origin;
      for (int l = s.lo[2]; l <= s.hi[2]; ++l)
        for (int k = s.lo[1]; k <= s.hi[1]; ++k)
          for (int j = s.lo[0]; j <= s.hi[0]; ++j) {
            double* p = f + j + sx * k + sy * l;
            *p = *p + spread_term(s, y, type, reach, fb[(long long)c * n + m], vol[m], j, k, l);
          }
    }
  }
  return wide;
}
