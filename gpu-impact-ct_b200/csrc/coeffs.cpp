// coeffs.cpp -- host-side grid and finite-difference coefficient generation (set-up time).
//
// Restates, for periodic boundaries and mapping_yes = T (prog/config.txt), the parts of
// IMPACT's set-up that produce the hot path's inputs:
//   coordinates          mod_geometry.f90:37-120, usr_geometry.f90:93-156, coord_tanh usr_func.f90:1964
//   FD_coeffs            mod_coeffs.f90:37-112 (interior stencil widths ncb*(4), mod_dims.f90)
//   diff_coeffs          mod_coeffs.f90:200-597 (stencil placement, xi-mapping of derivatives)
//   diff_coeffs_exact    mod_coeffs.f90:598-751 (equidistant weights; here formed exactly)
//   get_stencil          mod_coeffs.f90:1048-1259 (compact Laplacian cdg, level 1)
// The equidistant weights are the Lagrange-polynomial derivatives, evaluated in exact integer
// arithmetic and rounded once, which reproduces the reference's rational table bit for bit.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/impact_b200.h"

int impact_set_error_msg(int code, const char* msg);

namespace {

int64_t gcd_ll(int64_t a, int64_t b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b != 0) {
    const int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// derivative order `abl` at 0 of the Lagrange basis through x_j = x0 + j, j < n
int exact_weights(int abl, int n, double x0, double* w) {
  if (n < 1 || n > 12 || abl < 0 || abl >= n) return -1;
  int64_t s2[12];  // doubled abscissae (integers for integer or half-integer x0)
  for (int j = 0; j < n; ++j) s2[j] = static_cast<int64_t>(std::llround(2.0 * (x0 + j)));
  int64_t scale = 1;  // abl! * 2^abl
  for (int q = 1; q <= abl; ++q) scale *= 2 * q;
  for (int j = 0; j < n; ++j) {
    std::vector<int64_t> poly(n + 1, 0);
    poly[0] = 1;
    int deg = 0;
    int64_t den = 1;
    for (int m = 0; m < n; ++m) {
      if (m == j) continue;
      for (int q = deg + 1; q >= 1; --q) poly[q] = poly[q - 1] - s2[m] * poly[q];
      poly[0] = -s2[m] * poly[0];
      ++deg;
      den *= (s2[j] - s2[m]);
    }
    int64_t num = poly[abl] * scale;
    int64_t g = gcd_ll(num, den);
    if (g == 0) g = 1;
    num /= g;
    den /= g;
    if (den < 0) {
      den = -den;
      num = -num;
    }
    w[j] = static_cast<double>(num) / static_cast<double>(den);
  }
  return 0;
}

double coord(int kind, int M, double L, double s) {
  if (kind == 0) return (s - 1.0) * L / (static_cast<double>(M) - 1.0);
  const double t = (s - 1.0) / (static_cast<double>(M) - 1.0);
  return 0.5 * L * (1.0 + std::sinh(2.0 * (t - 0.5)) / std::sinh(1.0));
}

// grid types of diff_coeffs: 0 p->p, 1 u->u, 2 p->u, 3 u->p
int diff_coeffs(int abl, int upwind, int grid_type, int N, int bL, int bU, int n_int, const double* xC,
                double* cc) {
  const int nrow = bU - bL + 1;
  const int i0 = (grid_type == 0 || grid_type == 3) ? 1 : 0;
  std::memset(cc, 0, sizeof(double) * static_cast<size_t>(nrow) * (N + 1));
  for (int i = i0; i <= N; ++i) {
    int n = n_int;
    int right = (grid_type <= 1) ? (n - 1) / 2 : (grid_type == 2 ? n / 2 : n / 2 - 1);
    int left = right - n + 1;
    if (upwind == -1) {
      --n;
      ++left;
    } else if (upwind == 1) {
      --n;
      --right;
    }
    if (left < bL || right > bU) return -3;
    const double x0 = grid_type == 2 ? left - 0.5 : (grid_type == 3 ? left + 0.5 : static_cast<double>(left));
    double w[12];
    if (abl == 0) {
      exact_weights(0, n, x0, w);
    } else {
      double c1[12], c2[12];
      exact_weights(1, n, x0, c1);
      double d1 = 0.0, d2 = 0.0;  // x'(xi), x''(xi) from the same stencils
      for (int l = left; l <= right; ++l) d1 = d1 + c1[l - left] * xC[i + l + 3];
      if (abl == 2) {
        exact_weights(2, n, x0, c2);
        for (int l = left; l <= right; ++l) d2 = d2 + c2[l - left] * xC[i + l + 3];
      }
      for (int l = left; l <= right; ++l) {
        if (abl == 1)
          w[l - left] = c1[l - left] / d1;
        else
          w[l - left] = c2[l - left] / (d1 * d1) - c1[l - left] * d2 / (d1 * d1 * d1);
      }
    }
    for (int l = left; l <= right; ++l) cc[static_cast<size_t>(i) * nrow + (l - bL)] = w[l - left];
  }
  return 0;
}

}  // namespace

extern "C" int impact_b200_fd_exact(int abl, int n, double deltaX0, double* cc) {
  if (!cc) return impact_set_error_msg(-1, "impact_b200_fd_exact: null output");
  if (exact_weights(abl, n, deltaX0, cc) != 0) return impact_set_error_msg(-1, "impact_b200_fd_exact: bad stencil");
  return 0;
}

extern "C" int impact_b200_axis_coords(int M, double L, int kind, double* xp, double* xu) {
  if (M < 9 || !xp || !xu || (kind != 0 && kind != 1) || !(L > 0.0))
    return impact_set_error_msg(-1, "impact_b200_axis_coords: bad arguments (need M >= 9, L > 0, kind 0/1)");
  for (int i = 0; i < M + 7; ++i) xp[i] = xu[i] = 0.0;
  for (int i = 1; i <= M; ++i) xp[i + 3] = coord(kind, M, L, i);
  for (int i = 0; i <= M; ++i) xu[i + 3] = coord(kind, M, L, i + 0.5);
  // periodic continuation, mod_geometry.f90:95-103
  for (int i = -3; i <= 0; ++i) {
    xp[i + 3] = xp[M - 1 + i + 3] - L;
    xu[i + 3] = xu[M - 1 + i + 3] - L;
  }
  for (int i = M; i <= M + 3; ++i) {
    xp[i + 3] = xp[i - M + 1 + 3] + L;
    xu[i + 3] = xu[i - M + 1 + 3] + L;
  }
  return 0;
}

extern "C" int impact_b200_axis_coeffs(int M, const double* xp, const double* xu, impact_b200_axis_tables* t) {
  if (M < 9 || !xp || !xu || !t) return impact_set_error_msg(-1, "impact_b200_axis_coeffs: bad arguments");
  double* need[] = {t->cG, t->cD, t->cIpu, t->cIup, t->cNpU, t->cNpD, t->cNuU, t->cNuD, t->cp1, t->cpp, t->cuu, t->cdg};
  for (double* p : need)
    if (!p) return impact_set_error_msg(-1, "impact_b200_axis_coeffs: null table pointer");
  // interior widths: ncb*c(4) = 7 central (6 upwind), ncb*g(4) = 6, ncb*d(4) = 6 (mod_dims.f90)
  int rc = 0;
  rc |= diff_coeffs(1, -1, 0, M, -3, 3, 7, xp, t->cNpD);
  rc |= diff_coeffs(1, 1, 0, M, -3, 3, 7, xp, t->cNpU);
  rc |= diff_coeffs(1, -1, 1, M, -3, 3, 7, xu, t->cNuD);
  rc |= diff_coeffs(1, 1, 1, M, -3, 3, 7, xu, t->cNuU);
  rc |= diff_coeffs(1, 0, 0, M, -3, 3, 7, xp, t->cp1);
  rc |= diff_coeffs(2, 0, 0, M, -3, 3, 7, xp, t->cpp);
  rc |= diff_coeffs(2, 0, 1, M, -3, 3, 7, xu, t->cuu);
  rc |= diff_coeffs(1, 0, 2, M, -2, 3, 6, xp, t->cG);
  rc |= diff_coeffs(1, 0, 3, M, -3, 2, 6, xu, t->cD);
  rc |= diff_coeffs(0, 0, 2, M, -2, 3, 6, xp, t->cIpu);
  rc |= diff_coeffs(0, 0, 3, M, -3, 2, 6, xu, t->cIup);
  if (rc) return impact_set_error_msg(-1, "impact_b200_axis_coeffs: stencil does not fit");
  // compact Laplacian (get_stencil, periodic branch)
  std::vector<double> dm(M + 1), dp(M + 1), gm(M + 1), gp(M + 1);
  for (int i = 1; i <= M; ++i) {
    dm[i] = -1.0 / (xu[i + 3] - xu[i - 1 + 3]);
    dp[i] = 1.0 / (xu[i + 3] - xu[i - 1 + 3]);
  }
  for (int i = 0; i <= M; ++i) {
    gm[i] = -1.0 / (xp[i + 1 + 3] - xp[i + 3]);
    gp[i] = 1.0 / (xp[i + 1 + 3] - xp[i + 3]);
  }
  for (int i = 1; i <= M; ++i) {
    t->cdg[3 * (i - 1) + 0] = dm[i] * gm[i - 1];
    t->cdg[3 * (i - 1) + 1] = dm[i] * gp[i - 1] + dp[i] * gm[i];
    t->cdg[3 * (i - 1) + 2] = dp[i] * gp[i];
  }
  return 0;
}

// ---------------------------------------------------------------------------------------
// multigrid hierarchy (periodic)
// ---------------------------------------------------------------------------------------
#include "mg_host.h"

namespace impact {

static void compact_laplacian(int M, const double* xp, const double* xu, double* cdg) {
  std::vector<double> dm(M + 1), dp(M + 1), gm(M + 1), gp(M + 1);
  for (int i = 1; i <= M; ++i) {
    dm[i] = -1.0 / (xu[i + 3] - xu[i - 1 + 3]);
    dp[i] = 1.0 / (xu[i + 3] - xu[i - 1 + 3]);
  }
  for (int i = 0; i <= M; ++i) {
    gm[i] = -1.0 / (xp[i + 1 + 3] - xp[i + 3]);
    gp[i] = 1.0 / (xp[i + 1 + 3] - xp[i + 3]);
  }
  for (int i = 1; i <= M; ++i) {
    cdg[3 * (i - 1) + 0] = dm[i] * gm[i - 1];
    cdg[3 * (i - 1) + 1] = dm[i] * gp[i - 1] + dp[i] * gm[i];
    cdg[3 * (i - 1) + 2] = dp[i] * gp[i];
  }
}

std::vector<MGHostLevel> build_mg_hierarchy(const int N[3], const double* const xp[3], const double* const xu[3],
                                            const double L[3], int n_grids_limit) {
  constexpr int GMAX = 15;
  int MM[GMAX][3];
  for (int m = 0; m < 3; ++m) MM[0][m] = N[m];
  int ng = 1;
  for (int g = 1; g < GMAX; ++g)
    for (int m = 0; m < 3; ++m) {
      if ((MM[g - 1][m] - 1) % 2 == 0 && MM[g - 1][m] >= 5) {  // 5 = 2 (Nmin - 1) + 1
        MM[g][m] = (MM[g - 1][m] - 1) / 2 + 1;
        ng = g + 1;
      } else {
        MM[g][m] = MM[g - 1][m];
      }
    }
  if (n_grids_limit < 1) n_grids_limit = 1;
  if (ng > n_grids_limit) ng = n_grids_limit;
  std::vector<MGHostLevel> lv(ng);
  for (int g = 0; g < ng; ++g)
    for (int m = 0; m < 3; ++m) {
      const int M = MM[g][m];
      MGHostLevel& L_ = lv[g];
      L_.M[m] = M;
      L_.ratio[m] = (g + 1 < ng) ? (MM[g][m] - 1) / (MM[g + 1][m] - 1) : 1;
      const double* y1p = xp[m];
      std::vector<double> p(M + 7, 0.0), u(M + 7, 0.0);
      const int di = (MM[0][m] - 1) / (M - 1);  // level spacing in finest-grid points
      if (g == 0) {
        p.assign(xp[m], xp[m] + M + 7);
        u.assign(xu[m], xu[m] + M + 7);
      } else {
        for (int i = 1; i <= M; ++i) p[i + 3] = y1p[1 + di * i - di + 3];
        for (int i = 1; i <= M - 1; ++i) u[i + 3] = y1p[1 + di * i - di / 2 + 3];
        for (int i = -3; i <= 0; ++i) {
          p[i + 3] = p[M - 1 + i + 3] - L[m];
          u[i + 3] = u[M - 1 + i + 3] - L[m];
        }
        for (int i = M; i <= M + 3; ++i) {
          p[i + 3] = p[i - M + 1 + 3] + L[m];
          u[i + 3] = u[i - M + 1 + 3] + L[m];
        }
      }
      L_.cdg[m].assign(3 * M, 0.0);
      compact_laplacian(M, p.data(), u.data(), L_.cdg[m].data());
      L_.cI[m].assign(2 * (M + 1), 0.0);
      if (g + 1 < ng) {
        for (int i = 2; i <= M - 1; i += 2) {
          const int i0 = 1 + (i - 1) * di;
          const double Dx10 = y1p[i0 + 3] - y1p[i0 - di + 3];
          const double Dx12 = y1p[i0 + di + 3] - y1p[i0 - di + 3];
          L_.cI[m][2 * i + 0] = 1. - Dx10 / Dx12;
          L_.cI[m][2 * i + 1] = Dx10 / Dx12;
        }
      }
    }
  return lv;
}

}  // namespace impact
