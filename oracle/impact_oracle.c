/*
 * impact_oracle.c -- CPU FP64 oracle for the IMPACT fractional-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see impact_oracle.h).  Each routine names the reference
 * routine it restates.  Loop order, summation order and the stencil index ranges follow
 * the reference so that FP64 results agree to rounding; the only structural additions
 * are OpenMP over the slowest axis and per-plane partial sums for the reductions (a
 * deterministic, thread-count independent order).
 */
#include "impact_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846

/* RK3 coefficients (mod_vars.f90:774-775). */
static const double aRK[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double bRK[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

/* ------------------------------------------------------------------------------------ */
/* layout helpers                                                                       */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  int N1, N2, N3;
  size_t sx, sy; /* strides of j and k */
} dims_t;

static inline dims_t mkdims(int N1, int N2, int N3) {
  dims_t d;
  d.N1 = N1;
  d.N2 = N2;
  d.N3 = N3;
  d.sx = (size_t)(N1 + 7);
  d.sy = d.sx * (size_t)(N2 + 7);
  return d;
}
static inline size_t IX(const dims_t* d, int i, int j, int k) {
  return (size_t)(i + 3) + d->sx * (size_t)(j + 3) + d->sy * (size_t)(k + 3);
}
static inline size_t field_size(const dims_t* d) { return d->sy * (size_t)(d->N3 + 7); }
/* coefficient c(l, i) of a table with lower bound lo and n per row */
#define CF(tab, lo, n, l, i) ((tab)[(size_t)(i) * (n) + ((l) - (lo))])
#define CDG(tab, l, i) ((tab)[(size_t)((i)-1) * 3 + ((l) + 1)])

/* ------------------------------------------------------------------------------------ */
/* coordinates (mod_geometry.f90:37, usr_geometry.f90:93-156)                           */
/* ------------------------------------------------------------------------------------ */
static double coord_fn(int kind, int M, double L, double s) {
  /* s is the 1-based point index (half-integer for velocity points) */
  if (kind == 0) return (s - 1.0) * L / ((double)M - 1.0); /* coord_tanh, equidistant branch */
  double t = (s - 1.0) / ((double)M - 1.0);
  return 0.5 * L * (1.0 + sinh(2.0 * (t - 0.5)) / sinh(1.0));
}

void orc_coords(int M, double L, int kind, double* xp, double* xu) {
  /* arrays cover indices -3..M+3 (offset 3) */
  for (int i = -3; i <= M + 3; i++) {
    xp[i + 3] = 0.0;
    xu[i + 3] = 0.0;
  }
  for (int i = 1; i <= M; i++) xp[i + 3] = coord_fn(kind, M, L, (double)i);
  for (int i = 0; i <= M; i++) xu[i + 3] = coord_fn(kind, M, L, (double)i + 0.5);
  /* periodic continuation (mod_geometry.f90:95-103): lower ghosts from M-4..M-1, upper from 1..4 */
  for (int i = -3; i <= 0; i++) {
    xp[i + 3] = xp[(M - 1 + i) + 3] - L;
    xu[i + 3] = xu[(M - 1 + i) + 3] - L;
  }
  for (int i = M; i <= M + 3; i++) {
    xp[i + 3] = xp[(i - M + 1) + 3] + L;
    xu[i + 3] = xu[(i - M + 1) + 3] + L;
  }
}

/* ------------------------------------------------------------------------------------ */
/* exact equidistant FD weights (diff_coeffs_exact, mod_coeffs.f90:598-751)             */
/* ------------------------------------------------------------------------------------ */
static int64_t gcd64(int64_t a, int64_t b) {
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

int orc_fd_exact(int abl, int n, double deltaX0, double* cc) {
  /* Lagrange weights of derivative order abl at 0 for points x_j = deltaX0 + j, computed in
   * exact integer arithmetic on the doubled offsets s_j = 2 x_j, then rounded once. */
  if (n < 1 || n > 12 || abl < 0 || abl >= n) return -1;
  int64_t s[12];
  for (int j = 0; j < n; j++) s[j] = (int64_t)llround(2.0 * (deltaX0 + (double)j));
  int64_t fact = 1, pow2 = 1;
  for (int q = 1; q <= abl; q++) {
    fact *= q;
    pow2 *= 2;
  }
  for (int j = 0; j < n; j++) {
    /* poly(t) = prod_{m != j} (t - s_m), coefficients in increasing power */
    int64_t poly[13] = {0};
    poly[0] = 1;
    int deg = 0;
    int64_t den = 1;
    for (int m = 0; m < n; m++) {
      if (m == j) continue;
      for (int q = deg + 1; q >= 1; q--) poly[q] = poly[q - 1] - s[m] * poly[q];
      poly[0] = -s[m] * poly[0];
      deg++;
      den *= (s[j] - s[m]);
    }
    int64_t num = poly[abl] * fact * pow2;
    int64_t g = gcd64(num, den);
    if (g == 0) g = 1;
    num /= g;
    den /= g;
    if (den < 0) {
      den = -den;
      num = -num;
    }
    cc[j] = (double)num / (double)den;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* diff_coeffs (mod_coeffs.f90:200-597), periodic boundaries, mapping_yes = T           */
/* ------------------------------------------------------------------------------------ */
int orc_diff_coeffs(int abl, int upwind, int grid_type, int N, int bL, int bU, int n_coeff,
                    const double* xC, const double* xE, double* cc) {
  (void)xE;
  const int nrow = bU - bL + 1;
  const int iStart = (grid_type == 0 || grid_type == 3) ? 1 : 0;
  memset(cc, 0, sizeof(double) * (size_t)nrow * (size_t)(N + 1));
  for (int i = iStart; i <= N; i++) {
    int n = n_coeff;
    if (!(n > 0 && n > abl)) continue;
    int right;
    if (grid_type == 0 || grid_type == 1) {
      if (n % 2 == 0) return -2; /* central stencils need an odd count */
      right = (n - 1) / 2;
    } else if (grid_type == 2) {
      if (n % 2 != 0) return -2;
      right = n / 2;
    } else {
      if (n % 2 != 0) return -2;
      right = n / 2 - 1;
    }
    int left = right - n + 1;
    if (upwind == -1) {
      n -= 1;
      left += 1;
    }
    if (upwind == 1) {
      n -= 1;
      right -= 1;
    }
    if (right > bU || left < bL) return -3;
    double dx0;
    if (grid_type == 2)
      dx0 = (double)left - 0.5;
    else if (grid_type == 3)
      dx0 = (double)left + 0.5;
    else
      dx0 = (double)left;
    double w[12];
    if (abl == 1 || abl == 2) {
      double cxi[2][12];
      double dxi[2] = {0.0, 0.0};
      for (int k = 1; k <= abl; k++) {
        orc_fd_exact(k, n, dx0, cxi[k - 1]);
        for (int ii = left; ii <= right; ii++) dxi[k - 1] = dxi[k - 1] + cxi[k - 1][ii - left] * xC[i + ii + 3];
      }
      for (int ii = left; ii <= right; ii++) {
        if (abl == 1)
          w[ii - left] = cxi[0][ii - left] / dxi[0];
        else
          w[ii - left] = cxi[1][ii - left] / (dxi[0] * dxi[0]) -
                         cxi[0][ii - left] * dxi[1] / (dxi[0] * dxi[0] * dxi[0]);
      }
    } else if (abl == 0 && (grid_type == 2 || grid_type == 3)) {
      orc_fd_exact(0, n, dx0, w);
    } else {
      return -4; /* filters / integrators are not on the hot path */
    }
    for (int ii = left; ii <= right; ii++) cc[(size_t)i * nrow + (ii - bL)] = w[ii - left];
  }
  return 0;
}

/* get_stencil (mod_coeffs.f90:1048-1259), level 1, periodic branch */
void orc_get_stencil(int N, const double* xp, const double* xu, double* cdg) {
  double* cD = (double*)calloc((size_t)2 * (N + 1), sizeof(double)); /* cDu1R(-1:0, 0:N) */
  double* cG = (double*)calloc((size_t)2 * (N + 1), sizeof(double)); /* cGp1R(0:1, 0:N) */
  for (int i = 1; i <= N; i++) {
    cD[2 * i + 0] = -1.0 / (xu[i + 3] - xu[i - 1 + 3]);
    cD[2 * i + 1] = 1.0 / (xu[i + 3] - xu[i - 1 + 3]);
  }
  for (int i = 1; i <= N - 1; i++) {
    cG[2 * i + 0] = -1.0 / (xp[i + 1 + 3] - xp[i + 3]);
    cG[2 * i + 1] = 1.0 / (xp[i + 1 + 3] - xp[i + 3]);
  }
  cG[0] = -1.0 / (xp[1 + 3] - xp[0 + 3]);
  cG[1] = 1.0 / (xp[1 + 3] - xp[0 + 3]);
  cG[2 * N + 0] = -1.0 / (xp[N + 1 + 3] - xp[N + 3]);
  cG[2 * N + 1] = 1.0 / (xp[N + 1 + 3] - xp[N + 3]);
  for (int i = 1; i <= N; i++) {
    CDG(cdg, -1, i) = cD[2 * i + 0] * cG[2 * (i - 1) + 0];
    CDG(cdg, 0, i) = cD[2 * i + 0] * cG[2 * (i - 1) + 1] + cD[2 * i + 1] * cG[2 * i + 0];
    CDG(cdg, 1, i) = cD[2 * i + 1] * cG[2 * i + 1];
  }
  free(cD);
  free(cG);
}

/* RK3 stability limits along the rays z = r (-sin t + i cos t), t = n pi/80, n = 0..40:
 * the first r where |1 + z + z^2/2 + z^3/6| = 1 (the quantity tabulated at mod_vars.f90:785). */
static double amp2(double r, double t) {
  double zr = -r * sin(t), zi = r * cos(t);
  double z2r = zr * zr - zi * zi, z2i = 2.0 * zr * zi;
  double z3r = z2r * zr - z2i * zi, z3i = z2r * zi + z2i * zr;
  double re = 1.0 + zr + 0.5 * z2r + z3r / 6.0;
  double im = zi + 0.5 * z2i + z3i / 6.0;
  return re * re + im * im - 1.0;
}
void orc_stability_limits(double* lim41) {
  for (int n = 0; n <= 40; n++) {
    double t = (double)n * PI_D / 80.0;
    double lo = 1e-3, hi = lo;
    while (amp2(hi, t) < 0.0 && hi < 10.0) {
      lo = hi;
      hi += 1e-3;
    }
    for (int it = 0; it < 200; it++) {
      double mid = 0.5 * (lo + hi);
      if (amp2(mid, t) < 0.0)
        lo = mid;
      else
        hi = mid;
    }
    lim41[n] = 0.5 * (lo + hi);
  }
}

/* ------------------------------------------------------------------------------------ */
/* ghost fill (mod_exchange.f90:133-140), periodic branch                               */
/* ------------------------------------------------------------------------------------ */
void orc_exchange(int dir, int N1, int N2, int N3, double* phi) {
  dims_t d = mkdims(N1, N2, N3);
  if (dir == 1) {
    for (int k = 1; k <= N3; k++)
      for (int j = 1; j <= N2; j++) {
        for (int i = -3; i <= -1; i++) phi[IX(&d, 1 + i, j, k)] = phi[IX(&d, N1 + i, j, k)];
        for (int i = 1; i <= 3; i++) phi[IX(&d, N1 - 1 + i, j, k)] = phi[IX(&d, i, j, k)];
      }
  } else if (dir == 2) {
    for (int k = 1; k <= N3; k++)
      for (int i = 1; i <= N1; i++) {
        for (int j = -3; j <= -1; j++) phi[IX(&d, i, 1 + j, k)] = phi[IX(&d, i, N2 + j, k)];
        for (int j = 1; j <= 3; j++) phi[IX(&d, i, N2 - 1 + j, k)] = phi[IX(&d, i, j, k)];
      }
  } else {
    for (int j = 1; j <= N2; j++)
      for (int i = 1; i <= N1; i++) {
        for (int k = -3; k <= -1; k++) phi[IX(&d, i, j, 1 + k)] = phi[IX(&d, i, j, N3 + k)];
        for (int k = 1; k <= 3; k++) phi[IX(&d, i, j, N3 - 1 + k)] = phi[IX(&d, i, j, k)];
      }
  }
}
static void exchange_all(int N1, int N2, int N3, double* phi) {
  orc_exchange(1, N1, N2, N3, phi);
  orc_exchange(2, N1, N2, N3, phi);
  orc_exchange(3, N1, N2, N3, phi);
}

/* ------------------------------------------------------------------------------------ */
/* 1-D stencil helper: out = sum_l c(l, row) * phi(point + l*stride)                    */
/* ------------------------------------------------------------------------------------ */
static inline double stencil1(const double* tab, int lo, int hi, int row, const double* phi,
                              size_t p, ptrdiff_t stride) {
  const int n = hi - lo + 1;
  double s = CF(tab, lo, n, lo, row) * phi[(ptrdiff_t)p + (ptrdiff_t)lo * stride];
  for (int l = lo + 1; l <= hi; l++) s = s + CF(tab, lo, n, l, row) * phi[(ptrdiff_t)p + (ptrdiff_t)l * stride];
  return s;
}
static inline ptrdiff_t axis_stride(const dims_t* d, int a) {
  return a == 1 ? (ptrdiff_t)1 : (a == 2 ? (ptrdiff_t)d->sx : (ptrdiff_t)d->sy);
}
static inline int axis_row(int a, int i, int j, int k) { return a == 1 ? i : (a == 2 ? j : k); }

/* ------------------------------------------------------------------------------------ */
/* operators (mod_diff.f90)                                                             */
/* ------------------------------------------------------------------------------------ */
/* gradient (mod_diff.f90:309-414) */
void orc_gradient(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* grad) {
  dims_t d = mkdims(N1, N2, N3);
  orc_exchange(m, N1, N2, N3, phi);
  const double* tab = c->cG[m - 1];
  const ptrdiff_t st = axis_stride(&d, m);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        grad[p] = stencil1(tab, ORC_G_LO, ORC_G_HI, axis_row(m, i, j, k), phi, p, st);
      }
}

/* divergence (mod_diff.f90:52-118): m = 1 overwrites, m = 2, 3 accumulate */
void orc_divergence(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* div) {
  dims_t d = mkdims(N1, N2, N3);
  orc_exchange(m, N1, N2, N3, phi);
  const double* tab = c->cD[m - 1];
  const ptrdiff_t st = axis_stride(&d, m);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        int row = axis_row(m, i, j, k);
        if (m == 1) {
          div[p] = stencil1(tab, ORC_D_LO, ORC_D_HI, row, phi, p, st);
        } else {
          double s = div[p];
          for (int l = ORC_D_LO; l <= ORC_D_HI; l++)
            s = s + CF(tab, ORC_D_LO, ORC_ND, l, row) * phi[(ptrdiff_t)p + (ptrdiff_t)l * st];
          div[p] = s;
        }
      }
}

/* divergence2 (mod_diff.f90:130-215) */
void orc_divergence2(int N1, int N2, int N3, const orc_coeffs* c, double* u, double* v, double* w,
                     double* div) {
  dims_t d = mkdims(N1, N2, N3);
  orc_exchange(1, N1, N2, N3, u);
  orc_exchange(2, N1, N2, N3, v);
  orc_exchange(3, N1, N2, N3, w);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        double s = stencil1(c->cD[0], ORC_D_LO, ORC_D_HI, i, u, p, 1);
        for (int l = ORC_D_LO; l <= ORC_D_HI; l++)
          s = s + CF(c->cD[1], ORC_D_LO, ORC_ND, l, j) * v[(ptrdiff_t)p + (ptrdiff_t)l * (ptrdiff_t)d.sx];
        for (int l = ORC_D_LO; l <= ORC_D_HI; l++)
          s = s + CF(c->cD[2], ORC_D_LO, ORC_ND, l, k) * w[(ptrdiff_t)p + (ptrdiff_t)l * (ptrdiff_t)d.sy];
        div[p] = s;
      }
}

/* Helmholtz_explicit (mod_diff.f90:549-762): nl_m -= multL * (d2/dx2 + d2/dy2 + d2/dz2) u_m */
void orc_helmholtz(int m, int N1, int N2, int N3, const orc_coeffs* c, double multL, double* vel,
                   double* nl) {
  dims_t d = mkdims(N1, N2, N3);
  exchange_all(N1, N2, N3, vel);
  const double* cx = (m == 1) ? c->cuu[0] : c->cpp[0];
  const double* cy = (m == 2) ? c->cuu[1] : c->cpp[1];
  const double* cz = (m == 3) ? c->cuu[2] : c->cpp[2];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        double dd1 = stencil1(cx, ORC_B_LO, ORC_B_HI, i, vel, p, 1);
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++)
          dd1 = dd1 + CF(cy, ORC_B_LO, ORC_NB, l, j) * vel[(ptrdiff_t)p + (ptrdiff_t)l * (ptrdiff_t)d.sx];
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++)
          dd1 = dd1 + CF(cz, ORC_B_LO, ORC_NB, l, k) * vel[(ptrdiff_t)p + (ptrdiff_t)l * (ptrdiff_t)d.sy];
        nl[p] = nl[p] - multL * dd1;
      }
}

/* interpolate2_pre_vel (mod_diff.f90:1567-1648): pressure points -> u_m points */
void orc_interpolate_pre_vel(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi,
                             double* inter) {
  dims_t d = mkdims(N1, N2, N3);
  orc_exchange(m, N1, N2, N3, phi);
  const ptrdiff_t st = axis_stride(&d, m);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        inter[p] = stencil1(c->cIpu[m - 1], ORC_G_LO, ORC_G_HI, axis_row(m, i, j, k), phi, p, st);
      }
}

/* interpolate2_vel_pre (mod_diff.f90:1740-1825): u_m points -> pressure points */
void orc_interpolate_vel_pre(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi,
                             double* inter) {
  dims_t d = mkdims(N1, N2, N3);
  orc_exchange(m, N1, N2, N3, phi);
  const ptrdiff_t st = axis_stride(&d, m);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        inter[p] = stencil1(c->cIup[m - 1], ORC_D_LO, ORC_D_HI, axis_row(m, i, j, k), phi, p, st);
      }
}

/* one upwind term of nonlinear (mod_diff.f90:784-1424); component_id = 3*(m-1) + a */
void orc_nonlinear_upwind(int component_id, int N1, int N2, int N3, const orc_coeffs* c,
                          const double* pp, double* vel, double* nl) {
  dims_t d = mkdims(N1, N2, N3);
  const int m = (component_id - 1) / 3 + 1;
  const int a = (component_id - 1) % 3 + 1;
  orc_exchange(a, N1, N2, N3, vel);
  const double* cU = (a == m) ? c->cNuU[a - 1] : c->cNpU[a - 1];
  const double* cDn = (a == m) ? c->cNuD[a - 1] : c->cNpD[a - 1];
  const ptrdiff_t st = axis_stride(&d, a);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        int row = axis_row(a, i, j, k);
        double dd1 = (pp[p] >= 0.0) ? stencil1(cU, ORC_B_LO, ORC_B_HI, row, vel, p, st)
                                    : stencil1(cDn, ORC_B_LO, ORC_B_HI, row, vel, p, st);
        if (a == 1)
          nl[p] = dd1 * pp[p];
        else
          nl[p] = nl[p] + dd1 * pp[p];
      }
}

void orc_nonlinear(int m, int N1, int N2, int N3, const orc_coeffs* c, double* vel_m,
                   double* work1, double* work2, double* work3, double* pp, double* nl_m) {
  double* wk[3] = {work1, work2, work3};
  for (int a = 1; a <= 3; a++) {
    orc_interpolate_pre_vel(m, N1, N2, N3, c, wk[a - 1], pp);
    orc_nonlinear_upwind(3 * (m - 1) + a, N1, N2, N3, c, pp, vel_m, nl_m);
  }
}

/* axpby (axpby_kernel.cu:6-17 / mod_solvers.f90:281) */
void orc_axpby(int N1, int N2, int N3, double a, double b, const double* x, const double* y,
               double* z) {
  dims_t d = mkdims(N1, N2, N3);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        z[p] = a * x[p] + b * y[p];
      }
}

/* ------------------------------------------------------------------------------------ */
/* Laplacians and relaxation (mod_laplace.f90)                                          */
/* ------------------------------------------------------------------------------------ */
/* product_div_grad (mod_laplace.f90:38-197) */
void orc_product_div_grad(int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* dig,
                          double* lap) {
  for (int m = 1; m <= 3; m++) {
    orc_gradient(m, N1, N2, N3, c, phi, dig);
    orc_divergence(m, N1, N2, N3, c, dig, lap);
  }
}

/* product_div_grad_relax (mod_laplace.f90:216-327) */
void orc_product_dg_relax(int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* lap) {
  dims_t d = mkdims(N1, N2, N3);
  exchange_all(N1, N2, N3, phi);
  const ptrdiff_t sx = (ptrdiff_t)d.sx, sy = (ptrdiff_t)d.sy;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        lap[p] = CDG(c->cdg[0], -1, i) * phi[p - 1] + CDG(c->cdg[0], 1, i) * phi[p + 1] +
                 CDG(c->cdg[1], -1, j) * phi[p - sx] + CDG(c->cdg[1], 1, j) * phi[p + sx] +
                 CDG(c->cdg[2], -1, k) * phi[p - sy] + CDG(c->cdg[2], 1, k) * phi[p + sy] +
                 (CDG(c->cdg[0], 0, i) + CDG(c->cdg[1], 0, j) + CDG(c->cdg[2], 0, k)) * phi[p];
      }
}

/* relaxation_div_grad, Jacobi branch (mod_laplace.f90:339-613) */
void orc_jacobi(int N1, int N2, int N3, const orc_coeffs* c, int init_yes, int n_relax,
                double omega, const double* bb, double* rel, double* comp) {
  dims_t d = mkdims(N1, N2, N3);
  const ptrdiff_t sx = (ptrdiff_t)d.sx, sy = (ptrdiff_t)d.sy;
  for (int r = 1; r <= n_relax; r++) {
    if (r == 1 && init_yes) {
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= N3 - 1; k++)
        for (int j = 1; j <= N2 - 1; j++)
          for (int i = 1; i <= N1 - 1; i++) {
            size_t p = IX(&d, i, j, k);
            rel[p] = omega * bb[p] / (CDG(c->cdg[0], 0, i) + CDG(c->cdg[1], 0, j) + CDG(c->cdg[2], 0, k));
          }
    } else {
      exchange_all(N1, N2, N3, rel);
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= N3 - 1; k++)
        for (int j = 1; j <= N2 - 1; j++)
          for (int i = 1; i <= N1 - 1; i++) {
            size_t p = IX(&d, i, j, k);
            comp[p] = omega *
                          (bb[p] - CDG(c->cdg[0], -1, i) * rel[p - 1] - CDG(c->cdg[0], 1, i) * rel[p + 1] -
                           CDG(c->cdg[1], -1, j) * rel[p - sx] - CDG(c->cdg[1], 1, j) * rel[p + sx] -
                           CDG(c->cdg[2], -1, k) * rel[p - sy] - CDG(c->cdg[2], 1, k) * rel[p + sy]) /
                          (CDG(c->cdg[0], 0, i) + CDG(c->cdg[1], 0, j) + CDG(c->cdg[2], 0, k)) +
                      (1.0 - omega) * rel[p];
          }
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= N3 - 1; k++)
        for (int j = 1; j <= N2 - 1; j++)
          for (int i = 1; i <= N1 - 1; i++) {
            size_t p = IX(&d, i, j, k);
            rel[p] = comp[p];
          }
    }
  }
}

/* apply_pressure_BC_CT (usr_func.f90:857-897) with the label set of set_pressure_BC_kernel.cu */
void orc_pressure_bc(int N1, int N2, int N3, const uint8_t* label, int k_start_index,
                     double p_inlet, double p_outlet, double p_outlet2, double* rel) {
  dims_t d = mkdims(N1, N2, N3);
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        if (label[p] == 5 && k == k_start_index - 1) rel[p] = p_inlet;
        if (label[p] == 9 && k == k_start_index - 1) rel[p] = p_outlet;
        if (label[p] == 11) rel[p] = p_outlet2;
      }
}

/* ------------------------------------------------------------------------------------ */
/* reductions (mod_solvers.f90:2319-2470)                                               */
/* ------------------------------------------------------------------------------------ */
double orc_product_scalar(int N1, int N2, int N3, const double* a, const double* b) {
  dims_t d = mkdims(N1, N2, N3);
  double* part = (double*)calloc((size_t)N3, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++) {
    double s = 0.0;
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        s = s + a[p] * b[p];
      }
    part[k] = s;
  }
  double s = 0.0;
  for (int k = 1; k <= N3 - 1; k++) s += part[k];
  free(part);
  return s;
}

void orc_norms(int N1, int N2, int N3, const double* a, double* norm_inf, double* norm_two_sq) {
  dims_t d = mkdims(N1, N2, N3);
  double* pi = (double*)calloc((size_t)N3, sizeof(double));
  double* p2 = (double*)calloc((size_t)N3, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++) {
    double mi = 0.0, s = 0.0;
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        double v = a[IX(&d, i, j, k)];
        mi = fmax(fabs(v), mi);
        s = s + v * v;
      }
    pi[k] = mi;
    p2[k] = s;
  }
  double mi = 0.0, s = 0.0;
  for (int k = 1; k <= N3 - 1; k++) {
    mi = fmax(pi[k], mi);
    s += p2[k];
  }
  *norm_inf = mi;
  *norm_two_sq = s;
  free(pi);
  free(p2);
}

/* ------------------------------------------------------------------------------------ */
/* BiCGstab_orig (mod_solvers.f90:1509-1935), problem_type 2                            */
/* ------------------------------------------------------------------------------------ */
static void copy_interior(const dims_t* d, const double* src, double* dst) {
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= d->N3 - 1; k++)
    for (int j = 1; j <= d->N2 - 1; j++)
      for (int i = 1; i <= d->N1 - 1; i++) dst[IX(d, i, j, k)] = src[IX(d, i, j, k)];
}

typedef void (*precond_fn)(const void* ctx, double* v, double* z, double* comp);
typedef struct {
  int N1, N2, N3;
  const orc_coeffs* c;
  const orc_solver_opts* o;
} jac_ctx;
static void precond_jacobi(const void* ctx, double* v, double* z, double* comp) {
  /* single-level multigridV (mod_solvers.f90:456-585 with n_grids = 1): Jacobi sweeps from zero */
  const jac_ctx* j = (const jac_ctx*)ctx;
  orc_jacobi(j->N1, j->N2, j->N3, j->c, 1, j->o->n_sweeps, j->o->omega, v, z, comp);
}

static int converged(const orc_solver_opts* o, double ninf, double n2sq, double b2) {
  if (o->tol_abs_inf > 0.0 && ninf < o->tol_abs_inf) return 1;
  if (o->tol_rel > 0.0 && sqrt(n2sq) <= o->tol_rel * b2) return 1;
  return 0;
}

static void bicgstab_impl(int N1, int N2, int N3, const orc_coeffs* c, const orc_solver_opts* o,
                          precond_fn pfn, const void* pctx, double* bb, double* phi, double* work,
                          orc_solver_result* res) {
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  double* rr = work + 0 * fs;
  double* rh = work + 1 * fs;
  double* pp = work + 2 * fs;
  double* Ap = work + 3 * fs;
  double* Ar = work + 4 * fs;
  double* z1 = work + 5 * fs;
  double* z2 = work + 6 * fs;
  double* comp = work + 7 * fs;
  double* dig = work + 8 * fs;
  const int pre_on = pfn != NULL;
  const int init_yes = o->init_yes;
  double norm_inf = 0.0, norm2 = 0.0, b2sq = 0.0, dummy;
  double rhr = 0.0, rhr_prev, alpha = 0.0, omega = 0.0, beta, rhAp, rAr, ArAr;

  orc_norms(N1, N2, N3, bb, &dummy, &b2sq);
  const double b2 = sqrt(b2sq);
  if (!init_yes) {
    orc_product_div_grad(N1, N2, N3, c, phi, dig, rr);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= N3 - 1; k++)
      for (int j = 1; j <= N2 - 1; j++)
        for (int i = 1; i <= N1 - 1; i++) {
          size_t p = IX(&d, i, j, k);
          rr[p] = bb[p] - rr[p];
          rh[p] = rr[p];
        }
    orc_norms(N1, N2, N3, rr, &norm_inf, &norm2);
  } else {
    orc_norms(N1, N2, N3, bb, &norm_inf, &norm2);
  }
  res->status = 1;
  int counter = 0;
  for (;;) {
    int exit_yes = converged(o, norm_inf, norm2, b2) || counter == o->max_it;
    if (counter < 1 && norm_inf != 0.0 && counter != o->max_it) exit_yes = 0;
    if (exit_yes) {
      if (counter == 0 && init_yes) {
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= N3 - 1; k++)
          for (int j = 1; j <= N2 - 1; j++)
            for (int i = 1; i <= N1 - 1; i++) phi[IX(&d, i, j, k)] = 0.0;
      }
      res->status = converged(o, norm_inf, norm2, b2) ? 0 : 1;
      break;
    }
    if (!isfinite(norm_inf)) {
      res->status = 3;
      break;
    }
    counter++;
    rhr_prev = rhr;
    if (init_yes)
      rhr = (counter == 1) ? norm2 : orc_product_scalar(N1, N2, N3, rr, bb);
    else
      rhr = orc_product_scalar(N1, N2, N3, rr, rh);
    if (fabs(rhr) == 0.0) {
      copy_interior(&d, rr, rh);
      rhr = orc_product_scalar(N1, N2, N3, rr, rh);
    }
    if (counter >= 2) {
      if (omega == 0.0 || rhr_prev == 0.0) {
        res->status = 2;
        break;
      }
      beta = (alpha / omega) * (rhr / rhr_prev);
      omega = -beta * omega;
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= N3 - 1; k++)
        for (int j = 1; j <= N2 - 1; j++)
          for (int i = 1; i <= N1 - 1; i++) {
            size_t p = IX(&d, i, j, k);
            pp[p] = rr[p] + beta * pp[p] + omega * Ap[p];
          }
    } else {
      copy_interior(&d, (init_yes && counter == 1) ? bb : rr, pp);
    }
    if (pre_on) {
      pfn(pctx, pp, z1, comp);
      orc_product_div_grad(N1, N2, N3, c, z1, dig, Ap);
    } else {
      orc_product_div_grad(N1, N2, N3, c, pp, dig, Ap);
    }
    rhAp = orc_product_scalar(N1, N2, N3, Ap, init_yes ? bb : rh);
    if (fabs(rhAp) == 0.0) {
      res->status = 2;
      break;
    }
    alpha = rhr / rhAp;
    {
      const double* src = (init_yes && counter == 1) ? bb : rr;
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= N3 - 1; k++)
        for (int j = 1; j <= N2 - 1; j++)
          for (int i = 1; i <= N1 - 1; i++) {
            size_t p = IX(&d, i, j, k);
            rr[p] = src[p] - alpha * Ap[p];
          }
    }
    if (pre_on) {
      pfn(pctx, rr, z2, comp);
      orc_product_div_grad(N1, N2, N3, c, z2, dig, Ar);
    } else {
      orc_product_div_grad(N1, N2, N3, c, rr, dig, Ar);
    }
    rAr = orc_product_scalar(N1, N2, N3, rr, Ar);
    ArAr = orc_product_scalar(N1, N2, N3, Ar, Ar);
    if (fabs(ArAr) == 0.0) {
      res->status = 2;
      break;
    }
    omega = rAr / ArAr;
    const int first = (counter == 1 && init_yes);
    const double* zA = pre_on ? z1 : pp;
    const double* zB = pre_on ? z2 : rr;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= N3 - 1; k++)
      for (int j = 1; j <= N2 - 1; j++)
        for (int i = 1; i <= N1 - 1; i++) {
          size_t p = IX(&d, i, j, k);
          if (first)
            phi[p] = alpha * zA[p] + omega * zB[p];
          else
            phi[p] = phi[p] + omega * zB[p] + alpha * zA[p];
          rr[p] = rr[p] - omega * Ar[p];
        }
    orc_norms(N1, N2, N3, rr, &norm_inf, &norm2);
  }
  res->iterations = counter;
  res->res_inf = norm_inf;
  res->res_two = sqrt(norm2);
  res->b_two = b2;
}

static void precond_mg(const void* ctx, double* v, double* z, double* comp);
typedef struct {
  const orc_mg* mg;
  int n_down, n_up, n_bottom;
  double omega;
} mg_ctx;

void orc_bicgstab(int N1, int N2, int N3, const orc_coeffs* c, const orc_solver_opts* o,
                  double* bb, double* phi, double* work, orc_solver_result* res) {
  if (o->precond == 1 && o->mg != NULL) {
    mg_ctx m = {o->mg, o->mg_down, o->mg_up, o->mg_bottom, o->omega};
    bicgstab_impl(N1, N2, N3, c, o, precond_mg, &m, bb, phi, work, res);
    return;
  }
  jac_ctx j = {N1, N2, N3, c, o};
  bicgstab_impl(N1, N2, N3, c, o, o->n_sweeps > 0 ? precond_jacobi : NULL, &j, bb, phi, work, res);
}

/* ------------------------------------------------------------------------------------ */
/* geometric multigrid, periodic (mod_setup.f90:95-143 level sizes, mod_geometry.f90:66-103 */
/* level coordinates, get_stencil per level, interp_coeffs mod_coeffs.f90:1683-1746,     */
/* restr_coeffs :1879-2100 (constant 1/4 1/2 1/4 for periodic axes), multigridV /       */
/* restrict / interpolate mod_solvers.f90:353-1150)                                       */
/* ------------------------------------------------------------------------------------ */
static void jacobi_cdg(int N1, int N2, int N3, const double* const* cdg, int init_yes, int n_relax,
                       double omega, const double* bb, double* rel, double* comp) {
  orc_coeffs c;
  memset(&c, 0, sizeof(c));
  for (int a = 0; a < 3; a++) c.cdg[a] = cdg[a];
  orc_jacobi(N1, N2, N3, &c, init_yes, n_relax, omega, bb, rel, comp);
}
static void dg_relax_cdg(int N1, int N2, int N3, const double* const* cdg, double* phi, double* lap) {
  orc_coeffs c;
  memset(&c, 0, sizeof(c));
  for (int a = 0; a < 3; a++) c.cdg[a] = cdg[a];
  orc_product_dg_relax(N1, N2, N3, &c, phi, lap);
}

int orc_mg_build(int N1, int N2, int N3, const double* const* xp, const double* const* xu, const double* L,
                 int n_grids_limit, orc_mg* mg) {
  memset(mg, 0, sizeof(*mg));
  int MM[ORC_MG_MAX][3];
  MM[0][0] = N1;
  MM[0][1] = N2;
  MM[0][2] = N3;
  int ng = 1;
  for (int g = 1; g < ORC_MG_MAX; g++)
    for (int m = 0; m < 3; m++) {
      if ((MM[g - 1][m] - 1) % 2 == 0 && MM[g - 1][m] >= 5) {
        MM[g][m] = (MM[g - 1][m] - 1) / 2 + 1;
        ng = g + 1;
      } else {
        MM[g][m] = MM[g - 1][m];
      }
    }
  if (ng > n_grids_limit) ng = n_grids_limit;
  if (ng < 1) ng = 1;
  mg->n_grids = ng;
  for (int g = 0; g < ng; g++)
    for (int m = 0; m < 3; m++) {
      const int M = MM[g][m];
      mg->M[g][m] = M;
      mg->ratio[g][m] = (g + 1 < ng) ? (MM[g][m] - 1) / (MM[g + 1][m] - 1) : 1;
      double* p = (double*)calloc((size_t)M + 7, sizeof(double));
      double* u = (double*)calloc((size_t)M + 7, sizeof(double));
      const double* y1p = xp[m]; /* finest, offset 3 */
      if (g == 0) {
        memcpy(p, xp[m], sizeof(double) * (size_t)(M + 7));
        memcpy(u, xu[m], sizeof(double) * (size_t)(M + 7));
      } else {
        const int di = (MM[0][m] - 1) / (M - 1);
        for (int i = 1; i <= M; i++) p[i + 3] = y1p[1 + di * i - di + 3];
        for (int i = 1; i <= M - 1; i++) u[i + 3] = y1p[1 + di * i - di / 2 + 3];
        for (int i = -3; i <= 0; i++) {
          p[i + 3] = p[(M - 1 + i) + 3] - L[m];
          u[i + 3] = u[(M - 1 + i) + 3] - L[m];
        }
        for (int i = M; i <= M + 3; i++) {
          p[i + 3] = p[(i - M + 1) + 3] + L[m];
          u[i + 3] = u[(i - M + 1) + 3] + L[m];
        }
      }
      mg->xp[g][m] = p;
      mg->xu[g][m] = u;
      double* cdg = (double*)calloc((size_t)3 * M, sizeof(double));
      orc_get_stencil(M, p, u, cdg);
      mg->cdg[g][m] = cdg;
      double* ci = (double*)calloc((size_t)2 * (M + 1), sizeof(double));
      if (g + 1 < ng) {
        const int di = (MM[0][m] - 1) / (M - 1);
        for (int i = 2; i <= M - 1; i += 2) {
          const int i0 = 1 + (i - 1) * di;
          const double Dx10 = y1p[i0 + 3] - y1p[i0 - di + 3];
          const double Dx12 = y1p[i0 + di + 3] - y1p[i0 - di + 3];
          ci[2 * i + 0] = 1. - Dx10 / Dx12;
          ci[2 * i + 1] = Dx10 / Dx12;
        }
      }
      mg->cI[g][m] = ci;
    }
  for (int g = 1; g < ng; g++) {
    const size_t fs = (size_t)(mg->M[g][0] + 7) * (size_t)(mg->M[g][1] + 7) * (size_t)(mg->M[g][2] + 7);
    for (int q = 0; q < 3; q++) mg->f[g][q] = (double*)calloc(fs, sizeof(double));
  }
  return 0;
}

void orc_mg_free(orc_mg* mg) {
  for (int g = 0; g < ORC_MG_MAX; g++)
    for (int m = 0; m < 3; m++) {
      free(mg->xp[g][m]);
      free(mg->xu[g][m]);
      free(mg->cdg[g][m]);
      free(mg->cI[g][m]);
      free(mg->f[g][m]);
    }
  memset(mg, 0, sizeof(*mg));
}

/* restrict(.TRUE., g, coarse, fine1, fine2): coarse = R (fine1 - fine2), cR = 1/4, 1/2, 1/4 */
static void mg_restrict(const orc_mg* mg, int g, const double* fine1, const double* fine2, double* coarse) {
  const int* Mf = mg->M[g];
  const int* Mc = mg->M[g + 1];
  dims_t df = mkdims(Mf[0], Mf[1], Mf[2]);
  dims_t dc = mkdims(Mc[0], Mc[1], Mc[2]);
  const int r1 = mg->ratio[g][0], r2 = mg->ratio[g][1], r3 = mg->ratio[g][2];
  const int n1 = Mf[0] - 1, n2 = Mf[1] - 1, n3 = Mf[2] - 1;
  const double cm = 1. / 4., c0 = 2. / 4., cp = 1. / 4.;
#define WR(q, n) ((q) < 1 ? (q) + (n) : ((q) > (n) ? (q) - (n) : (q)))
#define DF(i, j, k) (fine1[IX(&df, WR(i, n1), WR(j, n2), WR(k, n3))] - fine2[IX(&df, WR(i, n1), WR(j, n2), WR(k, n3))])
#pragma omp parallel for schedule(static)
  for (int kk = 1; kk <= Mc[2] - 1; kk++)
    for (int jj = 1; jj <= Mc[1] - 1; jj++)
      for (int ii = 1; ii <= Mc[0] - 1; ii++) {
        const int i = r1 * (ii - 1) + 1, j = r2 * (jj - 1) + 1, k = r3 * (kk - 1) + 1;
        coarse[IX(&dc, ii, jj, kk)] = ((c0 + c0 + c0) * DF(i, j, k) + cm * DF(i - 1, j, k) + cp * DF(i + 1, j, k) +
                                       cm * DF(i, j - 1, k) + cp * DF(i, j + 1, k) + cm * DF(i, j, k - 1) +
                                       cp * DF(i, j, k + 1)) /
                                      3.;
      }
#undef DF
}

/* interpolate(.TRUE., g, coarse, fine, work): fine += P coarse (z, then y, then x passes) */
static void mg_interpolate_add(const orc_mg* mg, int g, double* coarse, double* fine, double* work) {
  const int* Mf = mg->M[g];
  const int* Mc = mg->M[g + 1];
  dims_t df = mkdims(Mf[0], Mf[1], Mf[2]);
  dims_t dc = mkdims(Mc[0], Mc[1], Mc[2]);
  const int di = mg->ratio[g][0], dj = mg->ratio[g][1], dk = mg->ratio[g][2];
  const int imax = Mf[0], jmax = Mf[1], kmax = Mf[2];
  exchange_all(Mc[0], Mc[1], Mc[2], coarse); /* exchange_relax: coarse(Mc) = coarse(1) */
  for (int kk = 1; kk <= Mc[2]; kk++)
    for (int jj = 1; jj <= Mc[1]; jj++)
      for (int ii = 1; ii <= Mc[0]; ii++)
        work[IX(&df, di * (ii - 1) + 1, dj * (jj - 1) + 1, dk * (kk - 1) + 1)] = coarse[IX(&dc, ii, jj, kk)];
  const double* c1 = mg->cI[g][0];
  const double* c2 = mg->cI[g][1];
  const double* c3 = mg->cI[g][2];
  if (dk != 1)
    for (int k = 2; k <= kmax - 1; k += dk)
      for (int j = 1; j <= jmax; j += dj)
        for (int i = 1; i <= imax; i += di)
          work[IX(&df, i, j, k)] = c3[2 * k] * work[IX(&df, i, j, k - 1)] + c3[2 * k + 1] * work[IX(&df, i, j, k + 1)];
  if (dj != 1)
    for (int k = 1; k <= kmax; k++)
      for (int j = 2; j <= jmax - 1; j += dj)
        for (int i = 1; i <= imax; i += di)
          work[IX(&df, i, j, k)] = c2[2 * j] * work[IX(&df, i, j - 1, k)] + c2[2 * j + 1] * work[IX(&df, i, j + 1, k)];
  if (di != 1)
    for (int k = 1; k <= kmax; k++)
      for (int j = 1; j <= jmax; j++)
        for (int i = 2; i <= imax - 1; i += di)
          work[IX(&df, i, j, k)] = c1[2 * i] * work[IX(&df, i - 1, j, k)] + c1[2 * i + 1] * work[IX(&df, i + 1, j, k)];
  for (int k = 1; k <= kmax - 1; k++)
    for (int j = 1; j <= jmax - 1; j++)
      for (int i = 1; i <= imax - 1; i++) fine[IX(&df, i, j, k)] = fine[IX(&df, i, j, k)] + work[IX(&df, i, j, k)];
}

void orc_mg_vcycle(const orc_mg* mg, int n_down, int n_up, int n_bottom, double omega, double* bb, double* phi,
                   double* work) {
  const int ng = mg->n_grids;
  double* A[ORC_MG_MAX];
  double* B[ORC_MG_MAX];
  double* Cw[ORC_MG_MAX];
  A[0] = bb;
  B[0] = phi;
  Cw[0] = work;
  for (int g = 1; g < ng; g++) {
    A[g] = mg->f[g][0];
    B[g] = mg->f[g][1];
    Cw[g] = mg->f[g][2];
  }
  for (int g = 0; g < ng - 1; g++) { /* relax_restrict */
    const int* M = mg->M[g];
    jacobi_cdg(M[0], M[1], M[2], (const double* const*)mg->cdg[g], 1, n_down, omega, A[g], B[g], Cw[g]);
    dg_relax_cdg(M[0], M[1], M[2], (const double* const*)mg->cdg[g], B[g], Cw[g]);
    mg_restrict(mg, g, A[g], Cw[g], A[g + 1]);
  }
  { /* relax_bottom */
    const int* M = mg->M[ng - 1];
    jacobi_cdg(M[0], M[1], M[2], (const double* const*)mg->cdg[ng - 1], 1, n_bottom, omega, A[ng - 1], B[ng - 1],
               Cw[ng - 1]);
    jacobi_cdg(M[0], M[1], M[2], (const double* const*)mg->cdg[ng - 1], 0, n_bottom, omega, A[ng - 1], B[ng - 1],
               Cw[ng - 1]);
  }
  for (int g = ng - 2; g >= 0; g--) { /* interpolate_relax */
    const int* M = mg->M[g];
    mg_interpolate_add(mg, g, B[g + 1], B[g], Cw[g]);
    jacobi_cdg(M[0], M[1], M[2], (const double* const*)mg->cdg[g], 0, n_up, omega, A[g], B[g], Cw[g]);
  }
}

static void precond_mg(const void* ctx, double* v, double* z, double* comp) {
  const mg_ctx* m = (const mg_ctx*)ctx;
  orc_mg_vcycle(m->mg, m->n_down, m->n_up, m->n_bottom, m->omega, v, z, comp);
}

void orc_bicgstab_mg(int N1, int N2, int N3, const orc_coeffs* c, const orc_mg* mg, const orc_solver_opts* o,
                     int n_down, int n_up, int n_bottom, double* bb, double* phi, double* work,
                     orc_solver_result* res) {
  mg_ctx m = {mg, n_down, n_up, n_bottom, o->omega};
  bicgstab_impl(N1, N2, N3, c, o, precond_mg, &m, bb, phi, work, res);
}

/* ------------------------------------------------------------------------------------ */
/* time step pieces                                                                      */
/* ------------------------------------------------------------------------------------ */
double orc_get_dtime(int N1, int N2, int N3, const orc_coeffs* c, const double* stab41,
                     double Re, double CFL, double dtime_max, double* vel, double* work) {
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  for (int m = 1; m <= 3; m++) orc_interpolate_vel_pre(m, N1, N2, N3, c, vel + (size_t)(m - 1) * fs, work + (size_t)(m - 1) * fs);
  double* part = (double*)calloc((size_t)N3, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= N3 - 1; k++) {
    double beta1 = 0.0;
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        double are = 0.0;
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) are = are + fabs(CF(c->cpp[0], ORC_B_LO, ORC_NB, l, i));
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) are = are + fabs(CF(c->cpp[1], ORC_B_LO, ORC_NB, l, j));
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) are = are + fabs(CF(c->cpp[2], ORC_B_LO, ORC_NB, l, k));
        are = are / Re;
        double dd1 = 0.0;
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) dd1 = dd1 + fabs(CF(c->cp1[0], ORC_B_LO, ORC_NB, l, i));
        double aim = dd1 * fabs(work[p]);
        dd1 = 0.0;
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) dd1 = dd1 + fabs(CF(c->cp1[1], ORC_B_LO, ORC_NB, l, j));
        aim = aim + dd1 * fabs(work[fs + p]);
        dd1 = 0.0;
        for (int l = ORC_B_LO; l <= ORC_B_HI; l++) dd1 = dd1 + fabs(CF(c->cp1[2], ORC_B_LO, ORC_NB, l, k));
        aim = aim + dd1 * fabs(work[2 * fs + p]);
        double angle = (fabs(aim) < 1e-16) ? PI_D / 2.0 : atan(are / aim);
        double radius = sqrt(are * are + aim * aim);
        long idx = lround(2.0 * 40.0 * angle / PI_D);
        if (idx < 0) idx = 0;
        if (idx > 40) idx = 40;
        beta1 = fmax(beta1, radius / stab41[idx]);
      }
    part[k] = beta1;
  }
  double beta1 = 0.0;
  for (int k = 1; k <= N3 - 1; k++) beta1 = fmax(beta1, part[k]);
  free(part);
  double dinv = beta1 / CFL;
  if (fabs(dinv) < 1.0 / dtime_max) return dtime_max;
  return 1.0 / dinv;
}

void orc_mask_forcing(int N1, int N2, int N3, const uint8_t* label, double u_inflow, double* vel) {
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) {
        size_t p = IX(&d, i, j, k);
        uint8_t lb = label[p];
        if (lb == 0 || lb == 7) {
          vel[p] = 0.0;
          vel[fs + p] = 0.0;
          vel[2 * fs + p] = 0.0;
        } else if (lb == 5) {
          vel[2 * fs + p] = u_inflow;
          vel[fs + p] = 0.0;
          vel[p] = 0.0;
        }
      }
}

void orc_level_pressure(int N1, int N2, int N3, double* pre) {
  dims_t d = mkdims(N1, N2, N3);
  double pre0 = 0.0;
  for (int k = 1; k <= N3 - 1; k++) {
    double s = 0.0;
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) s = s + pre[IX(&d, i, j, k)];
    pre0 += s;
  }
  pre0 = pre0 / (double)(N1 - 1) / (double)(N2 - 1) / (double)(N3 - 1);
  for (int k = 1; k <= N3 - 1; k++)
    for (int j = 1; j <= N2 - 1; j++)
      for (int i = 1; i <= N1 - 1; i++) pre[IX(&d, i, j, k)] = pre[IX(&d, i, j, k)] - pre0;
}

/* one time step (mod_timeint.f90:242-578, substeps :275-377; rhs_vel mod_rhs.f90:35-140;
 * explicit mod_solvers.f90:64-346) */
void orc_time_step(int N1, int N2, int N3, const orc_coeffs* c, const orc_step_params* p,
                   const double* stab41, const uint8_t* label, double* vel, double* nl, double* pre,
                   double* scratch, orc_step_state* st) {
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  double* rhs = scratch + 0 * fs;  /* 3 fields */
  double* work = scratch + 3 * fs; /* 3 fields */
  double* res = scratch + 6 * fs;
  double* pp = scratch + 7 * fs;
  double* sol = scratch + 8 * fs; /* 9 fields for the solver */

  double dt = orc_get_dtime(N1, N2, N3, c, stab41, p->Re, p->CFL, p->dtime_max, vel, work);
  if (st->timestep == 0 && dt > p->dtime0) dt = p->dtime0;
  st->dtime = dt;
  const double multL = 1.0 / p->Re;

  for (int s = 0; s < 3; s++) {
    /* exchange_all_all + interpolate_vel */
    for (int m = 0; m < 3; m++) exchange_all(N1, N2, N3, vel + m * fs);
    for (int m = 1; m <= 3; m++) {
      orc_interpolate_vel_pre(m, N1, N2, N3, c, vel + (m - 1) * fs, work + (m - 1) * fs);
      exchange_all(N1, N2, N3, work + (m - 1) * fs);
    }
    /* rhs_vel */
    for (int m = 0; m < 3; m++) copy_interior(&d, vel + m * fs, rhs + m * fs);
    if (s != 0) {
      const double mult = dt * bRK[s];
      for (int m = 0; m < 3; m++) {
        double* r = rhs + m * fs;
        const double* q = nl + m * fs;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= N3 - 1; k++)
          for (int j = 1; j <= N2 - 1; j++)
            for (int i = 1; i <= N1 - 1; i++) {
              size_t x = IX(&d, i, j, k);
              r[x] = r[x] - mult * q[x];
            }
      }
    }
    for (int m = 1; m <= 3; m++)
      orc_nonlinear(m, N1, N2, N3, c, vel + (m - 1) * fs, work, work + fs, work + 2 * fs, pp, nl + (m - 1) * fs);
    for (int m = 1; m <= 3; m++) orc_helmholtz(m, N1, N2, N3, c, multL, vel + (m - 1) * fs, nl + (m - 1) * fs);
    {
      const double mult = dt * aRK[s];
      for (int m = 0; m < 3; m++) {
        double* r = rhs + m * fs;
        const double* q = nl + m * fs;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= N3 - 1; k++)
          for (int j = 1; j <= N2 - 1; j++)
            for (int i = 1; i <= N1 - 1; i++) {
              size_t x = IX(&d, i, j, k);
              r[x] = r[x] - mult * q[x];
            }
      }
    }
    /* pressure pre-scaling (mod_timeint.f90:318) */
    const double ab = aRK[s] + bRK[s];
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= N3 - 1; k++)
      for (int j = 1; j <= N2 - 1; j++)
        for (int i = 1; i <= N1 - 1; i++) {
          size_t x = IX(&d, i, j, k);
          pre[x] = pre[x] * ab * dt;
        }
    /* explicit */
    for (int m = 0; m < 3; m++) copy_interior(&d, rhs + m * fs, vel + m * fs);
    orc_divergence2(N1, N2, N3, c, vel, vel + fs, vel + 2 * fs, res);
    orc_solver_result r;
    orc_bicgstab(N1, N2, N3, c, &p->poisson, res, pre, sol, &r);
    st->poisson_iterations[s] = r.iterations;
    st->poisson_status[s] = r.status;
    st->poisson_res_rel[s] = r.b_two > 0.0 ? r.res_two / r.b_two : 0.0;
    for (int m = 1; m <= 3; m++) {
      double* g = pp;
      orc_gradient(m, N1, N2, N3, c, pre, g);
      orc_axpby(N1, N2, N3, 1.0, -1.0, vel + (m - 1) * fs, g, vel + (m - 1) * fs);
    }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= N3 - 1; k++)
      for (int j = 1; j <= N2 - 1; j++)
        for (int i = 1; i <= N1 - 1; i++) {
          size_t x = IX(&d, i, j, k);
          pre[x] = pre[x] / ab / dt;
        }
  }
  st->timestep += 1;
  st->time += dt;
  const double u_in = p->U0 * (1.0 + 0.5 * sin(2.0 * PI_D * st->time / p->T_pulse));
  orc_mask_forcing(N1, N2, N3, label, u_in, vel);
  if (p->level_pressure) orc_level_pressure(N1, N2, N3, pre);
}

/* ------------------------------------------------------------------------------------ */
/* diffuse-interface immersed boundary transfers (mod_ibm.f90)                            */
/* ------------------------------------------------------------------------------------ */

/* discrete_delta (mod_ibm.f90:2021-2075).  pi = 2 |acos(0)| (FP64: the reference builds with
 * -fdefault-real-8).  A distance past the reach -- the reference's sentinel L1*L2*L3 for an
 * empty vicinity among them -- gives 0. */
double orc_ibm_delta(int type, double reach, double distance) {
  const double pi = 2.0 * fabs(acos(0.0));
  const double ad = fabs(distance);
  double delta = 0.0;
  if (type == 1) {
    if (ad <= reach) delta = (1.0 + cos(pi * ad / reach)) / (2.0 * reach);
  } else if (type == 2) {
    if (ad <= reach) delta = (reach - ad) / (reach * reach);
  } else if (type == 3) {
    if (ad <= reach / 2.0) {
      const double q = distance / (reach / 2.0);
      delta = (1.0 - q * q) / (reach / 2.0);
    } else if (ad > reach / 2.0 && ad <= reach) {
      const double q = distance / (reach / 2.0);
      delta = (2.0 - fabs(3.0 * distance / (reach / 2.0)) + q * q) / (reach / 2.0);
    }
  } else if (type == 4) {
    if (ad <= reach / 2.0) {
      const double t = ad / (reach / 2.0);
      delta = (3.0 - 2.0 * ad / (reach / 2.0) + sqrt(1.0 + 4.0 * ad / (reach / 2.0) - 4.0 * (t * t))) / (4.0 * reach);
    } else if (ad > reach / 2.0 && ad <= reach) {
      const double t = ad / (reach / 2.0);
      delta = (5.0 - 2.0 * ad / (reach / 2.0) - sqrt(-7.0 + 12.0 * ad / (reach / 2.0) - 4.0 * (t * t))) / (4.0 * reach);
    }
  }
  return delta;
}

/* find_vicinity_coordinates (mod_ibm.f90:743-876) along one axis: the first point of S..N
 * within the reach of y, and the last one before the first point beyond it; -1 / -1 when no
 * point is within reach.  x is a coordinate array over -3..N+3 (C offset 3). */
static void ibm_vicinity(const double* x, int S, int N, double y, double reach, int ind[2]) {
  ind[0] = ind[1] = -1;
  for (int i = S; i <= N; i++) {
    if (fabs(y - x[i + 3]) <= reach) {
      ind[0] = i;
      for (int j = i; j <= N; j++) {
        if (x[j + 3] - y > reach) {
          ind[1] = j - 1;
          return;
        } else if (j == N) {
          ind[1] = j;
          return;
        }
      }
    }
  }
}

/* The cell widths of mod_geometry.f90:193-204 on a periodic axis: dxp(i) = xu(i) - xu(i-1),
 * dxu(i) = xp(i+1) - xp(i), i = 1..N-1 (index i at offset i). */
static void ibm_widths(const double* xp, const double* xu, int N, double* dxp, double* dxu) {
  for (int i = 1; i <= N - 1; i++) {
    dxp[i] = xu[i + 3] - xu[i - 1 + 3];
    dxu[i] = xp[i + 1 + 3] - xp[i + 3];
  }
}

/* Shared walk of interpolate_vel_to_ib and spread_force_dens_to_vel_grid: for marker m and
 * velocity component c (0..2) the vicinity of every axis -- on the velocity grid xu along
 * axis c, on the pressure grid xp along the others -- and the distances yb - x.  Returns 0
 * when an axis has no point within reach: the reference then loops over the single index -1
 * with the sentinel distance, whose weight is 0, so every term it adds is a zero (it reads
 * vel(-1) and dx(-1) there, outside the interior); the restatement skips those terms. */
typedef struct {
  int lo[3], hi[3];
  double* dist[3];
  const double* dx[3];
} ibm_walk;

static int ibm_setup(const double* const* xp, const double* const* xu, double* const* dxp, double* const* dxu,
                     const int* N, double reach, int n, const double* yb, int m, int c, ibm_walk* w) {
  for (int a = 0; a < 3; a++) {
    const double* x = (a == c) ? xu[a] : xp[a];
    int ind[2];
    const double y = yb[(size_t)a * n + m];
    ibm_vicinity(x, 1, N[a] - 1, y, reach, ind);
    if (ind[0] == -1) return 0;
    w->lo[a] = ind[0];
    w->hi[a] = ind[1];
    for (int i = ind[0]; i <= ind[1]; i++) w->dist[a][i - ind[0]] = y - x[i + 3];
    w->dx[a] = (a == c) ? dxu[a] : dxp[a];
  }
  return 1;
}

static void ibm_alloc(const int* N, double** dxp, double** dxu, double** dist) {
  for (int a = 0; a < 3; a++) {
    dxp[a] = (double*)calloc((size_t)N[a] + 1, sizeof(double));
    dxu[a] = (double*)calloc((size_t)N[a] + 1, sizeof(double));
    dist[a] = (double*)calloc((size_t)N[a] + 1, sizeof(double));
  }
}
static void ibm_free(double** dxp, double** dxu, double** dist) {
  for (int a = 0; a < 3; a++) {
    free(dxp[a]);
    free(dxu[a]);
    free(dist[a]);
  }
}

/* interpolate_vel_to_ib (mod_ibm.f90:589-737), one block: ub(i, c) = sum over l, k, j of
 * delta(d1) * delta(d2) * delta(d3) * vel(j, k, l, c) * dx1(j) * dx2(k) * dx3(l), in that order. */
void orc_ibm_interpolate(int N1, int N2, int N3, const double* const* xp, const double* const* xu,
                         const double* L, int delta_type, double reach, int n, const double* yb,
                         const uint8_t* skip, const double* vel, double* ub) {
  (void)L;
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  const int N[3] = {N1, N2, N3};
  double *dxp[3], *dxu[3], *dist[3];
  ibm_alloc(N, dxp, dxu, dist);
  for (int a = 0; a < 3; a++) ibm_widths(xp[a], xu[a], N[a], dxp[a], dxu[a]);
  for (size_t q = 0; q < (size_t)3 * n; q++) ub[q] = 0.0;
  for (int m = 0; m < n; m++) {
    if (skip && skip[m]) continue;
    for (int c = 0; c < 3; c++) {
      ibm_walk w;
      for (int a = 0; a < 3; a++) w.dist[a] = dist[a];
      if (!ibm_setup(xp, xu, dxp, dxu, N, reach, n, yb, m, c, &w)) continue;
      double* u = &ub[(size_t)c * n + m];
      for (int l = w.lo[2]; l <= w.hi[2]; l++)
        for (int k = w.lo[1]; k <= w.hi[1]; k++)
          for (int j = w.lo[0]; j <= w.hi[0]; j++)
            *u = *u + orc_ibm_delta(delta_type, reach, w.dist[0][j - w.lo[0]]) *
                          orc_ibm_delta(delta_type, reach, w.dist[1][k - w.lo[1]]) *
                          orc_ibm_delta(delta_type, reach, w.dist[2][l - w.lo[2]]) *
                          vel[(size_t)c * fs + IX(&d, j, k, l)] * w.dx[0][j] * w.dx[1][k] * w.dx[2][l];
    }
  }
  ibm_free(dxp, dxu, dist);
}

/* spread_force_dens_to_vel_grid (mod_ibm.f90:428-583), one block: fd = 0, then
 * fd(j, k, l, c) += fb(i, c) * delta(d1) * delta(d2) * delta(d3) * node_vol(i) over the markers in
 * order.  The exchange_part calls that follow add the ghost planes 0 and N into the planes 1
 * and N-1 (mod_exchange.f90:1565-1568); those ghost planes hold zeros here (the vicinity search
 * visits only the points 1..N-1), so they change nothing and are not restated. */
void orc_ibm_spread(int N1, int N2, int N3, const double* const* xp, const double* const* xu, const double* L,
                    int delta_type, double reach, int n, const double* yb, const uint8_t* skip,
                    const double* fb, const double* node_vol, double* fd) {
  (void)L;
  dims_t d = mkdims(N1, N2, N3);
  const size_t fs = field_size(&d);
  const int N[3] = {N1, N2, N3};
  double *dxp[3], *dxu[3], *dist[3];
  ibm_alloc(N, dxp, dxu, dist);
  for (int a = 0; a < 3; a++) ibm_widths(xp[a], xu[a], N[a], dxp[a], dxu[a]);
  memset(fd, 0, 3 * fs * sizeof(double));
  for (int m = 0; m < n; m++) {
    if (skip && skip[m]) continue;
    for (int c = 0; c < 3; c++) {
      ibm_walk w;
      for (int a = 0; a < 3; a++) w.dist[a] = dist[a];
      if (!ibm_setup(xp, xu, dxp, dxu, N, reach, n, yb, m, c, &w)) continue;
      const double f = fb[(size_t)c * n + m];
      for (int l = w.lo[2]; l <= w.hi[2]; l++)
        for (int k = w.lo[1]; k <= w.hi[1]; k++)
          for (int j = w.lo[0]; j <= w.hi[0]; j++) {
            double* p = &fd[(size_t)c * fs + IX(&d, j, k, l)];
            *p = *p + f * orc_ibm_delta(delta_type, reach, w.dist[0][j - w.lo[0]]) *
                          orc_ibm_delta(delta_type, reach, w.dist[1][k - w.lo[1]]) *
                          orc_ibm_delta(delta_type, reach, w.dist[2][l - w.lo[2]]) * node_vol[m];
          }
    }
  }
  ibm_free(dxp, dxu, dist);
}

/* Host threads of the OpenMP loops above (test infrastructure: the CPU baseline reports single-
 * and all-core times).  n <= 0 leaves the setting unchanged; returns the threads now in use. */
#ifdef _OPENMP
#include <omp.h>
#endif
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
