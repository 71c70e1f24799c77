// mg.cu -- geometric multigrid V-cycle of the pressure Poisson preconditioner (periodic).
//
//   relaxation_div_grad     mod_laplace.f90:339-613   damped Jacobi sweeps on level g
//   product_div_grad_relax  mod_laplace.f90:216-327   residual of level g (fused: C = A - cdg(B))
//   restrict                mod_solvers.f90:588-808   coarse = R (bb - work), cR = 1/4 1/2 1/4
//   interpolate             mod_solvers.f90:955-1141  fine += P coarse (z, then y, then x passes)
//   multigridV              mod_solvers.f90:456-585   V-cycle with gstart = 1, init_yes = .TRUE.
#include "mg.cuh"
#include "prof.cuh"

namespace impact {

namespace {
constexpr int BX = 32, BY = 8, NT = BX * BY;
inline dim3 grid3(const Geom& g) { return dim3((g.n1 + BX - 1) / BX, (g.n2 + BY - 1) / BY, g.n3); }
__device__ __forceinline__ bool mg_halted(const SolverScalars* sc) { return sc != nullptr && (sc->done | sc->status); }
#define MG_PT                                        \
  const int i = blockIdx.x * BX + threadIdx.x + 1;   \
  const int j = blockIdx.y * BY + threadIdx.y + 1;   \
  const int k = blockIdx.z + 1;                      \
  if (i > g.n1 || j > g.n2) return;                  \
  const long long p = off(g, i, j, k);
}  // namespace

// init: out = omega bb / diag; otherwise one damped-Jacobi sweep of rel
template <typename T>
__global__ void __launch_bounds__(NT) k_mg_jacobi(Geom g, const T* __restrict__ c1, const T* __restrict__ c2,
                                                  const T* __restrict__ c3, T omega, const SolverScalars* __restrict__ sc,
                                                  int init, const T* __restrict__ bb, const T* __restrict__ rel,
                                                  T* __restrict__ out) {
  if (mg_halted(sc)) return;
  MG_PT
  const T* a = c1 + 3 * (i - 1);
  const T* b = c2 + 3 * (j - 1);
  const T* c = c3 + 3 * (k - 1);
  if (init) {
    out[p] = omega * bb[p] / (a[1] + b[1] + c[1]);
    return;
  }
  const T xw = __ldg(rel + off(g, wrapi(i - 1, g.n1), j, k)), xe = __ldg(rel + off(g, wrapi(i + 1, g.n1), j, k));
  const T xs = __ldg(rel + off(g, i, wrapi(j - 1, g.n2), k)), xn = __ldg(rel + off(g, i, wrapi(j + 1, g.n2), k));
  const T xm = __ldg(rel + off(g, i, j, wrapi(k - 1, g.n3))), xp = __ldg(rel + off(g, i, j, wrapi(k + 1, g.n3)));
  out[p] = omega * (bb[p] - a[0] * xw - a[2] * xe - b[0] * xs - b[2] * xn - c[0] * xm - c[2] * xp) / (a[1] + b[1] + c[1]) +
           (T(1) - omega) * __ldg(rel + p);
}

// C = A - cdg(B): the residual that restrict forms as fine1 - fine2 with fine2 = product_div_grad_relax
template <typename T>
__global__ void __launch_bounds__(NT) k_mg_residual(Geom g, const T* __restrict__ c1, const T* __restrict__ c2,
                                                    const T* __restrict__ c3, const SolverScalars* __restrict__ sc,
                                                    const T* __restrict__ A, const T* __restrict__ B, T* __restrict__ C) {
  if (mg_halted(sc)) return;
  MG_PT
  const T* a = c1 + 3 * (i - 1);
  const T* b = c2 + 3 * (j - 1);
  const T* c = c3 + 3 * (k - 1);
  const T lap = a[0] * __ldg(B + off(g, wrapi(i - 1, g.n1), j, k)) + a[2] * __ldg(B + off(g, wrapi(i + 1, g.n1), j, k)) +
                b[0] * __ldg(B + off(g, i, wrapi(j - 1, g.n2), k)) + b[2] * __ldg(B + off(g, i, wrapi(j + 1, g.n2), k)) +
                c[0] * __ldg(B + off(g, i, j, wrapi(k - 1, g.n3))) + c[2] * __ldg(B + off(g, i, j, wrapi(k + 1, g.n3))) +
                (a[1] + b[1] + c[1]) * __ldg(B + p);
  C[p] = A[p] - lap;
}

// coarse(ii,jj,kk) = (1.5 d(c) + sum over the six fine neighbours of 1/4 d) / 3, d = fine residual
template <typename T>
__global__ void __launch_bounds__(NT) k_mg_restrict(Geom gf, Geom g, int r1, int r2, int r3,
                                                   const SolverScalars* __restrict__ sc, const T* __restrict__ d,
                                                   T* __restrict__ coarse) {
  if (mg_halted(sc)) return;
  MG_PT
  const int fi = r1 * (i - 1) + 1, fj = r2 * (j - 1) + 1, fk = r3 * (k - 1) + 1;
  const T cm = T(1) / T(4), c0 = T(2) / T(4), cp = T(1) / T(4);
  const T v = (c0 + c0 + c0) * __ldg(d + off(gf, fi, fj, fk)) + cm * __ldg(d + off(gf, wrapi(fi - 1, gf.n1), fj, fk)) +
              cp * __ldg(d + off(gf, wrapi(fi + 1, gf.n1), fj, fk)) + cm * __ldg(d + off(gf, fi, wrapi(fj - 1, gf.n2), fk)) +
              cp * __ldg(d + off(gf, fi, wrapi(fj + 1, gf.n2), fk)) + cm * __ldg(d + off(gf, fi, fj, wrapi(fk - 1, gf.n3))) +
              cp * __ldg(d + off(gf, fi, fj, wrapi(fk + 1, gf.n3)));
  coarse[p] = v / T(3);
}

// fine += P coarse, evaluated per fine point exactly as the sequential z, y, x passes would
template <typename T>
__global__ void __launch_bounds__(NT) k_mg_prolong_add(Geom g, Geom gc, int r1, int r2, int r3, const T* __restrict__ cI1,
                                                       const T* __restrict__ cI2, const T* __restrict__ cI3,
                                                       const SolverScalars* __restrict__ sc, const T* __restrict__ coarse,
                                                       T* __restrict__ fine) {
  if (mg_halted(sc)) return;
  MG_PT
  // coarse indices bracketing each fine index (lo == hi for coincident points)
  auto br = [](int q, int r, int nc, int& lo, int& hi, bool& mid) {
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
  };
  int xl, xh, yl, yh, zl, zh;
  bool mx, my, mz;
  br(i, r1, gc.n1, xl, xh, mx);
  br(j, r2, gc.n2, yl, yh, my);
  br(k, r3, gc.n3, zl, zh, mz);
  auto Z = [&](int cx, int cy) -> T {
    if (!mz) return __ldg(coarse + off(gc, cx, cy, zl));
    return cI3[2 * k] * __ldg(coarse + off(gc, cx, cy, zl)) + cI3[2 * k + 1] * __ldg(coarse + off(gc, cx, cy, zh));
  };
  auto Y = [&](int cx) -> T {
    if (!my) return Z(cx, yl);
    return cI2[2 * j] * Z(cx, yl) + cI2[2 * j + 1] * Z(cx, yh);
  };
  const T w = mx ? cI1[2 * i] * Y(xl) + cI1[2 * i + 1] * Y(xh) : Y(xl);
  fine[p] = fine[p] + w;
}

template <typename T>
__global__ void __launch_bounds__(NT) k_mg_copy(Geom g, const SolverScalars* __restrict__ sc, const T* __restrict__ a,
                                                T* __restrict__ b) {
  if (mg_halted(sc)) return;
  MG_PT
  b[p] = a[p];
}

// `sweeps` relaxation steps on level l (the first one the init step when init); the result in B
template <typename T>
static void smooth(const MGLevel<T>& L, const SolverScalars* sc, T omega, int init, int sweeps, const T* A, T* B, T* C,
                   cudaStream_t s) {
  if (sweeps <= 0) return;
  const dim3 gr = grid3(L.g), bl(BX, BY);
  // targets alternate so that the last write lands in B; the first write may not read its target
  T* buf[2] = {B, C};
  int tgt = (sweeps % 2 == 1) ? 0 : 1;
  const T* src = B;
  int w = 0;
  if (init) {
    k_mg_jacobi<T><<<gr, bl, 0, s>>>(L.g, L.cdg[0], L.cdg[1], L.cdg[2], omega, sc, 1, A, nullptr, buf[tgt]);
    src = buf[tgt];
    tgt ^= 1;
    ++w;
  } else if (tgt == 0) {  // odd number of plain sweeps: stage the start in C first
    k_mg_copy<T><<<gr, bl, 0, s>>>(L.g, sc, B, C);
    src = C;
    prof::count(1);
  }
  for (; w < sweeps; ++w) {
    k_mg_jacobi<T><<<gr, bl, 0, s>>>(L.g, L.cdg[0], L.cdg[1], L.cdg[2], omega, sc, 0, A, src, buf[tgt]);
    src = buf[tgt];
    tgt ^= 1;
  }
  prof::count(sweeps);
}

template <typename T>
void mg_vcycle(const MGData<T>& mg, const SolverScalars* sc, const T* v, T* z, T* work0, cudaStream_t s) {
  const int n = mg.n;
  const T om = (T)mg.omega;
  const T* A[MG_MAX_LEVELS];
  T* B[MG_MAX_LEVELS];
  T* C[MG_MAX_LEVELS];
  for (int g = 0; g < n; ++g) {
    A[g] = g == 0 ? v : mg.lv[g].A;
    B[g] = g == 0 ? z : mg.lv[g].B;
    C[g] = g == 0 ? work0 : mg.lv[g].C;
  }
  for (int g = 0; g + 1 < n; ++g) {  // relax_restrict
    const MGLevel<T>& L = mg.lv[g];
    smooth<T>(L, sc, om, 1, mg.n_down, A[g], B[g], C[g], s);
    k_mg_residual<T><<<grid3(L.g), dim3(BX, BY), 0, s>>>(L.g, L.cdg[0], L.cdg[1], L.cdg[2], sc, A[g], B[g], C[g]);
    const MGLevel<T>& Lc = mg.lv[g + 1];
    k_mg_restrict<T><<<grid3(Lc.g), dim3(BX, BY), 0, s>>>(L.g, Lc.g, L.ratio[0], L.ratio[1], L.ratio[2], sc, C[g],
                                                          mg.lv[g + 1].A);
    prof::count(2);
  }
  {  // relax_bottom
    const MGLevel<T>& L = mg.lv[n - 1];
    smooth<T>(L, sc, om, 1, mg.n_bottom, A[n - 1], B[n - 1], C[n - 1], s);
    smooth<T>(L, sc, om, 0, mg.n_bottom, A[n - 1], B[n - 1], C[n - 1], s);
  }
  for (int g = n - 2; g >= 0; --g) {  // interpolate_relax
    const MGLevel<T>& L = mg.lv[g];
    const MGLevel<T>& Lc = mg.lv[g + 1];
    k_mg_prolong_add<T><<<grid3(L.g), dim3(BX, BY), 0, s>>>(L.g, Lc.g, L.ratio[0], L.ratio[1], L.ratio[2], L.cI[0],
                                                            L.cI[1], L.cI[2], sc, B[g + 1], B[g]);
    prof::count(1);
    smooth<T>(L, sc, om, 0, mg.n_up, A[g], B[g], C[g], s);
  }
}

template void mg_vcycle<double>(const MGData<double>&, const SolverScalars*, const double*, double*, double*,
                                cudaStream_t);
template void mg_vcycle<float>(const MGData<float>&, const SolverScalars*, const float*, float*, float*, cudaStream_t);

}  // namespace impact
