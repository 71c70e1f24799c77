// ibm.cu -- immersed-boundary transfers of a resident case (mod_ibm.f90): the velocity at the
// Lagrangian markers (interpolate_vel_to_ib, :589-737) and the force density of the marker
// forces on the three staggered velocity grids (spread_force_dens_to_vel_grid, :428-583).
//
// Markers are few next to the grid (a surface mesh against a volume), so both kernels are
// latency-bound gathers and scatters: one thread per (component, marker) walks the support in
// the reference's order for the velocity, which keeps it bit-identical to the sequential loop;
// one warp per (component, marker) spreads the support's points with FP64 atomics, so the
// force density equals the sequential sum up to the order of the additions.
#include <cmath>
#include <cstring>
#include <vector>

#include "case.cuh"
#include "ibm.cuh"

using namespace impact;

namespace {

struct IbmArgs {
  ibm::Axis ax[3];
  const double* yb;
  const uint8_t* skip;  // nullptr: no marker skipped
  int n;
  int type;
  double reach;
};

constexpr int INT = 128;  // threads per block of the velocity kernel
constexpr int SPT = 256;  // threads per block of the spreading kernel (8 markers)

__global__ void __launch_bounds__(INT) k_ibm_interp(IbmArgs A, const double* __restrict__ u,
                                                    const double* __restrict__ v, const double* __restrict__ w,
                                                    long long sx, long long sy, double* __restrict__ ub,
                                                    int* flag) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // c * n + m
  if (t >= 3LL * A.n) return;
  const int c = (int)(t / A.n), m = (int)(t - (long long)c * A.n);
  double r = 0.0;
  if (!(A.skip && A.skip[m])) {
    const double y[3] = {A.yb[m], A.yb[A.n + m], A.yb[2LL * A.n + m]};
    const double* f = c == 0 ? u : (c == 1 ? v : w);
    int wide = 0;
    r = ibm::gather(A.ax, y, A.type, A.reach, c, f, sx, sy, &wide);
    if (wide) atomicOr(flag, 1);
  }
  ub[t] = r;
}

__global__ void __launch_bounds__(SPT) k_ibm_spread(IbmArgs A, const double* __restrict__ fb,
                                                    const double* __restrict__ vol, double* fu, double* fv,
                                                    double* fw, long long sx, long long sy, int* flag) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // c * n + m
  const int lane = threadIdx.x & 31;
  if (gw >= 3LL * A.n) return;
  const int c = (int)(gw / A.n), m = (int)(gw - (long long)c * A.n);
  if (A.skip && A.skip[m]) return;
  const double y[3] = {A.yb[m], A.yb[A.n + m], A.yb[2LL * A.n + m]};
  ibm::Support s;
  const int ok = ibm::support(A.ax, y, A.reach, c, s);
  if (ok < 0 && lane == 0) atomicOr(flag, 1);
  if (ok <= 0) return;
  const int n0 = s.hi[0] - s.lo[0] + 1, n1 = s.hi[1] - s.lo[1] + 1, n2 = s.hi[2] - s.lo[2] + 1;
  const double fc = fb[(long long)c * A.n + m], vm = vol[m];
  double* f = c == 0 ? fu : (c == 1 ? fv : fw);
  for (int p = lane; p < n0 * n1 * n2; p += 32) {
    const int j = s.lo[0] + p % n0, q = p / n0;
    const int k = s.lo[1] + q % n1, l = s.lo[2] + q / n1;
    atomicAdd(f + j + sx * k + sy * l, ibm::spread_term(s, y, A.type, A.reach, fc, vm, j, k, l));
  }
}

// Device view of the marker state: the geometry buffer holds, axis after axis, the four
// arrays xp, xu, dxp, dxu of N entries each.
IbmArgs ibm_args(const CaseState& s) {
  IbmArgs A{};
  const int N[3] = {s.g.n1 + 1, s.g.n2 + 1, s.g.n3 + 1};
  const double* p = s.ibm.geom;
  for (int a = 0; a < 3; ++a) {
    A.ax[a].n = N[a] - 1;
    A.ax[a].xp = p;
    A.ax[a].xu = p + N[a];
    A.ax[a].dxp = p + 2 * (size_t)N[a];
    A.ax[a].dxu = p + 3 * (size_t)N[a];
    p += 4 * (size_t)N[a];
  }
  A.yb = s.ibm.yb;
  A.skip = s.ibm.has_skip ? s.ibm.skip : nullptr;
  A.n = s.ibm.n;
  A.type = s.ibm.type;
  A.reach = s.ibm.reach;
  return A;
}

// Reads the kernels' flag (the case stream is idle when this is called) and clears it.
int ibm_flag_check(CaseState& s, const char* who) {
  int h = 0;
  IMPACT_CUDA_CHECK(cudaMemcpy(&h, s.ibm.flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (!h) return 0;
  IMPACT_CUDA_CHECK(cudaMemset(s.ibm.flag, 0, sizeof(int)));
  return impact_set_error_msg(-1, who);
}

}  // namespace

extern "C" int impact_b200_case_set_markers(impact_b200_case* c, int n, const double* yb, const uint8_t* skip,
                                            double reach, int delta_type) {
  if (!c || n < 0 || (n > 0 && !yb) || delta_type < 1 || delta_type > 4 || !std::isfinite(reach) || !(reach > 0.0))
    return impact_set_error_msg(-1, "impact_b200_case_set_markers: bad arguments");
  CaseState& s = c->s;
  if (s.xp[0].empty())
    return impact_set_error_msg(-1, "impact_b200_case_set_markers: the case was created without coordinates");
  for (long long q = 0; q < 3LL * n; ++q)
    if (!std::isfinite(yb[q])) return impact_set_error_msg(-1, "impact_b200_case_set_markers: non-finite position");
  const int N[3] = {s.g.n1 + 1, s.g.n2 + 1, s.g.n3 + 1};
  std::vector<double> geom;
  for (int a = 0; a < 3; ++a) {
    const size_t at = geom.size();
    ibm::axis_tables(s.xp[a].data(), s.xu[a].data(), N[a], geom);
    if (ibm::widest_support(geom.data() + at, N[a], reach) > ibm::MAXW)
      return impact_set_error_msg(-1, "impact_b200_case_set_markers: the reach spans more than 16 grid points");
  }
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  if (!s.ibm.geom) {
    if (case_alloc(s, (void**)&s.ibm.geom, geom.size() * sizeof(double))) return -1;
    if (case_alloc(s, (void**)&s.ibm.flag, sizeof(int))) return -1;
    IMPACT_CUDA_CHECK(cudaMemsetAsync(s.ibm.flag, 0, sizeof(int), s.stream));
  }
  IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.ibm.geom, geom.data(), geom.size() * sizeof(double), cudaMemcpyHostToDevice,
                                    s.stream));
  if (n > s.ibm.cap) {  // grow (the old buffers stay with the case until it is destroyed)
    double *yb_d = nullptr, *buf_d = nullptr;
    uint8_t* skip_d = nullptr;
    if (case_alloc(s, (void**)&yb_d, (size_t)3 * n * sizeof(double)) ||
        case_alloc(s, (void**)&buf_d, (size_t)4 * n * sizeof(double)) || case_alloc(s, (void**)&skip_d, (size_t)n))
      return -1;  // the previous marker set stays in force
    s.ibm.yb = yb_d;
    s.ibm.buf = buf_d;
    s.ibm.skip = skip_d;
    s.ibm.cap = n;
  }
  if (n > 0) {
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.ibm.yb, yb, (size_t)3 * n * sizeof(double), cudaMemcpyHostToDevice, s.stream));
    if (skip)
      IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.ibm.skip, skip, (size_t)n, cudaMemcpyHostToDevice, s.stream));
  }
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));  // the host arrays are free again
  s.ibm.n = n;
  s.ibm.type = delta_type;
  s.ibm.reach = reach;
  s.ibm.has_skip = skip != nullptr;
  return 0;
}

extern "C" int impact_b200_case_ibm_interpolate(impact_b200_case* c, double* ub) {
  if (!c || (c->s.ibm.n > 0 && !ub)) return impact_set_error_msg(-1, "impact_b200_case_ibm_interpolate: bad arguments");
  CaseState& s = c->s;
  if (!s.ibm.geom) return impact_set_error_msg(-1, "impact_b200_case_ibm_interpolate: no markers set");
  if (s.ibm.n == 0) return 0;
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  const IbmArgs A = ibm_args(s);
  const long long origin = 3 + 3LL * s.g.nx + 3LL * s.g.nxy;  // point (0, 0, 0) of a padded field
  const long long threads = 3LL * s.ibm.n;
  k_ibm_interp<<<(unsigned)((threads + INT - 1) / INT), INT, 0, s.stream>>>(
      A, s.f[IMPACT_B200_VEL1] + origin, s.f[IMPACT_B200_VEL2] + origin, s.f[IMPACT_B200_VEL3] + origin,
      s.g.nx, s.g.nxy, s.ibm.buf, s.ibm.flag);
  IMPACT_CUDA_CHECK(cudaGetLastError());
  IMPACT_CUDA_CHECK(cudaMemcpyAsync(ub, s.ibm.buf, (size_t)threads * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  return ibm_flag_check(s, "impact_b200_case_ibm_interpolate: a marker support exceeded 16 points");
}

extern "C" int impact_b200_case_ibm_spread(impact_b200_case* c, const double* fb, const double* node_vol,
                                           int field_first) {
  if (!c || (c->s.ibm.n > 0 && (!fb || !node_vol)) ||
      (field_first != IMPACT_B200_NL1 && field_first != IMPACT_B200_RHS1))
    return impact_set_error_msg(-1, "impact_b200_case_ibm_spread: bad arguments (field_first: NL1 or RHS1)");
  CaseState& s = c->s;
  if (!s.ibm.geom) return impact_set_error_msg(-1, "impact_b200_case_ibm_spread: no markers set");
  IMPACT_CUDA_CHECK(cudaSetDevice(s.device));
  const size_t fbytes = (size_t)s.g.nfield * sizeof(double);
  for (int q = 0; q < 3; ++q) IMPACT_CUDA_CHECK(cudaMemsetAsync(s.f[field_first + q], 0, fbytes, s.stream));
  const int n = s.ibm.n;
  if (n > 0) {
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.ibm.buf, fb, (size_t)3 * n * sizeof(double), cudaMemcpyHostToDevice, s.stream));
    IMPACT_CUDA_CHECK(cudaMemcpyAsync(s.ibm.buf + 3LL * n, node_vol, (size_t)n * sizeof(double),
                                      cudaMemcpyHostToDevice, s.stream));
    const IbmArgs A = ibm_args(s);
    const long long origin = 3 + 3LL * s.g.nx + 3LL * s.g.nxy;
    const long long threads = 3LL * n * 32;
    k_ibm_spread<<<(unsigned)((threads + SPT - 1) / SPT), SPT, 0, s.stream>>>(
        A, s.ibm.buf, s.ibm.buf + 3LL * n, s.f[field_first] + origin, s.f[field_first + 1] + origin,
        s.f[field_first + 2] + origin, s.g.nx, s.g.nxy, s.ibm.flag);
    IMPACT_CUDA_CHECK(cudaGetLastError());
  }
  IMPACT_CUDA_CHECK(cudaStreamSynchronize(s.stream));
  return ibm_flag_check(s, "impact_b200_case_ibm_spread: a marker support exceeded 16 points");
}
