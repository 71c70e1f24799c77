// case.cuh -- one simulation case resident on one GPU (internal).
#pragma once
#include <vector>

#include "../../include/impact_b200.h"
#include "common.cuh"
#include "engine.cuh"
#include "mg.cuh"
#include "solver.cuh"

namespace impact {

// per-axis row sums used by get_dtime: sum_l |cpp(l,i)| and sum_l |cp1(l,i)|
struct DtRows {
  const double* spp[3];
  const double* sp1[3];
};

struct CaseState {
  int device = 0;
  int precision = 0;
  Geom g{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // coefficient tables, FP64 and FP32 copies, in one allocation each
  double* coef64 = nullptr;
  float* coef32 = nullptr;
  Coeffs<double> c64{};
  Coeffs<float> c32{};
  DtRows dt{};
  // fields
  double* f[IMPACT_B200_NFIELDS] = {};
  double* work[3] = {};   // velocities interpolated to pressure points
  // mixed precision: the interpolated velocities and the nonlinear term of the time step in FP32
  // (the FP32 rhs_vel pass reads and writes these; nl1..3 of such a case are not kept)
  float* work32[3] = {};
  float* nl32[3] = {};
  uint8_t* label = nullptr;
  // FP64 Krylov work (8 fields), or the mixed-precision set
  KrylovWork<double> kw64{};
  MixedWork mw{};
  // multigrid hierarchy (levels >= 1 own their fields); FP64 for plain cases, FP32 for the
  // inner solve of mixed-precision cases
  int mg_levels = 0;
  MGData<double> mg64{};
  MGData<float> mg32{};
  double* partial = nullptr;     // reduction scratch of the step kernels
  double* dscal = nullptr;       // small device scalars (dt, mean pressure, ...)
  double* hscal = nullptr;       // pinned host mirror
  SolverScalars* scal_host = nullptr;
  // product_div_grad collapsed to 11-point stencils per axis, FP64 and FP32 (rows 1..n)
  const double* W64[3] = {};
  const float* W32[3] = {};
  int zuni = 0;      // every z row of the collapsed weights is the same (uniform z spacing)
  int xuni = 0;      // every x row of the collapsed weights is the same (uniform x spacing)
  int cdg_zuni = 0;  // every z row of the fine compact Laplacian is the same
  // Poisson engines (a batch of one), built on first use and rebuilt when the solver
  // parameters or the right-hand side / solution fields change
  Engine<double>* e64 = nullptr;
  MixedEngine* emx = nullptr;
  const double* eng_b = nullptr;
  double* eng_x = nullptr;
  std::vector<void*> allocs;
  cudaEvent_t pre_wait = nullptr;  // the next step waits for it before it first reads the pressure
  // snapshot: device copies of fields taken on the case stream, read back on a copy stream
  double* snap = nullptr;  // snap_cap fields (case pool)
  int snap_cap = 0;
  cudaEvent_t snap_taken = nullptr, snap_read = nullptr;
  bool snap_pending = false;  // snap_read marks the last read-back of the buffer
  // measured inflow waveform (nondimensional time, velocity); empty: the sinusoidal inflow
  std::vector<double> inflow_t, inflow_u;
  bool pooled = false;  // allocs come from the per-device case pool (freed stream-ordered)
  // global coordinates over -3..N+3 per axis (host copies; empty when the case was created
  // without them)
  std::vector<double> xp[3], xu[3];
  // immersed-boundary markers (impact_b200_case_set_markers), device side
  struct {
    int n = 0, cap = 0, type = 0;
    double reach = 0.0;
    bool has_skip = false;
    double* geom = nullptr;   // per axis: xp, xu, dxp, dxu over the points 0..N-1 (0 unused)
    double* yb = nullptr;     // positions, column-major (cap, 3)
    uint8_t* skip = nullptr;  // cap flags
    double* buf = nullptr;    // 4 cap: marker velocities, or forces and node volumes
    int* flag = nullptr;      // set by a kernel that met a support wider than its limit
  } ibm;
};

}  // namespace impact

struct impact_b200_case {
  impact::CaseState s;
};

// Device memory owned by the case (freed with it), from the per-device case pool.
int case_alloc(impact::CaseState& s, void** p, size_t bytes);
