// engine.cuh -- the batched pressure Poisson engine (internal).
//
// Every kernel of the solve runs over a *job list*: an array of jobs in device memory, one per
// grid (a case's fine grid, or one multigrid level of a case), each cut into tiles of
// ETX x ETY columns and `kc` z-planes.  A launch walks the tiles of all its jobs (grid-stride
// over the concatenated tile range), so one launch per operator advances every case of a
// batch, whatever their sizes; a single case is a batch of one.  Inside a tile every thread
// owns one (i, j) column and marches along z, keeping the z-neighbours in registers.
//
// Per-case solver scalars live in device memory (SolverScalars), one per job; every kernel of a
// case that has converged or broken down is a no-op, so the host only polls all flags every
// `check_every` iterations and a converged case costs nothing while others continue.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "mg.cuh"
#include "prof.cuh"
#include "solver.cuh"

namespace impact {

constexpr int ETX = 32, ETY = 8, ENT = ETX * ETY;
constexpr int AXW = 11;     // product_div_grad collapsed to an 11-point stencil per axis (-5..5)
constexpr int KC_MAX = 64;  // largest tile depth

inline int tiles_xy(const Geom& g) { return ((g.n1 + ETX - 1) / ETX) * ((g.n2 + ETY - 1) / ETY); }
inline int tiles_of(const Geom& g, int kc, int vw = 1) {
  return ((g.n1 + ETX * vw - 1) / (ETX * vw)) * ((g.n2 + ETY - 1) / ETY) * ((g.n3 + kc - 1) / kc);
}
// Tile geometry of the fused smoothing kernel k_lv_multi (MNT threads): a block's input region
// is 16 V x (MNT / 16) columns (V = 16 bytes / element size consecutive columns per thread, one
// row per half-warp); with S stencil stages it yields (16 V - 2S) x (MNT / 16 - 2S) output
// columns, kc planes deep.
constexpr int MNT = 512;
// fast: the aligned path (every job with n1 divisible by V = 16 / sz and uniform z), whose x halo
// is S rounded up to V
inline int tiles_multi(const Geom& g, int kc, int sz, int S, bool fast) {
  const int V = 16 / sz, HX = fast ? (S + V - 1) / V * V : S;
  const int X = 16 * V - 2 * HX, Y = MNT / 16 - 2 * S;
  return ((g.n1 + X - 1) / X) * ((g.n2 + Y - 1) / Y) * ((g.n3 + kc - 1) / kc);
}

// one multigrid level of one case
template <typename T>
struct LevelJob {
  Geom g;
  int kc;
  int zuni;         // 1: every z row of cdg[2] is the same: 1/diag is constant along a column
  int vw;           // columns per thread: 16 / sizeof(T) when n1 is a multiple of it, else 1
  const T* cdg[3];  // compact Laplacian of this level
  const T* A;       // right-hand side
  T* B;             // iterate
  T* C;             // work (sweep partner, residual)
  // restriction into this level from the next finer one
  Geom gf;
  int rf[3];
  const T* Cf;
  // prolongation into this level from the next coarser one
  Geom gc;
  int rc[3];
  const T* cI[3];
  const T* Bc;
  const SolverScalars* sc;
};

// the fine grid of one case inside BiCGstab
template <typename T>
struct KrylovJob {
  Geom g;
  int kc;
  const T* W[3];  // collapsed product_div_grad weights, row (i-1) holds offsets -5..5
  int zuni;       // 1: every z row of W[2] is the same (uniform z spacing)
  int xuni;       // 1: every x row of W[0] is the same (uniform x spacing)
  int vec;        // FP32: the operator of this job runs in the 4-point vector kernel
  const T* bb;
  T* phi;
  T *rr, *rh, *pp, *Ap, *Ar, *z1, *z2;
  float* r32;  // mixed precision: FP32 image of the FP64 outer residual (the inner solve's bb = rh)
  float* r32p; // and its second copy, the inner solve's first search direction pp (null: none)
  SolverScalars* sc;
};

// FP64 outer loop of the mixed-precision solve for one case
struct MixJob {
  Geom g;
  int kc;
  const double* bb;
  double* x;
  double* r64;
  float* r32;
  float* e32;
  const double* q;     // [max|r|, sum r^2, sum b^2] of this case's outer residual
  const SolverScalars* isc;  // inner solve scalars (correction applied only when status is 0 or 1)
};

struct DevList {
  int njobs = 0, ntiles = 0;
  const int* ts = nullptr;    // tile prefix sums (njobs + 1)
  const void* jobs = nullptr;
};

// what the engine needs to know about one case
template <typename T>
struct EngineCase {
  Geom g;
  const T* W[3];         // collapsed operator weights (device)
  int zuni;              // 1: every z row of W[2] is the same
  int xuni = 0;          // 1: every x row of W[0] is the same
  const T* cdg[3];       // fine-level compact Laplacian (device)
  int cdg_zuni;          // 1: every z row of cdg[2] is the same
  const MGData<T>* mg;   // multigrid hierarchy (level >= 1 fields owned by the case), or null
  const T* bb;
  T* phi;
  T *rr, *rh, *pp, *Ap, *Ar, *z1, *z2, *comp;
};

struct EngineParams {
  int precond = 1;   // 0: n_sweeps damped-Jacobi sweeps from zero (none if 0); 1: multigrid V-cycle
  int n_sweeps = 0;
  int mg_down = 4, mg_up = 4, mg_bottom = 4;
  double omega = 0.8;
  int check_every = 2;
  int kc = 16;       // z-planes per tile
  int use_graph = 1; // replay each chunk of iterations as a captured CUDA graph
  int fuse = 1;      // V-cycle smoothing phases as fused multi-sweep kernels
  int bottom_cheb = 0;  // > 0: Chebyshev steps on a tail's coarsest level instead of Jacobi sweeps
  bool operator==(const EngineParams& o) const {
    return precond == o.precond && n_sweeps == o.n_sweeps && mg_down == o.mg_down && mg_up == o.mg_up &&
           mg_bottom == o.mg_bottom && omega == o.omega && check_every == o.check_every && kc == o.kc &&
           use_graph == o.use_graph && fuse == o.fuse && bottom_cheb == o.bottom_cheb;
  }
};

struct Phase {
  int kind;  // PH_*
  int list;
  int flip;
};
// PH_PRE: init + (mg_down - 1) sweeps + residual in one kernel; PH_POST: mg_up sweeps in one
// kernel (after a PH_PROLONG with flip = 1, which writes its result into C); for 2 or 3 sweeps
// PH_TAIL: the coarsest levels of every case of the list in one block per case (k_lv_tail)
enum { PH_INIT = 0, PH_SWEEP, PH_COPY, PH_RESID, PH_RESTRICT, PH_PROLONG, PH_PRE, PH_POST, PH_TAIL };

// device arena of job lists built on the host
struct ListArena {
  std::vector<unsigned char> host;
  std::vector<DevList> lists;
  std::vector<size_t> ts_off, job_off;
  unsigned char* dev = nullptr;
  template <typename J>
  int add(const std::vector<J>& jobs, const std::vector<int>& tiles);
  int upload(cudaStream_t s);
  void release();
};

template <typename T>
class Engine {
 public:
  Engine() = default;
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  ~Engine() { release(); }

  int build(const std::vector<EngineCase<T>>& cs, const EngineParams& p, cudaStream_t s);
  // BiCGstab on every case.  init[c] carries tol_rel, tol_abs_inf and max_it of case c; a case
  // with init[c].done = 1 is skipped.  zero_phi: 1 start from phi = 0 (init_yes); 2 the same
  // without writing phi = 0 (the first x update starts from 0; a solve that ends before it
  // leaves phi unwritten and SolverScalars::phi_zero set).  ext_ts / ext_partial (with zero_phi,
  // rh sharing bb's buffer): the caller's tile partials [max|r|, -, -, sum bb^2] (tile offsets
  // ext_ts) replace the init pass; the caller wrote r0 to pp as well and left rr unwritten: the
  // first iteration keeps pp and reads r0 from rh (SolverScalars::rr_in_rh).
  int solve(const std::vector<SolverScalars>& init, int zero_phi, std::vector<SolverResult>& res,
            const int* ext_ts = nullptr, const double* ext_partial = nullptr);
  // one application of the preconditioner of every case: z1 = M pp
  int apply_precond();
  // one application of the operator of every case: rr = A phi
  int apply_operator();
  // measurement: `iters` launches of one kernel kind on the finest level of every case
  // (0 sweep, 1 init, 2 residual, 3 prolongation, 4 restriction to level 2, 5 A x + dot,
  //  6 A x + 2 dots, 7 x update, 8 p update, 9 r update, 10 one V-cycle, 11 one BiCGstab
  //  iteration, 12 fused pre-smoothing + residual, 13 fused post-smoothing); returns ms per
  //  launch and the algorithmic bytes of one launch
  int bench(int kind, int iters, double* ms, double* bytes);
  int ncases() const { return (int)cs_.size(); }
  const EngineParams& params() const { return p_; }
  SolverScalars* scal_dev() const { return scal_; }
  bool built() const { return built_; }
  void release();
  long long launches_per_iteration() const { return launches_iter_; }

 private:
  void enqueue_precond(int variant);
  void enqueue_iteration();
  void enqueue_phase(const Phase& ph);
  void smooth(std::vector<Phase>& out, int list, int init, int sweeps);
  int poll(bool& all_done);

  std::vector<EngineCase<T>> cs_;
  EngineParams p_{};
  cudaStream_t s_ = nullptr;
  bool built_ = false;
  ListArena arena_;
  int kr_list_ = -1;
  int down0_ = -1, rs1_ = -1;  // finest-level list of the first schedule, restriction to level 2
  int pre0_ = -1, post0_ = -1; // its fused pre- and post-smoothing lists (-1: not fused)
  std::vector<Phase> vc_[2];  // preconditioner schedules: z1 = M pp, z2 = M rr
  double* partial_ = nullptr;
  SolverScalars* scal_ = nullptr;
  SolverScalars* scal_host_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  bool graph_prof_ = false;          // the graph holds profiler event nodes
  std::vector<prof::Pair> gpairs_;   // those nodes' events
  long long launches_iter_ = 0;
  // per list: cells of its grids, of the next finer and of the next coarser grids (bytes for
  // the profiler)
  std::vector<double> cells_, cells_f_, cells_c_;
  std::vector<char> fast_;  // per list: every job vectorised with uniform z (k_lv_fast)
  int kr_vec_ = 0;          // FP32 Krylov list: jobs in the vector kernel -- 0 none, 1 all, 2 some
};

// Mixed precision: FP64 residual and correction around the FP32 engine.
class MixedEngine {
 public:
  struct Case {
    Geom g;
    const double* W64[3];
    int zuni;
    int xuni = 0;
    const double* bb;
    double* x;
    double* r64;
    float* r32;
    float* e32;
    EngineCase<float> inner;  // bb = rh = r32, phi = e32
  };
  MixedEngine() = default;
  MixedEngine(const MixedEngine&) = delete;
  MixedEngine& operator=(const MixedEngine&) = delete;
  ~MixedEngine() { release(); }
  int build(const std::vector<Case>& cs, const EngineParams& p, cudaStream_t s);
  // outer[c]: tol_rel, tol_abs_inf, max_it (outer passes); inner_tol, inner_max_it for every case
  int solve(const std::vector<SolverScalars>& outer, double inner_tol, int inner_max_it, int zero_x,
            std::vector<SolverResult>& res, std::vector<int>& inner_its);
  bool built() const { return built_; }
  const EngineParams& params() const { return inner_.params(); }
  Engine<float>& inner() { return inner_; }
  void release();

 private:
  std::vector<Case> cs_;
  Engine<float> inner_;
  cudaStream_t s_ = nullptr;
  bool built_ = false;
  ListArena arena_;
  int ax_list_ = -1, mix_list_ = -1;
  int ax_vec_ = 0;  // outer residual jobs in the FP64 vector kernel: 0 none, 1 all, 2 some
  double* partial_ = nullptr;
  double* q_ = nullptr;       // device, 4 per case
  double* q_host_ = nullptr;  // pinned
  SolverScalars* oscal_ = nullptr;  // outer scalars (only done/status are used by the kernels)
};

// collapsed product_div_grad weights of one axis: W(i, o) = sum_{a+b=o} cD(a, i) cG(b, wrap(i+a)),
// rows i = 1..n, o = -5..5 (cG rows hold offsets -2..3, cD rows -3..2, both rows 0..M)
void collapse_divgrad(int M, const double* cG, const double* cD, std::vector<double>& W);

}  // namespace impact
