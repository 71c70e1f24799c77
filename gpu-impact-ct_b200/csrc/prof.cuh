// prof.cuh -- in-library kernel timing (CUDA events on the launching stream) and launch
// counting, read by the benchmark through impact_b200_profile_* / impact_b200_launch_count.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace impact {
namespace prof {

enum Kid {
  K_PC_SWEEP = 0,  // damped-Jacobi sweep of the preconditioner
  K_PC_INIT2,      // fused init + first sweep
  K_DIVGRAD,       // high-order Laplacian with fused inner products
  K_X_UPDATE,      // BiCGstab solution / residual update with norms
  K_P_UPDATE,
  K_R_UPDATE,
  K_NL_RHS,        // advection + Helmholtz + RK update of one component
  K_PROJECT,       // vel = rhs - G pre
  K_DIV2,          // divergence of rhs
  K_MG_SWEEP,      // multigrid damped-Jacobi sweep (every level)
  K_MG_INIT,       // multigrid init sweep
  K_MG_RESID,      // multigrid residual
  K_MG_OTHER,      // restriction, prolongation, copies
  K_MG_PRE,        // fused init + sweeps + residual of one V-cycle level
  K_MG_POST,       // fused sweeps after the prolongation
  K_MX_RESID,      // mixed precision: FP64 outer residual b - A x and its FP32 image
  K_MX_APPLY,      // mixed precision: x += e in FP64
  K_MG_TAIL,       // the coarsest levels' part of a V-cycle in one block per case
  K_KR_INIT,       // BiCGstab start: r = b - A x (or b), shadow residual, norms
  K_COUNT
};

bool enabled();
// returns a token (or -1 when profiling is off); bytes = algorithmic bytes of the launch
int begin(cudaStream_t s);
void end(int token, int kid, double bytes, cudaStream_t s);
// resolve every recorded pair whose stream has been synchronised
void flush();
void count(long long n);  // kernel launches issued by the library

// CUDA graphs: between capture_begin() and capture_end() the timed pairs become event-record
// nodes of the graph being captured; after every replay of that graph has completed,
// graph_account() adds their times, and graph_release() returns the events.
struct Pair {
  int kid;
  double bytes;
  cudaEvent_t a, b;
};
void capture_begin();
std::vector<Pair> capture_end();
void graph_account(const std::vector<Pair>& pairs);
void graph_release(std::vector<Pair>& pairs);

}  // namespace prof
}  // namespace impact

#define IMPACT_PROF(kid, bytes, stream, ...)                  \
  do {                                                        \
    const int _tok = impact::prof::begin(stream);             \
    __VA_ARGS__;                                              \
    impact::prof::end(_tok, (kid), (bytes), (stream));        \
    impact::prof::count(1);                                   \
  } while (0)
