// prof.cuh -- in-library kernel timing (CUDA events on the launching stream) and launch
// counting, read by the benchmark through impact_b200_profile_* / impact_b200_launch_count.
#pragma once
#include <cuda_runtime.h>

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
  K_COUNT
};

bool enabled();
// returns a token (or -1 when profiling is off); bytes = algorithmic bytes of the launch
int begin(cudaStream_t s);
void end(int token, int kid, double bytes, cudaStream_t s);
// resolve every recorded pair whose stream has been synchronised
void flush();
void count(long long n);  // kernel launches issued by the library

}  // namespace prof
}  // namespace impact

#define IMPACT_PROF(kid, bytes, stream, ...)                  \
  do {                                                        \
    const int _tok = impact::prof::begin(stream);             \
    __VA_ARGS__;                                              \
    impact::prof::end(_tok, (kid), (bytes), (stream));        \
    impact::prof::count(1);                                   \
  } while (0)
