// mg.cuh -- the multigrid hierarchy of a case on the device: per level its geometry, tables and
// fields (the V-cycle itself runs in the engine, engine.cu).
#pragma once
#include "common.cuh"

namespace impact {

constexpr int MG_MAX_LEVELS = 15;

template <typename T>
struct MGLevel {
  Geom g;
  const T* cdg[3];  // compact Laplacian of the level
  int zuni = 0;     // 1: every z row of cdg[2] is the same (uniform z spacing on this level)
  const T* cI[3];   // interpolation weights cI(1:2, 0:M) of the level
  int ratio[3];     // coarsening factor to the next level
  T *A, *B, *C;     // right-hand side, solution, work (levels >= 1)
  double lmin = 0;  // estimate of the smallest nonzero eigenvalue of diag(cdg)^-1 cdg on this level
};

template <typename T>
struct MGData {
  int n = 0;
  MGLevel<T> lv[MG_MAX_LEVELS];
  int n_down = 4, n_up = 4, n_bottom = 4;
  double omega = 0.8;
};

}  // namespace impact
