// capi.cu -- the C ABI: the reference's launcher FFI (src/*_launcher.cu, bound by the unchanged
// src/*_host.f90 wrappers) and library control / device-resident solve entry points.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/impact_b200.h"
#include "common.cuh"
#include "kernels.cuh"
#include "solver.cuh"

using namespace impact;

// ---------------------------------------------------------------------------------------
// errors (the reference prints and continues, grad_host.f90:7-30; here the message is kept
// and every int entry point returns a status)
// ---------------------------------------------------------------------------------------
static thread_local std::string g_err;

int impact_set_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_err = buf;
  return -static_cast<int>(e) - 1000;
}
int impact_set_error_msg(int code, const char* msg) {
  g_err = msg;
  return code;
}

extern "C" const char* impact_b200_last_error(void) { return g_err.c_str(); }
extern "C" void impact_b200_clear_error(void) { g_err.clear(); }
extern "C" int impact_b200_version(void) { return 10000; }

static cudaStream_t g_stream = nullptr;  // legacy default stream, as the reference launchers
extern "C" void impact_b200_set_stream(void* s) { g_stream = static_cast<cudaStream_t>(s); }
extern "C" int impact_b200_sync(void) {
  cudaError_t e = cudaStreamSynchronize(g_stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return impact_set_error(e, "impact_b200_sync", __FILE__, __LINE__);
  return 0;
}

static bool check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    impact_set_error(e, what, __FILE__, __LINE__);
    return false;
  }
  return true;
}

// padded extents -> geometry; the reference requires nx_dev - 8 cells per axis
static bool geom_from_dev(int nx, int ny, int nz, Geom* g, const char* who) {
  if (nx < 16 || ny < 16 || nz < 16) {
    impact_set_error_msg(-1, (std::string(who) + ": padded extents must be >= 16 (8 unique points)").c_str());
    return false;
  }
  *g = make_geom(nx - 7, ny - 7, nz - 7);
  return true;
}

// Library-owned scratch (jor_launcher_ output, product_scalar partials, the JOR solve's
// workspace), one buffer per (device, stream) so that launchers issued on different streams
// never share memory.  A buffer is allocated on the first use from its stream and regrown (after
// its stream has drained) when a larger grid arrives; it is kept until the process exits.
namespace {
struct ScratchSlot {
  int dev;
  cudaStream_t stream;
  void* ptr;
  size_t bytes;
};
std::mutex g_scratch_mu;
std::vector<ScratchSlot> g_scratch_slots;
}  // namespace

static void* scratch(size_t bytes, cudaStream_t s) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    impact_set_error_msg(-1, "library scratch: cudaGetDevice failed");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchSlot* slot = nullptr;
  for (auto& x : g_scratch_slots)
    if (x.dev == dev && x.stream == s) slot = &x;
  if (!slot) {
    g_scratch_slots.push_back({dev, s, nullptr, 0});
    slot = &g_scratch_slots.back();
  }
  if (bytes > slot->bytes) {
    if (slot->ptr) {
      cudaStreamSynchronize(s);
      cudaFree(slot->ptr);
    }
    slot->ptr = nullptr;
    slot->bytes = 0;
    if (cudaMalloc(&slot->ptr, bytes) != cudaSuccess) {
      slot->ptr = nullptr;
      impact_set_error_msg(-1, "library scratch allocation failed");
      return nullptr;
    }
    slot->bytes = bytes;
  }
  return slot->ptr;
}

// the Part 1 launchers' stream, for the other translation units of the C ABI
cudaStream_t impact_launcher_stream() { return g_stream; }

// ---------------------------------------------------------------------------------------
// Part 1: reference launchers
// ---------------------------------------------------------------------------------------
extern "C" void gradient_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_grad_coef,
                                   int* ny_grad_coef, double** phi_grad_dev, double** cGp_dev, double** grad_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "gradient_launcher_")) return;
  if (*nx_grad_coef != NG || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "gradient_launcher_: expects 6 coefficients per row and dimension_id 1..3");
    return;
  }
  (void)ny_grad_coef;
  launch_gradient<double>(*dimension_id, g, *cGp_dev, *phi_grad_dev, *grad_dev, g_stream);
  check_launch("gradient_launcher_");
}

extern "C" void divergence_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef,
                                     int* ny_div_coef, double** phi_div_dev, double** div_dev, double** cD_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "divergence_launcher_")) return;
  if (*nx_div_coef != ND || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "divergence_launcher_: expects 6 coefficients per row and dimension_id 1..3");
    return;
  }
  (void)ny_div_coef;
  launch_divergence<double>(*dimension_id, g, *cD_dev, *phi_div_dev, *div_dev, g_stream);
  check_launch("divergence_launcher_");
}

extern "C" void divergence2_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef1, int* nx_div_coef2,
                                      int* nx_div_coef3, double** phi_div2_dev, double** div2_dev, double** cDu1_dev,
                                      double** cDv2_dev, double** cDw3_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "divergence2_launcher_")) return;
  if (*nx_div_coef1 != ND || *nx_div_coef2 != ND || *nx_div_coef3 != ND) {
    impact_set_error_msg(-1, "divergence2_launcher_: expects 6 coefficients per row");
    return;
  }
  const double* u = *phi_div2_dev;
  launch_divergence2<double>(g, *cDu1_dev, *cDv2_dev, *cDw3_dev, u, u + g.nfield, u + 2 * g.nfield, *div2_dev,
                             g_stream);
  check_launch("divergence2_launcher_");
}

extern "C" void helmholtz_explicit_launcher_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxs1,
                                             int* nxs2, int* nxs3, double* multL, double** vel1_dev, double** helm_dev,
                                             double** cS1_helm_dev, double** cS2_helm_dev, double** cS3_helm_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "helmholtz_explicit_launcher_")) return;
  if (*nxs1 != NB || *nxs2 != NB || *nxs3 != NB) {
    impact_set_error_msg(-1, "helmholtz_explicit_launcher_: expects 7 coefficients per row");
    return;
  }
  launch_helmholtz<double>(*component_id, g, *cS1_helm_dev, *cS2_helm_dev, *cS3_helm_dev, *multL, *vel1_dev,
                           *helm_dev, g_stream);
  check_launch("helmholtz_explicit_launcher_");
}

extern "C" void nonlinear_upwind_launcher_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxn1,
                                           int* nyn1, double** pp_dev, double** vel_dev, double** nl_dev,
                                           double** cN1_dev, double** cN21_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "nonlinear_upwind_launcher_")) return;
  if (*nxn1 != NB || *component_id < 1 || *component_id > 9) {
    impact_set_error_msg(-1, "nonlinear_upwind_launcher_: expects 7 coefficients per row and component_id 1..9");
    return;
  }
  (void)nyn1;
  launch_nonlinear_upwind<double>(*component_id, g, *cN1_dev, *cN21_dev, *pp_dev, *vel_dev, *nl_dev, g_stream);
  check_launch("nonlinear_upwind_launcher_");
}

extern "C" void interpolate2_pre_vel_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIpu1,
                                               int* nyIpu1, double** phi_inter_pv_dev, double** cIpu_dev,
                                               double** inter_pv_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "interpolate2_pre_vel_launcher_")) return;
  if (*nxIpu1 != NG || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "interpolate2_pre_vel_launcher_: expects 6 coefficients per row, dimension_id 1..3");
    return;
  }
  (void)nyIpu1;
  launch_interp_pre_vel<double>(*dimension_id, g, *cIpu_dev, *phi_inter_pv_dev, *inter_pv_dev, g_stream);
  check_launch("interpolate2_pre_vel_launcher_");
}

extern "C" void interpolate2_vel_pre_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIup1,
                                               int* nyIup1, double** phi_inter_vp_dev, double** cIup_dev,
                                               double** inter_vp_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "interpolate2_vel_pre_launcher_")) return;
  if (*nxIup1 != ND || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "interpolate2_vel_pre_launcher_: expects 6 coefficients per row, dimension_id 1..3");
    return;
  }
  (void)nyIup1;
  launch_interp_vel_pre<double>(*dimension_id, g, *cIup_dev, *phi_inter_vp_dev, *inter_vp_dev, g_stream);
  check_launch("interpolate2_vel_pre_launcher_");
}

extern "C" void axpby_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, double* a, double* b, double** d_x, double** d_y,
                                double** d_z) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "axpby_launcher_")) return;
  launch_axpby<double>(g, *a, *b, *d_x, *d_y, *d_z, g_stream);
  check_launch("axpby_launcher_");
}

extern "C" void jor_launcher_(int* grid_id, int* nx_dev, int* ny_dev, int* nz_dev, int* ny_cdg1, int* ny_cdg2,
                              int* ny_cdg3, int* nx_cdg1, double* omega, double** cdg1_dev, double** cdg2_dev,
                              double** cdg3_dev, double** rel_dev, double** bb_dev, double** rear_ghost_dev,
                              double** front_ghost_dev, double** upper_ghost_dev, double** lower_ghost_dev,
                              double** west_ghost_dev, double** east_ghost_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "jor_launcher_")) return;
  if (*nx_cdg1 != 3 || *grid_id < 1) {
    impact_set_error_msg(-1, "jor_launcher_: expects cdg(-1:1,...) tables and grid_id >= 1");
    return;
  }
  double* out = static_cast<double*>(scratch((size_t)g.nfield * sizeof(double), g_stream));
  if (!out) return;
  launch_jor_faces(g, *ny_cdg1, *ny_cdg2, *ny_cdg3, *grid_id, *omega, *cdg1_dev, *cdg2_dev, *cdg3_dev, *rel_dev,
                   *bb_dev, *rear_ghost_dev, *front_ghost_dev, *upper_ghost_dev, *lower_ghost_dev, *west_ghost_dev,
                   *east_ghost_dev, out, g_stream);
  launch_copy_interior(g, out, *rel_dev, g_stream);
  check_launch("jor_launcher_");
}

extern "C" void get_ghost_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, double** rel_dev, double** rear_ghost_dev,
                                    double** front_ghost_dev, double** upper_ghost_dev, double** lower_ghost_dev,
                                    double** west_ghost_dev, double** east_ghost_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "get_ghost_launcher_")) return;
  launch_get_ghost(g, *rel_dev, *rear_ghost_dev, *front_ghost_dev, *upper_ghost_dev, *lower_ghost_dev,
                   *west_ghost_dev, *east_ghost_dev, g_stream);
  check_launch("get_ghost_launcher_");
}

// Plane of the inlet / first-outlet condition: 0 (default) Fortran index k == k_start_index - 1, the
// test of apply_pressure_BC_CT (usr_func.f90:857-897); 1 the plane of the reference GPU kernel,
// whose C-index test (k+4) == k_start_index - 1 (set_pressure_BC_kernel.cu:26) selects Fortran
// index k_start_index - 4.
static std::atomic<int> g_pbc_plane{0};
extern "C" int impact_b200_set_pressure_bc_plane(int mode) {
  if (mode != 0 && mode != 1)
    return impact_set_error_msg(-1, "impact_b200_set_pressure_bc_plane: mode 0 (CPU routine) or 1 (reference GPU kernel)");
  g_pbc_plane.store(mode);
  return 0;
}
extern "C" int impact_b200_pressure_bc_plane(void) { return g_pbc_plane.load(); }
// k_start_index as the kernels take it (they test Fortran index k == ks - 1)
static int pbc_ks(int k_start_index) { return g_pbc_plane.load() == 1 ? k_start_index - 3 : k_start_index; }

extern "C" void pressure_bc_launcher_(int* type_id1, int* type_id2, int* type_id3, int* k_start_index, int* nx_dev,
                                      int* ny_dev, int* nz_dev, double* pre_inlet, double* pre_outlet,
                                      double* pre_outlet_2, double** ct_geometry_dev, double** rel_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "pressure_bc_launcher_")) return;
  launch_pressure_bc_f64label(g, *type_id1, *type_id2, *type_id3, pbc_ks(*k_start_index), *pre_inlet, *pre_outlet,
                              *pre_outlet_2, *ct_geometry_dev, *rel_dev, g_stream);
  check_launch("pressure_bc_launcher_");
}

static bool cdg_level(int grid_id, int nx_cdg, const char* who) {
  if (nx_cdg != 3 || grid_id < 1) {
    impact_set_error_msg(-1, (std::string(who) + ": expects cdg(-1:1,...) tables and grid_id >= 1").c_str());
    return false;
  }
  return true;
}

extern "C" void jacobi_launcher_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g,
                                 int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g, double* omega_g, double** cdg1_dev3,
                                 double** cdg2_dev3, double** cdg3_dev3, double** rel_dev3, double** bb_dev3,
                                 double** comp_dev3) {
  Geom g;
  if (!geom_from_dev(*nx_dev_g, *ny_dev_g, *nz_dev_g, &g, "jacobi_launcher_")) return;
  if (!cdg_level(*grid_id, *nx_cdg1_g, "jacobi_launcher_")) return;
  const long long lv = *grid_id - 1;
  launch_jacobi<double>(g, *cdg1_dev3 + lv * *ny_cdg1_g * 3, *cdg2_dev3 + lv * *ny_cdg2_g * 3,
                        *cdg3_dev3 + lv * *ny_cdg3_g * 3, *omega_g, *bb_dev3, *rel_dev3, *comp_dev3, g_stream);
  check_launch("jacobi_launcher_");
}

extern "C" void product_dg_relax_launcher_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g,
                                           int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g, double** cdg1_dev2,
                                           double** cdg2_dev2, double** cdg3_dev2, double** rel_dev2,
                                           double** comp_dev2) {
  Geom g;
  if (!geom_from_dev(*nx_dev_g, *ny_dev_g, *nz_dev_g, &g, "product_dg_relax_launcher_")) return;
  if (!cdg_level(*grid_id, *nx_cdg1_g, "product_dg_relax_launcher_")) return;
  const long long lv = *grid_id - 1;
  launch_dg_relax<double>(g, *cdg1_dev2 + lv * *ny_cdg1_g * 3, *cdg2_dev2 + lv * *ny_cdg2_g * 3,
                          *cdg3_dev2 + lv * *ny_cdg3_g * 3, *rel_dev2, *comp_dev2, g_stream);
  check_launch("product_dg_relax_launcher_");
}

// ---------------------------------------------------------------------------------------
// Part 1b: FP32 launchers.  The reference's FP32 prior art (jor_kernel_v2_sp.cu,
// jacobi_solver_host_v3_sp.f90:25-56) casts the fields and tables to real*4 and launches a
// kernel named with the suffix _sp; these are the operator launchers above with that suffix:
// same arguments, every array (fields and coefficient tables) and scalar in FP32, FP32
// arithmetic and accumulation.
// ---------------------------------------------------------------------------------------
extern "C" void gradient_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_grad_coef,
                                      int* ny_grad_coef, float** phi_grad_dev, float** cGp_dev, float** grad_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "gradient_launcher_sp_")) return;
  if (*nx_grad_coef != NG || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "gradient_launcher_sp_: expects 6 coefficients per row and dimension_id 1..3");
    return;
  }
  (void)ny_grad_coef;
  launch_gradient<float>(*dimension_id, g, *cGp_dev, *phi_grad_dev, *grad_dev, g_stream);
  check_launch("gradient_launcher_sp_");
}

extern "C" void divergence_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef,
                                        int* ny_div_coef, float** phi_div_dev, float** div_dev, float** cD_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "divergence_launcher_sp_")) return;
  if (*nx_div_coef != ND || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "divergence_launcher_sp_: expects 6 coefficients per row and dimension_id 1..3");
    return;
  }
  (void)ny_div_coef;
  launch_divergence<float>(*dimension_id, g, *cD_dev, *phi_div_dev, *div_dev, g_stream);
  check_launch("divergence_launcher_sp_");
}

extern "C" void divergence2_launcher_sp_(int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef1, int* nx_div_coef2,
                                         int* nx_div_coef3, float** phi_div2_dev, float** div2_dev, float** cDu1_dev,
                                         float** cDv2_dev, float** cDw3_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "divergence2_launcher_sp_")) return;
  if (*nx_div_coef1 != ND || *nx_div_coef2 != ND || *nx_div_coef3 != ND) {
    impact_set_error_msg(-1, "divergence2_launcher_sp_: expects 6 coefficients per row");
    return;
  }
  const float* u = *phi_div2_dev;
  launch_divergence2<float>(g, *cDu1_dev, *cDv2_dev, *cDw3_dev, u, u + g.nfield, u + 2 * g.nfield, *div2_dev,
                            g_stream);
  check_launch("divergence2_launcher_sp_");
}

extern "C" void helmholtz_explicit_launcher_sp_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxs1,
                                                int* nxs2, int* nxs3, float* multL, float** vel1_dev, float** helm_dev,
                                                float** cS1_helm_dev, float** cS2_helm_dev, float** cS3_helm_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "helmholtz_explicit_launcher_sp_")) return;
  if (*nxs1 != NB || *nxs2 != NB || *nxs3 != NB) {
    impact_set_error_msg(-1, "helmholtz_explicit_launcher_sp_: expects 7 coefficients per row");
    return;
  }
  launch_helmholtz<float>(*component_id, g, *cS1_helm_dev, *cS2_helm_dev, *cS3_helm_dev, *multL, *vel1_dev, *helm_dev,
                          g_stream);
  check_launch("helmholtz_explicit_launcher_sp_");
}

extern "C" void nonlinear_upwind_launcher_sp_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxn1,
                                              int* nyn1, float** pp_dev, float** vel_dev, float** nl_dev,
                                              float** cN1_dev, float** cN21_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "nonlinear_upwind_launcher_sp_")) return;
  if (*nxn1 != NB || *component_id < 1 || *component_id > 9) {
    impact_set_error_msg(-1, "nonlinear_upwind_launcher_sp_: expects 7 coefficients per row and component_id 1..9");
    return;
  }
  (void)nyn1;
  launch_nonlinear_upwind<float>(*component_id, g, *cN1_dev, *cN21_dev, *pp_dev, *vel_dev, *nl_dev, g_stream);
  check_launch("nonlinear_upwind_launcher_sp_");
}

extern "C" void interpolate2_pre_vel_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev,
                                                  int* nxIpu1, int* nyIpu1, float** phi_inter_pv_dev, float** cIpu_dev,
                                                  float** inter_pv_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "interpolate2_pre_vel_launcher_sp_")) return;
  if (*nxIpu1 != NG || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "interpolate2_pre_vel_launcher_sp_: expects 6 coefficients per row, dimension_id 1..3");
    return;
  }
  (void)nyIpu1;
  launch_interp_pre_vel<float>(*dimension_id, g, *cIpu_dev, *phi_inter_pv_dev, *inter_pv_dev, g_stream);
  check_launch("interpolate2_pre_vel_launcher_sp_");
}

extern "C" void interpolate2_vel_pre_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev,
                                                  int* nxIup1, int* nyIup1, float** phi_inter_vp_dev, float** cIup_dev,
                                                  float** inter_vp_dev) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "interpolate2_vel_pre_launcher_sp_")) return;
  if (*nxIup1 != ND || *dimension_id < 1 || *dimension_id > 3) {
    impact_set_error_msg(-1, "interpolate2_vel_pre_launcher_sp_: expects 6 coefficients per row, dimension_id 1..3");
    return;
  }
  (void)nyIup1;
  launch_interp_vel_pre<float>(*dimension_id, g, *cIup_dev, *phi_inter_vp_dev, *inter_vp_dev, g_stream);
  check_launch("interpolate2_vel_pre_launcher_sp_");
}

extern "C" void axpby_launcher_sp_(int* nx_dev, int* ny_dev, int* nz_dev, float* a, float* b, float** d_x, float** d_y,
                                   float** d_z) {
  Geom g;
  if (!geom_from_dev(*nx_dev, *ny_dev, *nz_dev, &g, "axpby_launcher_sp_")) return;
  launch_axpby<float>(g, *a, *b, *d_x, *d_y, *d_z, g_stream);
  check_launch("axpby_launcher_sp_");
}

extern "C" void jacobi_launcher_sp_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g,
                                    int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g, float* omega_g, float** cdg1_dev3,
                                    float** cdg2_dev3, float** cdg3_dev3, float** rel_dev3, float** bb_dev3,
                                    float** comp_dev3) {
  Geom g;
  if (!geom_from_dev(*nx_dev_g, *ny_dev_g, *nz_dev_g, &g, "jacobi_launcher_sp_")) return;
  if (!cdg_level(*grid_id, *nx_cdg1_g, "jacobi_launcher_sp_")) return;
  const long long lv = *grid_id - 1;
  launch_jacobi<float>(g, *cdg1_dev3 + lv * *ny_cdg1_g * 3, *cdg2_dev3 + lv * *ny_cdg2_g * 3,
                       *cdg3_dev3 + lv * *ny_cdg3_g * 3, *omega_g, *bb_dev3, *rel_dev3, *comp_dev3, g_stream);
  check_launch("jacobi_launcher_sp_");
}

extern "C" void product_dg_relax_launcher_sp_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g,
                                              int* ny_cdg1_g, int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g,
                                              float** cdg1_dev2, float** cdg2_dev2, float** cdg3_dev2,
                                              float** rel_dev2, float** comp_dev2) {
  Geom g;
  if (!geom_from_dev(*nx_dev_g, *ny_dev_g, *nz_dev_g, &g, "product_dg_relax_launcher_sp_")) return;
  if (!cdg_level(*grid_id, *nx_cdg1_g, "product_dg_relax_launcher_sp_")) return;
  const long long lv = *grid_id - 1;
  launch_dg_relax<float>(g, *cdg1_dev2 + lv * *ny_cdg1_g * 3, *cdg2_dev2 + lv * *ny_cdg2_g * 3,
                         *cdg3_dev2 + lv * *ny_cdg3_g * 3, *rel_dev2, *comp_dev2, g_stream);
  check_launch("product_dg_relax_launcher_sp_");
}

// ---------------------------------------------------------------------------------------
// Part 2: device_jacobi_solver replacement (jacobi_solver_host_v4.f90:5-717)
// ---------------------------------------------------------------------------------------
namespace {
constexpr int BX = 32, BY = 8;
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// residual inf-norm of bb - cdg(rel) and sum |rel - rel_old|; rel_old <- rel
__global__ void __launch_bounds__(BX* BY) k_jor_check(Geom g, const double* __restrict__ c1, const double* __restrict__ c2,
                                                      const double* __restrict__ c3, const double* __restrict__ rel,
                                                      const double* __restrict__ bb, double* __restrict__ rel_old,
                                                      double* __restrict__ partial) {
  const int i = blockIdx.x * BX + threadIdx.x + 1, j = blockIdx.y * BY + threadIdx.y + 1, k = blockIdx.z + 1;
  double rmax = 0.0, dsum = 0.0;
  if (i <= g.n1 && j <= g.n2) {
    const long long p = off(g, i, j, k);
    const double* a = c1 + 3 * (i - 1);
    const double* b = c2 + 3 * (j - 1);
    const double* c = c3 + 3 * (k - 1);
    const double r = bb[p] - a[0] * rel[off(g, wrapi(i - 1, g.n1), j, k)] - a[2] * rel[off(g, wrapi(i + 1, g.n1), j, k)] -
                     b[0] * rel[off(g, i, wrapi(j - 1, g.n2), k)] - b[2] * rel[off(g, i, wrapi(j + 1, g.n2), k)] -
                     c[0] * rel[off(g, i, j, wrapi(k - 1, g.n3))] - c[2] * rel[off(g, i, j, wrapi(k + 1, g.n3))] -
                     (a[1] + b[1] + c[1]) * rel[p];
    rmax = fabs(r);
    dsum = fabs(rel[p] - rel_old[p]);
    rel_old[p] = rel[p];
  }
  __shared__ double sh[2][8];
  const int tid = threadIdx.x + BX * threadIdx.y;
  rmax = wmax(rmax);
  dsum = wsum(dsum);
  if ((tid & 31) == 0) {
    sh[0][tid >> 5] = rmax;
    sh[1][tid >> 5] = dsum;
  }
  __syncthreads();
  if (tid < 32) {
    double x = tid < 8 ? sh[0][tid] : 0.0, y = tid < 8 ? sh[1][tid] : 0.0;
    x = wmax(x);
    y = wsum(y);
    if (tid == 0) {
      const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
      partial[2 * bid] = x;
      partial[2 * bid + 1] = y;
    }
  }
}
__global__ void __launch_bounds__(1024) k_jor_check_fin(const double* __restrict__ partial, long long nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[2][32];
  double x = 0.0, y = 0.0;
  for (long long b = threadIdx.x; b < nb; b += blockDim.x) {
    x = fmax(x, partial[2 * b]);
    y += partial[2 * b + 1];
  }
  x = wmax(x);
  y = wsum(y);
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = x;
    sh[1][threadIdx.x >> 5] = y;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    x = wmax(sh[0][threadIdx.x]);
    y = wsum(sh[1][threadIdx.x]);
    if (threadIdx.x == 0) {
      out[0] = x;
      out[1] = y;
    }
  }
}
}  // namespace

namespace {
// Labels and values of the CT pressure boundary condition applied inside the JOR loop.
struct JorBc {
  const uint8_t* labels;  // host, padded layout; nullptr: none
  int k_start_index, t1, t2, t3;
  double p_in, p_out, p_out2;
};

int jacobi_solve_impl(int N1, int N2, int N3, int M1, int M2, int M3, double omega, const double* cdg1,
                      const double* cdg2, const double* cdg3, double* rel, const double* bb, int mode_j,
                      double tol_abs_inf, int max_sweeps, int* sweeps, double* res_inf, const JorBc& bc) {
  const Geom g = make_geom(N1, N2, N3);
  const size_t fb = (size_t)g.nfield * sizeof(double);
  const dim3 gr((g.n1 + BX - 1) / BX, (g.n2 + BY - 1) / BY, g.n3), bl(BX, BY);
  const long long nb = (long long)gr.x * gr.y * gr.z;
  cudaStream_t s = g_stream;
  int rc = 0;
  auto fail = [&](cudaError_t e, const char* w) {
    rc = impact_set_error(e, w, __FILE__, __LINE__);
  };
  // workspace: four fields, the cdg tables, the check partials and the labels, carved from the
  // stream's library scratch (allocated once, regrown only for a larger grid)
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_c = up(3 * sizeof(double) * (N1 + N2 + N3)), b_part = up((2 * nb + 8) * sizeof(double));
  const size_t b_lab = bc.labels ? up((size_t)g.nfield) : 0;
  unsigned char* ws = static_cast<unsigned char*>(scratch(4 * up(fb) + b_c + b_part + b_lab, s));
  if (!ws) return -1;
  double* d_rel = reinterpret_cast<double*>(ws);
  double* d_tmp = reinterpret_cast<double*>(ws + up(fb));
  double* d_bb = reinterpret_cast<double*>(ws + 2 * up(fb));
  double* d_old = reinterpret_cast<double*>(ws + 3 * up(fb));
  double* d_c = reinterpret_cast<double*>(ws + 4 * up(fb));
  double* d_part = reinterpret_cast<double*>(ws + 4 * up(fb) + b_c);
  uint8_t* d_lab = bc.labels ? ws + 4 * up(fb) + b_c + b_part : nullptr;
  cudaError_t e = cudaSuccess;
  const double pi_ref = 3.1415;  // the constant of the reference's stop test (jacobi_solver_host_v4.f90:383)
  const double thresh =
      20. * mode_j * 8. * 1. / 3.0 * 0.8 * pi_ref * pi_ref * (1. / ((double)M1 * M1) + 1. / ((double)M2 * M2) + 1. / ((double)M3 * M3));
  int done_sweeps = 0;
  double last_res = 0.0;
  if (!rc) {
    cudaMemcpyAsync(d_rel, rel, fb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_tmp, rel, fb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_bb, bb, fb, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_old, 0, fb, s);
    cudaMemcpyAsync(d_c, cdg1, 3 * sizeof(double) * N1, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_c + 3 * N1, cdg2, 3 * sizeof(double) * N2, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_c + 3 * (N1 + N2), cdg3, 3 * sizeof(double) * N3, cudaMemcpyHostToDevice, s);
    if (d_lab) cudaMemcpyAsync(d_lab, bc.labels, (size_t)g.nfield, cudaMemcpyHostToDevice, s);
    const double* c1 = d_c;
    const double* c2 = d_c + 3 * N1;
    const double* c3 = d_c + 3 * (N1 + N2);
    double err_old = 0.0;
    bool have_old = false;
    double h[2];
    for (int iter = 1; iter <= max_sweeps; ++iter) {
      // the boundary values first, before the stop test and the sweep of this iteration
      if (d_lab)
        launch_pressure_bc(g, bc.t1, bc.t2, bc.t3, pbc_ks(bc.k_start_index), bc.p_in, bc.p_out, bc.p_out2, d_lab, d_rel, s);
      if (iter % mode_j == 1 || mode_j == 1) {
        k_jor_check<<<gr, bl, 0, s>>>(g, c1, c2, c3, d_rel, d_bb, d_old, d_part);
        k_jor_check_fin<<<1, 1024, 0, s>>>(d_part, nb, d_part + 2 * nb);
        e = cudaMemcpyAsync(h, d_part + 2 * nb, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
          fail(e, "impact_b200_jacobi_solve check");
          break;
        }
        last_res = h[0];
        if (tol_abs_inf > 0.0 && h[0] < tol_abs_inf) break;
        if (have_old && h[1] > 0.0 && err_old > 0.0) {
          const double rel_err = std::fabs(std::log(err_old / h[1]));
          if (rel_err <= thresh) break;
        }
        err_old = h[1];
        have_old = true;
      }
      launch_jacobi<double>(g, c1, c2, c3, omega, d_bb, d_rel, d_tmp, s);
      std::swap(d_rel, d_tmp);
      done_sweeps = iter;
    }
    if (!rc) {
      e = cudaMemcpyAsync(rel, d_rel, fb, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) fail(e, "impact_b200_jacobi_solve result");
    }
  }
  if (sweeps) *sweeps = done_sweeps;
  if (res_inf) *res_inf = last_res;
  return rc;
}
}  // namespace

extern "C" int impact_b200_jacobi_solve(int N1, int N2, int N3, int M1, int M2, int M3, double omega,
                                        const double* cdg1, const double* cdg2, const double* cdg3, double* rel,
                                        const double* bb, int mode_j, double tol_abs_inf, int max_sweeps, int* sweeps,
                                        double* res_inf) {
  if (N1 < 9 || N2 < 9 || N3 < 9 || !cdg1 || !cdg2 || !cdg3 || !rel || !bb || mode_j < 1 || max_sweeps < 1)
    return impact_set_error_msg(-1, "impact_b200_jacobi_solve: bad arguments");
  const JorBc none{nullptr, 0, 0, 0, 0, 0.0, 0.0, 0.0};
  return jacobi_solve_impl(N1, N2, N3, M1, M2, M3, omega, cdg1, cdg2, cdg3, rel, bb, mode_j, tol_abs_inf, max_sweeps,
                           sweeps, res_inf, none);
}

extern "C" int impact_b200_jacobi_solve_bc(int N1, int N2, int N3, int M1, int M2, int M3, double omega,
                                           const double* cdg1, const double* cdg2, const double* cdg3, double* rel,
                                           const double* bb, int mode_j, double tol_abs_inf, int max_sweeps,
                                           int* sweeps, double* res_inf, const uint8_t* labels, int k_start_index,
                                           int type_id1, int type_id2, int type_id3, double p_inlet,
                                           double p_outlet, double p_outlet_2) {
  if (N1 < 9 || N2 < 9 || N3 < 9 || !cdg1 || !cdg2 || !cdg3 || !rel || !bb || mode_j < 1 || max_sweeps < 1 ||
      !labels)
    return impact_set_error_msg(-1, "impact_b200_jacobi_solve_bc: bad arguments");
  const JorBc bc{labels, k_start_index, type_id1, type_id2, type_id3, p_inlet, p_outlet, p_outlet_2};
  return jacobi_solve_impl(N1, N2, N3, M1, M2, M3, omega, cdg1, cdg2, cdg3, rel, bb, mode_j, tol_abs_inf, max_sweeps,
                           sweeps, res_inf, bc);
}

extern "C" int impact_b200_product_scalar(int N1, int N2, int N3, const double* a_dev, const double* b_dev,
                                          double* result) {
  if (N1 < 9 || N2 < 9 || N3 < 9 || !a_dev || !b_dev || !result)
    return impact_set_error_msg(-1, "impact_b200_product_scalar: bad arguments");
  const Geom g = make_geom(N1, N2, N3);
  const long long nd = reduce_partial_doubles(g, 1);
  double* part = static_cast<double*>(scratch((size_t)(nd + 8) * sizeof(double), g_stream));
  if (!part) return -1;
  double* out = part + nd;
  reduce_dot<double>(g, a_dev, b_dev, part, out, g_stream);
  cudaError_t e = cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, g_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) return impact_set_error(e, "impact_b200_product_scalar", __FILE__, __LINE__);
  return 0;
}
