/*
 * impact_b200.h -- C ABI of the B200 (sm_100a) implementation of IMPACT's fractional-step
 * hot path (GPU-IMPACT-CT).  Plain pointers and sizes only; no C++ or torch types.
 *
 * Part 1 -- the reference's own FFI.  IMPACT's Fortran wrappers (src/*_host.f90) bind the
 * trailing-underscore launchers of src/*_launcher.cu through gfortran's implicit interface:
 * every argument by reference, device arrays as double** (the Fortran c_ptr variables of
 * mod_vars_GPU.f90).  This library exports the same symbols with the same arguments, so the
 * unchanged *_host.f90 files link against it instead of the reference's .cu objects.  Arrays
 * use the reference layout: column-major phi(-3:N1+3,-3:N2+3,-3:N3+3), nx_dev = N1+7;
 * coefficient tables c(lo:hi,0:N) as c[i*nx_coef + (l-lo)]; cdg(-1:1,1:N,1:n_grids).
 * Boundaries are periodic in all directions (the only case the reference kernels cover).
 * The launchers run asynchronously on the library's current stream (impact_b200_set_stream,
 * default: the legacy default stream, as the reference) and report errors through
 * impact_b200_last_error(); like the reference launchers they return nothing.  jor_launcher_,
 * impact_b200_product_scalar and impact_b200_jacobi_solve(_bc) use a library scratch buffer of
 * the calling (device, stream) pair, allocated on first use and regrown for a larger grid: calls
 * on different streams never share scratch; calls on one stream from several host threads at
 * once are not supported.
 *
 * Part 2 -- device-resident entry points that replace whole Fortran loops (the GPU
 * Poisson solve of jacobi_solver_host_v4.f90, BiCGstab_orig, one RK3 time step), so that
 * fields stay in HBM between calls instead of crossing PCIe on every operator call.
 *
 * All functions returning int return 0 on success and a negative code on error; the
 * message is available from impact_b200_last_error().
 */
#ifndef IMPACT_B200_H
#define IMPACT_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ========================================================================================
 * Part 1: reference launcher ABI
 * ====================================================================================== */

/* gradient_kernel_launcher.cu:12 -- grad = G_m phi (pressure -> velocity point m) */
void gradient_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_grad_coef,
                        int* ny_grad_coef, double** phi_grad_dev, double** cGp_dev, double** grad_dev);
/* divergence_kernel_launcher.cu:12 -- div (=, m=1 / +=, m=2,3) D_m phi */
void divergence_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef,
                          int* ny_div_coef, double** phi_div_dev, double** div_dev, double** cD_dev);
/* divergence2_kernel_launcher.cu:12 -- div = D1 u + D2 v + D3 w, phi = vel(:,:,:,1:3) packed */
void divergence2_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef1, int* nx_div_coef2,
                           int* nx_div_coef3, double** phi_div2_dev, double** div2_dev, double** cDu1_dev,
                           double** cDv2_dev, double** cDw3_dev);
/* helmholtz_explicit_kernel_launcher.cu:12 -- helm -= multL (cS1 u_xx + cS2 u_yy + cS3 u_zz) */
void helmholtz_explicit_launcher_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxs1, int* nxs2,
                                  int* nxs3, double* multL, double** vel1_dev, double** helm_dev,
                                  double** cS1_helm_dev, double** cS2_helm_dev, double** cS3_helm_dev);
/* Nonlinear_upwind_kernel_launcher.cu:12 -- nl (=/+=) pp * D^{up|down}_a vel, component_id = 3(m-1)+a;
 * cN1 holds the table used where pp >= 0, cN21 the one used where pp < 0 */
void nonlinear_upwind_launcher_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxn1, int* nyn1,
                                double** pp_dev, double** vel_dev, double** nl_dev, double** cN1_dev,
                                double** cN21_dev);
/* interpolate2_pre_vel_kernel_launcher.cu:12 -- pressure -> velocity point m */
void interpolate2_pre_vel_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIpu1,
                                    int* nyIpu1, double** phi_inter_pv_dev, double** cIpu_dev,
                                    double** inter_pv_dev);
/* interpolate2_vel_pre_kernel_launcher.cu:12 -- velocity point m -> pressure */
void interpolate2_vel_pre_launcher_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIup1,
                                    int* nyIup1, double** phi_inter_vp_dev, double** cIup_dev,
                                    double** inter_vp_dev);
/* axpby_kernel_launcher.cu:12 -- z = a x + b y */
void axpby_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, double* a, double* b, double** d_x, double** d_y,
                     double** d_z);
/* jor_kernel_launcher.cu:12 -- one JOR sweep of the compact Laplacian cdg, boundary neighbours
 * taken from the six ghost-face arrays.  The reference updates rel in place (a data race between
 * neighbouring threads); this implementation is deterministic: it sweeps out of place into a
 * library-owned buffer and copies the result back into rel. */
void jor_launcher_(int* grid_id, int* nx_dev, int* ny_dev, int* nz_dev, int* ny_cdg1, int* ny_cdg2, int* ny_cdg3,
                   int* nx_cdg1, double* omega, double** cdg1_dev, double** cdg2_dev, double** cdg3_dev,
                   double** rel_dev, double** bb_dev, double** rear_ghost_dev, double** front_ghost_dev,
                   double** upper_ghost_dev, double** lower_ghost_dev, double** west_ghost_dev,
                   double** east_ghost_dev);
/* get_ghost_launcher.cu:12 -- copy the six boundary planes of rel into the face arrays */
void get_ghost_launcher_(int* nx_dev, int* ny_dev, int* nz_dev, double** rel_dev, double** rear_ghost_dev,
                         double** front_ghost_dev, double** upper_ghost_dev, double** lower_ghost_dev,
                         double** west_ghost_dev, double** east_ghost_dev);
/* set_pressure_BC_kernel_launcher.cu:12 -- Dirichlet pressure on labelled cells (labels as FP64,
 * the ct_geometry array of the reference).  By default planes are matched with the Fortran
 * index test k == k_start_index-1 of apply_pressure_BC_CT (usr_func.f90:857-897); see
 * impact_b200_set_pressure_bc_plane for the reference GPU kernel's plane. */
void pressure_bc_launcher_(int* type_id1, int* type_id2, int* type_id3, int* k_start_index, int* nx_dev,
                           int* ny_dev, int* nz_dev, double* pre_inlet, double* pre_outlet, double* pre_outlet_2,
                           double** ct_geometry_dev, double** rel_dev);
/* Plane of the inlet (label 5) and first-outlet (label 9) conditions of pressure_bc_launcher_ and
 * impact_b200_jacobi_solve_bc.  mode 0 (default): Fortran index k == k_start_index - 1, the test
 * of apply_pressure_BC_CT (usr_func.f90:857-897).  mode 1: the plane the reference GPU kernel
 * sets, whose C-index test (k+4) == k_start_index - 1 (set_pressure_BC_kernel.cu:26) selects
 * Fortran index k_start_index - 4, three planes below the CPU routine's.  Process-wide; returns
 * -1 for any other mode.  No counterpart in the reference (its two paths simply differ). */
int impact_b200_set_pressure_bc_plane(int mode);
int impact_b200_pressure_bc_plane(void);
/* jacobi_kernel_launcher.cu:12 -- comp = one damped-Jacobi sweep of rel (multigrid level grid_id) */
void jacobi_launcher_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g, int* ny_cdg2_g,
                      int* ny_cdg3_g, int* nx_cdg1_g, double* omega_g, double** cdg1_dev3, double** cdg2_dev3,
                      double** cdg3_dev3, double** rel_dev3, double** bb_dev3, double** comp_dev3);
/* product_dg_relax_kernel_launcher.cu:12 -- comp = cdg Laplacian of rel (level grid_id) */
void product_dg_relax_launcher_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g,
                                int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g, double** cdg1_dev2,
                                double** cdg2_dev2, double** cdg3_dev2, double** rel_dev2, double** comp_dev2);

/* ---- Part 1b: FP32 launchers ------------------------------------------------------------
 * The reference's FP32 prior art (jor_kernel_v2_sp.cu:5, jacobi_solver_host_v3_sp.f90:25-56)
 * casts the fields and tables to real*4 and launches kernels suffixed _sp.  These are the
 * operator launchers above with that suffix: the same arguments, every array (fields and
 * coefficient tables c(lo:hi,0:N)) and scalar in FP32, FP32 arithmetic and accumulation.  No
 * FP32 launcher of these operators exists in the reference; they replace the FP64 ones where a
 * caller stages its fields in real*4. */
void gradient_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_grad_coef,
                           int* ny_grad_coef, float** phi_grad_dev, float** cGp_dev, float** grad_dev);
void divergence_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef,
                             int* ny_div_coef, float** phi_div_dev, float** div_dev, float** cD_dev);
void divergence2_launcher_sp_(int* nx_dev, int* ny_dev, int* nz_dev, int* nx_div_coef1, int* nx_div_coef2,
                              int* nx_div_coef3, float** phi_div2_dev, float** div2_dev, float** cDu1_dev,
                              float** cDv2_dev, float** cDw3_dev);
void helmholtz_explicit_launcher_sp_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxs1, int* nxs2,
                                     int* nxs3, float* multL, float** vel1_dev, float** helm_dev,
                                     float** cS1_helm_dev, float** cS2_helm_dev, float** cS3_helm_dev);
void nonlinear_upwind_launcher_sp_(int* component_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxn1, int* nyn1,
                                   float** pp_dev, float** vel_dev, float** nl_dev, float** cN1_dev,
                                   float** cN21_dev);
void interpolate2_pre_vel_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIpu1,
                                       int* nyIpu1, float** phi_inter_pv_dev, float** cIpu_dev,
                                       float** inter_pv_dev);
void interpolate2_vel_pre_launcher_sp_(int* dimension_id, int* nx_dev, int* ny_dev, int* nz_dev, int* nxIup1,
                                       int* nyIup1, float** phi_inter_vp_dev, float** cIup_dev,
                                       float** inter_vp_dev);
void axpby_launcher_sp_(int* nx_dev, int* ny_dev, int* nz_dev, float* a, float* b, float** d_x, float** d_y,
                        float** d_z);
void jacobi_launcher_sp_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g, int* ny_cdg2_g,
                         int* ny_cdg3_g, int* nx_cdg1_g, float* omega_g, float** cdg1_dev3, float** cdg2_dev3,
                         float** cdg3_dev3, float** rel_dev3, float** bb_dev3, float** comp_dev3);
void product_dg_relax_launcher_sp_(int* grid_id, int* nx_dev_g, int* ny_dev_g, int* nz_dev_g, int* ny_cdg1_g,
                                   int* ny_cdg2_g, int* ny_cdg3_g, int* nx_cdg1_g, float** cdg1_dev2,
                                   float** cdg2_dev2, float** cdg3_dev2, float** rel_dev2, float** comp_dev2);

/* ========================================================================================
 * Part 2: library control and device-resident entry points
 * ====================================================================================== */

/* sticky message of the last error of the calling process ("" if none) */
const char* impact_b200_last_error(void);
void impact_b200_clear_error(void);
int impact_b200_version(void);
/* stream (a cudaStream_t) used by the Part 1 launchers; NULL = legacy default stream */
void impact_b200_set_stream(void* stream);
/* synchronise the launcher stream; returns the first pending CUDA error, if any */
int impact_b200_sync(void);

/* ---- grid set-up (mod_geometry.f90:37 / usr_geometry.f90:93; mod_coeffs.f90:37, 1048) ----
 * Coordinates of one periodic axis with M points: xp, xu over indices -3..M+3 (M+7 values).
 * kind 0 equidistant, 1 x(s) = L/2 (1 + sinh(2(s/(M-1) - 1/2)) / sinh 1). */
int impact_b200_axis_coords(int M, double L, int kind, double* xp, double* xu);

/* Every coefficient table of one periodic axis, FD_coeffs with mapping_yes = T.  Each pointer
 * is caller memory: 6*(M+1) doubles for cG, cD, cIpu, cIup; 7*(M+1) for cNpU, cNpD, cNuU,
 * cNuD, cp1, cpp, cuu; 3*M for cdg. */
typedef struct {
  double *cG, *cD, *cIpu, *cIup, *cNpU, *cNpD, *cNuU, *cNuD, *cp1, *cpp, *cuu, *cdg;
} impact_b200_axis_tables;
int impact_b200_axis_coeffs(int M, const double* xp, const double* xu, impact_b200_axis_tables* out);

/* Exact equidistant finite-difference weights (diff_coeffs_exact, mod_coeffs.f90:598-751). */
int impact_b200_fd_exact(int abl, int n, double deltaX0, double* cc);

/* ---- one simulation case resident on one GPU ----------------------------------------- */
typedef struct impact_b200_case impact_b200_case;

typedef struct {
  int N1, N2, N3;  /* IMPACT point counts; N-1 unique periodic points per axis */
  int precision;   /* 0: FP64 throughout (plain drop-in); 1: mixed (FP32 inner Poisson solve,
                      FP64 outer residual, correction, inner products and RHS operators) */
  int device;      /* CUDA device ordinal */
  void* stream;    /* cudaStream_t to run on; NULL: the case creates its own stream */
} impact_b200_case_desc;

typedef struct {
  const impact_b200_axis_tables* axis[3]; /* host tables of the three axes (copied to the GPU) */
  /* optional: the grid coordinates x1p/x1u.. over -3..N+3 and the box lengths; when given, the
   * case also builds the multigrid hierarchy of the pressure Poisson preconditioner */
  const double* xp[3];
  const double* xu[3];
  double L[3];
} impact_b200_coeffs;

/* field ids of impact_b200_case_upload/download/field_ptr */
enum {
  IMPACT_B200_VEL1 = 0, IMPACT_B200_VEL2 = 1, IMPACT_B200_VEL3 = 2, IMPACT_B200_PRE = 3,
  IMPACT_B200_NL1 = 4, IMPACT_B200_NL2 = 5, IMPACT_B200_NL3 = 6, IMPACT_B200_RES = 7,
  IMPACT_B200_RHS1 = 8, IMPACT_B200_RHS2 = 9, IMPACT_B200_RHS3 = 10, IMPACT_B200_NFIELDS = 11
};

int impact_b200_case_create(const impact_b200_case_desc* desc, const impact_b200_coeffs* coeffs,
                            impact_b200_case** out);
int impact_b200_case_destroy(impact_b200_case* c);
/* device bytes held by a case of this size and precision (admission control) */
long long impact_b200_case_bytes(int N1, int N2, int N3, int precision);
/* whole padded field (nx*ny*nz doubles, reference layout) host <-> device, on the case stream */
int impact_b200_case_upload(impact_b200_case* c, int field, const double* host);
int impact_b200_case_download(impact_b200_case* c, int field, double* host);
/* Elements [first, first + count) of the field (linear index of the padded layout; `host` is the
 * base of the whole host field) copied on `stream` (a cudaStream_t; NULL: the case stream), the
 * call returning at once: with pinned host memory the copies overlap other copies and kernels, and
 * ranges of one field let its download and the next upload pipeline against each other.  Ordering
 * against the case stream (its time steps) is the caller's, by events; the host range must stay
 * untouched until the copy has completed.  No counterpart in the reference (its wrappers copy
 * whole fields synchronously). */
int impact_b200_case_upload_async(impact_b200_case* c, int field, const double* host, size_t first, size_t count,
                                  void* stream);
int impact_b200_case_download_async(impact_b200_case* c, int field, double* host, size_t first, size_t count,
                                    void* stream);
/* Snapshot of resident fields (output and restart off the hot path, mod_inout.f90:78-500 without
 * HDF5): device copies of fields[0..nfields-1] are taken on the case stream at this point of its
 * work, then read back into host[q] (whole padded fields, pinned for overlap) on `stream` (NULL:
 * the case stream) while later steps run.  The call returns at once; the host buffers hold the
 * snapshot once `stream` has reached this point (synchronise it or an event recorded on it).  A
 * later snapshot of the case waits for the read-back of the previous one.  The copy buffer comes
 * from the case's memory pool on the first call (and grows to the largest field count asked for).
 * No counterpart in the reference (its output writes HDF5 from the host arrays). */
int impact_b200_case_snapshot(impact_b200_case* c, int nfields, const int* fields, double* const* host, void* stream);
/* wait until the case stream has finished its work */
int impact_b200_case_synchronize(impact_b200_case* c);
/* The next time step of the case waits for `event` (a cudaEvent_t the caller recorded, e.g. after
 * an asynchronous upload of the pressure) only where it first reads the pressure -- after the
 * explicit part of its first substep -- instead of before it starts, so that the pressure upload
 * overlaps that part of the step.  The event is consumed by that step and must stay valid until
 * the step call has returned.  No counterpart in the reference (its wrappers copy whole fields
 * synchronously). */
int impact_b200_case_defer_pressure(impact_b200_case* c, void* event);
/* Measured inflow waveform of the label-5 voxels (read_velocity_waveform / convert_waveform,
 * usr_func.f90:574-651, as apply_CT_forcing :923-945 uses it): n (time, velocity) pairs in
 * nondimensional units, times non-decreasing, the last one the pulse length.  At the end of every
 * step the time is shifted into the current pulse and the inflow voxels take the value at the
 * start of the last table interval that holds it (none does: they keep their velocity).  n = 0
 * restores the default inflow U0 (1 + sin(2 pi t / T_pulse) / 2). */
int impact_b200_case_set_inflow_waveform(impact_b200_case* c, int n, const double* time, const double* velocity);
/* Diffuse-interface immersed boundary (mod_ibm.f90).  n Lagrangian markers at positions yb, a
 * column-major (n, 3) array (all x, then all y, then all z: the reference's yb(1:M_bound, 1:3)),
 * in the units of the case's coordinates; skip[i] != 0 excludes marker i (its index is listed in
 * ebcs(:, 1)), skip = NULL excludes none.  delta_type 1..4 and reach are ddf_type and reach of
 * discrete_delta (mod_ibm.f90:2021-2075); a reach whose vicinity could span more than 16 points
 * of an axis is rejected.  The case must have been created with coordinates (xp, xu). */
int impact_b200_case_set_markers(impact_b200_case* c, int n, const double* yb, const uint8_t* skip, double reach,
                                 int delta_type);
/* interpolate_vel_to_ib (mod_ibm.f90:589-737): ub (host, column-major (n, 3)) = the velocity of
 * the resident fields at every marker, the sum of delta * u * cell volume over its vicinity on
 * each component's staggered grid; skipped markers get 0.  Returns when ub is written. */
int impact_b200_case_ibm_interpolate(impact_b200_case* c, double* ub);
/* spread_force_dens_to_vel_grid (mod_ibm.f90:428-583): the three fields field_first..+2
 * (IMPACT_B200_NL1 or IMPACT_B200_RHS1) are zeroed and receive the force density of the marker
 * forces fb (host, column-major (n, 3)) times the node volumes node_vol (host, n) spread with the
 * delta kernel.  The additions of overlapping supports are atomic, so the order of the sum at a
 * point is not fixed. */
int impact_b200_case_ibm_spread(impact_b200_case* c, const double* fb, const double* node_vol, int field_first);
/* voxel labels (padded layout, one byte per point): 0 solid, 1 fluid, 5 inflow, 7 wall, 9/11 outlets */
int impact_b200_case_set_labels(impact_b200_case* c, const uint8_t* host_labels);
double* impact_b200_case_field_ptr(impact_b200_case* c, int field);
void* impact_b200_case_stream(impact_b200_case* c);

typedef struct {
  double tol_rel;      /* ||b - A x||_2 <= tol_rel ||b||_2 (0 = off) */
  double tol_abs_inf;  /* ||b - A x||_inf < tol_abs_inf (0 = off; the reference's epsU) */
  int max_it;          /* BiCGstab iterations (outer refinements in mixed precision) */
  int n_sweeps;        /* damped-Jacobi sweeps per preconditioner application (0 = none) */
  double omega;        /* their relaxation factor (0.8 for the BiCGstab preconditioner) */
  int init_yes;        /* 1: start from x = 0 */
  int check_every;     /* iterations between host polls of the device convergence flag */
  double inner_tol_rel;/* mixed precision: relative tolerance of each FP32 inner solve */
  int inner_max_it;    /* mixed precision: iteration cap of each inner solve */
  int precond;         /* 0: n_sweeps damped-Jacobi sweeps; 1: multigrid V-cycle (multigridV,
                          mod_solvers.f90:456-585; needs the coordinates at case creation) */
  int mg_down, mg_up, mg_bottom; /* V-cycle sweeps (n_relax_down / _up / _bottom), relaxation omega */
  int tile_kc;         /* z-planes per tile of the solver kernels (0: library default); chosen by
                          the autotuner of the Python package, no counterpart in the reference */
  int smooth_unfused;  /* 0 (default): the sweeps of each V-cycle smoothing phase (and, before a
                          restriction, the residual after them) run as one z-marching kernel;
                          1: one sweep per launch.  Same results bit for bit; no counterpart in
                          the reference */
  int bottom_cheb;     /* 0 (default): the coarsest level of the V-cycle gets mg_bottom damped-Jacobi
                          sweeps, then mg_bottom more (relax_bottom, mod_solvers.f90:420-450);
                          d > 0: d steps of the Chebyshev semi-iteration of the Jacobi-scaled
                          coarsest operator from x = 0 instead (a fixed polynomial in A, so the
                          preconditioner stays linear), in the one-block coarse tail, on cases whose
                          coarsest level fits there.  For hierarchies that stop at a large coarsest
                          level (n = 8 x odd); no counterpart in the reference */
} impact_b200_solver_params;

typedef struct {
  int iterations;       /* BiCGstab iterations (mixed: outer refinements) */
  int inner_iterations; /* mixed precision: FP32 BiCGstab iterations summed over refinements */
  int status;           /* 0 converged, 1 iteration cap, 2 breakdown, 3 non-finite */
  double res_inf, res_two, b_two;
} impact_b200_solver_result;

/* Pressure Poisson solve A x = b on resident fields (BiCGstab_orig, mod_solvers.f90:1509-1935;
 * A = product_div_grad, preconditioner = Jacobi sweeps of the compact cdg Laplacian). */
int impact_b200_case_poisson(impact_b200_case* c, int field_b, int field_x, const impact_b200_solver_params* p,
                             impact_b200_solver_result* r);

/* Apply the preconditioner of p once: field_out = M field_in.  FP64 cases: the FP64
 * preconditioner; mixed-precision cases: the FP32 preconditioner of the inner solve (field_in
 * rounded to FP32, the result widened to FP64). */
int impact_b200_case_precond(impact_b200_case* c, int field_in, int field_out, const impact_b200_solver_params* p);
/* op 0: field_out = A field_in, product_div_grad (mod_laplace.f90:38-197), the operator of the
 * pressure Poisson solve; op 1: field_out = divergence2 of the resident velocity (mod_diff.f90:
 * 130-215; field_in unused).  FP64, on the resident fields.  op 2: op 0 in FP32 (field_in
 * rounded to FP32, the FP32 weights and kernel of the mixed solve's inner iteration, the result
 * widened to FP64). */
int impact_b200_case_apply(impact_b200_case* c, int op, int field_in, int field_out);
/* levels of the multigrid hierarchy of the case (0 when it has none) */
int impact_b200_case_mg_levels(impact_b200_case* c);

typedef struct {
  double Re, CFL, dtime_max, dtime0; /* get_dtime (mod_lib.f90:46-250), timeint_mode 1 */
  double U0, T_pulse;                /* inflow u_z = U0 (1 + 0.5 sin(2 pi t / T)) on label 5 */
  int level_pressure;                /* subtract the mean pressure after each step */
  impact_b200_solver_params poisson;
  /* mixed-precision cases only: 1 = rhs_vel (advection, Helmholtz, the RK update's nonlinear
   * terms) as the FP32 pass -- FP32 interpolated velocities, nonlinear term, coefficients and
   * accumulation, the velocity and rhs FP64; 0 (default) = the FP64 pass.  No counterpart in the
   * reference. */
  int explicit_fp32;
} impact_b200_step_params;

typedef struct {
  double time, dtime;
  int timestep;
  int poisson_iterations[3];
  int inner_iterations[3];
  double poisson_res_rel[3];
  int poisson_status[3];
} impact_b200_step_state;

/* nsteps RK3 time steps (mod_timeint.f90:242-578) on the resident fields. */
int impact_b200_case_step(impact_b200_case* c, const impact_b200_step_params* p, impact_b200_step_state* st,
                          int nsteps);

/* ---- batches (no counterpart in the reference) ------------------------------------------
 * A batch advances several cases of one device and one precision together, each with its own
 * grid size, parameters and time step: every kernel of the pressure solve is one launch over
 * the tiles of all cases (converged cases drop out on the device), and each chunk of solver
 * iterations is replayed as a captured CUDA graph.  The solver structure (preconditioner,
 * sweeps, omega, check_every) comes from p[0].poisson; tolerances and max_it from each p[c].
 * A case must not be stepped on its own while it belongs to a batch that is stepping. */
typedef struct impact_b200_batch impact_b200_batch;
int impact_b200_batch_create(impact_b200_case* const* cases, int ncases, impact_b200_batch** out);
int impact_b200_batch_destroy(impact_b200_batch* b);
/* nsteps RK3 steps of every case; p and st hold one entry per case, in creation order. */
int impact_b200_batch_step(impact_b200_batch* b, const impact_b200_step_params* p, impact_b200_step_state* st,
                           int nsteps);
int impact_b200_batch_size(impact_b200_batch* b);
void* impact_b200_batch_stream(impact_b200_batch* b);

/* ---- device_jacobi_solver (jacobi_solver_host_v4.f90:5) replacement -------------------
 * Host arrays rel (in/out) and bb in the reference layout.  Deterministic out-of-place JOR
 * sweeps of the compact Laplacian on the device, periodic neighbours read in place (no ghost
 * faces cross PCIe), stopping on the reference's heuristic relative-change test evaluated every
 * mode_j sweeps, or when ||bb - A rel||_inf < tol_abs_inf (if > 0), or after max_sweeps.
 * cdg1..3: host tables cdg(-1:1,1:N) of level 1.  Returns the sweeps done in *sweeps.  Runs on
 * the library's current stream; its device workspace (four fields, the tables, the labels) is the
 * stream's library scratch, so repeated solves allocate nothing after the first on a grid size. */
int impact_b200_jacobi_solve(int N1, int N2, int N3, int M1, int M2, int M3, double omega, const double* cdg1,
                             const double* cdg2, const double* cdg3, double* rel, const double* bb, int mode_j,
                             double tol_abs_inf, int max_sweeps, int* sweeps, double* res_inf);
/* The same solve in the third RK substep of a CT case (jacobi_solver_host_v4.f90:302-305): at the
 * start of every iteration, before its stop test and sweep, the CT pressure condition
 * (pressure_bc_launcher_) sets rel on the labelled points -- type_id1: label 5 on plane
 * k_start_index - 1 to p_inlet, type_id2: label 9 on that plane to p_outlet, type_id3: every
 * label 11 to p_outlet_2 (the reference passes 1, 1, 0 and values already multiplied by
 * (aRK + bRK) dt).  labels: host, one byte per point in the padded layout. */
int impact_b200_jacobi_solve_bc(int N1, int N2, int N3, int M1, int M2, int M3, double omega, const double* cdg1,
                                const double* cdg2, const double* cdg3, double* rel, const double* bb, int mode_j,
                                double tol_abs_inf, int max_sweeps, int* sweeps, double* res_inf,
                                const uint8_t* labels, int k_start_index, int type_id1, int type_id2, int type_id3,
                                double p_inlet, double p_outlet, double p_outlet_2);

/* Deterministic FP64 inner product over the unique periodic points (product_scalar,
 * mod_solvers.f90:2319-2354) of two device fields of a grid with N1 x N2 x N3 points.
 * The block partials live in a library scratch buffer, allocated on the first call from a
 * (device, stream) pair and regrown for larger grids; runs on the library's current stream
 * (impact_b200_set_stream) and returns once *result (host memory) is written. */
int impact_b200_product_scalar(int N1, int N2, int N3, const double* a_dev, const double* b_dev, double* result);

/* The same inner product for callers that cannot let the library allocate device memory: a
 * host code whose GPU memory is all claimed by its own allocator, or a loop that cannot pay for
 * cudaMalloc/cudaFree (they can synchronise the device).  No counterpart in the reference.  Its
 * scratch is a fixed 128 KiB array in device memory, held by every GPU that loads the library
 * until exit; grids with more than 16384 unique z-planes (N3 > 16385) are rejected.  The first
 * call on a device resolves the array's address (make it before any stream capture there); calls
 * whose kernels overlap on the GPU share the array and race, so serialise them.  Runs on the
 * library's current stream (impact_b200_set_stream), so it is ordered after the launchers queued
 * there; fields written on any other stream (a case stream, a caller's non-blocking stream) must
 * be complete before the call.  The sum runs per z-plane and then over the planes: deterministic,
 * and equal to impact_b200_product_scalar's result up to rounding, not bit for bit.  Returns
 * once *result (host memory) is written. */
int impact_b200_product_scalar_noalloc(int N1, int N2, int N3, const double* a_dev, const double* b_dev,
                                       double* result);

/* ---- measurement hooks -----------------------------------------------------------------
 * When enabled, the library records CUDA events on the launching stream around its hot kernels
 * and accumulates, per kernel kind kid (0 jacobi_sweep, 1 jacobi_init2, 2 div_grad_dot,
 * 3 x_update, 4 p_update, 5 r_update, 6 nl_rhs, 7 project, 8 divergence2, 9 mg_sweep,
 * 10 mg_init, 11 mg_residual, 12 mg_transfer, 13 mg_pre_smooth, 14 mg_post_smooth,
 * 15 mx_residual, 16 mx_apply, 17 mg_coarse_tail, 18 kr_init), the launches, the elapsed
 * milliseconds and the algorithmic bytes moved.  launch_count counts every kernel
 * launch the library has issued since load. */
void impact_b200_profile_enable(int enable);
void impact_b200_profile_reset(void);
int impact_b200_profile_read(int kid, long long* launches, double* total_ms, double* total_bytes, const char** name);
long long impact_b200_launch_count(void);
/* launch one hot kernel iters times on the case's resident fields (kid 0 Jacobi sweep, 1 fused
 * init + sweep, 2 A x with a fused inner product, 3 A x, 4 one-thread-per-point Jacobi sweep, in
 * the case's precision; FP64 passes of the time step: 10..12 rhs_vel of component 1..3 (reads
 * vel_m, work1..3, nl_m; writes nl_m, rhs_m; 1/Re = 2e-3, dt bRK = -0.01, dt aRK = 0.02), 13 interpolate_vel (vel -> work), 14 projection
 * (vel = rhs - G pre), 15 divergence2 of rhs into res); *ms_per_launch = average device time
 * (CUDA events on the case stream) */
int impact_b200_case_kernel_bench(impact_b200_case* c, int kid, int iters, double* ms_per_launch);
/* Measurement: iters launches of one kernel of the Poisson engine on the case's finest level, in
 * the solve precision (FP64, or FP32 for the inner solve of a mixed case), the engine built with
 * the solver parameters p.  kind: 0 sweep, 1 init sweep, 2 residual, 3 prolongation,
 * 4 restriction, 5 A x + inner product, 6 A x + two inner products, 7 x update, 8 p update,
 * 9 r update, 10 one V-cycle, 11 one BiCGstab iteration, 12 fused pre-smoothing (init sweep,
 * mg_down - 1 sweeps and the residual in one kernel), 13 fused post-smoothing (mg_up sweeps).
 * Returns the average ms per launch (CUDA events on the case stream) and the algorithmic bytes of
 * one launch (0 for 10, 11). */
int impact_b200_case_engine_bench(impact_b200_case* c, int kind, int iters, const impact_b200_solver_params* p,
                                  double* ms, double* bytes);

#ifdef __cplusplus
}
#endif
#endif
