/*
 * impact_oracle.h -- CPU FP64 oracle for the IMPACT fractional-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of IMPACT's CPU
 * routines (mod_diff.f90, mod_laplace.f90, mod_solvers.f90, mod_rhs.f90,
 * mod_coeffs.f90, mod_timeint.f90, usr_func.f90, mod_lib.f90).  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg may load
 * it, and only as the checker or the timed CPU baseline.  The CUDA product never
 * links or calls anything in this directory.
 *
 * Parity pins: the exact finite-difference weights are checked against the
 * reference's own table (mod_coeffs.f90:598-751, diff_coeffs_exact) through the
 * fixture tests/golden/fd_exact_table.json; the RK3 stability limits against the
 * reference's table (mod_vars.f90:785-795) through tests/golden/stability_limit.json;
 * and the operator restatements against the reference's own CUDA kernels (built
 * from the reference sources by oracle/build_ref.sh into oracle/_ref) on a GPU.
 *
 * Layout (mod_vars.f90:476-518, mod_mem_GPU.f90:27-31): every field is a
 * column-major FP64 array phi(-3:N1+3, -3:N2+3, -3:N3+3); Fortran index i maps to
 * C offset i+3, so nx = N1+7.  Only all-periodic boundaries are covered
 * (BC_*_global = -1, prog/config.txt:38-45): the unique points are 1..N-1 per axis.
 *
 * Coefficient tables c(lo:hi, 0:N) are stored as c[i*(hi-lo+1) + (l-lo)];
 * the compact Laplacian cdg(-1:1, 1:N) as cdg[(i-1)*3 + (l+1)].
 */
#ifndef IMPACT_ORACLE_H
#define IMPACT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Stencil widths of IMPACT (mod_vars.f90:157-214): b = -3..3, d = -3..2, g = -2..3. */
#define ORC_B_LO (-3)
#define ORC_B_HI 3
#define ORC_D_LO (-3)
#define ORC_D_HI 2
#define ORC_G_LO (-2)
#define ORC_G_HI 3
#define ORC_NB 7 /* b/n tables: 7 coefficients per row */
#define ORC_ND 6 /* d tables: 6 */
#define ORC_NG 6 /* g tables: 6 */

/* All coefficient tables of one grid, one pointer per axis (a = 0,1,2 for x,y,z). */
typedef struct {
  const double* cG[3];   /* cGp1,cGp2,cGp3   g-range, rows 0..N   (pressure -> velocity derivative) */
  const double* cD[3];   /* cDu1,cDv2,cDw3   d-range, rows 0..N   (velocity -> pressure derivative) */
  const double* cIpu[3]; /* cIpu,cIpv,cIpw   g-range              (pressure -> velocity interpolation) */
  const double* cIup[3]; /* cIup,cIvp,cIwp   d-range              (velocity -> pressure interpolation) */
  const double* cNpU[3]; /* cNp1U..cNp3U     b-range, pressure grid upwind (used where pp >= 0) */
  const double* cNpD[3]; /* cNp1D..cNp3D     b-range, pressure grid downwind (pp < 0) */
  const double* cNuU[3]; /* cNu1U,cNv2U,cNw3U b-range, velocity grid upwind */
  const double* cNuD[3]; /* cNu1D,cNv2D,cNw3D */
  const double* cp1[3];  /* cp1,cp2,cp3      b-range, first derivative on the pressure grid */
  const double* cpp[3];  /* cp11,cp22,cp33   b-range, second derivative on the pressure grid */
  const double* cuu[3];  /* cu11,cv22,cw33   b-range, second derivative on the velocity grid */
  const double* cdg[3];  /* cdg1,cdg2,cdg3   (-1:1, 1:N) compact Laplacian */
} orc_coeffs;

/* ---------------- grid and coefficient generation ---------------- */
/* Global coordinates of one periodic axis with M points: xp/xu hold indices -3..M+3
 * (offset 3).  kind 0 = equidistant (usr_geometry.f90:93-156 with coord_tanh,
 * usr_func.f90:1964), kind 1 = x(s) = L/2 (1 + sinh(2(s/(M-1) - 1/2))/sinh(1)).
 * Periodic continuation as mod_geometry.f90:95-103. */
void orc_coords(int M, double L, int kind, double* xp, double* xu);

/* Exact equidistant FD weights (diff_coeffs_exact, mod_coeffs.f90:598-751): derivative
 * order abl of the polynomial through the n points deltaX0 + 0..n-1, at 0.  Returns 0. */
int orc_fd_exact(int abl, int n, double deltaX0, double* cc);

/* diff_coeffs (mod_coeffs.f90:200-597) for periodic boundaries and mapping_yes = T.
 * grid_type 0 p->p, 1 u->u, 2 p->u, 3 u->p; upwind -1/0/+1; n_coeff = interior width.
 * xC/xE: coordinate arrays over -3..N+3 (offset 3).  cc: (bU-bL+1)*(N+1). */
int orc_diff_coeffs(int abl, int upwind, int grid_type, int N, int bL, int bU, int n_coeff,
                    const double* xC, const double* xE, double* cc);

/* get_stencil (mod_coeffs.f90:1048-1259), grid level 1, periodic: cdg(-1:1,1:N). */
void orc_get_stencil(int N, const double* xp, const double* xu, double* cdg);

/* RK3 stability limit along 41 rays (the quantity tabulated in mod_vars.f90:785). */
void orc_stability_limits(double* lim41);

/* ---------------- ghost fill ---------------- */
/* exchange (mod_exchange.f90:133-140 and the dir 2/3 analogues), periodic branch. */
void orc_exchange(int dir, int N1, int N2, int N3, double* phi);

/* ---------------- operators (mod_diff.f90) ---------------- */
void orc_gradient(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* grad);
void orc_divergence(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* div);
void orc_divergence2(int N1, int N2, int N3, const orc_coeffs* c, double* u, double* v, double* w,
                     double* div);
void orc_helmholtz(int m, int N1, int N2, int N3, const orc_coeffs* c, double multL, double* vel,
                   double* nl);
void orc_interpolate_pre_vel(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi,
                             double* inter);
void orc_interpolate_vel_pre(int m, int N1, int N2, int N3, const orc_coeffs* c, double* phi,
                             double* inter);
/* One upwind term (component_id 1..9 = (m,a) pairs, Nonlinear_upwind_host.f90:6):
 * nl_m (=, first axis) / (+=) dd1(a)*pp with pp already interpolated. */
void orc_nonlinear_upwind(int component_id, int N1, int N2, int N3, const orc_coeffs* c,
                          const double* pp, double* vel, double* nl);
/* Full nonlinear term of component m from vel_m and work1..3 (mod_diff.f90:784-1424). */
void orc_nonlinear(int m, int N1, int N2, int N3, const orc_coeffs* c, double* vel_m,
                   double* work1, double* work2, double* work3, double* pp_scratch, double* nl_m);
void orc_axpby(int N1, int N2, int N3, double a, double b, const double* x, const double* y,
               double* z);

/* ---------------- Laplacians / relaxation (mod_laplace.f90) ---------------- */
void orc_product_div_grad(int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* dig,
                          double* lap);
void orc_product_dg_relax(int N1, int N2, int N3, const orc_coeffs* c, double* phi, double* lap);
/* Damped Jacobi / JOR sweeps (relaxation_div_grad, mod_laplace.f90:339-613):
 * init_yes: the first sweep is rel = omega*bb/diag. comp is a work field. */
void orc_jacobi(int N1, int N2, int N3, const orc_coeffs* c, int init_yes, int n_relax,
                double omega, const double* bb, double* rel, double* comp);
/* Pressure Dirichlet values on labelled planes (apply_pressure_BC_CT, usr_func.f90:857-897). */
void orc_pressure_bc(int N1, int N2, int N3, const uint8_t* label, int k_start_index,
                     double p_inlet, double p_outlet, double p_outlet2, double* rel);

/* ---------------- reductions (mod_solvers.f90:2319-2470) ---------------- */
double orc_product_scalar(int N1, int N2, int N3, const double* a, const double* b);
void orc_norms(int N1, int N2, int N3, const double* a, double* norm_inf, double* norm_two_sq);

/* ---------------- solvers ---------------- */
typedef struct {
  double tol_rel;     /* stop when ||r||_2 <= tol_rel * ||b||_2 (0 = off) */
  double tol_abs_inf; /* stop when ||r||_inf < tol_abs_inf (0 = off; the reference's epsU) */
  int max_it;
  int n_sweeps;       /* Jacobi sweeps per preconditioner application (0 = none) */
  double omega;       /* Jacobi/JOR relaxation of the preconditioner */
  int init_yes;       /* 1: start from phi = 0 as BiCGstab_orig with init_yes */
  int precond;        /* 0: n_sweeps Jacobi sweeps; 1: multigrid V-cycle (mg) */
  const struct orc_mg_s* mg;
  int mg_down, mg_up, mg_bottom;
} orc_solver_opts;

typedef struct {
  int iterations;
  int status;        /* 0 converged, 1 max iterations, 2 breakdown, 3 non-finite */
  double res_inf;    /* recursive residual at exit */
  double res_two;    /* sqrt of sum of squares */
  double b_two;
} orc_solver_result;

/* BiCGstab_orig (mod_solvers.f90:1509-1935), problem_type 2, with the Jacobi preconditioner
 * of opts and the high-order operator product_div_grad. work: 9 fields of the padded size. */
void orc_bicgstab(int N1, int N2, int N3, const orc_coeffs* c, const orc_solver_opts* o,
                  double* bb, double* phi, double* work, orc_solver_result* res);

/* ---------------- one fractional time step (mod_timeint.f90:242-578) ---------------- */
typedef struct {
  double Re;
  double CFL;
  double dtime_max;
  double dtime0;     /* cap for the first step (timestep == 0) */
  double U0;         /* inflow amplitude: u_z = U0 (1 + 0.5 sin(2 pi t / T)) on label 5 */
  double T_pulse;
  int level_pressure; /* subtract the mean pressure after every step (Int_lev_pre = 1) */
  orc_solver_opts poisson;
} orc_step_params;

typedef struct {
  double time;
  double dtime;
  int timestep;
  int poisson_iterations[3];
  double poisson_res_rel[3];
  int poisson_status[3];
} orc_step_state;

/* Fields: vel (3 padded fields), nl (3), rhs (3), pre, work (3), res, plus solver work (9).
 * scratch must hold 11 padded fields. label: padded uint8 labels. */
void orc_time_step(int N1, int N2, int N3, const orc_coeffs* c, const orc_step_params* p,
                   const double* stab41, const uint8_t* label, double* vel, double* nl, double* pre,
                   double* scratch, orc_step_state* st);

/* get_dtime (mod_lib.f90:46-250) for timeint_mode 1. work: 3 padded fields. */
double orc_get_dtime(int N1, int N2, int N3, const orc_coeffs* c, const double* stab41,
                     double Re, double CFL, double dtime_max, double* vel, double* work);

/* Mask forcing (apply_CT_forcing, usr_func.f90:909-1049, idealized branch). */
void orc_mask_forcing(int N1, int N2, int N3, const uint8_t* label, double u_inflow, double* vel);
/* level_pressure (mod_lib.f90:507-537). */
void orc_level_pressure(int N1, int N2, int N3, double* pre);


/* ---------------- geometric multigrid (mod_solvers.f90:353-1150, mod_setup.f90:95-143,
 * mod_geometry.f90:66-103, mod_coeffs.f90:1048-1259 and 1683-2100), periodic ---------------- */
#define ORC_MG_MAX 15
typedef struct orc_mg_s {
  int n_grids;
  int M[ORC_MG_MAX][3];     /* points per axis (NN) of every level */
  int ratio[ORC_MG_MAX][3]; /* coarsening factor from level g to g+1 (2 or 1) */
  double* xp[ORC_MG_MAX][3]; /* level coordinates over -3..M+3 */
  double* xu[ORC_MG_MAX][3];
  double* cdg[ORC_MG_MAX][3]; /* compact Laplacian cdg(-1:1,1:M) of the level */
  double* cI[ORC_MG_MAX][3];  /* interpolation weights cI(1:2, 0:M) of the level (even points) */
  double* f[ORC_MG_MAX][3];   /* level fields: bb, phi, work (padded, level 1 unused) */
} orc_mg;

/* Build the hierarchy of a periodic grid from its finest global coordinates (xp/xu over
 * -3..N+3 per axis) and box lengths; n_grids_limit caps the number of levels. */
int orc_mg_build(int N1, int N2, int N3, const double* const* xp, const double* const* xu, const double* L,
                 int n_grids_limit, orc_mg* mg);
void orc_mg_free(orc_mg* mg);
/* multigridV(init_yes = .TRUE., gstart = 1, bb, phi) with damped-Jacobi smoothing
 * (n_down / n_up / n_bottom sweeps, relaxation omega); work: one padded level-1 field. */
void orc_mg_vcycle(const orc_mg* mg, int n_down, int n_up, int n_bottom, double omega, double* bb, double* phi,
                   double* work);
/* BiCGstab_orig with the multigrid V-cycle preconditioner (precond_Poisson = 1). */
void orc_bicgstab_mg(int N1, int N2, int N3, const orc_coeffs* c, const orc_mg* mg, const orc_solver_opts* o,
                     int n_down, int n_up, int n_bottom, double* bb, double* phi, double* work,
                     orc_solver_result* res);

/* ---------------- diffuse-interface immersed boundary transfers (mod_ibm.f90), periodic ----------
 * n Lagrangian markers; yb, ub, fb are column-major (n, 3) arrays (all x, then all y, then all z:
 * the reference's yb(1:M_bound, 1:3)).  skip[i] != 0 excludes marker i (its index is in
 * ebcs(:, 1)).  xp / xu are the global coordinates over -3..N+3 per axis, L the box lengths.
 * delta_type 1..4 and reach as ddf_type and reach of the reference. */
double orc_ibm_delta(int delta_type, double reach, double distance);
/* interpolate_vel_to_ib (mod_ibm.f90:589-737): ub = sum of delta * vel * cell volume, per component */
void orc_ibm_interpolate(int N1, int N2, int N3, const double* const* xp, const double* const* xu,
                         const double* L, int delta_type, double reach, int n, const double* yb,
                         const uint8_t* skip, const double* vel, double* ub);
/* spread_force_dens_to_vel_grid (mod_ibm.f90:428-583): fd (three padded fields) = 0, then the
 * delta-weighted marker forces times node volumes */
void orc_ibm_spread(int N1, int N2, int N3, const double* const* xp, const double* const* xu, const double* L,
                    int delta_type, double reach, int n, const double* yb, const uint8_t* skip,
                    const double* fb, const double* node_vol, double* fd);

/* OpenMP threads of the oracle's loops; n <= 0 queries.  Returns the threads in use. */
int orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
