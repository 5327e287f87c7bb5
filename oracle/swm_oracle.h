/*
 * swm_oracle.h -- CPU FP64 oracle for the mPDeC5 shallow-water time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, the smoke() check and bench.py's CPU-baseline
 * leg use it, and only as the checker / the timed CPU restatement.
 *
 * It restates, routine by routine and in the same loop and summation order,
 * the Fortran hot path of accdavlo/sw-mpdec (fv-solver-sw/src/):
 *   timediscretization.f90:458-566 (mPDeC5), :571-664 (mPDeC2),
 *   :771-908 (Patankar assembly), :913-924 (PATANKAR_DIV);
 *   jacobi_iteration.f90:25-87; finitevolume.f90:219-271 (CSR pattern),
 *   :402-540 (RHS + P/D), :546-640 (fluxes), :646-757 (limiter);
 *   reconstruction.f90:54-184, :408-514, :673-755, :999-1136 (WENO5);
 *   equation.f90:284-413 (source), :515-785 (periodic BC), :791-906 (dt),
 *   :912-1106 (variable maps, flux, Rusanov); mesh.f90:58-146,157-170.
 * Arithmetic follows the Fortran source expression order with no FMA
 * contraction (build with -ffp-contract=off), i.e. the reference's default
 * `COMPILER=GNU DEBUG` (-O0) build semantics.
 *
 * Parity pinning: no Fortran compiler exists in this image or on the GPU
 * hosts, and the reference ships no golden vectors, so this restatement is
 * pinned by the known answers derivable from the reference source (WENO
 * stencil/weight sums, Gauss weights, theta row sums, exact preservation of
 * constant states, well-balancing of the lake at rest, the 5th-order
 * convergence of the smooth vortex with an exact solution, positivity and
 * mass conservation of the Patankar/Jacobi update).  Against the Fortran
 * binary itself the oracle is "parity unpinned".
 */
#ifndef SWM_ORACLE_H
#define SWM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc_t;

/* Bathymetry flags: 0 flat, 1 and 2 as equation.f90:428-442, 3 Gaussian
 * b = A exp(-(ax (x-cx)^2 + ay (y-cy)^2)), par = {A, ax, cx, ay, cy}. */
typedef struct orc_params {
  int nx, ny;
  double x0[2], x1[2];
  double g, cfl;
  int timescheme;       /* 1 FE, 2 SSPRK(5,4), 3 RK65, 4 DeC5, 5 mPDeC5, 6 mPEuler, 7 mPDeC2 */
  int bathy_flag;
  double bathy_par[5];
  int well_balanced;
  int jacobi_maxiter;   /* 1000 in the reference */
  double jacobi_tol;    /* 1e-16 in the reference */
  int mpdec2_compat;    /* 1: reproduce the hp(2,nx,ny) sequence-association read of mPDeC2 */
} orc_params;

orc_t *orc_create(const orc_params *p);
void orc_destroy(orc_t *o);

/* Initial conditions (cell averages by 4x4 Gauss quadrature, finitevolume.f90:314-330).
 * ic 1..6: ExactFunction cases of equation.f90:109-206 (t = 0).
 * ic 101 vortex: par {cx, cy, eps, ub, vb, R}
 * ic 102 lake + pulse: par {pulse_amp, x_lo, x_hi}     (bathymetry from params)
 * ic 103 circular dam break: par {cx, cy, radius, h_in}
 * ic 104 wave over island: par {amp, xc, width}       (bathymetry from params)
 * ic 105 still water h = max(level - b, MIN_DEPTH): par {level}
 * Writes the interior of U; ghosts are left zero (BC fills them). */
int orc_fill_ic(orc_t *o, int ic, const double *par);
/* Well-balanced init (finitevolume.f90:339-396): U := cell average of the WB
 * state ic, then one RHS; FXWB, FYWB, SWB are stored.  U is zeroed after. */
int orc_init_wb(orc_t *o, int ic, const double *par);
/* The same from given cell averages [3][ny][nx]. */
int orc_init_wb_planes(orc_t *o, const double *planes);
/* PostProcessing (postprocessing.f90:23-60): L1 error of U against the Gauss average
 * of ExactFunction(ic, t) (case 1 advected to time t), times dx dy, per variable. */
int orc_l1_error(const orc_t *o, int ic, const double *par, double t, double out[3]);

/* Ghosted state (3, nx+6, ny+6), var fastest (Fortran U(1:3,-2:nx+3,-2:ny+3)). */
void orc_set_state(orc_t *o, const double *U);
void orc_get_state(const orc_t *o, double *U, double *V);
/* Interior state as three planes [3][ny][nx] (x fastest). */
void orc_get_planes(const orc_t *o, double *out);
void orc_set_planes(orc_t *o, const double *in);

double orc_timestep(orc_t *o);                    /* equation.f90:791-837 */
int orc_step(orc_t *o, double t, double dt);      /* one mPDeC5/mPDeC2 step */
/* Driver loop of timediscretization.f90:46-95 without I/O; returns steps. */
int orc_run(orc_t *o, double tend, int n_outputs, double *t_out);

/* One RHS (FVTimeDerivative).  Outputs (nullable):
 * Ut (3,nx,ny), FX (3,0:nx,1:ny), FY (3,1:nx,0:ny), S (3,nx,ny),
 * prod/dest (5N).  Input: current ghosted state. */
void orc_rhs(orc_t *o, double *Ut, double *FX, double *FY, double *S,
             double *prod, double *dest);

/* Jacobi on a user system in the reference CSR layout (1-based RowStart and
 * ColumnsVector are the ones built at create); mass has 5N values. */
int orc_jacobi(orc_t *o, const double *mass, const double *diag,
               const double *rhs, double *sol);

/* CSR pattern access (1-based values as in the reference). */
const int *orc_rowstart(const orc_t *o);
const int *orc_columns(const orc_t *o);

/* Statistics of the last step. */
int orc_last_jacobi_iters(const orc_t *o, int *iters, int max);
long long orc_total_jacobi_iters(const orc_t *o);
double orc_mesh_dx(const orc_t *o, int d);

/* Elementary routines exposed for unit tests. */
void orc_weno5_first(const double q[5], double *wm, double *wp);
void orc_weno5_second(const double q[5], double w[4]);
void orc_quadrature(double nodes[4], double weights[4]);
void orc_theta_mpdec5(double theta[16], double beta[4]);
double orc_patankar_div(double prod, double h);

/* Bathymetry b, b_x, b_y for a parameter set (used by IC fill and tests). */
void orc_bathymetry(const orc_params *p, double x, double y, double *b,
                    double *bx, double *by);

/* Threads used by the timing build (1 for the reference build). */
int orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
