/*
 * swm.h -- C ABI of the B200 (sm_100a) mPDeC5 shallow-water time step.
 *
 * This is the drop-in boundary for the reference's time step in
 * accdavlo/sw-mpdec (Fortran 90).  The reference exposes the step as two
 * module procedures that share all state through module globals:
 *   REAL FUNCTION TimeStep()                        equation.f90:791-837
 *   SUBROUTINE TimeDiscretizationByMPDeC5(t)        timediscretization.f90:458-566
 *   SUBROUTINE TimeDiscretizationByMPDeC2(t)        timediscretization.f90:571-664
 * called from the driver loop at timediscretization.f90:58,71-72,75-76.
 * The Fortran driver keeps t, dt, output cadence and I/O; it calls these
 * entry points through ISO_C_BINDING (sw-mpdec_b200/fortran/mod_swm_capi.f90).
 *
 * Conventions
 *  - Every call returns an int status: 0 ok, >0 warning, <0 error.
 *  - Host arrays are owned by the caller and are copied in/out; the library
 *    never retains a host pointer.  The library owns all device memory, its
 *    stream and its CUDA graphs.  State stays on the device between steps.
 *  - Ghosted state arrays use the reference's layout U(1:3,-2:nx+3,-2:ny+3):
 *    column-major, variable fastest, 3*(nx+6)*(ny+6) doubles
 *    (finitevolume.f90:139).  Only the interior is read on input.
 *  - One handle per host thread; calls on a handle are synchronous unless
 *    documented otherwise.
 */
#ifndef SWM_H
#define SWM_H

#if defined(__GNUC__)
#define SWM_API __attribute__((visibility("default")))
#else
#define SWM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SWM_OK 0
#define SWM_WARN_JACOBI_MAXITER 1 /* jacobi_iteration.f90:83-85 prints and continues */
#define SWM_ERR_PARAM (-1)        /* invalid parameters (parameters.f90:123-126 STOPs) */
#define SWM_ERR_CUDA (-2)         /* CUDA runtime error */
#define SWM_ERR_NAN (-3)          /* non-finite state detected */
#define SWM_ERR_WATCHDOG (-4)     /* a bounded device wait gave up */
#define SWM_ERR_ALLOC (-5)        /* device or host allocation failed */
#define SWM_ERR_STATE (-6)        /* call out of order (e.g. no state set) */
#define SWM_ERR_UNSUPPORTED (-7)  /* option not available on this device */

/* ---- option enums ---- */
/* The reference's WENO weights use eps = 1e-24 on absolute values, so where a
 * stencil varies by less than ~1e-7 its smoothness indicators are rounding noise
 * and any change of arithmetic (FMA contraction, reciprocals) moves face values by
 * up to that variation.  Parity at relative L1 1e-12 therefore needs the
 * reference's own expression order: that is the plain FP64 form. */
#define SWM_PREC_FP64 0     /* FP64 in the reference's expression order, no contraction */
#define SWM_PREC_SPLIT 1    /* FP32 WENO on deviations from the cell value, FP64 rest */
#define SWM_PREC_FP64_FMA 2 /* FP64 with FMA contraction and shared reciprocals */

#define SWM_SOLVER_CSR 0     /* Jacobi on the reference CSR layout (finitevolume.f90:219-271) */
#define SWM_SOLVER_STENCIL 1 /* matrix-free 5-point Jacobi, shared-memory temporal blocking */

#define SWM_BATHY_FLAT 0
#define SWM_BATHY_SINCOS 1 /* equation.f90:430 */
#define SWM_BATHY_BUMP 2   /* equation.f90:433-438 */
#define SWM_BATHY_GAUSS 3  /* A exp(-(ax (x-cx)^2 + ay (y-cy)^2)); par = {A, ax, cx, ay, cy} */

typedef struct swm_params {
  int nx, ny;            /* nElemsX, nElemsY (parameters.f90:66-120) */
  double x0[2], x1[2];   /* MESH_X0, MESH_X1 */
  double g;              /* Gravity */
  double cfl;            /* CFL (parameters.f90:139) */
  int timescheme;        /* parameters.f90:144 (timediscretization.f90:60-79):
                          * 5 mPDeC5, 7 mPDeC2, 6 mPEuler (Patankar, h >= 0);
                          * 1 forward Euler, 2 SSPRK(5,4), 3 RK65, 4 DeC5 (explicit,
                          * as the reference built without -DPATANKAR: Ut(1) from the
                          * mass fluxes) */
  int bathy_flag;        /* BathymetryFlag */
  double bathy_par[5];   /* SWM_BATHY_GAUSS parameters */
  int well_balanced;     /* -DWELLBALANCED (src/makefile:48) */
  int precision;         /* SWM_PREC_* */
  int solver;            /* SWM_SOLVER_* */
  int jacobi_maxiter;    /* maxIter = 1000 (jacobi_iteration.f90:64) */
  double jacobi_tol;     /* tolerance = 1e-16 (jacobi_iteration.f90:63) */
  int jacobi_block;      /* stencil solver: Jacobi sweeps per pass (1..8), 0 = auto */
  int mpdec2_compat;     /* 1: reproduce the hp(2,nx,ny) read of Up(:,1,:,:) of mPDeC2 and mPEuler */
  int use_graph;         /* capture each step into a CUDA graph (1 = default) */
  int device;            /* CUDA device ordinal */
  int source_table;      /* FP64 form, Gaussian and sin/cos bathymetries: 1 (default) reads
                          * b_x, b_y tabulated with the host libm at the 16 interior Gauss
                          * points of every cell (256 B per cell and RHS; the reference's
                          * source term bit for bit, equation.f90:380-388,451-509); 0 forms
                          * the source from per-column and per-row factors of the separable
                          * gradient (no per-cell table; equal to the reference's up to
                          * rounding).  The split and FMA forms always use the factors. */
} swm_params;

typedef struct swm_stats {
  int status;                 /* status of the last step */
  int n_solves;               /* Patankar solves in the last step (13 for mPDeC5) */
  int jacobi_iters[16];       /* Jacobi iterations of each solve of the last step */
  int jacobi_iters_min, jacobi_iters_max;
  long long jacobi_iters_total; /* over all steps */
  long long steps;            /* steps taken */
  double lambda_max[2];       /* LambdaMaxX, LambdaMaxY of the last swm_timestep */
} swm_stats;

typedef struct swm_solver *swm_handle;

/* Fill *p with the reference defaults (CFL 1.0, mPDeC5, tol 1e-16, maxIter 1000,
 * FP64, CSR solver, graphs on) for an nx*ny grid on [x0,x1]. */
SWM_API int swm_params_default(swm_params *p, int nx, int ny, double x00, double x01, double x10,
                       double x11);

/* Allocate device state for one grid (replaces InitializeFiniteVolume's
 * allocation and CSR pattern build, finitevolume.f90:129-271). */
SWM_API int swm_create(const swm_params *p, swm_handle *out);
SWM_API int swm_destroy(swm_handle h);

/* Copy the state U (ghosted layout) to the device. */
SWM_API int swm_set_state(swm_handle h, const double *U_ghosted);
/* Copy the device state back; V_ghosted (nullable) receives ConsToPrim of the
 * state with periodic ghosts, as BoundaryConditions leaves V (equation.f90:778-782). */
SWM_API int swm_get_state(swm_handle h, double *U_ghosted, double *V_ghosted);
/* Interior state as three planes [3][ny][nx] (x fastest); host arrays. */
SWM_API int swm_set_planes(swm_handle h, const double *planes);
SWM_API int swm_get_planes(swm_handle h, double *planes);

/* Well-balanced reference state (InitializeWBVariables, finitevolume.f90:339-396):
 * runs one RHS on Uwb with the live kernel and precision and keeps FXWB, FYWB, SWB. */
SWM_API int swm_set_wb_state(swm_handle h, const double *Uwb_ghosted);

/* ---- driver-side initialisation and post-processing on the device ----
 * Initial condition `ic` evaluated by ExactFunction (equation.f90:70-230) and
 * averaged with the 4x4 Gauss rule of FillInitialConditions (finitevolume.f90:281-333):
 *   ic 1..6   the reference's cases (1 the smooth vortex, 2 sin/cos lake, 3 and 6
 *             perturbations over the bathymetry, 4 and 5 circular dam breaks);
 *   ic 101    vortex            par {cx, cy, eps, ub, vb, R}
 *   ic 102    lake + pulse      par {amp, x_lo, x_hi}   (bathymetry from the params)
 *   ic 103    dam break         par {cx, cy, radius, h_in}
 *   ic 104    wave over island  par {amp, xc, width}    (bathymetry from the params)
 *   ic 105    still water       par {level}
 * par holds npar <= 8 values (nullable when npar = 0).  Transcendental functions are
 * CUDA's, so cell averages match a host evaluation to the last few bits. */
/* U := the cell averages of ic (replaces CALL FillInitialConditions, main.f90:23). */
SWM_API int swm_fill_ic(swm_handle h, int ic, const double *par, int npar);
/* InitializeWBVariables (finitevolume.f90:339-396) from ic: the WB fluxes and source
 * of its cell averages with the live kernel; the state is left unchanged. */
SWM_API int swm_init_wb_ic(swm_handle h, int ic, const double *par, int npar);
/* PostProcessing (postprocessing.f90:23-60): l1[v] = sum_cells |U - Uexact(ic, t)| dx dy
 * for v = h, hu, hv (case 1 is advected to time t; the others do not depend on t). */
SWM_API int swm_l1_error(swm_handle h, int ic, const double *par, int npar, double t,
                         double l1[3]);

/* WriteSolutionToDisk(t) (output.f90:29-185), formatted on the device: SOLUTION_* and
 * ERROR_* files in `directory` named as TIMESTAMP does, Tecplot (which_output 2),
 * Octave (1) or both (3), every value as (SP,ES21.14E2) with |v| < 1e-70 printed as 0.
 * SOLUTION holds the barycentres, V = ConsToPrim(U) and the cell-averaged bathymetry;
 * ERROR holds U - Uexact(ic, t) (par/npar as for swm_fill_ic).  flags
 * SWM_OUT_V_LAST_RHS writes, for mPDeC5, the V the reference's BoundaryConditions left
 * behind: that of the last RHS input of the step (Ua(4) of correction 4). */
#define SWM_OUT_V_LAST_RHS 1
SWM_API int swm_write_output(swm_handle h, double t, int which_output, int ic, const double *par,
                             int npar, const char *directory, int flags);
/* WriteMeshToDisk (output.f90:190-231): MESH_CoordinateX.dat, MESH_CoordinateY.dat. */
SWM_API int swm_write_mesh(swm_handle h, const char *directory);
/* n values as 21-character (SP,ES21.14E2) fields, back to back in out[21*n] (no NUL). */
SWM_API int swm_debug_format(swm_handle h, const double *x, int n, char *out);

/* TimeStep() (equation.f90:791-837): CFL time step of the current state. */
SWM_API int swm_timestep(swm_handle h, double *dt_min);

/* One mPDeC5 (or mPDeC2) step of size dt from time t; the state is updated on
 * the device.  Replaces TimeDiscretizationByMPDeC5(t) (timediscretization.f90:458-566).
 * Returns SWM_WARN_JACOBI_MAXITER if a solve stopped at maxIter, and SWM_ERR_NAN if
 * the new state holds a non-finite value or a negative depth: the step ends with
 * TimeStep()'s reduction of the new state, which the next swm_timestep reuses. */
SWM_API int swm_step(swm_handle h, double t, double dt);

/* Steps from t to t_end with dt = min(TimeStep(), t_out - t, t_end - t), restating
 * the driver loop of timediscretization.f90:57-95 (output times every
 * t_end/n_outputs) without I/O; returns the number of steps in *n_steps. */
SWM_API int swm_run(swm_handle h, double t_end, int n_outputs, int *n_steps, double *t_reached);

SWM_API int swm_get_stats(swm_handle h, swm_stats *s);
/* Device-side totals of the state: mass sum(h), min(h), for invariant checks. */
SWM_API int swm_state_summary(swm_handle h, double *mass, double *min_h);

/* The cudaStream_t the handle launches on (for CUDA-event timing by the caller). */
SWM_API int swm_get_stream(swm_handle h, void **stream);
/* One step like swm_step, launched eagerly with CUDA events around every kernel:
 * ms[0..3] = device milliseconds spent in the RHS, assembly and Jacobi kernels and
 * the whole step; launches[0..2] = launches of each of the three classes. */
SWM_API int swm_profile_step(swm_handle h, double t, double dt, float *ms, int *launches);

/* Message for the last error on this thread (static storage). */
SWM_API const char *swm_last_error(void);
SWM_API const char *swm_strerror(int status);

/* ---- diagnostics (parity tests) ---- */
/* One RHS (FVTimeDerivative, finitevolume.f90:402-540) of the ghosted input
 * state.  Outputs (nullable, column-major like the reference):
 * Ut(3,nx,ny) [Ut(1) as the build without PATANKAR forms it (finitevolume.f90:530-533);
 * the Patankar schemes use Ut(2:3) and the mass fluxes only],
 * FX(3,0:nx,1:ny), FY(3,1:nx,0:ny), S(3,nx,ny): WB-subtracted when WB is on. */
SWM_API int swm_debug_rhs(swm_handle h, const double *U_ghosted, double *Ut, double *FX, double *FY,
                  double *S);
/* Jacobi (jacobi_iteration.f90:52-87) on a user system given in the reference's
 * CSR values: mass[5N] (slot order S,W,C,E,N), diag[N], rhs[N] -> sol[N];
 * runs the handle's solver (CSR or stencil) and returns the iteration count. */
SWM_API int swm_debug_jacobi(swm_handle h, const double *mass, const double *diag, const double *rhs,
                     double *sol, int *iters);

/* Failure paths a test can reach without a GPU fault.
 * swm_debug_set_spin_limit: polls each grid-barrier wait of the handle's Jacobi
 * launches makes before it gives up with SWM_ERR_WATCHDOG (default 2^26, about a
 * second); limit <= 0 makes every wait that is not already open give up at once.
 * The step's graph is rebuilt with the new limit.  Every step and debug solve
 * starts from a cleared control block, so a handle stays usable after a watchdog.
 * swm_debug_inject_alloc_failure: from now on the library's nth device or
 * pinned-host allocation (process-wide, counted from this call) fails as if the
 * allocator had; 0 disables.  *counted (nullable) receives the number of
 * allocations made since the previous call. */
SWM_API int swm_debug_set_spin_limit(swm_handle h, long long limit);
/* RHS tile loads: enable = 1 (default) stages the haloed state tiles that lie inside
 * the grid by TMA tensor copies (even nx), 0 loads every tile with wrapped-index
 * loads.  Both give bit-identical results; the step's graph is rebuilt. */
SWM_API int swm_debug_set_tma(swm_handle h, int enable);
SWM_API int swm_debug_inject_alloc_failure(long long nth, long long *counted);

/* ---- allocation-free Jacobi solve ----
 * No counterpart in the reference (its jacobi() works on module arrays).  For
 * callers that cannot let a library allocate device memory -- drivers that own
 * every byte through their own pool or share a hard memory cap between solvers,
 * and loops that must not pay the device-wide synchronisation of cudaMalloc and
 * cudaFree.  Solves one Patankar system (x <- (rhs - S x_S - W x_W - E x_E - N x_N)/D
 * on the periodic nx*ny grid, stop rule of jacobi_iteration.f90:52-87) with the
 * matrix-free stencil kernel, `block` sweeps per pass (1..8).  All arrays are the
 * caller's device memory, nx*ny doubles each, [ny][nx] row-major; sol is written
 * while the others are read, so it must not overlap rhs or any coefficient plane
 * (SWM_ERR_PARAM otherwise).  Scratch is a static device array sized for at most
 * 1,048,576 cells (8 MiB plus a small control block), held on every GPU that
 * loads the library until the process exits; larger grids are rejected with
 * SWM_ERR_PARAM.  The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress) and the kernel's resident grid; make that first
 * call before any stream capture.  Every call shares the scratch: calls whose
 * work overlaps on the GPU (other streams, other host threads) race.  Runs on
 * `stream` (a cudaStream_t, 0 = legacy default), then synchronises that stream to
 * read the iteration count back, so a stream that is being captured is refused
 * with SWM_ERR_STATE; returns after the solve with the count in *iters. */
SWM_API int swm_jacobi_noalloc(int nx, int ny, const double *cS, const double *cW,
                               const double *cE, const double *cN, const double *cD,
                               const double *rhs, double *sol, int maxiter, double tol,
                               int block, int *iters, void *stream);

/* Checked build only (libswm_checked.so, -DSWM_CHECKED): the device-side index checks
 * at the kernels' wrapped-index sites record a failure instead of touching memory out
 * of range.  Returns, and clears, the site of the first failing check (0 none; 1 RHS
 * tile load, 2/3 Jacobi tile loads, 4 CSR columns, 5 mPDeC2 compatibility read, 6
 * ensemble work item) and the number of failing checks; SWM_ERR_UNSUPPORTED in the
 * normal build. */
SWM_API int swm_debug_checked_status(int *site, unsigned long long *count);

/* ---- batched ensembles ---- */
typedef struct swm_batch *swm_batch_handle;
/* n problems of independent size and parameters, stepped together (the
 * reference's time loop, timediscretization.f90:57-95, over an ensemble): a whole
 * mPDeC5 step of every problem is one cooperative persistent launch (TimeStep, the
 * RHS of every tile, and per correction the assembly of its three substeps and one
 * batched Jacobi solve of all their systems, each with its own stop rule), captured
 * with its memsets as a CUDA graph.  All problems share precision and jacobi_block
 * (taken from p[0]); mPDeC5 only, no well-balanced reference; the stencil solver is
 * always used.  jacobi_block = 0 lets the first step time the schedules (2, 4 and 8
 * sweeps per pass, one or two CTAs per SM) on the initial state and keep the
 * fastest; every schedule gives the same results. */
SWM_API int swm_batch_create(int n, const swm_params *p, swm_batch_handle *out);
SWM_API int swm_batch_destroy(swm_batch_handle b);
SWM_API int swm_batch_set_planes(swm_batch_handle b, int i, const double *planes);
SWM_API int swm_batch_get_planes(swm_batch_handle b, int i, double *planes);
/* One step of every problem, each with its own dt = TimeStep() (computed on
 * the device); dt_out[n] (nullable) receives the steps taken. */
SWM_API int swm_batch_step(swm_batch_handle b, double *dt_out);
SWM_API int swm_batch_cells(swm_batch_handle b, long long *cells);
/* Sweeps per Jacobi pass in use (chosen by the first step when jacobi_block was 0),
 * Jacobi sweeps summed over all steps and problems, and (nullable) the sweeps of
 * the last step, [13][n] (solve-major). */
SWM_API int swm_batch_get_stats(swm_batch_handle b, int *jacobi_block, long long *iters_total,
                                int *last_iters);
/* The cudaStream_t the ensemble launches on (for CUDA-event timing by the caller). */
SWM_API int swm_batch_get_stream(swm_batch_handle b, void **stream);
/* The step form.  per_phase = 1: a kernel per phase, captured in one graph (17 per
 * step for the split and FMA forms: TimeStep (2), the RHS of U^n, per correction
 * 1..4 the fused assembly of its three substeps, one batched Jacobi solve of their
 * systems and one RHS launch over the new substeps, then the last correction's
 * assembly and solve; 25 for FP64, whose three assemblies are separate); 0: the one
 * persistent launch; < 0: the autotuner's choice (with jacobi_block = 0 the first
 * step times both forms; without it the persistent launch).  Results are identical.
 * Resets the captured graph. */
SWM_API int swm_batch_debug_set_launches(swm_batch_handle b, int per_phase);
/* Measurement: one step of every problem (it advances the state) in the current form,
 * recording when its phases end (the persistent launch by a global timer read at each
 * phase's closing barrier, the per-phase form by CUDA events between its kernels);
 * ms[0..n-1] (cap >= 16) receive the phase durations: TimeStep, RHS of U^n, then per
 * correction k = 1..5 the assembly, the Jacobi solve and (k < 5) the RHS of the new
 * substeps. */
SWM_API int swm_batch_debug_phase_times(swm_batch_handle b, double *ms, int cap, int *n);
/* Debug: polls of every grid-barrier wait of the ensemble's kernels before the step
 * gives up with SWM_ERR_WATCHDOG (default 2^26; <= 0: at once).  Resets the graph. */
SWM_API int swm_batch_debug_set_spin_limit(swm_batch_handle b, long long limit);
/* Launches of the ensemble's own kernels in one step (1, or 17 / 25 per phase) and
 * the CTAs of the persistent launch (0 when per phase). */
SWM_API int swm_batch_get_launch_info(swm_batch_handle b, int *launches_per_step, int *ctas);

#ifdef __cplusplus
}
#endif
#endif /* SWM_H */
