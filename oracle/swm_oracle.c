/*
 * swm_oracle.c -- CPU FP64 oracle for the mPDeC5 shallow-water time step.
 *
 * TEST INFRASTRUCTURE ONLY (see swm_oracle.h).  Every routine restates the
 * Fortran routine named in its comment, keeping the reference's array shapes
 * (1-based, ghosted, variable-fastest), loop nesting and expression order so
 * that rounding matches the reference's unoptimised build.  Deviations that
 * cannot change a non-zero result are listed where they occur (dropped
 * `0.0*Q(k)` terms of the WENO stencils, the identity rotations of the
 * Riemann solver), and the source term reconstructs only the depth it uses.
 *
 * Build:  gcc -O2 -ffp-contract=off -fPIC -shared (reference semantics), or
 *         add -fopenmp -DORC_OMP for the threaded timing build (identical
 *         per-cell arithmetic; only the Jacobi residual sum is reassociated).
 */
#include "swm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef ORC_OMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

/* finitevolume_vars.f90:96-106 */
#define MIN_DEPTH 1.0e-6
#define WENOEPS 1.0e-24
#define MIN_TIMESTEP 1.0e-30
static const double wLobatto = 1. / 12.;

struct orc {
  orc_params p;
  int nx, ny, N;
  double sx[2], dx[2];
  double qn[4], qw[4], wgp[4][4];
  double *U, *V;           /* (3,-2:nx+3,-2:ny+3) */
  double *WM, *WP;         /* (3,4,0:nx+1,0:ny+1) */
  double *FX, *FY;         /* (3,0:nx,1:ny), (3,1:nx,0:ny) */
  double *FluxX, *FluxY;   /* (3,4,0:nx,1:ny), (3,4,1:nx,0:ny) */
  double *S, *Ut;          /* (3,1:nx,1:ny) */
  double *FXWB, *FYWB, *SWB;
  int have_wb;
  double *Ua, *Up, *FUp;   /* (4,3,1:nx,1:ny) */
  double *Prod, *Dest;     /* (1:5N) */
  double *ProdUp, *DestUp; /* (4,1:5N) */
  int *RowStart, *Cols, *SIM;
  double *Vtemp;           /* (4,-2:nx+3,1:ny), depth only */
  double *mass, *diag, *rhs, *havec, *solp, *hpk;
  double *EK; /* explicit schemes: 8 stage arrays (3,1:nx,1:ny) */
  double dt;
  int iters[64];
  int nsolves;
  long long total_iters;
};

/* ---- index helpers (Fortran bounds) ---- */
#define NX (o->nx)
#define NY (o->ny)
#define IU(v, i, j) ((v) + 3 * (((i) + 2) + (NX + 6) * ((j) + 2)))
#define IW(v, g, i, j) ((v) + 3 * ((g) - 1) + 12 * ((i) + (NX + 2) * (j)))
#define IFX(v, i, j) ((v) + 3 * ((i) + (NX + 1) * ((j) - 1)))
#define IFY(v, i, j) ((v) + 3 * ((i) - 1 + NX * (j)))
#define IFLX(v, g, i, j) ((v) + 3 * ((g) - 1) + 12 * ((i) + (NX + 1) * ((j) - 1)))
#define IFLY(v, g, i, j) ((v) + 3 * ((g) - 1) + 12 * ((i) - 1 + NX * (j)))
#define IC3(v, i, j) ((v) + 3 * ((i) - 1 + NX * ((j) - 1)))
#define I4(m, v, i, j) (((m) - 1) + 4 * ((v) + 3 * ((i) - 1 + NX * ((j) - 1))))
#define IPU(r, s) (((r) - 1) + 4 * ((s) - 1))
#define ISIM(K, c) (((K) - 1) + o->N * ((c) - 1))
#define IVT(g, i, j) (((g) - 1) + 4 * (((i) + 2) + (NX + 6) * ((j) - 1)))

/* Fortran MODULO for integers (result has the sign of the divisor). */
static inline int fmodulo(int a, int p) {
  int r = a % p;
  return (r < 0) ? r + p : r;
}
/* mesh.f90:157-170 GlobalElem */
static inline int global_elem(const orc_t *o, int ii, int jj) {
  return fmodulo(jj - 1, o->ny) * o->nx + fmodulo(ii - 1, o->nx) + 1;
}
static inline double fmax2(double a, double b) { return (a > b) ? a : b; }
static inline double fmin2(double a, double b) { return (a < b) ? a : b; }

/* mesh.f90:126-129, CASE(4) */
void orc_quadrature(double qn[4], double qw[4]) {
  qw[0] = (18. - sqrt(30.)) / 72.;
  qw[1] = (18. + sqrt(30.)) / 72.;
  qw[2] = (18. + sqrt(30.)) / 72.;
  qw[3] = (18. - sqrt(30.)) / 72.;
  qn[0] = -(0.5 * sqrt(3. / 7. + 2. / 7. * sqrt(6. / 5.)));
  qn[1] = -(0.5 * sqrt(3. / 7. - 2. / 7. * sqrt(6. / 5.)));
  qn[2] = 0.5 * sqrt(3. / 7. - 2. / 7. * sqrt(6. / 5.));
  qn[3] = 0.5 * sqrt(3. / 7. + 2. / 7. * sqrt(6. / 5.));
}

/* timediscretization.f90:491-511, thetaDeC(m,r) stored row-major th[(m-1)*4+(r-1)] */
void orc_theta_mpdec5(double th[16], double beta[4]) {
  static const double colmajor[16] = {
      0.0000000000000000000, 0.1103005664791649049, 0.0730327668541684294, 0.0833333333333333287,
      0.0000000000000000000, 0.1896994335208351257, 0.4505740308958107176, 0.4166666666666666852,
      0.0000000000000000000, -0.0339073642291439076, 0.2269672331458314485, 0.4166666666666666852,
      0.0000000000000000000, 0.0103005664791649201, -0.0269672331458315692, 0.0833333333333333287};
  for (int r = 0; r < 4; ++r)
    for (int m = 0; m < 4; ++m) th[m * 4 + r] = colmajor[r * 4 + m];
  beta[0] = 0.0000000000000000000;
  beta[1] = 0.2763932022500210639;
  beta[2] = 0.7236067977499789361;
  beta[3] = 1.0000000000000000000;
}

/* timediscretization.f90:913-924 */
double orc_patankar_div(double prod, double h) {
  if (h < MIN_DEPTH) return 0.;
  return 2. * h * prod / (h * h + fmax2(h * h, MIN_DEPTH));
}

/* reconstruction.f90:673-755 WENO5_FirstSweep; q[0..4] = Q(-2..2) */
void orc_weno5_first(const double Q[5], double *WM, double *WP) {
  const double qm2 = Q[0], qm1 = Q[1], q0 = Q[2], qp1 = Q[3], qp2 = Q[4];
  double beta1 = (1.0 / 3.0) * (4.0 * qm2 * qm2 - 19.0 * qm2 * qm1 + 25.0 * qm1 * qm1 +
                                11.0 * qm2 * q0 - 31.0 * qm1 * q0 + 10.0 * q0 * q0);
  double beta2 = (1.0 / 3.0) * (4.0 * qm1 * qm1 - 13.0 * qm1 * q0 + 13.0 * q0 * q0 +
                                5.0 * qm1 * qp1 - 13.0 * q0 * qp1 + 4.0 * qp1 * qp1);
  double beta3 = (1.0 / 3.0) * (10.0 * q0 * q0 - 31.0 * q0 * qp1 + 25.0 * qp1 * qp1 +
                                11.0 * q0 * qp2 - 19.0 * qp1 * qp2 + 4.0 * qp2 * qp2);
  double t1 = WENOEPS + beta1, t2 = WENOEPS + beta2, t3 = WENOEPS + beta3;
  double d1 = t1 * t1, d2 = t2 * t2, d3 = t3 * t3;
  double a1, a2, a3, W1, W2, W3;
  /* WM: x_{i-1/2} */
  a1 = (3.0 / 10.0) / d1;
  a2 = (3.0 / 5.0) / d2;
  a3 = (1.0 / 10.0) / d3;
  W1 = (1.0 / 6.0) * (-qm2 + 5.0 * qm1 + 2.0 * q0);
  W2 = (1.0 / 6.0) * (2.0 * qm1 + 5.0 * q0 - qp1);
  W3 = (1.0 / 6.0) * (11.0 * q0 - 7.0 * qp1 + 2.0 * qp2);
  *WM = a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3;
  /* WP: x_{i+1/2} */
  a1 = (1.0 / 10.0) / d1;
  a2 = (3.0 / 5.0) / d2;
  a3 = (3.0 / 10.0) / d3;
  W1 = (1.0 / 6.0) * (2.0 * qm2 - 7.0 * qm1 + 11.0 * q0);
  W2 = (1.0 / 6.0) * (-qm1 + 5.0 * q0 + 2.0 * qp1);
  W3 = (1.0 / 6.0) * (2.0 * q0 + 5.0 * qp1 - qp2);
  *WP = a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3;
}

/* reconstruction.f90:999-1136 WENO5_SecondSweep (4 Gauss points).  The
 * reference's `0.0000000000000000 * Q(k)` terms are dropped: adding a signed
 * zero never changes a non-zero sum. */
void orc_weno5_second(const double Q[5], double W[4]) {
  const double qm2 = Q[0], qm1 = Q[1], q0 = Q[2], qp1 = Q[3], qp2 = Q[4];
  double beta1 = (1.0 / 3.0) * (4.0 * qm2 * qm2 - 19.0 * qm2 * qm1 + 25.0 * qm1 * qm1 +
                                11.0 * qm2 * q0 - 31.0 * qm1 * q0 + 10.0 * q0 * q0);
  double beta2 = (1.0 / 3.0) * (4.0 * qm1 * qm1 - 13.0 * qm1 * q0 + 13.0 * q0 * q0 +
                                5.0 * qm1 * qp1 - 13.0 * q0 * qp1 + 4.0 * qp1 * qp1);
  double beta3 = (1.0 / 3.0) * (10.0 * q0 * q0 - 31.0 * q0 * qp1 + 25.0 * qp1 * qp1 +
                                11.0 * q0 * qp2 - 19.0 * qp1 * qp2 + 4.0 * qp2 * qp2);
  double t1 = WENOEPS + beta1, t2 = WENOEPS + beta2, t3 = WENOEPS + beta3;
  double d1 = t1 * t1, d2 = t2 * t2, d3 = t3 * t3;
  double a1, a2, a3, W1, W2, W3;
  /* point x_{j-1/2 sqrt(3/7+2/7 sqrt(6/5))} */
  a1 = 0.2658420974778319 / d1;
  a2 = 0.6112504900322486 / d2;
  a3 = 0.1229074124899195 / d3;
  W1 = -0.1642562761719537 * qm2 + 0.7590807081409336 * qm1 + 0.4051755680310201 * q0;
  W2 = 0.2663118796250726 * qm1 + 0.8979443965468811 * q0 - 0.1642562761719537 * qp1;
  W3 = 1.6968800354220990 * q0 - 0.9631919150471715 * qp1 + 0.2663118796250726 * qp2;
  W[0] = (a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3);
  /* point x_{j-1/2 sqrt(3/7-2/7 sqrt(6/5))} */
  a1 = 0.1281641584355059 / d1;
  a2 = 0.5219691498503563 / d2;
  a3 = 0.3498666917141379 / d3;
  W1 = -0.1122135388132497 * qm2 + 0.3944175994189276 * qm1 + 0.7177959393943222 * q0;
  W2 = 0.0577769829791784 * qm1 + 1.0544365558340714 * q0 - 0.1122135388132497 * qp1;
  W3 = 1.2277675047716066 * q0 - 0.2855444877507849 * qp1 + 0.0577769829791784 * qp2;
  W[1] = (a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3);
  /* point x_{j+1/2 sqrt(3/7-2/7 sqrt(6/5))} */
  a1 = 0.3498666917141379 / d1;
  a2 = 0.5219691498503563 / d2;
  a3 = 0.1281641584355059 / d3;
  W1 = 0.0577769829791784 * qm2 - 0.2855444877507849 * qm1 + 1.2277675047716066 * q0;
  W2 = -0.1122135388132497 * qm1 + 1.0544365558340714 * q0 + 0.0577769829791784 * qp1;
  W3 = 0.7177959393943222 * q0 + 0.3944175994189276 * qp1 - 0.1122135388132497 * qp2;
  W[2] = (a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3);
  /* point x_{j+1/2 sqrt(3/7+2/7 sqrt(6/5))} */
  a1 = 0.1229074124899195 / d1;
  a2 = 0.6112504900322486 / d2;
  a3 = 0.2658420974778319 / d3;
  W1 = 0.2663118796250726 * qm2 - 0.9631919150471715 * qm1 + 1.6968800354220990 * q0;
  W2 = -0.1642562761719537 * qm1 + 0.8979443965468811 * q0 + 0.2663118796250726 * qp1;
  W3 = 0.4051755680310201 * q0 + 0.7590807081409336 * qp1 - 0.1642562761719537 * qp2;
  W[3] = (a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3);
}

/* equation.f90:419-509 Bathymetry, Bathymetry_X, Bathymetry_Y (+ Gaussian flag 3). */
void orc_bathymetry(const orc_params *p, double x, double y, double *b, double *bx,
                    double *by) {
  const double PI = acos(-1.0);
  double B = 0., BX = 0., BY = 0.;
  switch (p->bathy_flag) {
    case 1:
      B = 0.1 * sin(2. * PI * x) * cos(2. * PI * y);
      BX = 0.1 * 2. * PI * cos(2. * PI * x) * cos(2. * PI * y);
      BY = -(0.1 * 2. * PI * sin(2. * PI * x) * sin(2. * PI * y));
      break;
    case 2: {
      double r2 = x * x + y * y;
      if (r2 < 1) {
        double d = 1.0 - r2;
        double e = exp(1.0 - 1.0 / d);
        B = e;
        BX = -(2.0 * x / (d * d) * e);
        BY = -(2.0 * y / (d * d) * e);
      }
    } break;
    case 3: {
      const double A = p->bathy_par[0], ax = p->bathy_par[1], cx = p->bathy_par[2];
      const double ay = p->bathy_par[3], cy = p->bathy_par[4];
      double dxv = x - cx, dyv = y - cy;
      double e = exp(-(ax * (dxv * dxv) + ay * (dyv * dyv)));
      B = A * e;
      BX = (-2.0 * ax * dxv) * B;
      BY = (-2.0 * ay * dyv) * B;
    } break;
    default:
      break;
  }
  if (b) *b = B;
  if (bx) *bx = BX;
  if (by) *by = BY;
}

static double *dalloc(size_t n) {
  double *p = (double *)calloc(n ? n : 1, sizeof(double));
  return p;
}

orc_t *orc_create(const orc_params *p) {
  if (!p || p->nx < 3 || p->ny < 3) return NULL;
  orc_t *o = (orc_t *)calloc(1, sizeof(orc_t));
  if (!o) return NULL;
  o->p = *p;
  o->nx = p->nx;
  o->ny = p->ny;
  o->N = p->nx * p->ny;
  /* mesh.f90:58-60 */
  o->sx[0] = fabs(p->x1[0] - p->x0[0]);
  o->sx[1] = fabs(p->x1[1] - p->x0[1]);
  o->dx[0] = fabs(o->sx[0]) / ((double)o->nx);
  o->dx[1] = fabs(o->sx[1]) / ((double)o->ny);
  orc_quadrature(o->qn, o->qw);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) o->wgp[a][b] = o->qw[a] * o->qw[b]; /* mesh.f90:139 */
  const size_t nx = o->nx, ny = o->ny, N = o->N;
  o->U = dalloc(3 * (nx + 6) * (ny + 6));
  o->V = dalloc(3 * (nx + 6) * (ny + 6));
  o->WM = dalloc(12 * (nx + 2) * (ny + 2));
  o->WP = dalloc(12 * (nx + 2) * (ny + 2));
  o->FX = dalloc(3 * (nx + 1) * ny);
  o->FY = dalloc(3 * nx * (ny + 1));
  o->FluxX = dalloc(12 * (nx + 1) * ny);
  o->FluxY = dalloc(12 * nx * (ny + 1));
  o->S = dalloc(3 * N);
  o->Ut = dalloc(3 * N);
  o->FXWB = dalloc(3 * (nx + 1) * ny);
  o->FYWB = dalloc(3 * nx * (ny + 1));
  o->SWB = dalloc(3 * N);
  o->Ua = dalloc(12 * N);
  o->Up = dalloc(12 * N);
  o->FUp = dalloc(12 * N);
  o->Prod = dalloc(5 * N);
  o->Dest = dalloc(5 * N);
  o->ProdUp = dalloc(20 * N);
  o->DestUp = dalloc(20 * N);
  o->RowStart = (int *)calloc(N + 1, sizeof(int));
  o->Cols = (int *)calloc(5 * N, sizeof(int));
  o->SIM = (int *)calloc(5 * N, sizeof(int));
  o->Vtemp = dalloc(4 * (nx + 6) * ny);
  o->mass = dalloc(5 * N);
  o->diag = dalloc(N);
  o->rhs = dalloc(N);
  o->havec = dalloc(N);
  o->solp = dalloc(N);
  o->hpk = dalloc(4 * N);
  o->EK = dalloc(24 * N);
  if (!o->EK || !o->U || !o->V || !o->WM || !o->WP || !o->FX || !o->FY || !o->FluxX || !o->FluxY ||
      !o->S || !o->Ut || !o->FXWB || !o->FYWB || !o->SWB || !o->Ua || !o->Up || !o->FUp ||
      !o->Prod || !o->Dest || !o->ProdUp || !o->DestUp || !o->RowStart || !o->Cols || !o->SIM ||
      !o->Vtemp || !o->mass || !o->diag || !o->rhs || !o->havec || !o->solp || !o->hpk) {
    orc_destroy(o);
    return NULL;
  }
  /* finitevolume.f90:219-267 CSR pattern (1-based values) */
  int isv = 0, irs = 0;
  for (int jj = 1; jj <= o->ny; ++jj)
    for (int ii = 1; ii <= o->nx; ++ii) {
      int K = global_elem(o, ii, jj);
      isv += 1;
      irs += 1;
      o->RowStart[irs - 1] = isv;
      o->Cols[isv - 1] = global_elem(o, ii, jj - 1);
      o->SIM[ISIM(K, 1)] = isv;
      isv += 1;
      o->Cols[isv - 1] = global_elem(o, ii - 1, jj);
      o->SIM[ISIM(K, 2)] = isv;
      isv += 1;
      o->Cols[isv - 1] = global_elem(o, ii, jj);
      o->SIM[ISIM(K, 3)] = isv;
      isv += 1;
      o->Cols[isv - 1] = global_elem(o, ii + 1, jj);
      o->SIM[ISIM(K, 4)] = isv;
      isv += 1;
      o->Cols[isv - 1] = global_elem(o, ii, jj + 1);
      o->SIM[ISIM(K, 5)] = isv;
    }
  o->RowStart[o->N] = o->RowStart[o->N - 1] + 5;
  return o;
}

void orc_destroy(orc_t *o) {
  if (!o) return;
  double **arrs[] = {&o->U, &o->V, &o->WM, &o->WP, &o->FX, &o->FY, &o->FluxX, &o->FluxY,
                     &o->S, &o->Ut, &o->FXWB, &o->FYWB, &o->SWB, &o->Ua, &o->Up, &o->FUp,
                     &o->Prod, &o->Dest, &o->ProdUp, &o->DestUp, &o->Vtemp, &o->mass,
                     &o->diag, &o->rhs, &o->havec, &o->solp, &o->hpk, &o->EK};
  for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k) free(*arrs[k]);
  free(o->RowStart);
  free(o->Cols);
  free(o->SIM);
  free(o);
}

/* equation.f90:912-945 ConsToPrim */
static inline void cons_to_prim(const double *c, double *p) {
  double h = c[0], ht = h + MIN_DEPTH / h;
  p[0] = h;
  p[1] = c[1] / ht;
  p[2] = c[2] / ht;
}

/* equation.f90:515-785, periodic branches, then V = ConsToPrim(U) */
static void boundary_conditions(orc_t *o) {
  double *U = o->U;
  const int nx = NX, ny = NY;
  for (int jj = 1; jj <= ny; ++jj) /* left */
    for (int ii = 0; ii <= 2; ++ii)
      for (int v = 0; v < 3; ++v) U[IU(v, -2 + ii, jj)] = U[IU(v, nx - 2 + ii, jj)];
  for (int jj = 1; jj <= ny; ++jj) /* right */
    for (int ii = 1; ii <= 3; ++ii)
      for (int v = 0; v < 3; ++v) U[IU(v, nx + ii, jj)] = U[IU(v, ii, jj)];
  for (int ii = 1; ii <= nx; ++ii) /* top */
    for (int jj = 1; jj <= 3; ++jj)
      for (int v = 0; v < 3; ++v) U[IU(v, ii, ny + jj)] = U[IU(v, ii, jj)];
  for (int ii = 1; ii <= nx; ++ii) /* bottom */
    for (int jj = 0; jj <= 2; ++jj)
      for (int v = 0; v < 3; ++v) U[IU(v, ii, -2 + jj)] = U[IU(v, ii, ny - 2 + jj)];
  for (int pass = 0; pass < 2; ++pass) { /* upper corners */
    int jlo = pass ? ny + 1 : -2, jhi = pass ? ny + 3 : 0;
    for (int jj = jlo; jj <= jhi; ++jj)
      for (int ii = 0; ii <= 2; ++ii)
        for (int v = 0; v < 3; ++v) U[IU(v, -2 + ii, jj)] = U[IU(v, nx - 2 + ii, jj)];
  }
  for (int pass = 0; pass < 2; ++pass) { /* right corners */
    int jlo = pass ? ny + 1 : -2, jhi = pass ? ny + 3 : 0;
    for (int jj = jlo; jj <= jhi; ++jj)
      for (int ii = 1; ii <= 3; ++ii)
        for (int v = 0; v < 3; ++v) U[IU(v, nx + ii, jj)] = U[IU(v, ii, jj)];
  }
  OMP_FOR
  for (int jj = -2; jj <= ny + 3; ++jj)
    for (int ii = -2; ii <= nx + 3; ++ii) cons_to_prim(&U[IU(0, ii, jj)], &o->V[IU(0, ii, jj)]);
}

/* reconstruction.f90:54-116 (CASE 4) + WENO_XDIR :408-458 */
static void reconstruction_x(orc_t *o) {
  const int nx = NX, ny = NY;
  OMP_FOR
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 0; ii <= nx + 1; ++ii)
      for (int v = 0; v < 3; ++v) {
        double tm[5], tp[5], q[5], w[4];
        for (int jl = -2; jl <= 2; ++jl) {
          for (int k = 0; k < 5; ++k) q[k] = o->V[IU(v, ii - 2 + k, jj + jl)];
          orc_weno5_first(q, &tm[jl + 2], &tp[jl + 2]);
        }
        orc_weno5_second(tm, w);
        for (int g = 1; g <= 4; ++g) o->WM[IW(v, g, ii, jj)] = w[g - 1];
        orc_weno5_second(tp, w);
        for (int g = 1; g <= 4; ++g) o->WP[IW(v, g, ii, jj)] = w[g - 1];
      }
}

/* reconstruction.f90:122-184 (CASE 4) + WENO_YDIR :464-514 */
static void reconstruction_y(orc_t *o) {
  const int nx = NX, ny = NY;
  OMP_FOR
  for (int jj = 0; jj <= ny + 1; ++jj)
    for (int ii = 1; ii <= nx; ++ii)
      for (int v = 0; v < 3; ++v) {
        double tm[5], tp[5], q[5], w[4];
        for (int il = -2; il <= 2; ++il) {
          for (int k = 0; k < 5; ++k) q[k] = o->V[IU(v, ii + il, jj - 2 + k)];
          orc_weno5_first(q, &tm[il + 2], &tp[il + 2]);
        }
        orc_weno5_second(tm, w);
        for (int g = 1; g <= 4; ++g) o->WM[IW(v, g, ii, jj)] = w[g - 1];
        orc_weno5_second(tp, w);
        for (int g = 1; g <= 4; ++g) o->WP[IW(v, g, ii, jj)] = w[g - 1];
      }
}

/* finitevolume.f90:669-694 (x) and :730-754 (y), body shared */
static inline void limit_cell(const orc_t *o, double Vc, double *wm, double *wp, int stride) {
  double alpha = 0., beta = 0.;
  for (int g = 0; g < 4; ++g) {
    alpha = alpha + o->qw[g] * wm[g * stride];
    beta = beta + o->qw[g] * wp[g * stride];
  }
  double csi = (Vc - wLobatto * alpha - wLobatto * beta) / (1. - 2. * wLobatto);
  for (int g = 0; g < 4; ++g) {
    double mmin = csi;
    if (wm[g * stride] < mmin) mmin = wm[g * stride];
    if (wp[g * stride] < mmin) mmin = wp[g * stride];
    double theta;
    if (Vc == mmin)
      theta = 1.;
    else
      theta = fmin2(1., fabs((Vc - MIN_DEPTH) / (Vc - mmin)));
    wp[g * stride] = Vc + theta * (wp[g * stride] - Vc);
    wm[g * stride] = Vc + theta * (wm[g * stride] - Vc);
  }
}
static void positivity_limiter_x(orc_t *o) {
  OMP_FOR
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 0; ii <= NX; ++ii)
      limit_cell(o, o->V[IU(0, ii, jj)], &o->WM[IW(0, 1, ii, jj)], &o->WP[IW(0, 1, ii, jj)], 3);
}
static void positivity_limiter_y(orc_t *o) {
  OMP_FOR
  for (int jj = 0; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      limit_cell(o, o->V[IU(0, ii, jj)], &o->WM[IW(0, 1, ii, jj)], &o->WP[IW(0, 1, ii, jj)], 3);
}

/* equation.f90:988-1106 EvaluateFlux1D + WaveSpeeds1D + RiemannSolverByRusanov on the
 * face-normal frame.  The reference rotates with n=(1,0),t=(0,1) for x faces and
 * n=(0,1),t=(-1,0) for y faces (:1048-1069); those products with 0 and +-1 are exact,
 * so the x face uses (h,u,v) and the y face (h,v,u) with the flux components mapped
 * back as (F1, F3', F2'), value-identical to the rotated form. */
static inline void rusanov(double g, const double *PL, const double *PR, double *F) {
  double hL = PL[0], uL = PL[1], vL = PL[2];
  double hR = PR[0], uR = PR[1], vR = PR[2];
  double FL[3], FR[3], CL[3], CR[3];
  FL[0] = hL * uL;
  FL[1] = hL * (uL * uL) + 0.5 * g * (hL * hL);
  FL[2] = hL * uL * vL;
  FR[0] = hR * uR;
  FR[1] = hR * (uR * uR) + 0.5 * g * (hR * hR);
  FR[2] = hR * uR * vR;
  double fastL = uL + sqrt(g * hL), fastR = uR + sqrt(g * hR);
  double lam = fmax2(fabs(fastL), fabs(fastR));
  CL[0] = hL;
  CL[1] = hL * uL;
  CL[2] = hL * vL;
  CR[0] = hR;
  CR[1] = hR * uR;
  CR[2] = hR * vR;
  for (int v = 0; v < 3; ++v) F[v] = 0.5 * ((FL[v] + FR[v]) - lam * (CR[v] - CL[v]));
}

/* finitevolume.f90:546-590 NumericalFluxFX */
static void numerical_flux_x(orc_t *o) {
  const double g = o->p.g;
  OMP_FOR
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 0; ii <= NX; ++ii)
      for (int q = 1; q <= 4; ++q) {
        double PL[3], PR[3], F[3];
        for (int v = 0; v < 3; ++v) {
          PL[v] = o->WP[IW(v, q, ii, jj)];
          PR[v] = o->WM[IW(v, q, ii + 1, jj)];
        }
        rusanov(g, PL, PR, F);
        for (int v = 0; v < 3; ++v) o->FluxX[IFLX(v, q, ii, jj)] = F[v];
      }
  OMP_FOR
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 0; ii <= NX; ++ii)
      for (int v = 0; v < 3; ++v) {
        double s = 0.0;
        for (int q = 1; q <= 4; ++q) s = s + o->qw[q - 1] * o->FluxX[IFLX(v, q, ii, jj)];
        o->FX[IFX(v, ii, jj)] = s;
      }
}

/* finitevolume.f90:596-640 NumericalFluxFY */
static void numerical_flux_y(orc_t *o) {
  const double g = o->p.g;
  OMP_FOR
  for (int jj = 0; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int q = 1; q <= 4; ++q) {
        double PL[3], PR[3], F[3];
        PL[0] = o->WP[IW(0, q, ii, jj)];
        PL[1] = o->WP[IW(2, q, ii, jj)];
        PL[2] = o->WP[IW(1, q, ii, jj)];
        PR[0] = o->WM[IW(0, q, ii, jj + 1)];
        PR[1] = o->WM[IW(2, q, ii, jj + 1)];
        PR[2] = o->WM[IW(1, q, ii, jj + 1)];
        rusanov(g, PL, PR, F);
        o->FluxY[IFLY(0, q, ii, jj)] = F[0];
        o->FluxY[IFLY(1, q, ii, jj)] = F[2];
        o->FluxY[IFLY(2, q, ii, jj)] = F[1];
      }
  OMP_FOR
  for (int jj = 0; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int v = 0; v < 3; ++v) {
        double s = 0.0;
        for (int q = 1; q <= 4; ++q) s = s + o->qw[q - 1] * o->FluxY[IFLY(v, q, ii, jj)];
        o->FY[IFY(v, ii, jj)] = s;
      }
}

/* mesh.f90:62-72,142: x coordinate of Gauss node q (0-based) of column ii (1-based) */
static inline double gp_coord(const orc_t *o, int d, int ii, int q) {
  double node = o->p.x0[d] + ((double)(ii - 1)) * o->dx[d];
  double bary = node + 0.5 * o->dx[d];
  return bary + o->qn[q] * o->dx[d];
}

/* equation.f90:284-392 SourceTerms (CASE 4), :398-413 SourceFunc.  Only the depth is
 * reconstructed: SourceFunc reads Q(1) alone (:409-410). */
static void source_terms(orc_t *o) {
  const int nx = NX, ny = NY;
  memset(o->S, 0, sizeof(double) * 3 * o->N);
  if (o->p.bathy_flag <= 0) return;
  OMP_FOR
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = -2; ii <= nx + 3; ++ii) {
      double q[5], w[4];
      for (int k = 0; k < 5; ++k) q[k] = o->U[IU(0, ii, jj - 2 + k)];
      orc_weno5_second(q, w);
      for (int g = 1; g <= 4; ++g) o->Vtemp[IVT(g, ii, jj)] = w[g - 1];
    }
  const double grav = o->p.g;
  OMP_FOR
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii) {
      double sw[4][4][3]; /* SW(1:3, xGP, yGP) */
      for (int iGP = 1; iGP <= 4; ++iGP) {
        double q[5], w[4];
        for (int k = 0; k < 5; ++k) q[k] = o->Vtemp[IVT(iGP, ii - 2 + k, jj)];
        orc_weno5_second(q, w);
        for (int jGP = 1; jGP <= 4; ++jGP) {
          double X = gp_coord(o, 0, ii, jGP - 1), Y = gp_coord(o, 1, jj, iGP - 1);
          double bx, by;
          orc_bathymetry(&o->p, X, Y, NULL, &bx, &by);
          double h = w[jGP - 1];
          sw[jGP - 1][iGP - 1][0] = 0.;
          sw[jGP - 1][iGP - 1][1] = -(grav * h * bx);
          sw[jGP - 1][iGP - 1][2] = -(grav * h * by);
        }
      }
      for (int v = 0; v < 3; ++v) {
        double s = 0.0;
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b) s = s + o->wgp[a][b] * sw[a][b][v];
        o->S[IC3(v, ii, jj)] = s;
      }
    }
}

/* finitevolume.f90:446-540 UpdateTimeDerivative (PATANKAR [+WELLBALANCED]) */
static void update_time_derivative(orc_t *o, int wb) {
  const int nx = NX, ny = NY;
  if (wb) {
    for (size_t k = 0; k < (size_t)3 * (nx + 1) * ny; ++k) o->FX[k] = o->FX[k] - o->FXWB[k];
    for (size_t k = 0; k < (size_t)3 * nx * (ny + 1); ++k) o->FY[k] = o->FY[k] - o->FYWB[k];
    for (size_t k = 0; k < (size_t)3 * o->N; ++k) o->S[k] = o->S[k] - o->SWB[k];
  }
  const double dx = o->dx[0], dy = o->dx[1];
  OMP_FOR
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii) {
      size_t isv = (size_t)5 * ((jj - 1) * nx + (ii - 1)); /* 0-based slot of S neighbour */
      double f;
      f = o->FY[IFY(0, ii, jj - 1)];
      o->Prod[isv + 0] = fmax2(f, 0.) / dy;
      o->Dest[isv + 0] = -fmin2(f, 0.) / dy;
      f = o->FX[IFX(0, ii - 1, jj)];
      o->Prod[isv + 1] = fmax2(f, 0.) / dx;
      o->Dest[isv + 1] = -fmin2(f, 0.) / dx;
      o->Prod[isv + 2] = 0.;
      o->Dest[isv + 2] = 0.;
      f = -o->FX[IFX(0, ii, jj)];
      o->Prod[isv + 3] = fmax2(f, 0.) / dx;
      o->Dest[isv + 3] = -fmin2(f, 0.) / dx;
      f = -o->FY[IFY(0, ii, jj)];
      o->Prod[isv + 4] = fmax2(f, 0.) / dy;
      o->Dest[isv + 4] = -fmin2(f, 0.) / dy;
      /* Ut(2:3) in the PATANKAR build; Ut(1) as the build without it computes
       * (finitevolume.f90:530-533), used by the explicit schemes only */
      for (int v = 0; v < 3; ++v)
        o->Ut[IC3(v, ii, jj)] = o->S[IC3(v, ii, jj)] -
                                (o->FX[IFX(v, ii, jj)] - o->FX[IFX(v, ii - 1, jj)]) / dx -
                                (o->FY[IFY(v, ii, jj)] - o->FY[IFY(v, ii, jj - 1)]) / dy;
    }
}

/* finitevolume.f90:402-440 FVTimeDerivative (shock indicator and Fix pass omitted:
 * ReconstructionFix == Reconstruction makes them result-identical). */
static void fv_time_derivative(orc_t *o, int wb) {
  boundary_conditions(o);
  reconstruction_x(o);
  positivity_limiter_x(o);
  numerical_flux_x(o);
  reconstruction_y(o);
  positivity_limiter_y(o);
  numerical_flux_y(o);
  source_terms(o);
  update_time_derivative(o, wb);
}

void orc_rhs(orc_t *o, double *Ut, double *FX, double *FY, double *S, double *prod,
             double *dest) {
  fv_time_derivative(o, o->p.well_balanced && o->have_wb);
  const size_t N = o->N;
  if (Ut) memcpy(Ut, o->Ut, sizeof(double) * 3 * N);
  if (FX) memcpy(FX, o->FX, sizeof(double) * 3 * (o->nx + 1) * o->ny);
  if (FY) memcpy(FY, o->FY, sizeof(double) * 3 * o->nx * (o->ny + 1));
  if (S) memcpy(S, o->S, sizeof(double) * 3 * N);
  if (prod) memcpy(prod, o->Prod, sizeof(double) * 5 * N);
  if (dest) memcpy(dest, o->Dest, sizeof(double) * 5 * N);
}

/* equation.f90:791-837 TimeStep + WaveSpeeds2D :880-906 */
double orc_timestep(orc_t *o) {
  double LX = 0.0, LY = 0.0, ts = DBL_MAX;
  const double g = o->p.g;
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii) {
      double prim[3];
      cons_to_prim(&o->U[IU(0, ii, jj)], prim);
      double fx = prim[1] + sqrt(g * prim[0]);
      double fy = prim[2] + sqrt(g * prim[0]);
      LX = fmax2(LX, fabs(fx));
      LY = fmax2(LY, fabs(fy));
      double a = o->dx[0] / LX, b = o->dx[1] / LY;
      if (a < ts) ts = a;
      if (b < ts) ts = b;
    }
  ts = o->p.cfl * ts;
  if (ts < MIN_TIMESTEP) ts = MIN_TIMESTEP;
  return ts;
}

/* jacobi_iteration.f90:25-43 sparse_matmul and :52-87 jacobi */
static int jacobi_solve(orc_t *o, const double *mv, const double *diag, const double *rhs,
                        double *sol) {
  const int n = o->N;
  const int maxIter = o->p.jacobi_maxiter;
  const double tol = o->p.jacobi_tol;
  double *solp = o->solp;
  int k = 0;
  double residual = 0.;
  for (int i = 0; i < n; ++i) {
    solp[i] = rhs[i];
    sol[i] = 0.;
  }
  for (int i = 0; i < n; ++i) residual = residual + fabs(sol[i] - solp[i]);
  residual = residual / (double)n;
  while ((tol < residual) && (k < maxIter)) {
    k = k + 1;
    OMP_FOR
    for (int row = 1; row <= n; ++row) {
      double prod = 0.;
      for (int sp = o->RowStart[row - 1]; sp <= o->RowStart[row] - 1; ++sp)
        prod = prod + mv[sp - 1] * solp[o->Cols[sp - 1] - 1];
      sol[row - 1] = (rhs[row - 1] - prod) / diag[row - 1];
    }
    residual = 0.;
#ifdef ORC_OMP
#pragma omp parallel for reduction(+ : residual) schedule(static)
#endif
    for (int i = 0; i < n; ++i) residual = residual + fabs(sol[i] - solp[i]);
    residual = residual / (double)n;
    memcpy(solp, sol, sizeof(double) * n);
  }
  o->total_iters += k;
  if (o->nsolves < 64) o->iters[o->nsolves] = k;
  o->nsolves++;
  return k;
}

int orc_jacobi(orc_t *o, const double *mass, const double *diag, const double *rhs,
               double *sol) {
  return jacobi_solve(o, mass, diag, rhs, sol);
}

/* hp(m,i,j) read by MODIFIED_PATANKAR_MATRIX_INVERSION (timediscretization.f90:784).
 * msteps == 4: Up(m,1,i,j).  msteps == 2 with mpdec2_compat: the dummy hp(2,nx,ny)
 * associated with the packed (4,nx,ny) temporary of Up(:,1,:,:). */
static inline double hp_read(const orc_t *o, int msteps, int m, int i, int j) {
  if (msteps == 2 && o->p.mpdec2_compat) {
    long L = (long)(m - 1) + 2L * ((i - 1) + (long)o->nx * (j - 1));
    int a = (int)(L % 4) + 1;
    long c = L / 4;
    int ic = (int)(c % o->nx) + 1, jc = (int)(c / o->nx) + 1;
    return o->Up[I4(a, 0, ic, jc)];
  }
  return o->Up[I4(m, 0, i, j)];
}

/* timediscretization.f90:771-908 MODIFIED_PATANKAR_MATRIX_INVERSION */
static void patankar_inversion(orc_t *o, int m, int msteps, const double *theta /*[m][r] 4x4*/) {
  const int nx = NX, ny = NY;
  const double dt = o->dt;
  double *Mass = o->mass, *Diag = o->diag, *rhs = o->rhs;
  for (int k = 0; k < 5 * o->N; ++k) Mass[k] = 0.;
  for (int k = 0; k < o->N; ++k) Diag[k] = 1.;
  OMP_FOR
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii) {
      const int K = global_elem(o, ii, jj);
      const int nbr_i[4] = {ii, fmodulo(ii - 2, nx) + 1, fmodulo(ii, nx) + 1, ii};
      const int nbr_j[4] = {fmodulo(jj - 2, ny) + 1, jj, jj, fmodulo(jj, ny) + 1};
      const int slot[4] = {1, 2, 4, 5};
      const double hK = hp_read(o, msteps, m, ii, jj);
      for (int nb = 0; nb < 4; ++nb) {
        const int KL = o->SIM[ISIM(K, slot[nb])];
        const double hL = hp_read(o, msteps, m, nbr_i[nb], nbr_j[nb]);
        for (int rr = 1; rr <= msteps; ++rr) {
          const double th = theta[(m - 1) * 4 + (rr - 1)];
          if (th > 0.) {
            Mass[KL - 1] = Mass[KL - 1] - dt * th * (orc_patankar_div(o->ProdUp[IPU(rr, KL)], hL));
            Diag[K - 1] = Diag[K - 1] + dt * th * (orc_patankar_div(o->DestUp[IPU(rr, KL)], hK));
          } else {
            Diag[K - 1] = Diag[K - 1] - dt * th * (orc_patankar_div(o->ProdUp[IPU(rr, KL)], hK));
            Mass[KL - 1] = Mass[KL - 1] + dt * th * (orc_patankar_div(o->DestUp[IPU(rr, KL)], hL));
          }
        }
      }
      rhs[global_elem(o, ii, jj) - 1] = hp_read(o, msteps, 1, ii, jj);
    }
  for (int k = 0; k < o->N; ++k) o->havec[k] = 0.;
  jacobi_solve(o, Mass, Diag, rhs, o->havec);
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii) o->Ua[I4(m, 0, ii, jj)] = o->havec[global_elem(o, ii, jj) - 1];
}

static void store_rhs(orc_t *o, int m) {
  const int nx = NX, ny = NY;
  for (int jj = 1; jj <= ny; ++jj)
    for (int ii = 1; ii <= nx; ++ii)
      for (int v = 1; v < 3; ++v) o->FUp[I4(m, v, ii, jj)] = o->Ut[IC3(v, ii, jj)];
  for (int s = 1; s <= 5 * o->N; ++s) {
    o->ProdUp[IPU(m, s)] = o->Prod[s - 1];
    o->DestUp[IPU(m, s)] = o->Dest[s - 1];
  }
}

static void load_state_from_ua(orc_t *o, int m) {
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int v = 0; v < 3; ++v) o->U[IU(v, ii, jj)] = o->Ua[I4(m, v, ii, jj)];
}

static int explicit_step(orc_t *o, double dt);

/* timediscretization.f90:458-566 (mPDeC5: MSteps=4, KCorr=5), :571-664 (mPDeC2:
 * MSteps=2, KCorr=2), :671-764 (mPEuler: MSteps=2, KCorr=1); schemes 1-4 below. */
int orc_step(orc_t *o, double t, double dt) {
  (void)t; /* stage times are unused by the periodic BC and the source term */
  if (o->p.timescheme >= 1 && o->p.timescheme <= 4) return explicit_step(o, dt);
  const int nx = NX, ny = NY;
  int msteps, kcorr;
  double theta[16];
  memset(theta, 0, sizeof(theta));
  if (o->p.timescheme == 7 || o->p.timescheme == 6) {
    msteps = 2;
    kcorr = o->p.timescheme == 7 ? 2 : 1;
    theta[1 * 4 + 0] = 0.5; /* thetaDeC(2,1) */
    theta[1 * 4 + 1] = 0.5; /* thetaDeC(2,2) */
  } else {
    double beta[4];
    msteps = 4;
    kcorr = 5;
    orc_theta_mpdec5(theta, beta);
  }
  const int wb = o->p.well_balanced && o->have_wb;
  o->dt = dt;
  o->nsolves = 0;
  for (int m = 1; m <= msteps; ++m)
    for (int jj = 1; jj <= ny; ++jj)
      for (int ii = 1; ii <= nx; ++ii)
        for (int v = 0; v < 3; ++v) {
          o->Ua[I4(m, v, ii, jj)] = o->U[IU(v, ii, jj)];
          o->Up[I4(m, v, ii, jj)] = o->U[IU(v, ii, jj)];
        }
  fv_time_derivative(o, wb);
  for (int m = 1; m <= msteps; ++m) store_rhs(o, m);
  for (int kk = 1; kk <= kcorr; ++kk) {
    int mlo = (kk == kcorr) ? msteps : 2;
    for (int ii = mlo; ii <= msteps; ++ii) {
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int v = 1; v < 3; ++v) {
            double acc = o->Ua[I4(1, v, i, j)];
            for (int jj = 1; jj <= msteps; ++jj)
              acc = acc + dt * theta[(ii - 1) * 4 + (jj - 1)] * o->FUp[I4(jj, v, i, j)];
            o->Ua[I4(ii, v, i, j)] = acc;
          }
      patankar_inversion(o, ii, msteps, theta);
    }
    if (kk != kcorr) {
      for (int ii = 2; ii <= msteps; ++ii) {
        load_state_from_ua(o, ii);
        fv_time_derivative(o, wb);
        store_rhs(o, ii);
      }
    }
    memcpy(o->Up, o->Ua, sizeof(double) * 12 * o->N);
  }
  load_state_from_ua(o, msteps);
  int warn = 0;
  for (int s = 0; s < o->nsolves && s < 64; ++s)
    if (o->iters[s] >= o->p.jacobi_maxiter) warn = 1;
  return warn;
}

/* ---- explicit schemes (build without PATANKAR: Ut(1) from the mass fluxes) ---- */
static double *ek(orc_t *o, int k) { return o->EK + (size_t)k * 3 * o->N; }

static void copy_state_out(const orc_t *o, double *X) {
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int v = 0; v < 3; ++v) X[IC3(v, ii, jj)] = o->U[IU(v, ii, jj)];
}
static void copy_state_in(orc_t *o, const double *X) {
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int v = 0; v < 3; ++v) o->U[IU(v, ii, jj)] = X[IC3(v, ii, jj)];
}

/* TimeDiscretizationByForwardEuler :200-242, BySSPRK4 :104-195, ByRK65 :247-348,
 * ByDeC5 :353-451, each expression in the reference's evaluation order. */
static int explicit_step(orc_t *o, double dt) {
  const int wb = o->p.well_balanced && o->have_wb;
  const size_t n3 = (size_t)3 * o->N;
  const double *Ut = o->Ut;
  o->dt = dt;
  o->nsolves = 0;
  switch (o->p.timescheme) {
    case 1: { /* U = K0 + Ut dt */
      double *K0 = ek(o, 0);
      copy_state_out(o, K0);
      fv_time_derivative(o, wb);
      for (size_t k = 0; k < n3; ++k) K0[k] = K0[k] + Ut[k] * dt;
      copy_state_in(o, K0);
    } break;
    case 2: { /* SSPRK(5,4) */
      double *K0 = ek(o, 0), *K1 = ek(o, 1), *K2 = ek(o, 2), *K3 = ek(o, 3), *K4 = ek(o, 4),
             *K5 = ek(o, 5);
      copy_state_out(o, K0);
      fv_time_derivative(o, wb);
      for (size_t k = 0; k < n3; ++k)
        K1[k] = 1.00000000000000 * K0[k] + 0.39175222700392 * Ut[k] * dt;
      copy_state_in(o, K1);
      fv_time_derivative(o, wb);
      for (size_t k = 0; k < n3; ++k)
        K2[k] = 0.44437049406734 * K0[k] + 0.55562950593266 * K1[k] +
                0.36841059262959 * Ut[k] * dt;
      copy_state_in(o, K2);
      fv_time_derivative(o, wb);
      for (size_t k = 0; k < n3; ++k)
        K3[k] = 0.62010185138540 * K0[k] + 0.37989814861460 * K2[k] +
                0.25189177424738 * Ut[k] * dt;
      copy_state_in(o, K3);
      fv_time_derivative(o, wb);
      for (size_t k = 0; k < n3; ++k) {
        K4[k] = 0.17807995410773 * K0[k] + 0.82192004589227 * K3[k] +
                0.54497475021237 * Ut[k] * dt;
        K5[k] = Ut[k];
      }
      copy_state_in(o, K4);
      fv_time_derivative(o, wb);
      double *Un = ek(o, 6);
      for (size_t k = 0; k < n3; ++k)
        Un[k] = 0.00683325884039 * K0[k] + 0.51723167208978 * K2[k] + 0.12759831133288 * K3[k] +
                0.34833675773694 * K4[k] + 0.08460416338212 * K5[k] * dt +
                0.22600748319395 * Ut[k] * dt;
      copy_state_in(o, Un);
    } break;
    case 3: { /* RK65: ARK(6,5) column-major, bRK, cRK */
      static const double A[6][5] = {{0., 0., 0., 0., 0.},
                                     {0.25, 0., 0., 0., 0.},
                                     {0.125, 0.125, 0., 0., 0.},
                                     {0., 0., 0.5, 0., 0.},
                                     {0.1875, -0.375, 0.375, 0.5625, 0.},
                                     {-0.42857142857142855, 1.1428571428571428, 0.8571428571428571,
                                      -1.7142857142857142, 1.1428571428571428}};
      static const double b[6] = {0.077777777777777778, 0., 0.35555555555555556,
                                  0.13333333333333333, 0.35555555555555556, 0.077777777777777778};
      double *UN0 = ek(o, 6), *St = ek(o, 7);
      copy_state_out(o, UN0);
      fv_time_derivative(o, wb);
      memcpy(ek(o, 0), Ut, sizeof(double) * n3);
      for (int st = 1; st <= 5; ++st) { /* stage st uses K0..K(st-1) */
        for (size_t k = 0; k < n3; ++k) {
          double acc = A[st][0] * ek(o, 0)[k];
          for (int j = 1; j < st; ++j) acc = acc + A[st][j] * ek(o, j)[k];
          St[k] = UN0[k] + acc * dt;
        }
        copy_state_in(o, St);
        fv_time_derivative(o, wb);
        memcpy(ek(o, st), Ut, sizeof(double) * n3);
      }
      for (size_t k = 0; k < n3; ++k) {
        double acc = b[0] * ek(o, 0)[k];
        for (int j = 1; j < 6; ++j) acc = acc + b[j] * ek(o, j)[k];
        St[k] = UN0[k] + acc * dt;
      }
      copy_state_in(o, St);
    } break;
    case 4: { /* DeC5: MSteps 4, KCorr 5, the mPDeC5 theta table */
      double theta[16], beta[4];
      orc_theta_mpdec5(theta, beta);
      /* Ua(m) in ek(m-1), FUp(m) in o->FUp-like storage ek(4..7) */
      for (int m = 0; m < 4; ++m) copy_state_out(o, ek(o, m));
      fv_time_derivative(o, wb);
      for (int m = 0; m < 4; ++m) memcpy(ek(o, 4 + m), Ut, sizeof(double) * n3);
      for (int kk = 1; kk <= 5; ++kk) {
        const int mlo = (kk == 5) ? 4 : 2;
        for (int ii = mlo; ii <= 4; ++ii) {
          double *Ua = ek(o, ii - 1);
          const double *U1 = ek(o, 0);
          for (size_t k = 0; k < n3; ++k) {
            double acc = U1[k];
            for (int jj = 1; jj <= 4; ++jj)
              acc = acc + dt * theta[(ii - 1) * 4 + (jj - 1)] * ek(o, 3 + jj)[k];
            Ua[k] = acc;
          }
        }
        if (kk != 5)
          for (int ii = 2; ii <= 4; ++ii) {
            copy_state_in(o, ek(o, ii - 1));
            fv_time_derivative(o, wb);
            memcpy(ek(o, 3 + ii), Ut, sizeof(double) * n3);
          }
      }
      copy_state_in(o, ek(o, 3));
    } break;
    default:
      return -1;
  }
  return 0;
}

/* timediscretization.f90:46-95 without output */
int orc_run(orc_t *o, double tend, int n_outputs, double *t_out) {
  double t = 0.0;
  double dt_an = tend / (double)n_outputs;
  double t_an = t + dt_an;
  int steps = 0;
  if (t == tend) {
    if (t_out) *t_out = t;
    return 0;
  }
  for (;;) {
    double dt_min = orc_timestep(o);
    double a = fmin2(dt_min, t_an - t), b = fmin2(dt_min, tend - t);
    double dt = fmin2(a, b);
    orc_step(o, t, dt);
    steps++;
    t = t + dt;
    if (fabs(t_an - t) < 1.0e-10) {
      t_an = t_an + dt_an;
      if (t_an > tend) t_an = tend;
    }
    if (fabs(t - tend) < 1.0e-10) break;
  }
  if (t_out) *t_out = t;
  return steps;
}

/* ---------------- initial conditions (driver side) ---------------- */

/* Fortran MODULO for reals */
static inline double rmodulo(double a, double p) { return a - floor(a / p) * p; }

/* equation.f90:70-230 ExactFunction at time t (only case 1, the vortex advected by
 * (u_inf, v_inf), depends on t), plus the new benchmark cases. */
static void exact_function(const orc_t *o, int ic, const double *par, double t, double x,
                           double y, double cons[3]) {
  const double PI = acos(-1.0);
  const double g = o->p.g;
  double prim[3] = {0., 0., 0.};
  double b;
  switch (ic) {
    case 1: { /* unsteady smooth vortex */
      double u_inf = 2., v_inf = 3., H_inf = 1.;
      double xm0 = o->p.x0[0] + 0.5 * o->sx[0], xm1 = o->p.x0[1] + 0.5 * o->sx[1];
      double xc0 = rmodulo(x - u_inf * t - o->p.x0[0], o->sx[0]) + o->p.x0[0] - xm0;
      double xc1 = rmodulo(y - v_inf * t - o->p.x0[1], o->sx[1]) + o->p.x0[1] - xm1;
      double r = xc0 * xc0 + xc1 * xc1;
      prim[0] = H_inf;
      prim[1] = u_inf;
      prim[2] = v_inf;
      if (r < 1) {
        double ar = atan(r - 1.);
        double hd = 3. * 0.1 * exp(1. / pow(ar, 3.)) / (pow(ar, 4) * ((r - 1.) * (r - 1.) + 1.));
        double omega = sqrt(2. * g * hd);
        prim[0] = 1. - 0.1 * exp(-1. / pow(atan(1. - r), 3.));
        prim[1] = prim[1] + omega * (+xc1);
        prim[2] = prim[2] + omega * (-xc0);
      }
    } break;
    case 2:
      prim[0] = 1. - 0.1 * sin(2. * PI * x) * cos(2. * PI * y);
      break;
    case 3: {
      orc_bathymetry(&o->p, x, y, &b, NULL, NULL);
      prim[0] = fmax2(0.7 - b, MIN_DEPTH);
      double r2 = ((x + 2) * (x + 2) + (y - 0.5) * (y - 0.5)) * 9.;
      if (r2 < 1) prim[0] = prim[0] + 0.05 * exp(1. - 1. / ((1 - r2) * (1 - r2)));
    } break;
    case 4:
    case 5: {
      double xm0 = o->p.x0[0] + 0.5 * o->sx[0], xm1 = o->p.x0[1] + 0.5 * o->sx[1];
      double a = x - xm0, c = y - xm1;
      double r = sqrt(a * a + c * c);
      if (ic == 4) prim[0] = (r <= 7.) ? 2.5 : MIN_DEPTH;
      else prim[0] = (r <= 15.) ? 10. : 0.5;
    } break;
    case 6: {
      double r2 = (x + 2) * (x + 2);
      orc_bathymetry(&o->p, x, y, &b, NULL, NULL);
      prim[0] = fmax2(0.7 - b, MIN_DEPTH);
      if (r2 < 1) prim[0] = prim[0] + 0.5 * exp(1. - 1. / ((1 - r2) * (1 - r2)));
      prim[1] = (prim[0] > MIN_DEPTH * 10) ? 1.0 : 0.0;
    } break;
    case 101: { /* vortex: par {cx, cy, eps, ub, vb, R} */
      double rx = (x - par[0]) / par[5], ry = (y - par[1]) / par[5];
      double r2 = rx * rx + ry * ry;
      double e1 = exp(1. - r2);
      prim[0] = 1. - par[2] * par[2] / (4. * g) * (e1 * e1);
      prim[1] = par[3] - par[2] * ry * e1;
      prim[2] = par[4] + par[2] * rx * e1;
    } break;
    case 102: /* lake at rest + pulse: par {amp, xlo, xhi} */
      orc_bathymetry(&o->p, x, y, &b, NULL, NULL);
      prim[0] = fmax2(1. - b, MIN_DEPTH);
      if (x > par[1] && x < par[2]) prim[0] = prim[0] + par[0];
      break;
    case 103: { /* dam break: par {cx, cy, radius, h_in} */
      double a = x - par[0], c = y - par[1];
      prim[0] = (sqrt(a * a + c * c) < par[2]) ? par[3] : MIN_DEPTH;
    } break;
    case 104: { /* wave over island: par {amp, xc, width} */
      orc_bathymetry(&o->p, x, y, &b, NULL, NULL);
      double hs = fmax2(1. - b, MIN_DEPTH);
      double s = (x - par[1]) / par[2];
      double eta = par[0] * exp(-(s * s));
      prim[0] = hs + eta;
      cons[0] = prim[0];
      cons[1] = eta * sqrt(g * prim[0]);
      cons[2] = 0.;
      return;
    }
    case 105: /* still water: par {level} */
      orc_bathymetry(&o->p, x, y, &b, NULL, NULL);
      prim[0] = fmax2(par[0] - b, MIN_DEPTH);
      break;
    default:
      break;
  }
  cons[0] = prim[0]; /* PrimToCons, equation.f90:977-979 */
  cons[1] = prim[0] * prim[1];
  cons[2] = prim[0] * prim[2];
}

static int valid_ic(int ic) { return (ic >= 1 && ic <= 6) || (ic >= 101 && ic <= 105); }

/* finitevolume.f90:281-333 FillInitialConditions (U part) */
int orc_fill_ic(orc_t *o, int ic, const double *par) {
  if (!valid_ic(ic)) return -1;
  memset(o->U, 0, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
  OMP_FOR
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii)
      for (int iGP = 0; iGP < 4; ++iGP)
        for (int jGP = 0; jGP < 4; ++jGP) {
          double ut[3];
          exact_function(o, ic, par, 0.0, gp_coord(o, 0, ii, iGP), gp_coord(o, 1, jj, jGP), ut);
          for (int v = 0; v < 3; ++v)
            o->U[IU(v, ii, jj)] = o->U[IU(v, ii, jj)] + o->wgp[iGP][jGP] * ut[v];
        }
  return 0;
}

/* postprocessing.f90:23-60 PostProcessing: L1error(v) = sum_cells |U - Uexact(t)| dx dy,
 * Uexact the 4x4 Gauss average of ExactFunction(ic, t) (serial sum, cell order j, i). */
int orc_l1_error(const orc_t *o, int ic, const double *par, double t, double out[3]) {
  if (!valid_ic(ic)) return -1;
  double l1[3] = {0., 0., 0.};
  for (int jj = 1; jj <= NY; ++jj)
    for (int ii = 1; ii <= NX; ++ii) {
      double ue[3] = {0., 0., 0.};
      for (int iGP = 0; iGP < 4; ++iGP)
        for (int jGP = 0; jGP < 4; ++jGP) {
          double ut[3];
          exact_function(o, ic, par, t, gp_coord(o, 0, ii, iGP), gp_coord(o, 1, jj, jGP), ut);
          for (int v = 0; v < 3; ++v) ue[v] = ue[v] + o->wgp[iGP][jGP] * ut[v];
        }
      for (int v = 0; v < 3; ++v) l1[v] = l1[v] + fabs(o->U[IU(v, ii, jj)] - ue[v]);
    }
  for (int v = 0; v < 3; ++v) out[v] = l1[v] * o->dx[0] * o->dx[1];
  return 0;
}

/* finitevolume.f90:339-396 InitializeWBVariables */
int orc_init_wb(orc_t *o, int ic, const double *par) {
  if (orc_fill_ic(o, ic, par) != 0) return -1;
  fv_time_derivative(o, 0);
  memcpy(o->FXWB, o->FX, sizeof(double) * 3 * (o->nx + 1) * o->ny);
  memcpy(o->FYWB, o->FY, sizeof(double) * 3 * o->nx * (o->ny + 1));
  memcpy(o->SWB, o->S, sizeof(double) * 3 * o->N);
  o->have_wb = 1;
  memset(o->U, 0, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
  return 0;
}

/* InitializeWBVariables from given cell averages [3][ny][nx] */
int orc_init_wb_planes(orc_t *o, const double *planes) {
  orc_set_planes(o, planes);
  fv_time_derivative(o, 0);
  memcpy(o->FXWB, o->FX, sizeof(double) * 3 * (o->nx + 1) * o->ny);
  memcpy(o->FYWB, o->FY, sizeof(double) * 3 * o->nx * (o->ny + 1));
  memcpy(o->SWB, o->S, sizeof(double) * 3 * o->N);
  o->have_wb = 1;
  memset(o->U, 0, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
  return 0;
}

void orc_set_state(orc_t *o, const double *U) {
  memcpy(o->U, U, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
}
void orc_get_state(const orc_t *o, double *U, double *V) {
  if (U) memcpy(U, o->U, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
  if (V) memcpy(V, o->V, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
}
void orc_get_planes(const orc_t *o, double *out) {
  for (int v = 0; v < 3; ++v)
    for (int jj = 1; jj <= NY; ++jj)
      for (int ii = 1; ii <= NX; ++ii)
        out[(size_t)v * o->N + (size_t)(jj - 1) * NX + (ii - 1)] = o->U[IU(v, ii, jj)];
}
void orc_set_planes(orc_t *o, const double *in) {
  memset(o->U, 0, sizeof(double) * 3 * (o->nx + 6) * (o->ny + 6));
  for (int v = 0; v < 3; ++v)
    for (int jj = 1; jj <= NY; ++jj)
      for (int ii = 1; ii <= NX; ++ii)
        o->U[IU(v, ii, jj)] = in[(size_t)v * o->N + (size_t)(jj - 1) * NX + (ii - 1)];
}

const int *orc_rowstart(const orc_t *o) { return o->RowStart; }
const int *orc_columns(const orc_t *o) { return o->Cols; }
int orc_last_jacobi_iters(const orc_t *o, int *iters, int max) {
  int n = o->nsolves < max ? o->nsolves : max;
  for (int k = 0; k < n && k < 64; ++k) iters[k] = o->iters[k];
  return o->nsolves;
}
long long orc_total_jacobi_iters(const orc_t *o) { return o->total_iters; }
double orc_mesh_dx(const orc_t *o, int d) { return o->dx[d]; }
int orc_threads(void) {
#ifdef ORC_OMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
