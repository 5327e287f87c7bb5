// swm_host.h -- host-side set-up shared by the single-grid solver and the ensembles:
// mesh and quadrature (mesh.f90:58-70, :127-142) and the bathymetry tables the RHS
// kernels read.
#pragma once
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstddef>
#include <vector>

#include "../../include/swm.h"
#include "swm_device.cuh"
#include "swm_rhs.cuh"

namespace swm {

// NVTX range for the lifetime of the object: the C-ABI calls and, when a step is
// enqueued eagerly or captured, its phases show up by name in a profiler timeline
// (no cost without an attached tool).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// thetaDeC of mPDeC5 (timediscretization.f90:491-506), row m, column r, row-major [m][r]
inline constexpr double kTheta5[4][4] = {
    {0.0000000000000000000, 0.0000000000000000000, 0.0000000000000000000, 0.0000000000000000000},
    {0.1103005664791649049, 0.1896994335208351257, -0.0339073642291439076, 0.0103005664791649201},
    {0.0730327668541684294, 0.4505740308958107176, 0.2269672331458314485, -0.0269672331458315692},
    {0.0833333333333333287, 0.4166666666666666852, 0.4166666666666666852, 0.0833333333333333287}};

// 4-point Gauss-Legendre nodes on [-1/2, 1/2] and weights (mesh.f90:127-129).
inline void host_quadrature(double qn[4], double qw[4]) {
  qw[0] = (18. - sqrt(30.)) / 72.;
  qw[1] = (18. + sqrt(30.)) / 72.;
  qw[2] = (18. + sqrt(30.)) / 72.;
  qw[3] = (18. - sqrt(30.)) / 72.;
  qn[0] = -(0.5 * sqrt(3. / 7. + 2. / 7. * sqrt(6. / 5.)));
  qn[1] = -(0.5 * sqrt(3. / 7. - 2. / 7. * sqrt(6. / 5.)));
  qn[2] = 0.5 * sqrt(3. / 7. - 2. / 7. * sqrt(6. / 5.));
  qn[3] = 0.5 * sqrt(3. / 7. + 2. / 7. * sqrt(6. / 5.));
}

// Uniform mesh of the parameters (mesh.f90:58-60: dx = |x1 - x0| / nx).
inline Grid host_grid(const swm_params& p) {
  Grid gr{};
  gr.nx = p.nx;
  gr.ny = p.ny;
  gr.x0 = p.x0[0];
  gr.y0 = p.x0[1];
  gr.dx = fabs(fabs(p.x1[0] - p.x0[0])) / ((double)p.nx);
  gr.dy = fabs(fabs(p.x1[1] - p.x0[1])) / ((double)p.ny);
  gr.rdx = 1.0 / gr.dx;
  gr.rdy = 1.0 / gr.dy;
  gr.g = p.g;
  gr.bathy = p.bathy_flag;
  for (int k = 0; k < 5; ++k) gr.bp[k] = p.bathy_par[k];
  host_quadrature(gr.qn, gr.qw);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) gr.wgp[a][b] = gr.qw[a] * gr.qw[b];
  for (int q = 0; q < 4; ++q) gr.qwf[q] = (float)gr.qw[q];
  return gr;
}

// Gauss node q of cell c (0-based): node = x0 + c dx, bary = node + dx/2,
// gp = bary + qn dx (mesh.f90:64,70,142).
inline double host_gp(double x0, double h, int c, double q) {
  double node = x0 + ((double)c) * h;
  double bary = node + 0.5 * h;
  return bary + q * h;
}

// Bathymetry_X / Bathymetry_Y (equation.f90:451-509) and the Gaussian island/lake
// b = A exp(-(ax (x-cx)^2 + ay (y-cy)^2)).
inline void host_bathy_grad(const swm_params& p, double x, double y, double* bx, double* by) {
  const double PI = acos(-1.0);
  *bx = 0.;
  *by = 0.;
  if (p.bathy_flag == SWM_BATHY_SINCOS) {
    *bx = 0.1 * 2. * PI * cos(2. * PI * x) * cos(2. * PI * y);
    *by = -(0.1 * 2. * PI * sin(2. * PI * x) * sin(2. * PI * y));
  } else if (p.bathy_flag == SWM_BATHY_BUMP) {
    double r2 = x * x + y * y;
    if (r2 < 1) {
      double d = 1.0 - r2;
      double e = exp(1.0 - 1.0 / d);
      *bx = -(2.0 * x / (d * d) * e);
      *by = -(2.0 * y / (d * d) * e);
    }
  } else if (p.bathy_flag == SWM_BATHY_GAUSS) {
    const double A = p.bathy_par[0], ax = p.bathy_par[1], cx = p.bathy_par[2];
    const double ay = p.bathy_par[3], cy = p.bathy_par[4];
    double dxv = x - cx, dyv = y - cy;
    double e = exp(-(ax * (dxv * dxv) + ay * (dyv * dyv)));
    double B = A * e;
    *bx = (-2.0 * ax * dxv) * B;
    *by = (-2.0 * ay * dyv) * B;
  }
}

// A separable gradient (b_x = P(x) Q(y), b_y = R(x) T(y): the Gaussian and the sin/cos
// bathymetry) is evaluated from per-column and per-row factors, except in the FP64 form
// with source_table = 1, which reads b_x, b_y tabulated at every interior Gauss point
// (the reference's own products, bit for bit); the bump always takes the table.
inline bool separable_source(const swm_params& p) {
  return (p.bathy_flag == SWM_BATHY_GAUSS || p.bathy_flag == SWM_BATHY_SINCOS) &&
         (p.precision != SWM_PREC_FP64 || !p.source_table);
}

inline bool full_source_table(const swm_params& p) {
  return p.bathy_flag > 0 && !separable_source(p);
}

// b_x, b_y at the 16 interior Gauss points of every cell, planes [4][4][2][ny*nx]
// (x-GP a, y-GP b, component).
inline void host_bgrad_table(const swm_params& p, const Grid& gr, std::vector<double>& tab) {
  const size_t nx = p.nx, ny = p.ny, N = nx * ny;
  tab.assign(32 * N, 0.0);
  std::vector<double> X(4 * nx), Y(4 * ny);
  for (size_t i = 0; i < nx; ++i)
    for (int q = 0; q < 4; ++q) X[4 * i + q] = host_gp(gr.x0, gr.dx, (int)i, gr.qn[q]);
  for (size_t j = 0; j < ny; ++j)
    for (int q = 0; q < 4; ++q) Y[4 * j + q] = host_gp(gr.y0, gr.dy, (int)j, gr.qn[q]);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (size_t j = 0; j < ny; ++j)
        for (size_t i = 0; i < nx; ++i) {
          double bx, by;
          host_bathy_grad(p, X[4 * i + a], Y[4 * j + b], &bx, &by);
          tab[((a * 4 + b) * 2 + 0) * N + j * nx + i] = bx;
          tab[((a * 4 + b) * 2 + 1) * N + j * nx + i] = by;
        }
}

// Separable factors with the Gauss weights folded in:
//   col[i] = { w_a P(x_a) (a = 0..3), w_a R(x_a) },  row[j] = { w_b Q(y_b), w_b T(y_b) },
// so that S_hu = -g sum_a col.P_a sum_b row.Q_b h_ab and
//         S_hv = -g sum_b row.T_b sum_a col.R_a h_ab
// equal sum_ab W_ab (-g h_ab b_x|y) of equation.f90:380-388 up to rounding.
inline void host_source_factors(const swm_params& p, const Grid& gr, std::vector<double>& col,
                                std::vector<double>& row) {
  const int nx = p.nx, ny = p.ny;
  col.assign(8 * (size_t)nx, 0.0);
  row.assign(8 * (size_t)ny, 0.0);
  const double PI = acos(-1.0);
  for (int i = 0; i < nx; ++i)
    for (int q = 0; q < 4; ++q) {
      const double x = host_gp(gr.x0, gr.dx, i, gr.qn[q]);
      double P = 0., R = 0.;
      if (p.bathy_flag == SWM_BATHY_GAUSS) {
        const double d = x - p.bathy_par[2], e = exp(-(p.bathy_par[1] * (d * d)));
        P = p.bathy_par[0] * (-2.0 * p.bathy_par[1] * d) * e;
        R = p.bathy_par[0] * e;
      } else if (p.bathy_flag == SWM_BATHY_SINCOS) {
        P = 0.1 * 2. * PI * cos(2. * PI * x);
        R = -(0.1 * 2. * PI * sin(2. * PI * x));
      }
      col[8 * (size_t)i + q] = gr.qw[q] * P;
      col[8 * (size_t)i + 4 + q] = gr.qw[q] * R;
    }
  for (int j = 0; j < ny; ++j)
    for (int q = 0; q < 4; ++q) {
      const double y = host_gp(gr.y0, gr.dy, j, gr.qn[q]);
      double Q = 0., T = 0.;
      if (p.bathy_flag == SWM_BATHY_GAUSS) {
        const double d = y - p.bathy_par[4], e = exp(-(p.bathy_par[3] * (d * d)));
        Q = e;
        T = (-2.0 * p.bathy_par[3] * d) * e;
      } else if (p.bathy_flag == SWM_BATHY_SINCOS) {
        Q = cos(2. * PI * y);
        T = sin(2. * PI * y);
      }
      row[8 * (size_t)j + q] = gr.qw[q] * Q;
      row[8 * (size_t)j + 4 + q] = gr.qw[q] * T;
    }
}

// The split form's records of the same factors (SrcSplit): FP32 factors, the column's
// w R as (w R, w R) pairs, and the FP64 sums of each factor's four weights.
inline void host_source_split(const std::vector<double>& col, const std::vector<double>& row,
                              std::vector<SrcSplit>& cols, std::vector<SrcSplit>& rows) {
  const size_t nx = col.size() / 8, ny = row.size() / 8;
  cols.assign(nx, SrcSplit{});
  rows.assign(ny, SrcSplit{});
  for (size_t i = 0; i < nx; ++i) {
    const double* c = &col[8 * i];
    for (int q = 0; q < 4; ++q) {
      cols[i].a[q] = (float)c[q];
      cols[i].b[2 * q] = cols[i].b[2 * q + 1] = (float)c[4 + q];
    }
    cols[i].s[0] = ((c[0] + c[1]) + c[2]) + c[3];
    cols[i].s[1] = ((c[4] + c[5]) + c[6]) + c[7];
  }
  for (size_t j = 0; j < ny; ++j) {
    const double* r = &row[8 * j];
    for (int q = 0; q < 4; ++q) {
      rows[j].a[q] = (float)r[q];
      rows[j].b[q] = (float)r[4 + q];
    }
    rows[j].s[0] = ((r[0] + r[1]) + r[2]) + r[3];
    rows[j].s[1] = ((r[4] + r[5]) + r[6]) + r[7];
  }
}

}  // namespace swm
