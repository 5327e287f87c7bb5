// swm_ic.cu -- initial conditions and the L1 error on the device (sm_100a).
//
//   FillInitialConditions (finitevolume.f90:281-333): U = sum_{a,b} W_ab ExactFunction(x_a, y_b)
//   PostProcessing        (postprocessing.f90:23-60):  L1 = sum_cells |U - Uexact(t)| dx dy
//
// ExactFunction (equation.f90:70-230) cases 1..6 and the benchmark cases 101..105.
// Built with -fmad=false so that every expression rounds in the reference's order;
// the transcendental functions are CUDA's, so values agree with a host evaluation to
// the last few bits rather than bit for bit.
#include "swm_kernels.cuh"

namespace swm {

namespace {

// Bathymetry b(x, y) (equation.f90:419-450; flag 3: b = A exp(-(ax (x-cx)^2 + ay (y-cy)^2))).
__device__ double bathy_b(const Grid& gr, double x, double y) {
  const double PI = acos(-1.0);
  if (gr.bathy == BATHY_SINCOS) return 0.1 * sin(2. * PI * x) * cos(2. * PI * y);
  if (gr.bathy == BATHY_BUMP) {
    double r2 = x * x + y * y;
    if (r2 < 1) {
      double d = 1.0 - r2;
      return exp(1.0 - 1.0 / d);
    }
    return 0.;
  }
  if (gr.bathy == BATHY_GAUSS) {
    double dxv = x - gr.bp[2], dyv = y - gr.bp[4];
    return gr.bp[0] * exp(-(gr.bp[1] * (dxv * dxv) + gr.bp[3] * (dyv * dyv)));
  }
  return 0.;
}

// Fortran MODULO for reals
__device__ __forceinline__ double rmodulo(double a, double p) { return a - floor(a / p) * p; }

// ExactFunction(ic, t, (x, y)) -> conservative state
__device__ void exact_function(const IcArgs& a, double x, double y, double cons[3]) {
  const Grid& gr = a.gr;
  const double PI = acos(-1.0);
  const double g = gr.g;
  const double* par = a.par;
  double prim[3] = {0., 0., 0.};
  switch (a.ic) {
    case 1: {  // unsteady smooth vortex advected by (u_inf, v_inf) (equation.f90:109-133)
      const double u_inf = 2., v_inf = 3., H_inf = 1.;
      const double xm0 = gr.x0 + 0.5 * a.sx[0], xm1 = gr.y0 + 0.5 * a.sx[1];
      const double xc0 = rmodulo(x - u_inf * a.t - gr.x0, a.sx[0]) + gr.x0 - xm0;
      const double xc1 = rmodulo(y - v_inf * a.t - gr.y0, a.sx[1]) + gr.y0 - xm1;
      const double r = xc0 * xc0 + xc1 * xc1;
      prim[0] = H_inf;
      prim[1] = u_inf;
      prim[2] = v_inf;
      if (r < 1) {
        const double ar = atan(r - 1.);
        const double hd =
            3. * 0.1 * exp(1. / pow(ar, 3.)) / (pow(ar, 4.) * ((r - 1.) * (r - 1.) + 1.));
        const double omega = sqrt(2. * g * hd);
        prim[0] = 1. - 0.1 * exp(-1. / pow(atan(1. - r), 3.));
        prim[1] = prim[1] + omega * (+xc1);
        prim[2] = prim[2] + omega * (-xc0);
      }
    } break;
    case 2:  // (equation.f90:135-140)
      prim[0] = 1. - 0.1 * sin(2. * PI * x) * cos(2. * PI * y);
      break;
    case 3: {  // perturbed lake over the bump (equation.f90:141-150)
      prim[0] = dmax(0.7 - bathy_b(gr, x, y), kMinDepth);
      const double r2 = ((x + 2) * (x + 2) + (y - 0.5) * (y - 0.5)) * 9.;
      if (r2 < 1) prim[0] = prim[0] + 0.05 * exp(1. - 1. / ((1 - r2) * (1 - r2)));
    } break;
    case 4:
    case 5: {  // circular dam breaks (equation.f90:151-178)
      const double xm0 = gr.x0 + 0.5 * a.sx[0], xm1 = gr.y0 + 0.5 * a.sx[1];
      const double dx0 = x - xm0, dx1 = y - xm1;
      const double r = sqrt(dx0 * dx0 + dx1 * dx1);
      if (a.ic == 4)
        prim[0] = (r <= 7.) ? 2.5 : kMinDepth;
      else
        prim[0] = (r <= 15.) ? 10. : 0.5;
    } break;
    case 6: {  // wave towards the bump (equation.f90:179-190)
      const double r2 = (x + 2) * (x + 2);
      prim[0] = dmax(0.7 - bathy_b(gr, x, y), kMinDepth);
      if (r2 < 1) prim[0] = prim[0] + 0.5 * exp(1. - 1. / ((1 - r2) * (1 - r2)));
      prim[1] = (prim[0] > kMinDepth * 10) ? 1.0 : 0.0;
    } break;
    case 101: {  // vortex: par {cx, cy, eps, ub, vb, R}
      const double rx = (x - par[0]) / par[5], ry = (y - par[1]) / par[5];
      const double r2 = rx * rx + ry * ry;
      const double e1 = exp(1. - r2);
      prim[0] = 1. - par[2] * par[2] / (4. * g) * (e1 * e1);
      prim[1] = par[3] - par[2] * ry * e1;
      prim[2] = par[4] + par[2] * rx * e1;
    } break;
    case 102:  // lake at rest + pulse: par {amp, xlo, xhi}
      prim[0] = dmax(1. - bathy_b(gr, x, y), kMinDepth);
      if (x > par[1] && x < par[2]) prim[0] = prim[0] + par[0];
      break;
    case 103: {  // dam break: par {cx, cy, radius, h_in}
      const double dx0 = x - par[0], dx1 = y - par[1];
      prim[0] = (sqrt(dx0 * dx0 + dx1 * dx1) < par[2]) ? par[3] : kMinDepth;
    } break;
    case 104: {  // wave over the island: par {amp, xc, width}
      const double hs = dmax(1. - bathy_b(gr, x, y), kMinDepth);
      const double s = (x - par[1]) / par[2];
      const double eta = par[0] * exp(-(s * s));
      cons[0] = hs + eta;
      cons[1] = eta * sqrt(g * cons[0]);
      cons[2] = 0.;
      return;
    }
    case 105:  // still water: par {level}
      prim[0] = dmax(par[0] - bathy_b(gr, x, y), kMinDepth);
      break;
    default:
      break;
  }
  cons[0] = prim[0];  // PrimToCons (equation.f90:977-979)
  cons[1] = prim[0] * prim[1];
  cons[2] = prim[0] * prim[2];
}

// 4x4 Gauss average of the exact state over cell (i, j), 0-based (finitevolume.f90:314-330)
__device__ void cell_average(const IcArgs& a, int i, int j, double u[3]) {
  const Grid& gr = a.gr;
  u[0] = u[1] = u[2] = 0.;
#pragma unroll 1
  for (int ia = 0; ia < 4; ++ia) {
    const double x = (gr.x0 + ((double)i) * gr.dx + 0.5 * gr.dx) + gr.qn[ia] * gr.dx;
#pragma unroll 1
    for (int jb = 0; jb < 4; ++jb) {
      const double y = (gr.y0 + ((double)j) * gr.dy + 0.5 * gr.dy) + gr.qn[jb] * gr.dy;
      double ut[3];
      exact_function(a, x, y, ut);
#pragma unroll
      for (int v = 0; v < 3; ++v) u[v] = u[v] + gr.wgp[ia][jb] * ut[v];
    }
  }
}

constexpr int kIcThreads = 256;

__global__ void __launch_bounds__(kIcThreads) ic_fill_kernel(const IcArgs a) {
  const int n = a.gr.nx * a.gr.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double u[3];
    cell_average(a, c % a.gr.nx, c / a.gr.nx, u);
    a.h[c] = u[0];
    a.hu[c] = u[1];
    a.hv[c] = u[2];
  }
}

// Per-block sums of |U - Uexact| in a fixed order (thread-strided cells, then a
// tree over the block), written to partial[block][3].
__global__ void __launch_bounds__(kIcThreads) l1_partial_kernel(const IcArgs a, double* partial) {
  __shared__ double red[3][kIcThreads];
  const int n = a.gr.nx * a.gr.ny;
  double s[3] = {0., 0., 0.};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double ue[3];
    cell_average(a, c % a.gr.nx, c / a.gr.nx, ue);
    s[0] = s[0] + fabs(a.h[c] - ue[0]);
    s[1] = s[1] + fabs(a.hu[c] - ue[1]);
    s[2] = s[2] + fabs(a.hv[c] - ue[2]);
  }
  for (int v = 0; v < 3; ++v) red[v][threadIdx.x] = s[v];
  __syncthreads();
  for (int o = kIcThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int v = 0; v < 3; ++v) red[v][threadIdx.x] = red[v][threadIdx.x] + red[v][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int v = 0; v < 3; ++v) partial[3 * blockIdx.x + v] = red[v][0];
}

// Serial sum of the block partials (fixed order), then L1error * MESH_DX(1) * MESH_DX(2)
// (postprocessing.f90:50).
__global__ void l1_final_kernel(const double* partial, int nblk, double dx, double dy,
                                double* out) {
  if (threadIdx.x < 3) {
    double s = 0.;
    for (int b = 0; b < nblk; ++b) s = s + partial[3 * b + threadIdx.x];
    out[threadIdx.x] = s * dx * dy;
  }
}

__global__ void __launch_bounds__(kIcThreads) error_planes_kernel(const IcArgs a, double* e0,
                                                                   double* e1, double* e2) {
  const int n = a.gr.nx * a.gr.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double ue[3];
    cell_average(a, c % a.gr.nx, c / a.gr.nx, ue);
    e0[c] = a.h[c] - ue[0];
    e1[c] = a.hu[c] - ue[1];
    e2[c] = a.hv[c] - ue[2];
  }
}

__global__ void __launch_bounds__(kIcThreads) bath_average_kernel(const IcArgs a, double* b) {
  const Grid& gr = a.gr;
  const int n = gr.nx * gr.ny;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int i = c % gr.nx, j = c / gr.nx;
    double s = 0.;
    for (int ia = 0; ia < 4; ++ia) {
      const double x = (gr.x0 + ((double)i) * gr.dx + 0.5 * gr.dx) + gr.qn[ia] * gr.dx;
      for (int jb = 0; jb < 4; ++jb) {
        const double y = (gr.y0 + ((double)j) * gr.dy + 0.5 * gr.dy) + gr.qn[jb] * gr.dy;
        s = s + gr.wgp[ia][jb] * bathy_b(gr, x, y);
      }
    }
    b[c] = s;
  }
}

}  // namespace

cudaError_t launch_error_planes(const IcArgs& a, double* const e[3], cudaStream_t s) {
  error_planes_kernel<<<ic_blocks(a.gr.nx * a.gr.ny), kIcThreads, 0, s>>>(a, e[0], e[1], e[2]);
  return cudaGetLastError();
}

cudaError_t launch_bath_average(const IcArgs& a, double* b, cudaStream_t s) {
  bath_average_kernel<<<ic_blocks(a.gr.nx * a.gr.ny), kIcThreads, 0, s>>>(a, b);
  return cudaGetLastError();
}

int ic_blocks(int ncells) {
  int b = (ncells + kIcThreads - 1) / kIcThreads;
  return b < 1 ? 1 : (b > kIcMaxBlocks ? kIcMaxBlocks : b);
}

bool ic_supported(int ic) { return (ic >= 1 && ic <= 6) || (ic >= 101 && ic <= 105); }

cudaError_t launch_ic_fill(const IcArgs& a, cudaStream_t s) {
  ic_fill_kernel<<<ic_blocks(a.gr.nx * a.gr.ny), kIcThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_l1_error(const IcArgs& a, double* partial, double* out, cudaStream_t s) {
  const int nb = ic_blocks(a.gr.nx * a.gr.ny);
  l1_partial_kernel<<<nb, kIcThreads, 0, s>>>(a, partial);
  l1_final_kernel<<<1, 32, 0, s>>>(partial, nb, a.gr.dx, a.gr.dy, out);
  return cudaGetLastError();
}

}  // namespace swm
