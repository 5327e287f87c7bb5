// swm_device.cuh -- device building blocks of the mPDeC5 time step (sm_100a).
//
// The three precision forms share this code:
//   EXACT  (FP64, translation unit built with -fmad=false): the reference's
//          expression order and correctly rounded divisions (div_rn), so that
//          results match the CPU restatement of the Fortran bit for bit where no
//          libm call is involved;
//   FAST   (FP64, FMA contraction): WENO weights use one reciprocal per
//          smoothness indicator and one per Gauss point instead of six
//          divisions per point;
//   SPLIT  (FP32 WENO on deviations from the cell value, FP64 everywhere else).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#ifndef SWM_EXACT
#define SWM_EXACT 0
#endif

namespace swm {

// finitevolume_vars.f90:96-106
constexpr double kMinDepth = 1.0e-6;
constexpr double kWenoEps = 1.0e-24;
// FP32 WENO uses eps = 1e-18: (1e-24)^2 underflows to 0 in FP32, which would turn
// a flat stencil's weights into inf/inf.  (1e-18)^2 = 1e-36 is a normal float.
constexpr float kWenoEpsF = 1.0e-18f;
constexpr double kWLobatto = 1. / 12.;
// limiter denominator 1 - 2 wL and its correctly rounded reciprocal
constexpr double kCsiDen = 1. - 2. * kWLobatto;
constexpr double kCsiRcp = 1. / kCsiDen;

// Bathymetry kinds (swm.h SWM_BATHY_*)
enum { BATHY_FLAT = 0, BATHY_SINCOS = 1, BATHY_BUMP = 2, BATHY_GAUSS = 3 };

struct Grid {
  int nx, ny;
  double x0, y0;
  double dx, dy;
  double rdx, rdy;  // 1/dx, 1/dy (the split and FMA forms multiply by these)
  double g;
  int bathy;
  double bp[5];  // Gaussian A, ax, cx, ay, cy
  double qn[4];  // Gauss nodes on [-1/2, 1/2] (mesh.f90:128-129)
  double qw[4];  // Gauss weights (mesh.f90:127)
  double wgp[4][4];
  float qwf[4];  // the Gauss weights rounded to FP32 (split-form limiter)
};

__device__ __forceinline__ int wrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// Checked build (-DSWM_CHECKED): the wrapped-index sites of the kernels (tile and halo
// loads of the RHS and the Jacobi, CSR column reads, the mPDeC2 compatibility read,
// ensemble work items) check their index against the array's extent; a failing check
// records its site (the first one, and a count) and the access is skipped, so that a
// wrong index shows up as a status instead of a memory fault.  Without the flag the
// checks compile to nothing.
enum {
  kChkRhsLoad = 1, kChkJacPairs, kChkJacCells, kChkCsr, kChkCompat2, kChkEnsItem
};
#ifdef SWM_CHECKED
// one record per translation unit (each unit's device code is a module of its own)
static __device__ int g_swm_check_site;
static __device__ unsigned long long g_swm_check_count;
__device__ __forceinline__ bool swm_in_range(long long i, long long n, int site) {
  if (i >= 0 && i < n) return true;
  atomicCAS(&g_swm_check_site, 0, site);
  atomicAdd(&g_swm_check_count, 1ull);
  return false;
}
#define SWM_IN_RANGE(i, n, site) ::swm::swm_in_range((long long)(i), (long long)(n), (site))
// Host reader of this unit's record, read and cleared: site of the first failing check
// (0 none) and the number of failing checks.
#define SWM_CHECK_READER(fn)                                                             \
  int fn(int* site, unsigned long long* count) {                                       \
    int zero = 0;                                                                      \
    unsigned long long zc = 0;                                                         \
    cudaError_t e = cudaMemcpyFromSymbol(site, g_swm_check_site, sizeof(int));         \
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(count, g_swm_check_count, sizeof(zc)); \
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_swm_check_site, &zero, sizeof(int)); \
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_swm_check_count, &zc, sizeof(zc));  \
    return e == cudaSuccess ? 0 : -1;                                                  \
  }
#else
#define SWM_IN_RANGE(i, n, site) true
#define SWM_CHECK_READER(fn)                        \
  int fn(int* site, unsigned long long* count) {  \
    *site = -1;                                     \
    *count = 0;                                     \
    return 0;                                       \
  }
#endif
__device__ __forceinline__ double dmax(double a, double b) { return (a > b) ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return (a < b) ? a : b; }

// Reciprocals of the non-EXACT WENO weights: the correctly rounded FP64 reciprocal,
// and the hardware approximation in FP32 (relative error ~2^-23; its arguments are
// normal: eps_f^2 = 1e-36 <= d and the weight sums are bounded by 1/d).
__device__ __forceinline__ double rcp_(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// FP32 square root by the hardware approximation (relative error ~2^-23); for the
// split form's wave-speed bound, which only scales the Rusanov jump term.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Correctly rounded x / y from a shared correctly rounded reciprocal r = RN(1/y):
// two residual corrections with FMA (Markstein, IBM J. Res. Dev. 34(1), 1990;
// Theorem 8.10 of Muller et al., Handbook of Floating-Point Arithmetic): with r
// correctly rounded and q faithful, q + RN(x - q y) r rounds to RN(x / y), provided
// the residual x - q y is exact and the quotient normal.  mk_range() bounds the
// operands so that this holds: x, y in [2^-400, 2^400) gives quotients in
// (2^-800, 2^800) and residuals far above the subnormal range.
__device__ __forceinline__ bool mk_range(double x) {
  return ((unsigned)(__double2hiint(x) >> 20) & 0x7ffu) - 623u < 800u;
}
__device__ __forceinline__ double div_mk(double x, double y, double r) {
  double q = x * r;
  double e = fma(-q, y, x);
  q = fma(e, r, q);
  e = fma(-q, y, x);
  return fma(e, r, q);
}
// The IEEE division, kept out of line: it only serves operands outside mk_range.
static __device__ __noinline__ double div_ieee(double x, double y) { return x / y; }
// x / y for any operands; a zero numerator gives x * r, the correctly signed zero
// (NaN for y = 0 or NaN).
__device__ __forceinline__ double div_rn(double x, double y, double r) {
  if (__builtin_expect(mk_range(x) && mk_range(y), 1)) return div_mk(x, y, r);
  if (x == 0.0) return x * r;
  return div_ieee(x, y);
}

template <typename T>
__device__ __forceinline__ T weno_eps();
template <>
__device__ __forceinline__ double weno_eps<double>() { return kWenoEps; }
template <>
__device__ __forceinline__ float weno_eps<float>() { return kWenoEpsF; }

// Smoothness indicators (reconstruction.f90:699-704 and :1024-1029), squared with eps.
// EXACT keeps the reference's expanded quadratic forms.  The other forms use the
// identical sums of squares, e.g. 3*beta1 = 4a^2-19ab+25b^2+11ac-31bc+10c^2 =
// 3*(13/12 (a-2b+c)^2 + 1/4 (a-4b+3c)^2): non-negative by construction and free of
// the cancellation of the expanded form, which in FP32 can drive eps+beta to zero
// (and the weights to inf/inf) on nearly constant stencils.
template <typename T, bool EXACT>
__device__ __forceinline__ void weno_d(T qm2, T qm1, T q0, T qp1, T qp2, T& d1, T& d2, T& d3) {
  T beta1, beta2, beta3;
  if (EXACT) {
    beta1 = (T(1.0) / T(3.0)) * (T(4.0) * qm2 * qm2 - T(19.0) * qm2 * qm1 + T(25.0) * qm1 * qm1 +
                                 T(11.0) * qm2 * q0 - T(31.0) * qm1 * q0 + T(10.0) * q0 * q0);
    beta2 = (T(1.0) / T(3.0)) * (T(4.0) * qm1 * qm1 - T(13.0) * qm1 * q0 + T(13.0) * q0 * q0 +
                                 T(5.0) * qm1 * qp1 - T(13.0) * q0 * qp1 + T(4.0) * qp1 * qp1);
    beta3 = (T(1.0) / T(3.0)) * (T(10.0) * q0 * q0 - T(31.0) * q0 * qp1 + T(25.0) * qp1 * qp1 +
                                 T(11.0) * q0 * qp2 - T(19.0) * qp1 * qp2 + T(4.0) * qp2 * qp2);
  } else {
    const T c13 = T(13.0) / T(12.0), c4 = T(0.25);
    T s1 = qm2 - T(2.0) * qm1 + q0, r1 = qm2 - T(4.0) * qm1 + T(3.0) * q0;
    T s2 = qm1 - T(2.0) * q0 + qp1, r2 = qm1 - qp1;
    T s3 = q0 - T(2.0) * qp1 + qp2, r3 = T(3.0) * q0 - T(4.0) * qp1 + qp2;
    beta1 = c13 * (s1 * s1) + c4 * (r1 * r1);
    beta2 = c13 * (s2 * s2) + c4 * (r2 * r2);
    beta3 = c13 * (s3 * s3) + c4 * (r3 * r3);
  }
  T t1 = weno_eps<T>() + beta1, t2 = weno_eps<T>() + beta2, t3 = weno_eps<T>() + beta3;
  d1 = t1 * t1;
  d2 = t2 * t2;
  d3 = t3 * t3;
}

// How the WENO weights divide: products with reciprocals (non-EXACT forms), or the
// reference's quotients, correctly rounded from shared reciprocals (EXACT, when the
// smoothness indicators are in mk_range) or by IEEE division (EXACT otherwise).
enum { kDivRcp = 0, kDivMk = 1, kDivIeee = 2 };

// Nonlinear combination of one reconstruction point, i_k = RN(1/d_k).
//  EXACT: omega_k = alpha_k/(alpha1+alpha2+alpha3), alpha_k = gamma_k/d_k
//         (reconstruction.f90:716-728), literal order.  With d_k in
//         [2^-400, 2^400), alpha_k and their sum lie in [2^-405, 2^402], so every
//         quotient (>= 2^-807) and residual stays normal and div_mk is exact.
//  else : the same weights as products with the reciprocals.
template <typename T, int DIV>
__device__ __forceinline__ T weno_point(T g1, T g2, T g3, T d1, T d2, T d3, T i1, T i2, T i3, T W1,
                                        T W2, T W3) {
  if constexpr (DIV == kDivMk) {
    T a1 = div_mk(g1, d1, i1), a2 = div_mk(g2, d2, i2), a3 = div_mk(g3, d3, i3);
    const T s = a1 + a2 + a3, rs = rcp_(s);
    return div_mk(a1, s, rs) * W1 + div_mk(a2, s, rs) * W2 + div_mk(a3, s, rs) * W3;
  } else if constexpr (DIV == kDivIeee) {
    T a1 = g1 / d1, a2 = g2 / d2, a3 = g3 / d3;
    return a1 / (a1 + a2 + a3) * W1 + a2 / (a1 + a2 + a3) * W2 + a3 / (a1 + a2 + a3) * W3;
  } else {
    T a1 = g1 * i1, a2 = g2 * i2, a3 = g3 * i3;
    return (a1 * W1 + a2 * W2 + a3 * W3) * rcp_(a1 + a2 + a3);
  }
}

template <int DIV>
__device__ __forceinline__ bool div_ok(double d1, double d2, double d3) {
  return DIV != kDivMk || (mk_range(d1) && mk_range(d2) && mk_range(d3));
}
template <int DIV>
__device__ __forceinline__ bool div_ok(float, float, float) {
  return true;
}

// WENO5_FirstSweep (reconstruction.f90:673-755): cell-face means at x_{i-1/2},
// x_{i+1/2}.  Returns false (nothing written) when kDivMk's range check fails.
template <typename T, bool EXACT, int DIV>
__device__ __forceinline__ bool weno5_first_div(T qm2, T qm1, T q0, T qp1, T qp2, T& wm, T& wp) {
  T d1, d2, d3;
  weno_d<T, EXACT>(qm2, qm1, q0, qp1, qp2, d1, d2, d3);
  if (!div_ok<DIV>(d1, d2, d3)) return false;
  T i1 = T(0), i2 = T(0), i3 = T(0);
  if constexpr (DIV != kDivIeee) {
    i1 = rcp_(d1);
    i2 = rcp_(d2);
    i3 = rcp_(d3);
  }
  const T s6 = T(1.0) / T(6.0);
  T W1 = s6 * (-qm2 + T(5.0) * qm1 + T(2.0) * q0);
  T W2 = s6 * (T(2.0) * qm1 + T(5.0) * q0 - qp1);
  T W3 = s6 * (T(11.0) * q0 - T(7.0) * qp1 + T(2.0) * qp2);
  wm = weno_point<T, DIV>(T(3.0) / T(10.0), T(3.0) / T(5.0), T(1.0) / T(10.0), d1, d2, d3, i1, i2,
                          i3, W1, W2, W3);
  W1 = s6 * (T(2.0) * qm2 - T(7.0) * qm1 + T(11.0) * q0);
  W2 = s6 * (-qm1 + T(5.0) * q0 + T(2.0) * qp1);
  W3 = s6 * (T(2.0) * q0 + T(5.0) * qp1 - qp2);
  wp = weno_point<T, DIV>(T(1.0) / T(10.0), T(3.0) / T(5.0), T(3.0) / T(10.0), d1, d2, d3, i1, i2,
                          i3, W1, W2, W3);
  return true;
}

// WENO5_SecondSweep (reconstruction.f90:999-1136): values at the 4 Gauss nodes.
// Linear weights and sub-stencil coefficients are the reference's tabulated
// constants (generated offline by weno-weights/WENO_double.m); the reference's
// 0.0*Q(k) terms are omitted (they only change the sign of an exact zero).
template <typename T, bool EXACT, int DIV>
__device__ __forceinline__ bool weno5_second_div(T qm2, T qm1, T q0, T qp1, T qp2, T w[4]) {
  T d1, d2, d3;
  weno_d<T, EXACT>(qm2, qm1, q0, qp1, qp2, d1, d2, d3);
  if (!div_ok<DIV>(d1, d2, d3)) return false;
  T i1 = T(0), i2 = T(0), i3 = T(0);
  if constexpr (DIV != kDivIeee) {
    i1 = rcp_(d1);
    i2 = rcp_(d2);
    i3 = rcp_(d3);
  }
  T W1, W2, W3;
  W1 = T(-0.1642562761719537) * qm2 + T(0.7590807081409336) * qm1 + T(0.4051755680310201) * q0;
  W2 = T(0.2663118796250726) * qm1 + T(0.8979443965468811) * q0 - T(0.1642562761719537) * qp1;
  W3 = T(1.6968800354220990) * q0 - T(0.9631919150471715) * qp1 + T(0.2663118796250726) * qp2;
  w[0] = weno_point<T, DIV>(T(0.2658420974778319), T(0.6112504900322486), T(0.1229074124899195),
                            d1, d2, d3, i1, i2, i3, W1, W2, W3);
  W1 = T(-0.1122135388132497) * qm2 + T(0.3944175994189276) * qm1 + T(0.7177959393943222) * q0;
  W2 = T(0.0577769829791784) * qm1 + T(1.0544365558340714) * q0 - T(0.1122135388132497) * qp1;
  W3 = T(1.2277675047716066) * q0 - T(0.2855444877507849) * qp1 + T(0.0577769829791784) * qp2;
  w[1] = weno_point<T, DIV>(T(0.1281641584355059), T(0.5219691498503563), T(0.3498666917141379),
                            d1, d2, d3, i1, i2, i3, W1, W2, W3);
  W1 = T(0.0577769829791784) * qm2 - T(0.2855444877507849) * qm1 + T(1.2277675047716066) * q0;
  W2 = T(-0.1122135388132497) * qm1 + T(1.0544365558340714) * q0 + T(0.0577769829791784) * qp1;
  W3 = T(0.7177959393943222) * q0 + T(0.3944175994189276) * qp1 - T(0.1122135388132497) * qp2;
  w[2] = weno_point<T, DIV>(T(0.3498666917141379), T(0.5219691498503563), T(0.1281641584355059),
                            d1, d2, d3, i1, i2, i3, W1, W2, W3);
  W1 = T(0.2663118796250726) * qm2 - T(0.9631919150471715) * qm1 + T(1.6968800354220990) * q0;
  W2 = T(-0.1642562761719537) * qm1 + T(0.8979443965468811) * q0 + T(0.2663118796250726) * qp1;
  W3 = T(0.4051755680310201) * q0 + T(0.7590807081409336) * qp1 - T(0.1642562761719537) * qp2;
  w[3] = weno_point<T, DIV>(T(0.1229074124899195), T(0.6112504900322486), T(0.2658420974778319),
                            d1, d2, d3, i1, i2, i3, W1, W2, W3);
  return true;
}

// Out-of-line IEEE versions for EXACT reconstructions whose indicators leave mk_range
// (results by value, so that the callers' arrays stay in registers).
struct Weno2 {
  double m, p;
};
struct Weno4 {
  double w[4];
};
static __device__ __noinline__ Weno2 weno5_first_ieee(double qm2, double qm1, double q0, double qp1,
                                               double qp2) {
  Weno2 r;
  weno5_first_div<double, true, kDivIeee>(qm2, qm1, q0, qp1, qp2, r.m, r.p);
  return r;
}
static __device__ __noinline__ Weno4 weno5_second_ieee(double qm2, double qm1, double q0, double qp1,
                                                double qp2) {
  Weno4 r;
  weno5_second_div<double, true, kDivIeee>(qm2, qm1, q0, qp1, qp2, r.w);
  return r;
}

template <typename T, bool EXACT>
__device__ __forceinline__ void weno5_first(T qm2, T qm1, T q0, T qp1, T qp2, T& wm, T& wp) {
  if constexpr (EXACT) {
    if (!weno5_first_div<T, true, kDivMk>(qm2, qm1, q0, qp1, qp2, wm, wp)) {
      const Weno2 r = weno5_first_ieee(qm2, qm1, q0, qp1, qp2);
      wm = r.m;
      wp = r.p;
    }
  } else {
    weno5_first_div<T, false, kDivRcp>(qm2, qm1, q0, qp1, qp2, wm, wp);
  }
}

template <typename T, bool EXACT>
__device__ __forceinline__ void weno5_second(T qm2, T qm1, T q0, T qp1, T qp2, T w[4]) {
  if constexpr (EXACT) {
    if (!weno5_second_div<T, true, kDivMk>(qm2, qm1, q0, qp1, qp2, w)) {
      const Weno4 r = weno5_second_ieee(qm2, qm1, q0, qp1, qp2);
#pragma unroll
      for (int g = 0; g < 4; ++g) w[g] = r.w[g];
    }
  } else {
    weno5_second_div<T, false, kDivRcp>(qm2, qm1, q0, qp1, qp2, w);
  }
}

// ---------------------------------------------------------------------------------
// Packed FP32 pairs for the split form: sm_100's f32x2 add/sub/mul/fma instructions
// carry two independent reconstructions per issued instruction (the two faces of a
// cell, or two neighbouring stencils).  The smoothness indicators are the non-EXACT
// sums of squares above; the point values use the candidate-quadratic form below.
struct f2 {
  unsigned long long v;
};
__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ f2 f2_splat(float c) { return f2_pack(c, c); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ f2 rcp2(f2 a) {
  float lo, hi;
  f2_unpack(a, lo, hi);
  return f2_pack(rcp_(lo), rcp_(hi));
}
// Packed WENO5 in the candidate-quadratic form.  On the cell xi in [-1/2, 1/2] the
// quadratic whose cell averages match candidate stencil k is
//   p_1(xi) = q0 + hx r_1 + tau s_1,  p_2 = q0 - hx r_2 + tau s_2,  p_3 = q0 - hx r_3 + tau s_3,
// hx = xi/2, tau = (xi^2 - 1/12)/2, with the second differences s_1 = qm2 - 2qm1 + q0,
// s_2 = qm1 - 2q0 + qp1, s_3 = q0 - 2qp1 + qp2 and r_1 = qm2 - 4qm1 + 3q0,
// r_2 = qm1 - qp1, r_3 = 3q0 - 4qp1 + qp2: the same quantities the Jiang-Shu
// smoothness indicators beta_k = 13/12 s_k^2 + 1/4 r_k^2 square
// (reconstruction.f90:699-704).  With a_k = gamma_k i_k, i_k = 1/(eps + beta_k)^2,
//   sum_k omega_k p_k(xi) = q0 + sum_k gamma_k (+-hx u_k + tau v_k) / sum_k gamma_k i_k,
// u_k = i_k r_k, v_k = i_k s_k formed once per stencil: 10 packed operations per
// point where the tabulated three-term candidates take 18.  (hx, tau) of a point are
// read off the reference's tabulated candidate-2 coefficients c of qm1 and qp1:
// hx = (c_qp1 - c_qm1)/2, tau = (c_qm1 + c_qp1)/2.  Z: q0 is an exact zero (values
// taken as deviations from the stencil's own centre), whose terms are dropped.
struct WenoUV2 {
  f2 u1, u2, u3, v1, v2, v3, i1, i2, i3;
};

template <bool Z>
__device__ __forceinline__ WenoUV2 weno_uv_x2(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2) {
  const f2 m2 = f2_splat(-2.f), m4 = f2_splat(-4.f), c3 = f2_splat(3.f);
  f2 s1, r1, s2, r2, s3, r3;
  if constexpr (Z) {
    s1 = fma2(m2, qm1, qm2);
    r1 = fma2(m4, qm1, qm2);
    s2 = add2(qm1, qp1);
    s3 = fma2(m2, qp1, qp2);
    r3 = fma2(m4, qp1, qp2);
  } else {
    s1 = add2(fma2(m2, qm1, qm2), q0);
    r1 = fma2(c3, q0, fma2(m4, qm1, qm2));
    s2 = add2(fma2(m2, q0, qm1), qp1);
    s3 = add2(fma2(m2, qp1, q0), qp2);
    r3 = fma2(c3, q0, fma2(m4, qp1, qp2));
  }
  r2 = sub2(qm1, qp1);
  // eps + beta_k as a sum of squares: never below eps
  const f2 c13 = f2_splat(13.f / 12.f), c4 = f2_splat(0.25f), eps = f2_splat(kWenoEpsF);
  const f2 t1 = fma2(mul2(c13, s1), s1, fma2(mul2(c4, r1), r1, eps));
  const f2 t2 = fma2(mul2(c13, s2), s2, fma2(mul2(c4, r2), r2, eps));
  const f2 t3 = fma2(mul2(c13, s3), s3, fma2(mul2(c4, r3), r3, eps));
  WenoUV2 w;
  w.i1 = rcp2(mul2(t1, t1));
  w.i2 = rcp2(mul2(t2, t2));
  w.i3 = rcp2(mul2(t3, t3));
  w.u1 = mul2(w.i1, r1);
  w.u2 = mul2(w.i2, r2);
  w.u3 = mul2(w.i3, r3);
  w.v1 = mul2(w.i1, s1);
  w.v2 = mul2(w.i2, s2);
  w.v3 = mul2(w.i3, s3);
  return w;
}

// One reconstruction point: its linear weights gamma_k and (hx, tau), folded into
// FP32 coefficients at compile time.
struct WenoGp {
  float cu1, cu2, cu3, cv1, cv2, cv3, g1, g2, g3;
};
__host__ __device__ constexpr WenoGp weno_gp(double g1, double g2, double g3, double hx, double tau) {
  return {float(g1 * hx), float(-g2 * hx), float(-g3 * hx), float(g1 * tau), float(g2 * tau),
          float(g3 * tau), float(g1),      float(g2),       float(g3)};
}
// hx and tau of a second-sweep Gauss node from the candidate-2 coefficients
__host__ __device__ constexpr double gp_hx(double c_qm1, double c_qp1) { return 0.5 * (c_qp1 - c_qm1); }
__host__ __device__ constexpr double gp_tau(double c_qm1, double c_qp1) { return 0.5 * (c_qm1 + c_qp1); }

template <bool Z>
__device__ __forceinline__ f2 weno_gp_x2(const WenoUV2& t, f2 q0, const WenoGp c) {
  f2 num = mul2(f2_splat(c.cu1), t.u1);
  num = fma2(f2_splat(c.cu2), t.u2, num);
  num = fma2(f2_splat(c.cu3), t.u3, num);
  num = fma2(f2_splat(c.cv1), t.v1, num);
  num = fma2(f2_splat(c.cv2), t.v2, num);
  num = fma2(f2_splat(c.cv3), t.v3, num);
  const f2 den = fma2(f2_splat(c.g3), t.i3, fma2(f2_splat(c.g2), t.i2, mul2(f2_splat(c.g1), t.i1)));
  const f2 rd = rcp2(den);
  if constexpr (Z)
    return mul2(num, rd);
  else
    return fma2(num, rd, q0);
}

// Two first sweeps (reconstruction.f90:673-755): the faces xi = -1/2 (hx = -1/4,
// tau = 1/12, gamma = 3/10, 3/5, 1/10) and xi = +1/2 (mirrored).
template <bool Z = false>
__device__ __forceinline__ void weno5_first_x2(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2, f2& wm,
                                               f2& wp) {
  const WenoUV2 t = weno_uv_x2<Z>(qm2, qm1, q0, qp1, qp2);
  constexpr WenoGp cm = weno_gp(0.3, 0.6, 0.1, -0.25, 1.0 / 12.0);
  constexpr WenoGp cp = weno_gp(0.1, 0.6, 0.3, 0.25, 1.0 / 12.0);
  wm = weno_gp_x2<Z>(t, q0, cm);
  wp = weno_gp_x2<Z>(t, q0, cp);
}

// Two second sweeps (reconstruction.f90:999-1136): the 4 Gauss nodes with the
// reference's tabulated linear weights; (hx, tau) from its candidate-2 rows.
template <bool Z = false>
__device__ __forceinline__ void weno5_second_x2(f2 qm2, f2 qm1, f2 q0, f2 qp1, f2 qp2, f2 w[4]) {
  const WenoUV2 t = weno_uv_x2<Z>(qm2, qm1, q0, qp1, qp2);
  constexpr double a0 = 0.2663118796250726, b0 = -0.1642562761719537;  // node 0: c_qm1, c_qp1
  constexpr double a1 = 0.0577769829791784, b1 = -0.1122135388132497;  // node 1
  constexpr WenoGp c0 = weno_gp(0.2658420974778319, 0.6112504900322486, 0.1229074124899195,
                                gp_hx(a0, b0), gp_tau(a0, b0));
  constexpr WenoGp c1 = weno_gp(0.1281641584355059, 0.5219691498503563, 0.3498666917141379,
                                gp_hx(a1, b1), gp_tau(a1, b1));
  constexpr WenoGp c2 = weno_gp(0.3498666917141379, 0.5219691498503563, 0.1281641584355059,
                                gp_hx(b1, a1), gp_tau(b1, a1));
  constexpr WenoGp c3 = weno_gp(0.1229074124899195, 0.6112504900322486, 0.2658420974778319,
                                gp_hx(b0, a0), gp_tau(b0, a0));
  w[0] = weno_gp_x2<Z>(t, q0, c0);
  w[1] = weno_gp_x2<Z>(t, q0, c1);
  w[2] = weno_gp_x2<Z>(t, q0, c2);
  w[3] = weno_gp_x2<Z>(t, q0, c3);
}

// ConsToPrim (equation.f90:912-945): u = hu / (h + MIN_DEPTH / h).  EXACT rounds
// every quotient correctly (div_rn, one reciprocal of the desingularised depth for
// both velocities); the other forms multiply by the reciprocals.  h = 0 gives
// ht = inf and u = v = 0 in both.
template <bool EXACT>
__device__ __forceinline__ void cons_to_prim(double h, double hu, double hv, double& u, double& v) {
  if constexpr (EXACT) {
    const double ht = h + div_rn(kMinDepth, h, __drcp_rn(h)), rt = __drcp_rn(ht);
    u = div_rn(hu, ht, rt);
    v = div_rn(hv, ht, rt);
  } else {
    const double rt = __drcp_rn(h + kMinDepth * __drcp_rn(h));
    u = hu * rt;
    v = hv * rt;
  }
}

// Rusanov flux in the face-normal frame: EvaluateFlux1D + WaveSpeeds1D +
// RiemannSolverByRusanov (equation.f90:988-1106).  (hn = normal velocity,
// ht = tangential); the reference's rotations by n=(1,0)/(0,1) and t=(0,1)/(-1,0)
// multiply by exact 0 and +-1, so an x face passes (h,u,v) and a y face (h,v,u)
// with the tangential component mapped back.
// LAM32 (split form): the bound lam only scales the jump term lam*(UR-UL), so it is
// formed from FP32 square roots; the fluxes themselves stay FP64.
template <bool LAM32 = false>
__device__ __forceinline__ void rusanov(double g, double hL, double nL, double tL, double hR,
                                        double nR, double tR, double& F0, double& F1, double& F2) {
  double FL0 = hL * nL;
  double FL1 = hL * (nL * nL) + 0.5 * g * (hL * hL);
  double FL2 = hL * nL * tL;
  double FR0 = hR * nR;
  double FR1 = hR * (nR * nR) + 0.5 * g * (hR * hR);
  double FR2 = hR * nR * tR;
  double lam;
  if (LAM32) {
    float fl = (float)nL + sqrt_approx((float)(g * hL)),
          fr = (float)nR + sqrt_approx((float)(g * hR));
    lam = (double)fmaxf(fabsf(fl), fabsf(fr));
  } else {
    double fastL = nL + sqrt(g * hL), fastR = nR + sqrt(g * hR);
    lam = dmax(fabs(fastL), fabs(fastR));
  }
  F0 = 0.5 * ((FL0 + FR0) - lam * (hR - hL));
  F1 = 0.5 * ((FL1 + FR1) - lam * (hR * nR - hL * nL));
  F2 = 0.5 * ((FL2 + FR2) - lam * (hR * tR - hL * tL));
}

// Positivity limiter on the 4 face values of h of one cell
// (finitevolume.f90:671-691, identical for x and y).
__device__ __forceinline__ void limit_h(const Grid& gr, double Vc, double wm[4], double wp[4]) {
  double alpha = 0., beta = 0.;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    alpha = alpha + gr.qw[g] * wm[g];
    beta = beta + gr.qw[g] * wp[g];
  }
  double csi = div_rn(Vc - kWLobatto * alpha - kWLobatto * beta, kCsiDen, kCsiRcp);
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    double mmin = csi;
    if (wm[g] < mmin) mmin = wm[g];
    if (wp[g] < mmin) mmin = wp[g];
    // theta = min(1, |a/m|) is exactly 1 when |a| >= |m|: the quotient is then >= 1,
    // and rounding keeps it there; the division only runs when it can limit
    const double ta = Vc - kMinDepth, tm = Vc - mmin;
    double theta;
    if (Vc == mmin || fabs(ta) >= fabs(tm))
      theta = 1.;
    else
      theta = dmin(1., fabs(ta / tm));
    wp[g] = Vc + theta * (wp[g] - Vc);
    wm[g] = Vc + theta * (wm[g] - Vc);
  }
}

// The same limiter on deviations d = W - Vc (split form): csi - Vc =
// -(wL a' + wL b')/(1 - 2 wL) with a' = sum w_g dM_g, b' = sum w_g dP_g.  The sums,
// csi and the minimum are FP32 (they only pick the deviation that binds); theta is
// formed in FP64 from that deviation, so that the limited depth V + theta*d stays
// >= MIN_DEPTH up to FP64 rounding for every face value d >= mmin.
__device__ __forceinline__ void limit_h_dev(const Grid& gr, double Vc, const float dm[4],
                                            const float dp[4], double wm[4], double wp[4]) {
  float alpha = 0.f, beta = 0.f;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    alpha = fmaf(gr.qwf[g], dm[g], alpha);
    beta = fmaf(gr.qwf[g], dp[g], beta);
  }
  const float csi = -((float)kWLobatto * alpha + (float)kWLobatto * beta) * (float)kCsiRcp;
  const double ta = Vc - kMinDepth;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const double mmin = (double)fminf(csi, fminf(dm[g], dp[g]));
    double theta = 1.;
    if (mmin != 0. && fabs(ta) < fabs(mmin))  // else the quotient would be >= 1
      theta = dmin(1., fabs(ta / mmin));
    wp[g] = Vc + theta * (double)dp[g];
    wm[g] = Vc + theta * (double)dm[g];
  }
}

}  // namespace swm
