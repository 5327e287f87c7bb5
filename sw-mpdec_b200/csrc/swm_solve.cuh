// swm_solve.cuh -- device code of the Patankar assembly and of the Jacobi solver,
// shared by the single-grid and batched kernels (swm_kernels.cu, built with
// -fmad=false) and by the ensemble step kernels, which live in the RHS units
// (swm_rhs_fast.cu contracts, swm_rhs_exact.cu does not).  Every floating-point
// expression here that a compiler could contract into a fused multiply-add is
// written with explicit roundings (__dmul_rn, __dadd_rn, fma) or sits in a branch
// that only the -fmad=false units instantiate (the FP64 form's exact assembly), so the
// code gives the same bits in every unit.
#pragma once
#include <cstdint>

#include "swm_kernels.cuh"

namespace swm {

// ---------------------------------------------------------------------------
// Residual limbs: |dx| in units of 2^-100 as three 40-bit integers,
// X = floor(v * 2^100) = l2 * 2^80 + l1 * 2^40 + l0 (exact apart from the
// truncation below 2^-100), so the integer sum is order-independent.  X is taken
// from the bits of v: v = m * 2^(e - 1075) with the 53-bit significand m, hence
// X = m * 2^(e - 975) and each limb is m shifted by (e - 975 - 40k), masked --
// integer shifts only, no floating-point-to-integer conversions.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ unsigned long long shift_u64(unsigned long long m, int d) {
  return d >= 0 ? (d < 64 ? m << d : 0ull) : (d > -64 ? m >> -d : 0ull);
}

__host__ __device__ inline void residual_limbs(double v, unsigned long long& l2,
                                               unsigned long long& l1, unsigned long long& l0) {
  const unsigned long long m40 = (1ull << 40) - 1;
  if (!(v < 1048576.0)) {  // >= 2^20 or NaN: saturate (never converged)
    l2 = m40;
    l1 = m40;
    l0 = m40;
    return;
  }
#ifdef __CUDA_ARCH__
  const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
#else
  unsigned long long bits;
  memcpy(&bits, &v, sizeof bits);
#endif
  // v >= 0: no sign bit; e = 0 (zero, subnormal) scales as e = 1 without the hidden bit
  const int e = (int)(bits >> 52);
  const unsigned long long m = (bits & ((1ull << 52) - 1)) | (e ? (1ull << 52) : 0ull);
  const int s = (e ? e : 1) - 975;
  l2 = shift_u64(m, s - 80);  // < 2^40 since v < 2^20
  l1 = shift_u64(m, s - 40) & m40;
  l0 = shift_u64(m, s) & m40;
}


// total <= thresh for sums of limbs (each sum < 2^64): normalise carries, compare.
__device__ __forceinline__ bool limbs_le(unsigned long long s2, unsigned long long s1,
                                         unsigned long long s0, const unsigned long long* t) {
  const unsigned long long m40 = (1ull << 40) - 1;
  s1 += s0 >> 40;
  s0 &= m40;
  s2 += s1 >> 40;
  s1 &= m40;
  if (s2 != t[0]) return s2 < t[0];
  if (s1 != t[1]) return s1 < t[1];
  return s0 <= t[2];
}

// Approximate value of a limb sum (2^-100 units) for planning only.
__device__ __forceinline__ double limbs_value(unsigned long long s2, unsigned long long s1,
                                              unsigned long long s0) {
  return __dadd_rn(__dadd_rn(__dmul_rn((double)s2, 0x1p-20), __dmul_rn((double)s1, 0x1p-60)),
                   __dmul_rn((double)s0, 0x1p-100));
}

// Sweeps of the next pass: a pass costs mostly its tile loads, so one that runs
// past the stop (or is redone) is wasted.  The residual ratio of the last two
// sweeps (rT after rP) extrapolates the sweeps still needed to reach the threshold;
// the next pass runs that many, at most blk.  Iterates and stop indices do not
// depend on pass lengths: every sweep's residual is summed and checked in order.
__device__ __forceinline__ int plan_sweeps(double rT, double rP, double thresh_d, int blk) {
  int plan = blk;
  if (rP > 0. && rT > 0. && rT < rP && thresh_d > 0.) {
    const double need = log(thresh_d / rT) / log(rT / rP);
    if (need > 0. && need < (double)blk) plan = (int)ceil(need);
  }
  return plan < 1 ? 1 : plan;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Stage combination + Patankar assembly for substep m
//   Ua(m,2:3) = Ua(1,2:3) + sum_r dt theta(m,r) FUp(r,2:3)   timediscretization.f90:539-543
//   Mass/Diagonal of MODIFIED_PATANKAR_MATRIX_INVERSION       timediscretization.f90:795-885
// P/D entries are rebuilt from the stored mass fluxes with the same operations
// UpdateTimeDerivative uses (finitevolume.f90:500-523).
// ---------------------------------------------------------------------------
// PATANKAR_DIV(p, h) = 0 if h < MIN_DEPTH, else 2 h p / den(h) with
// den(h) = h^2 + max(h^2, MIN_DEPTH) (timediscretization.f90:913-924).
__device__ __forceinline__ double patankar_den(double h) {
  const double h2 = __dmul_rn(h, h);
  return __dadd_rn(h2, dmax(h2, kMinDepth));
}

// 1/x for the fast forms' Patankar denominators (>= MIN_DEPTH) and diagonals (>= 1):
// the FP32 hardware reciprocal of fl32(x) (relative error < 2^-22 against 1/x) refined
// by two Newton-Raphson steps in FP64, e <- 1 - x r, r <- r + r e, which square the
// error (2^-44, then below the final rounding).  The weights of a cell are the same
// function of its depth wherever they are formed, so production and destruction
// still cancel exactly.
__device__ __forceinline__ double rcp_fast(double x) {
  double r = (double)rcp_((float)x);
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ double hp_read(const AssembleArgs& a, int m, int i, int j) {
  // m, i, j 0-based
  if (a.msteps == 2 && a.compat2) {
    long long L = (long long)m + 2LL * ((long long)i + (long long)a.nx * j);
    int s = (int)(L % 4);
    long long c = L / 4;
    int ic = (int)(c % a.nx), jc = (int)(c / a.nx);
    if (s >= 2) return 0.0;  // Up(3:4,...) are never written by mPDeC2
    if (!SWM_IN_RANGE(jc, a.ny, kChkCompat2)) return 0.0;
    return a.hp[s][(size_t)jc * a.nx + ic];
  }
  return a.hp[m][(size_t)j * a.nx + i];
}

// Inputs of one cell shared by every substep m of a correction iteration.
template <int MS>
struct CellIn {
  double dt, fu[MS], fv[MS], fl[4][MS], hu_n, hv_n;
  double b;  // FAST: the solve's rhs hp(1,.) (timediscretization.f90:887)
};

template <bool FAST, int MS>
__device__ __forceinline__ void load_cell(const AssembleArgs& a, int i, int j, size_t k, size_t kx,
                                          CellIn<MS>& c) {
  c.dt = *a.dt;
  if constexpr (FAST) c.b = hp_read(a, 0, i, j);
#pragma unroll
  for (int r = 0; r < MS; ++r) {
    c.fu[r] = a.fu[r][k];
    c.fv[r] = a.fv[r][k];
    c.fl[0][r] = a.fym[r][k];            // S face, oriented into the cell
    c.fl[1][r] = a.fxm[r][kx];           // W
    c.fl[2][r] = -a.fxm[r][kx + 1];      // E
    c.fl[3][r] = -a.fym[r][k + a.nx];    // N
  }
  c.hu_n = a.hu_n[k];
  c.hv_n = a.hv_n[k];
}

// Outputs of one substep m: Ua(m, 2:3) and its Patankar system (stencil or CSR).
struct StageOut {
  double *hu, *hv, *cS, *cW, *cE, *cN, *cD;
};

// Combination + assembly of substep m (1-based) for one cell from its loaded inputs.
//  exact: the reference's branches and operation order; each quotient correctly
//         rounded (div_rn) from RN(1/len) and one RN(1/den(h)) per depth, i.e. equal
//         to the division it replaces;
//  FAST : weights w(h) = 2h/den(h) from one reciprocal per depth, 1/len folded into
//         them, dt theta_r formed once and every term added by a fused
//         multiply-add (split and FMA forms; the batched assembly shares this code,
//         so ensemble members match single grids).  For a face flux f only one of
//         max(f,0) and max(-f,0) is non-zero; the zero one adds an exact zero.
// hp(m) of the cell and of its S, W, E, N neighbours (m 1-based).
__device__ __forceinline__ void load_hp(const AssembleArgs& a, int m1, int i, int j, double& hK,
                                        double (&hL)[4]) {
  const int nx = a.nx, ny = a.ny, m = m1 - 1;
  const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1;
  const int jm = j == 0 ? ny - 1 : j - 1, jp = j == ny - 1 ? 0 : j + 1;
  hK = hp_read(a, m, i, j);
  hL[0] = hp_read(a, m, i, jm);
  hL[1] = hp_read(a, m, im, j);
  hL[2] = hp_read(a, m, ip, j);
  hL[3] = hp_read(a, m, i, jp);
}

template <bool FAST, int MS>
__device__ __forceinline__ void assemble_stage(const AssembleArgs& a, bool csr, int i, int j,
                                               const CellIn<MS>& c, const double hK,
                                               const double (&hL)[4], const double* theta,
                                               const StageOut& o) {
  const size_t k = (size_t)j * a.nx + i;
  const size_t kj = a.jpitch > 0 ? (size_t)j * a.jpitch + i : k;  // stencil planes
  const double dt = c.dt;
  double M[4] = {0., 0., 0., 0.};
  double D = 1.;
  if constexpr (FAST) {
    // the same sums with dt theta_r formed once, 1/len folded into the depth
    // weights, and each term added by one fused multiply-add
    double cr[MS];
#pragma unroll
    for (int r = 0; r < MS; ++r) cr[r] = dt * theta[r];
    double au = c.hu_n, av = c.hv_n;
#pragma unroll
    for (int r = 0; r < MS; ++r) {
      au = fma(cr[r], c.fu[r], au);
      av = fma(cr[r], c.fv[r], av);
    }
    o.hu[k] = au;
    o.hv[k] = av;
    const double wK = hK >= kMinDepth ? (2. * hK) * rcp_fast(patankar_den(hK)) : 0.;
#pragma unroll
    for (int nb = 0; nb < 4; ++nb) {
      const double ilen = (nb == 0 || nb == 3) ? a.inv_dy : a.inv_dx;
      const double h = hL[nb];
      const double wL = h >= kMinDepth ? (2. * h) * rcp_fast(patankar_den(h)) : 0.;
      const double aL = ilen * wL, aK = ilen * wK;
#pragma unroll
      for (int r = 0; r < MS; ++r) {
        const double f = c.fl[nb][r], pf = dmax(f, 0.), qf = dmax(-f, 0.);
        if (theta[r] > 0.) {
          M[nb] = fma(-(cr[r] * pf), aL, M[nb]);
          D = fma(cr[r] * qf, aK, D);
        } else {
          D = fma(-(cr[r] * pf), aK, D);
          M[nb] = fma(cr[r] * qf, aL, M[nb]);
        }
      }
    }
  } else {
    double au = c.hu_n, av = c.hv_n;
    // ---- explicit momentum (timediscretization.f90:539-543) ----
  #pragma unroll
    for (int r = 0; r < MS; ++r) {
      au = au + dt * theta[r] * c.fu[r];
      av = av + dt * theta[r] * c.fv[r];
    }
    o.hu[k] = au;
    o.hv[k] = av;
    // ---- Patankar weights (timediscretization.f90:795-885) ----
    const double denK = patankar_den(hK), rdenK = __drcp_rn(denK);
  #pragma unroll
    for (int nb = 0; nb < 4; ++nb) {
      const bool ydir = (nb == 0 || nb == 3);
      const double len = ydir ? a.dy : a.dx, ilen = ydir ? a.inv_dy : a.inv_dx;
      const double h = hL[nb], denL = patankar_den(h), rdenL = __drcp_rn(denL);
  #pragma unroll
      for (int r = 0; r < MS; ++r) {
        const double f = c.fl[nb][r], th = theta[r];
        if (f > 0.) {  // production P_KL = f/len
          const double P = div_rn(f, len, ilen);
          if (th > 0.) {
            const double pd = h < kMinDepth ? 0. : div_rn(2. * h * P, denL, rdenL);
            M[nb] = M[nb] - dt * th * pd;
          } else {
            const double pd = hK < kMinDepth ? 0. : div_rn(2. * hK * P, denK, rdenK);
            D = D - dt * th * pd;
          }
        } else if (f < 0.) {  // destruction D_KL = -f/len
          const double Q = div_rn(-f, len, ilen);
          if (th > 0.) {
            const double pd = hK < kMinDepth ? 0. : div_rn(2. * hK * Q, denK, rdenK);
            D = D + dt * th * pd;
          } else {
            const double pd = h < kMinDepth ? 0. : div_rn(2. * h * Q, denL, rdenL);
            M[nb] = M[nb] + dt * th * pd;
          }
        }
      }
    }
  }
  if (csr) {
    // CSR slots S, W, C, E, N of row K (finitevolume.f90:234-261)
    double* mv = a.csr_mass + 5 * k;
    mv[0] = M[0];
    mv[1] = M[1];
    mv[2] = 0.;
    mv[3] = M[2];
    mv[4] = M[3];
    a.csr_diag[k] = D;
  } else if constexpr (FAST) {
    // the fast stencil solver iterates x = b/D - sum (M/D) x: the row divided by its
    // Diagonal, the rhs b = hp(1,.) (timediscretization.f90:887) in the D plane
    const double rD = rcp_fast(D);
    o.cS[kj] = M[0] * rD;
    o.cW[kj] = M[1] * rD;
    o.cE[kj] = M[2] * rD;
    o.cN[kj] = M[3] * rD;
    o.cD[kj] = c.b * rD;
  } else {
    o.cS[kj] = M[0];
    o.cW[kj] = M[1];
    o.cE[kj] = M[2];
    o.cN[kj] = M[3];
    o.cD[kj] = D;
  }
}

// One cell of the combination + assembly of substep a.m.  Every shared input is
// loaded before any arithmetic (MS stages unrolled), so all of a thread's loads are
// in flight together.
template <bool FAST, int MS>
__device__ __forceinline__ void assemble_cell(const AssembleArgs& a, bool csr, const int i,
                                              const int j) {
  const size_t k = (size_t)j * a.nx + i, kx = (size_t)j * (a.nx + 1) + i;
  CellIn<MS> c;
  load_cell<FAST, MS>(a, i, j, k, kx, c);
  double hK, hL[4];
  load_hp(a, a.m, i, j, hK, hL);
  const StageOut o{a.hu_out, a.hv_out, a.cS, a.cW, a.cE, a.cN, a.cD};
  assemble_stage<FAST, MS>(a, csr, i, j, c, hK, hL, a.theta, o);
  if (a.rhs_out) {  // rhs = hp(1,.) (timediscretization.f90:887), in the planes' layout
    const size_t kj = a.jpitch > 0 ? (size_t)j * a.jpitch + i : k;
    a.rhs_out[kj] = hp_read(a, 0, i, j);
  }
}

// One cell of the fast forms' fused assembly of the kMaxFusedStages substeps of a
// correction (assemble_kernel's arithmetic per substep, shared inputs loaded once),
// plus the rhs in the planes' padded layout when rhs_out is set (odd nx, once per step).
__device__ __forceinline__ void assemble_multi_cell(const AssembleMultiArgs& am, const int i,
                                                    const int j) {
  const size_t kk = (size_t)j * am.base.nx + i, kx = (size_t)j * (am.base.nx + 1) + i;
  CellIn<4> cin;
  load_cell<true, 4>(am.base, i, j, kk, kx, cin);
  double hK[kMaxFusedStages], hL[kMaxFusedStages][4];
#pragma unroll
  for (int q = 0; q < kMaxFusedStages; ++q) load_hp(am.base, am.m[q], i, j, hK[q], hL[q]);
#pragma unroll
  for (int q = 0; q < kMaxFusedStages; ++q) {
    const StageOut o{am.hu_out[q], am.hv_out[q], am.cS[q], am.cW[q], am.cE[q], am.cN[q], am.cD[q]};
    assemble_stage<true, 4>(am.base, false, i, j, cin, hK[q], hL[q], am.theta[q], o);
  }
  if (am.base.rhs_out) {
    const size_t kj = am.base.jpitch > 0 ? (size_t)j * am.base.jpitch + i : kk;
    am.base.rhs_out[kj] = cin.b;
  }
}

// ---------------------------------------------------------------------------
// Jacobi (jacobi_iteration.f90:52-87): x^{k+1} = (b - L x^k)/D from x^0 = b,
// residual mean|x^{k+1}-x^k|, stop when <= tol or at maxIter.
// One cooperative persistent launch per solve; passes separated by a bounded
// grid barrier; the stop decision is taken identically by every CTA from the
// integer residual sums.
// ---------------------------------------------------------------------------
// C: JacobiCtl or JacBatchCtl (bar_count, bar_gen, status).
template <typename C>
__device__ bool grid_barrier(C* ctl, long long spin_limit, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &ctl->bar_gen;
    unsigned int gen = *vgen;
    __threadfence();
    unsigned int arrived = atomicAdd(&ctl->bar_count, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      atomicExch(&ctl->bar_count, 0u);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        if (++spins > spin_limit || spin_limit <= 0) {
          ok = 0;
          atomicExch(&ctl->status, -4);
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Stencil tile geometry
constexpr int JBX = 64, JBY = 16, JNT = 256;

template <int TB>
struct JTile {
  static constexpr int HX = JBX + 2 * TB, HY = JBY + 2 * TB, HN = HX * HY;
  static constexpr size_t bytes = sizeof(double) * 8 * HN;
};

// Asynchronous global->shared copies.  Both are weak reads in the memory model: a copy
// issued after a grid barrier (fence + atomics + bar.sync) observes every write made
// before it, such as the previous pass's iterate written by other CTAs.
// 16 bytes through L2 (cp.async.cg, the only form of that size that skips L1).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
// 8 bytes (cp.async.ca).
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}

// Per-thread residual sums for sweep 0 (initial residual) and sweeps 1..kMaxBlock.
// Each |dx| (capped at 2^20; NaN counts as 2^20) is rounded to a multiple of 2^-100
// and split exactly into parts h2 + h1 + h0, multiples of 2^-20, 2^-60 and 2^-100
// with |h1| <= 2^-21, |h0| <= 2^-61: x + C - C rounds x to a multiple of 2^k for
// C = 1.5 * 2^(52+k) and |x| < 2^(51+k), and the remainders are exact.  Each part
// has at most 40 significant bits in its unit, so up to 2^13 of them sum exactly in
// one FP64 accumulator (callers flush before that); the sums are exact integers in
// their units, hence independent of the order of summation.
struct Acc {
  double s2[kMaxBlock + 1], s1[kMaxBlock + 1], s0[kMaxBlock + 1];
};
constexpr int kAccFlushCells = 4096;  // values per thread between flushes, < 2^13

__device__ __forceinline__ void acc_zero(Acc& acc) {
#pragma unroll
  for (int t = 0; t <= kMaxBlock; ++t) {
    acc.s2[t] = 0.;
    acc.s1[t] = 0.;
    acc.s0[t] = 0.;
  }
}

template <int T>
__device__ __forceinline__ void acc_put(Acc& acc, double v) {
  const double a = v < 1048576.0 ? v : 1048576.0;
  const double C2 = 0x1.8p32, C1 = 0x1.8p-8, C0 = 0x1.8p-48;
  const double h2 = __dsub_rn(__dadd_rn(a, C2), C2);
  const double r = __dsub_rn(a, h2);
  const double h1 = __dsub_rn(__dadd_rn(r, C1), C1);
  const double h0 = __dsub_rn(__dadd_rn(__dsub_rn(r, h1), C0), C0);
  acc.s2[T] = __dadd_rn(acc.s2[T], h2);
  acc.s1[T] = __dadd_rn(acc.s1[T], h1);
  acc.s0[T] = __dadd_rn(acc.s0[T], h0);
}

// Every array a stencil pass copies with 16-byte cp.async starts on a 16-byte boundary.
__host__ __device__ __forceinline__ bool arrays_aligned16(const JacobiArgs& a, const double* xin) {
  const unsigned long long u = (unsigned long long)a.cS | (unsigned long long)a.cW |
                               (unsigned long long)a.cE | (unsigned long long)a.cN |
                               (unsigned long long)a.cD | (unsigned long long)a.b |
                               (unsigned long long)xin;
  return (u & 15ull) == 0;
}

// periodic index for -n <= g < 2n
__device__ __forceinline__ int wrap_near(int g, int n) {
  if (g < 0) g += n;
  if (g >= n) g -= n;
  return g;
}

// Sweep T (1..TB) of a pass over a tile in shared memory: the cells of rows
// T..HY-1-T and columns T..HX-1-T, from xp into xn.  The work unit is a pair of
// adjacent cells (lx even, lx + 1) of one row: 16-byte loads of the six
// coefficient pairs and of the centre, south and north pairs of x, 8-byte loads of
// the west and east neighbours.  For odd T the first and last pairs of a row reach
// one column past the region; those cells are computed and stored too, but no later
// sweep reads them (sweep T+1 reads columns T..HX-1-T only), and their neighbour
// loads stay inside the tile arrays since rows 0 and HY-1 are never swept.
// Residuals count the tile's own cells: (lx - TB, ly - TB) < (cx_lim, cy_lim).
// PART (a tile cut by the grid's edge, cx_lim < JBX or cy_lim < JBY): the units cover
// only the (cx_lim + 2 TB) x (cy_lim + 2 TB) box such a tile loads, so its cost
// follows its size; the same argument bounds its reads (the pair reaching one column
// past the region reads at most one unloaded column, and no later sweep reads it).
__device__ __forceinline__ double2 lds2(const double* p) {
  return *reinterpret_cast<const double2*>(p);
}

template <int TB, int T, bool RECIP, bool PART>
__device__ __forceinline__ void tile_sweep(const double* sm, const double* xp, double* xn,
                                           int cx_lim, int cy_lim, Acc& acc) {
  using G = JTile<TB>;
  constexpr int HX = G::HX, HN = G::HN;
  constexpr int P0 = T / 2, NP = (HX - T - 1) / 2 - P0 + 1;  // pairs covering [T, HX-T)
  constexpr int NU = NP * (G::HY - 2 * T), NQ = (NU + JNT - 1) / JNT;
  static_assert(HX % 2 == 0 && HN % 2 == 0, "16-byte pairs");
  // PART: np >= 1 pairs per row, nu units; u / np = (u * mul) >> 32 with
  // mul = floor(2^32 / np) + 1 (33 bits for np = 1), exact for u * np < 2^32
  int np = NP, nu = NU;
  unsigned long long mul = 0;
  if constexpr (PART) {
    np = (cx_lim + 2 * TB - T - 1) / 2 - P0 + 1;
    nu = np * (cy_lim + 2 * TB - 2 * T);
    mul = (1ull << 32) / (unsigned)np + 1ull;
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const int u = threadIdx.x + q * JNT;
    if (PART ? u >= nu : (NU % JNT != 0 && u >= NU)) break;
    int row, pr;
    if constexpr (PART) {
      row = (int)(((unsigned long long)u * mul) >> 32);
      pr = u - row * np;
    } else {
      row = u / NP;
      pr = u % NP;
    }
    const int ly = T + row, lx = 2 * (P0 + pr);
    const int c = ly * HX + lx;
    // RECIP (split form): the planes hold the row divided by its Diagonal and b/D
    const double2 cS = lds2(sm + c), cW = lds2(sm + HN + c), cE = lds2(sm + 2 * HN + c),
                  cN = lds2(sm + 3 * HN + c), cD = lds2(sm + 4 * HN + c),
                  cB = RECIP ? cD : lds2(sm + 5 * HN + c);
    const double2 xs = lds2(xp + c - HX), xc = lds2(xp + c), xq = lds2(xp + c + HX);
    const double xw = xp[c - 1], xe = xp[c + 2];
    // product = (((S x_S + W x_W) + E x_E) + N x_N); the zero centre slot of the
    // reference CSR row adds an exact zero and is skipped.
    double p0 = __dmul_rn(cS.x, xs.x), p1 = __dmul_rn(cS.y, xs.y);
    p0 = __dadd_rn(p0, __dmul_rn(cW.x, xw));
    p1 = __dadd_rn(p1, __dmul_rn(cW.y, xc.x));
    p0 = __dadd_rn(p0, __dmul_rn(cE.x, xc.y));
    p1 = __dadd_rn(p1, __dmul_rn(cE.y, xe));
    p0 = __dadd_rn(p0, __dmul_rn(cN.x, xq.x));
    p1 = __dadd_rn(p1, __dmul_rn(cN.y, xq.y));
    double2 v;
    v.x = RECIP ? __dsub_rn(cD.x, p0) : __ddiv_rn(__dsub_rn(cB.x, p0), cD.x);
    v.y = RECIP ? __dsub_rn(cD.y, p1) : __ddiv_rn(__dsub_rn(cB.y, p1), cD.y);
    *reinterpret_cast<double2*>(xn + c) = v;
    if ((unsigned)(ly - TB) < (unsigned)cy_lim) {
      if ((unsigned)(lx - TB) < (unsigned)cx_lim) acc_put<T>(acc, fabs(__dsub_rn(v.x, xc.x)));
      if ((unsigned)(lx + 1 - TB) < (unsigned)cx_lim) acc_put<T>(acc, fabs(__dsub_rn(v.y, xc.y)));
    }
  }
}

// Sweeps T..Tp of a pass, each followed by a block barrier; xp ends on the last iterate.
template <int TB, int T, bool RECIP, bool PART>
__device__ __forceinline__ void tile_sweeps(const double* sm, double*& xp, double*& xn, int Tp,
                                            int cx_lim, int cy_lim, Acc& acc) {
  if constexpr (T <= TB) {
    if (T <= Tp) {
      tile_sweep<TB, T, RECIP, PART>(sm, xp, xn, cx_lim, cy_lim, acc);
      __syncthreads();
      double* tmp = xp;
      xp = xn;
      // a first sweep that read x^0 = b from b's own tile hands over the x0 buffer
      xn = (tmp == sm + 5 * JTile<TB>::HN) ? const_cast<double*>(sm) + 6 * JTile<TB>::HN : tmp;
      tile_sweeps<TB, T + 1, RECIP, PART>(sm, xp, xn, Tp, cx_lim, cy_lim, acc);
    }
  }
}

// Block reduction of the per-thread sums into s_acc (sweeps 0..TB) as 40-bit limbs
// [2^80, 2^40, 1] of 2^-100 units.  The parts' sums are exact integers below 2^53
// in their units; carries normalise the (possibly negative) lower parts, and a
// thread's top limb is capped at 2^40 - 1 (its sum is then >= 2^20, far above any
// stop threshold).
template <int TB>
__device__ __forceinline__ void acc_reduce(Acc& acc, unsigned long long (*s_acc)[3]) {
  const long long m40 = (1ll << 40) - 1;
#pragma unroll
  for (int t = 0; t <= TB; ++t) {
    const long long S2 = __double2ll_rn(__dmul_rn(acc.s2[t], 0x1p20));
    const long long S1 = __double2ll_rn(__dmul_rn(acc.s1[t], 0x1p60));
    const long long S0 = __double2ll_rn(__dmul_rn(acc.s0[t], 0x1p100));
    const long long n1 = S1 + (S0 >> 40);  // arithmetic shifts: floor division
    const long long n2 = S2 + (n1 >> 40);
    const unsigned long long limb[3] = {(unsigned long long)(n2 < m40 ? n2 : m40),
                                        (unsigned long long)(n1 & m40),
                                        (unsigned long long)(S0 & m40)};
    acc.s2[t] = 0.;
    acc.s1[t] = 0.;
    acc.s0[t] = 0.;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      unsigned long long v = warp_sum_u64(limb[l]);
      if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_acc[t][l], v);
    }
  }
}

// The tile's haloed box (JBX + 2TB) x (JBY + 2TB) of the system and of the iterate
// into shared memory (b's tile holds x^0 on a first pass).  PART (a tile cut by the
// grid's edge): only the (cx_lim + 2TB) x (cy_lim + 2TB) box its sweeps read.
template <int TB, bool RECIP, bool PART>
__device__ __forceinline__ void tile_load(const JacobiArgs& a, const double* xin, double* sm,
                                          int i0, int j0, int cx_lim, int cy_lim, int pitch,
                                          bool pairs, bool small, bool from_b) {
  using G = JTile<TB>;
  constexpr int HX = G::HX, HY = G::HY, HN = G::HN, NW = JNT / 32;
  double* sS = sm;
  double* sW = sS + HN;
  double* sE = sW + HN;
  double* sN = sE + HN;
  double* sD = sN + HN;
  double* sB = sD + HN;
  double* x0 = sB + HN;
  const int nx = a.nx, ny = a.ny;
  // the system's arrays, read once: in the batched solver `a` is a descriptor staged
  // in shared memory, and a shared load per copy address made it 28% slower
  const double *pS = a.cS, *pW = a.cW, *pE = a.cE, *pN = a.cN, *pD = a.cD, *pB = a.b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wx = PART ? min(HX, cx_lim + 2 * TB) : HX, wy = PART ? min(HY, cy_lim + 2 * TB) : HY;
  if (pairs) {
    // even pitch, no multiple wrap: a pair (gi, gi + 1) with gi even and gi + 1 < nx
    // is one 16-byte copy per array.  With even nx that is every pair; with odd nx
    // (rows padded to an even pitch) the pair that reaches the seam, and the pairs
    // of a seam tile's wrapped halo (odd gi), take two 8-byte copies instead.
    for (int ly = warp; ly < wy; ly += NW) {
      const int gj = wrap_near(j0 - TB + ly, ny);
      const size_t row = (size_t)gj * pitch;
      for (int lp = lane; lp < (wx + 1) / 2; lp += 32) {
        const int lx = 2 * lp;
        const int gi = wrap_near(i0 - TB + lx, nx);
        const size_t g = row + gi;
        const int c = ly * HX + lx;
        if (!SWM_IN_RANGE(gi, nx, kChkJacPairs) || !SWM_IN_RANGE(gj, ny, kChkJacPairs))
          continue;
        if ((gi & 1) == 0 && gi + 1 < nx) {
          cp_async16(&sS[c], &pS[g]);
          cp_async16(&sW[c], &pW[g]);
          cp_async16(&sE[c], &pE[g]);
          cp_async16(&sN[c], &pN[g]);
          cp_async16(&sD[c], &pD[g]);
          if (!RECIP || from_b) cp_async16(&sB[c], &pB[g]);  // RECIP: b only for x^0
          if (!from_b) cp_async16(&x0[c], &xin[g]);
        } else {
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const size_t ge = e == 0 ? g : row + (gi + 1 < nx ? gi + 1 : 0);
            cp_async8(&sS[c + e], &pS[ge]);
            cp_async8(&sW[c + e], &pW[ge]);
            cp_async8(&sE[c + e], &pE[ge]);
            cp_async8(&sN[c + e], &pN[ge]);
            cp_async8(&sD[c + e], &pD[ge]);
            if (!RECIP || from_b) cp_async8(&sB[c + e], &pB[ge]);
            if (!from_b) cp_async8(&x0[c + e], &xin[ge]);
          }
        }
      }
    }
    cp_async_wait_all();
  } else {
    for (int ly = warp; ly < wy; ly += NW) {
      int gj = j0 - TB + ly;
      gj = small ? wrap(gj, ny) : wrap_near(gj, ny);
      const size_t row = (size_t)gj * pitch;
      for (int lx = lane; lx < wx; lx += 32) {
        int gi = i0 - TB + lx;
        gi = small ? wrap(gi, nx) : wrap_near(gi, nx);
        const size_t g = row + gi;
        const int c = ly * HX + lx;
        if (!SWM_IN_RANGE(gi, nx, kChkJacCells) || !SWM_IN_RANGE(gj, ny, kChkJacCells)) continue;
        cp_async8(&sS[c], &pS[g]);
        cp_async8(&sW[c], &pW[g]);
        cp_async8(&sE[c], &pE[g]);
        cp_async8(&sN[c], &pN[g]);
        cp_async8(&sD[c], &pD[g]);
        if (!RECIP || from_b) cp_async8(&sB[c], &pB[g]);
        if (!from_b) cp_async8(&x0[c], &xin[g]);
      }
    }
    cp_async_wait_all();
  }
}

// One stencil pass of Tp <= TB sweeps over every tile of this CTA.  A tile is a
// JBX x JBY block of cells plus a TB-cell halo in shared memory; sweep t updates
// the region shrunk by t, so after Tp sweeps the tile interior holds x^{k+Tp},
// bit-identical to Tp global sweeps.  Warps own rows, lanes own columns.
template <int TB, bool RECIP, bool ONE_TILE>
__device__ void stencil_tiles(const JacobiArgs& a, const double* xin, double* xout, int Tp,
                              bool first, Acc& acc, double* sm, int tile_first,
                              unsigned long long (*s_acc)[3]) {
  using G = JTile<TB>;
  constexpr int HX = G::HX, HY = G::HY, HN = G::HN, NW = JNT / 32;
  double* sB = sm + 5 * HN;
  double* x0 = sm + 6 * HN;
  double* x1 = sm + 7 * HN;
  const int nx = a.nx, ny = a.ny, pitch = a.pitch > 0 ? a.pitch : nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool small = (nx < HX) || (ny < HY);
  // 16-byte pairs need an even first column (i0 - TB), an even row pitch and 16-byte
  // aligned arrays (the allocation-free entry takes the caller's pointers as given)
  const bool pairs = (TB % 2 == 0) && !small && (pitch % 2 == 0) && arrays_aligned16(a, xin);
  // first pass: x^0 = b, already in the b tile (sweep 1 reads it there)
  const bool from_b = xin == a.b;
  const int tx = (nx + JBX - 1) / JBX, ty = (ny + JBY - 1) / JBY;
  // ONE_TILE: exactly tile `tile_first` (ensembles); else every CTA-strided tile
  const int t_end = ONE_TILE ? tile_first + 1 : tx * ty;
  const int t_step = ONE_TILE ? 1 : gridDim.x;
  // values a thread adds per sweep and tile: two per pair unit of sweep 1
  constexpr int kPerTile = 2 * ((((HX - 2) / 2 + 1) * (HY - 2) + JNT - 1) / JNT);
  int since_flush = 0;
  for (int tile = tile_first; tile < t_end; tile += t_step) {
    const int i0 = (tile % tx) * JBX, j0 = (tile / tx) * JBY;
    const int cx_lim = min(JBX, nx - i0), cy_lim = min(JBY, ny - j0);
    if (!ONE_TILE && (since_flush += kPerTile) > kAccFlushCells) {
      acc_reduce<TB>(acc, s_acc);  // keep the per-thread part sums exact
      since_flush = kPerTile;
    }
    // ensembles: a tile cut by the grid's edge loads and sweeps only the box it needs
    // (their grids are small, edge tiles common); the single-grid kernel keeps one
    // code path, which measured 2% faster with the partial variant compiled out
    const bool part = ONE_TILE && (cx_lim < JBX || cy_lim < JBY);
    if (part)
      tile_load<TB, RECIP, true>(a, xin, sm, i0, j0, cx_lim, cy_lim, pitch, pairs, small, from_b);
    else
      tile_load<TB, RECIP, false>(a, xin, sm, i0, j0, cx_lim, cy_lim, pitch, pairs, small, from_b);
    __syncthreads();
    if (first) {  // initial residual mean|0 - b| (jacobi_iteration.f90:69)
      for (int ly = TB + warp; ly < TB + JBY; ly += NW)
        for (int lx = TB + lane; lx < TB + JBX; lx += 32)
          if (i0 + lx - TB < nx && j0 + ly - TB < ny) acc_put<0>(acc, fabs(0. - sB[ly * HX + lx]));
    }
    double* xp = from_b ? sB : x0;
    double* xn = x1;
    if (part)
      tile_sweeps<TB, 1, RECIP, true>(sm, xp, xn, Tp, cx_lim, cy_lim, acc);
    else
      tile_sweeps<TB, 1, RECIP, false>(sm, xp, xn, Tp, cx_lim, cy_lim, acc);
    for (int ly = TB + warp; ly < TB + JBY; ly += NW) {
      const int gj = j0 + ly - TB;
      if (gj >= ny) continue;
      for (int lx = TB + lane; lx < TB + JBX; lx += 32) {
        const int gi = i0 + lx - TB;
        if (gi < nx) xout[(size_t)gj * pitch + gi] = xp[ly * HX + lx];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Ensembles: one cooperative launch solves the Patankar systems of every problem.
// Each pass visits the tiles of all still-active problems; residual limbs are
// flushed per tile into that problem's accumulators; after a grid barrier CTA 0
// applies the single-problem stop rule to every problem (stop, redo the pass with
// fewer sweeps, or continue), and a second barrier publishes the decisions.
// ---------------------------------------------------------------------------
// CTA 0: the stop rule of jacobi_iteration.f90:71-81 for every active system.
static __device__ void batch_decide(const JacobiBatchArgs& a, int blk, int* s_cnt) {
  if (threadIdx.x == 0) *s_cnt = 0;
  __syncthreads();
  int active = 0;
  const int nsys = a.nsets * a.nprob;
  for (int p = threadIdx.x; p < nsys; p += blockDim.x) {
    JacBatchState* S = &a.st[p];
    if (!__ldcg(&S->active)) continue;
    const JacobiArgs& d = a.descs[p];
    int k = __ldcg(&S->k), Tp = __ldcg(&S->Tp);
    const int xnext = __ldcg(&S->xnext);  // the buffer the pass just wrote
    const int first = __ldcg(&S->first), rollback = __ldcg(&S->rollback);
    int act = 1;
    if (rollback) {  // the redone pass delivered x^{final_k}
      act = 0;
      S->result = xnext;
    } else {
      int stop = -1;
      if (first && limbs_le(__ldcg(&S->acc[0][0]), __ldcg(&S->acc[0][1]),
                            __ldcg(&S->acc[0][2]), d.thresh)) {
        stop = 0;
      } else {
        for (int t = 1; t <= Tp; ++t)
          if (limbs_le(__ldcg(&S->acc[t][0]), __ldcg(&S->acc[t][1]), __ldcg(&S->acc[t][2]),
                       d.thresh)) {
            stop = t;
            break;
          }
      }
      S->first = 0;
      if (stop == 0) {
        act = 0;
        S->result = 0;
        S->final_k = 0;
      } else if (stop > 0) {
        S->final_k = k + stop;
        if (stop < Tp) {
          S->rollback = 1;
          S->Tp = stop;
        } else {
          act = 0;
          S->result = xnext;
        }
      } else {
        k += Tp;
        S->k = k;
        if (k >= d.maxiter) {
          act = 0;
          S->maxhit = 1;
          S->final_k = k;
          S->result = xnext;
        } else {
          S->cur = xnext;
          const double rT = limbs_value(__ldcg(&S->acc[Tp][0]), __ldcg(&S->acc[Tp][1]),
                                        __ldcg(&S->acc[Tp][2]));
          const double rP = Tp >= 2 ? limbs_value(__ldcg(&S->acc[Tp - 1][0]),
                                                  __ldcg(&S->acc[Tp - 1][1]),
                                                  __ldcg(&S->acc[Tp - 1][2]))
                                    : __ldcg(&S->r_prev);
          S->r_prev = rT;
          const double th = limbs_value(d.thresh[0], d.thresh[1], d.thresh[2]);
          const int plan = plan_sweeps(rT, rP, th, blk);
          S->Tp = (d.maxiter - k < plan) ? d.maxiter - k : plan;
          // the next pass writes the other ping-pong buffer or, when it is expected to
          // be the last, the destination itself (not the rhs, not the pass's input, and
          // only with unpadded rows), which saves copying the result there
          const bool expect_stop = rP > 0. && rT > 0. && rT < rP && th > 0. &&
                                   log(th / rT) / log(rT / rP) <= (double)blk;
          const int pitch = d.pitch > 0 ? d.pitch : d.nx;
          S->xnext = (expect_stop && pitch == d.nx && d.out != d.b && xnext != 3)
                         ? 3
                         : (xnext == 1 ? 2 : 1);
        }
      }
    }
    S->active = act;
    for (int q = 0; q < (kMaxBlock + 1) * 3; ++q) (&S->acc[0][0])[q] = 0ull;
    active += act;
  }
  if (active) atomicAdd(s_cnt, active);
  __syncthreads();
  if (threadIdx.x == 0) {
    a.ctl->n_active = *s_cnt;
    __threadfence();
  }
}

constexpr int kJacChunk = 4;  // work items per counter fetch of a batched solve

// One batched solve of a.nsets x a.nprob independent systems (system set q, problem
// p -> system q * nprob + p, descriptor descs[system]); every CTA of the grid takes
// part and every grid barrier is passed by all of them.  Returns false when a
// barrier wait gave up (status -4 recorded).  The final iterates are delivered to
// each system's destination before it returns (without a closing barrier).
template <int TB, bool RECIP>
__device__ __forceinline__ bool jacobi_batch_solve(const JacobiBatchArgs& a, double* jsm) {
  __shared__ unsigned long long s_acc[kMaxBlock + 1][3];
  __shared__ __align__(16) JacobiArgs sd;
  __shared__ int s_ok, s_cnt, s_p, s_active, s_Tp, s_first, s_cur, s_xnext, s_next;
  __shared__ int2 s_items[2][kJacChunk];  // (system, tile) items of two chunks
  __shared__ int s_claim[2];              // the chunk after the current one
  static_assert(sizeof(JacobiArgs) % 8 == 0 && sizeof(JacobiArgs) / 8 <= JNT, "descriptor copy");
  const int blk = a.block < 1 ? 1 : (a.block > TB ? TB : a.block);
  const int nsys = a.nsets * a.nprob, nwork = a.nsets * a.ntiles;
  if (a.work && blockIdx.x == 0 && threadIdx.x == 0) *a.work = 0u;  // visible after the barrier
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nsys; p += gridDim.x * blockDim.x) {
    JacBatchState* S = &a.st[p];
    const int mi = a.descs[p].maxiter;
    S->active = 1;
    S->k = 0;
    S->Tp = (mi < blk) ? mi : blk;
    S->rollback = 0;
    S->first = 1;
    S->cur = 0;
    S->xnext = 1;
    S->result = 0;
    S->final_k = 0;
    S->maxhit = 0;
    S->r_prev = -1.0;
    for (int q = 0; q < (kMaxBlock + 1) * 3; ++q) (&S->acc[0][0])[q] = 0ull;
  }
  if (!grid_barrier(a.ctl, a.spin_limit, &s_ok)) return false;
  Acc acc;
  acc_zero(acc);
  int loaded = -1;
  // values a thread adds per sweep slot and tile (as stencil_tiles counts them); the
  // part sums are flushed before they could exceed kAccFlushCells values
  constexpr int kPerTile =
      2 * ((((JTile<TB>::HX - 2) / 2 + 1) * (JTile<TB>::HY - 2) + JNT - 1) / JNT);
  // the staged system's sums go to its accumulators (a CTA-uniform call)
  auto flush = [&]() {
    if (s_active) {
      acc_reduce<TB>(acc, s_acc);
      __syncthreads();
      if (threadIdx.x < (TB + 1) * 3) {
        const unsigned long long v = (&s_acc[0][0])[threadIdx.x];
        if (v) atomicAdd(&(&a.st[s_p].acc[0][0])[threadIdx.x], v);
      }
    }
  };
  // stage system sys: its pass state, its descriptor, zeroed block sums
  auto stage = [&](int sys) {
    __syncthreads();  // the previous system's tiles and flush are done
    if (threadIdx.x == 0) {
      const JacBatchState* S = &a.st[sys];
      s_p = sys;
      s_active = __ldcg(&S->active);
      s_Tp = __ldcg(&S->Tp);
      s_first = __ldcg(&S->first);
      s_cur = __ldcg(&S->cur);
      s_xnext = __ldcg(&S->xnext);
    }
    if (sys != loaded) {
      if (threadIdx.x < sizeof(JacobiArgs) / 8)
        reinterpret_cast<unsigned long long*>(&sd)[threadIdx.x] =
            reinterpret_cast<const unsigned long long*>(&a.descs[sys])[threadIdx.x];
      loaded = sys;
    }
    if (threadIdx.x < (kMaxBlock + 1) * 3) (&s_acc[0][0])[threadIdx.x] = 0ull;
    __syncthreads();
  };
  auto tile = [&](int t) {
    const double* xin = s_cur == 0 ? sd.b : (s_cur == 1 ? sd.xa : (s_cur == 2 ? sd.xb : sd.out));
    double* xout = s_xnext == 1 ? sd.xa : (s_xnext == 2 ? sd.xb : sd.out);
    stencil_tiles<TB, RECIP, true>(sd, xin, xout, s_Tp, s_first != 0, acc, jsm, t, s_acc);
  };
  for (;;) {
    if (a.work) {
      // chunks of kJacChunk consecutive work items claimed from the shared counter
      // (dynamic balance) two ahead: while a chunk runs, the next chunk's items are
      // read into registers and the chunk after it is claimed; both are published at
      // the chunk's closing barrier, so no chunk waits on a global round trip.  A
      // system stays staged, and its sums in the thread accumulators, while
      // consecutive items belong to it.
      auto item = [&](int w) {  // (system, tile) of work item w < nwork
        const int set = w / a.ntiles;
        const int2 t = a.tiles[w - set * a.ntiles];
        return make_int2(set * a.nprob + t.x, t.y);
      };
      __syncthreads();
      if (threadIdx.x == 0) {
        s_next = (int)atomicAdd(a.work, 1u) * kJacChunk;
        s_claim[0] = (int)atomicAdd(a.work, 1u) * kJacChunk;
      }
      __syncthreads();
      if (threadIdx.x < kJacChunk && s_next + (int)threadIdx.x < nwork)
        s_items[0][threadIdx.x] = item(s_next + threadIdx.x);
      int cur = -1, since = 0, buf = 0;
      int w0 = s_next;
      __syncthreads();
      while (w0 < nwork) {
        const int wn = s_claim[buf];  // the next chunk
        int2 pre = make_int2(0, 0);   // its items, in flight while this chunk runs
        if (threadIdx.x < kJacChunk && wn + (int)threadIdx.x < nwork)
          pre = item(wn + threadIdx.x);
        int nxt = 0;  // the chunk after it
        if (threadIdx.x == 0) nxt = (int)atomicAdd(a.work, 1u) * kJacChunk;
        const int w1 = w0 + kJacChunk < nwork ? w0 + kJacChunk : nwork;
        for (int w = w0; w < w1; ++w) {
          const int2 it = s_items[buf][w - w0];  // (system, tile)
          const int sys = it.x;
          if (sys != cur || since + kPerTile > kAccFlushCells) {
            if (cur >= 0) flush();
            stage(sys);
            cur = sys;
            since = 0;
          }
          if (s_active) {
            tile(it.y);
            since += kPerTile;
          }
        }
        if (threadIdx.x < kJacChunk) s_items[buf ^ 1][threadIdx.x] = pre;
        if (threadIdx.x == 0) s_claim[buf ^ 1] = nxt;
        __syncthreads();  // the chunk is done; the next one's items and claim are visible
        buf ^= 1;
        w0 = wn;
      }
      if (cur >= 0) flush();
    } else {
      // work items strided by CTA, each system flushed per item
      for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int set = w / a.ntiles;
        const int2 t = a.tiles[w - set * a.ntiles];
        stage(set * a.nprob + t.x);
        if (s_active) {
          tile(t.y);
          flush();
        }
      }
    }
    if (!grid_barrier(a.ctl, a.spin_limit, &s_ok)) return false;
    if (blockIdx.x == 0) {
      batch_decide(a, blk, &s_cnt);
      if (a.work && threadIdx.x == 0) *a.work = 0u;  // the next pass's items start at 0
    }
    if (!grid_barrier(a.ctl, a.spin_limit, &s_ok)) return false;
    if (threadIdx.x == 0) s_cnt = __ldcg(&a.ctl->n_active);
    __syncthreads();
    if (s_cnt == 0) break;
  }
  // deliver every system's final iterate (haVec) to its destination, unless the last
  // pass wrote it there
  for (int p = 0; p < nsys; ++p) {
    const JacobiArgs& d = a.descs[p];
    const int res = __ldcg(&a.st[p].result);
    if (res == 3) continue;
    const double* src = res == 1 ? d.xa : d.xb;
    const int n = d.nx * d.ny, pitch = d.pitch > 0 ? d.pitch : d.nx;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
      const int s = pitch == d.nx ? q : (q / d.nx) * pitch + q % d.nx;  // padded rows
      d.out[q] = res == 0 ? 0. : __ldcg(&src[s]);
    }
  }
  if (blockIdx.x == 0) {
    for (int p = threadIdx.x; p < nsys; p += blockDim.x) {
      a.iters[p] = __ldcg(&a.st[p].final_k);
      if (__ldcg(&a.st[p].maxhit)) atomicMax(&a.ctl->status, 1);
    }
  }
  return true;
}

}  // namespace swm
