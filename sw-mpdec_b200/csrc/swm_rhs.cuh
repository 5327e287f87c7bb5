// swm_rhs.cuh -- fused FV right-hand side of one mPDeC stage (sm_100a).
//
// One CTA owns a TX x TY tile of cells and performs, in shared memory, everything
// FVTimeDerivative (finitevolume.f90:402-440) does for those cells:
//   periodic halo + ConsToPrim   (equation.f90:556-782; halo read with wrapped indices)
//   WENO5 x: first sweeps along x, second sweeps along y (reconstruction.f90:408-458)
//   positivity limiter on h     (finitevolume.f90:646-698; seam quirk kept: the
//                                wrapped cell to the right of the domain is not limited)
//   Rusanov at 4 Gauss points + Gauss sum (finitevolume.f90:546-590)
//   the same for y              (reconstruction.f90:464-514, finitevolume.f90:596-757)
//   bathymetry source           (equation.f90:284-413; depth only, 4x4 interior GPs)
//   WB subtraction + momentum update + mass face fluxes (finitevolume.f90:446-540)
// The first sweeps are computed once per (column,row) and shared by the five
// cells whose stencils use them (the reference recomputes them per cell).
//
// Outputs: momentum RHS (Ut(2:3)) and the WB-subtracted mass fluxes FX(1,.), FY(1,.),
// from which the Patankar production/destruction entries are formed exactly as
// UpdateTimeDerivative does (finitevolume.f90:500-523); optionally all flux
// components and the source (WB capture and diagnostics).
#pragma once
#include <type_traits>

#include "swm_device.cuh"
#include "swm_tma.cuh"

namespace swm {

// Split-form bathymetry factor record (64 bytes, 16-byte aligned).
struct SrcSplit {
  float a[4];
  float b[8];
  double s[2];
};

struct RhsArgs {
  Grid gr;
  const double* h;
  const double* hu;
  const double* hv;     // state planes [ny][nx]
  double* ut_hu;
  double* ut_hv;        // momentum RHS [ny][nx]
  double* ut_h;         // nullable: mass RHS Ut(1) (build without PATANKAR, explicit schemes)
  double* fxm;          // mass flux at x faces [ny][nx+1] (face f = left face of cell f)
  double* fym;          // mass flux at y faces [ny+1][nx]
  double* fx_full;      // nullable: [3][ny][nx+1]
  double* fy_full;      // nullable: [3][ny+1][nx]
  double* s_full;       // nullable: [3][ny][nx]
  const double* fx_wb;  // nullable: WB reference fluxes, same layouts
  const double* fy_wb;
  const double* s_wb;
  // nullable: separable source factors with the Gauss weights folded in,
  // src_col [nx][2][4] = {w_a P(x_a), w_a R(x_a)}, src_row [ny][2][4] =
  // {w_b Q(y_b), w_b T(y_b)} for b_x = P Q, b_y = R T (split and FMA forms)
  const double* src_col;
  const double* src_row;
  // nullable: the same factors for the split form as FP32 with their FP64 sums,
  // one record per column (a = w P, b = (w R, w R) pairs, s = sum w P, sum w R) and per
  // row (a = w Q, b = w T, s = sum w Q, sum w T)
  const SrcSplit* src_cols;
  const SrcSplit* src_rows;
  // nullable: b_x, b_y at the 16 interior Gauss points of every cell, evaluated on the
  // host with the analytic formula (equation.f90:451-509), planes [4][4][2][ny*nx]
  const double* bgrad;
  // nullable: status word set to -4 when a tile's TMA load did not complete in time
  int* status;
};

// 16 x 16 tiles: less vertical halo than 32 x 8 (the FP64 form is 4% faster, the split
// form the same) at 105 KB of shared memory, two CTAs per SM
constexpr int RHS_TX = 16;
constexpr int RHS_TY = 16;
constexpr int RHS_NT = 256;

// Shared-memory plan (element counts).
template <typename T>
struct RhsSmem {
  static constexpr int TX = RHS_TX, TY = RHS_TY;
  static constexpr int VX = TX + 6, VY = TY + 6;                  // V tile incl. 3-cell halo
  static constexpr int nV = 3 * VY * VX;                          // double
  static constexpr int F1X = (TY + 4) * (TX + 2);                 // x first sweeps
  static constexpr int F1Y = (TY + 2) * (TX + 4);                 // y first sweeps
  static constexpr int nF1 = 2 * 3 * (F1X > F1Y ? F1X : F1Y);     // T
  static constexpr int WX = TY * (TX + 2);                        // x face-value cells
  static constexpr int WY = (TY + 2) * TX;                        // y face-value cells
  static constexpr int nW = 2 * 3 * 4 * (WX > WY ? WX : WY);      // double
  static constexpr int nFX = 3 * TY * (TX + 1);                   // double
  static constexpr int nFY = 3 * (TY + 1) * TX;                   // double
  // split form: V also as interleaved FP32 (hi, lo) pairs (hi = fl32(V), lo = fl32(V - hi))
  static constexpr int nVF = std::is_same<T, float>::value ? 2 * nV : 0;  // float
  // split form: the source term's y sweeps [4][TY][TX+4] in a buffer of their own, so
  // they can run in the x second-sweep phase (the FP64 form reuses the first-sweep area)
  static constexpr int nVt = std::is_same<T, float>::value ? 4 * TY * (TX + 4) : 0;  // float
  static constexpr size_t bytes = sizeof(double) * (nV + nW + nFX + nFY) + sizeof(T) * nF1 +
                                  sizeof(float) * (nVF + nVt);
};

}  // namespace swm

#ifdef SWM_RHS_NS
// The kernel is compiled in two translation units (EXACT with -fmad=false, FAST
// with contraction); the namespace keeps their host stubs apart.
namespace swm {
namespace SWM_RHS_NS {

// Gauss sum over the four lanes 4k..4k+3 of a face, in the reference's order
// ((0 + t0) + t1) + t2) + t3 (finitevolume.f90:546-590); valid in lane 4k.  Every
// lane of the warp must call it.
__device__ __forceinline__ double quad_sum(double t) {
  const double t1 = __shfl_down_sync(0xffffffffu, t, 1);
  const double t2 = __shfl_down_sync(0xffffffffu, t, 2);
  const double t3 = __shfl_down_sync(0xffffffffu, t, 3);
  double s = __dadd_rn(0.0, t);
  s = __dadd_rn(s, t1);
  s = __dadd_rn(s, t2);
  return __dadd_rn(s, t3);
}

// Gauss-summed fluxes of NF faces: whole faces (4 Gauss points in one thread,
// conflict-free consecutive shared loads) while a full round of NT threads remains,
// then the rest as (face, Gauss point) items, four lanes per face.  flux(f, g, F...)
// evaluates one Gauss point, store(f, s0, s1, s2) keeps the sums.  Both paths round
// every product and sum (no contraction), so a face shared by two tiles gets the same
// flux from either, whichever path each tile takes for it.
template <int NF, int NT, typename Flux, typename Store>
__device__ __forceinline__ void face_pass(const Grid& gr, Flux&& flux, Store&& store) {
  const int tid = threadIdx.x;
  constexpr int FULL = (NF / NT) * NT, REST = NF - FULL;
  for (int f = tid; f < FULL; f += NT) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      double F0, F1, F2;
      flux(f, g, F0, F1, F2);
      s0 = __dadd_rn(s0, __dmul_rn(gr.qw[g], F0));
      s1 = __dadd_rn(s1, __dmul_rn(gr.qw[g], F1));
      s2 = __dadd_rn(s2, __dmul_rn(gr.qw[g], F2));
    }
    store(f, s0, s1, s2);
  }
  if constexpr (REST > 0) {
    static_assert((4 * REST) % 32 == 0, "whole warps in the remainder");
    for (int it0 = 0; it0 < 4 * REST; it0 += NT) {
      if (it0 + (tid & ~31) >= 4 * REST) break;  // warp-uniform
      const int it = it0 + tid, g = it & 3, f = FULL + (it >> 2);
      double F0, F1, F2;
      flux(f, g, F0, F1, F2);
      const double w = gr.qw[g];
      const double s0 = quad_sum(__dmul_rn(w, F0)), s1 = quad_sum(__dmul_rn(w, F1)),
                   s2 = quad_sum(__dmul_rn(w, F2));
      if (g == 0) store(f, s0, s1, s2);
    }
  }
}

// Split form: the first sweeps of two rows (wm, wp packed by row) stored as the (m, p)
// pairs of row 0 at p[0] and of row 1 at p[pitch].
__device__ __forceinline__ void store_mp(unsigned long long* p, int pitch, f2 wm, f2 wp) {
  float m0, m1, p0, p1;
  f2_unpack(wm, m0, m1);
  f2_unpack(wp, p0, p1);
  p[0] = f2_pack(m0, p0).v;
  p[pitch] = f2_pack(m1, p1).v;
}

// MODE: 0 FP64 (EXACT per translation unit), 1 SPLIT.  One CTA, tile origin (i0, j0).
// tm (nullable): tensor maps of the input planes; tiles whose haloed box lies inside
// the grid are then staged by TMA, the others (at the periodic seams) by wrapped loads.
template <int MODE>
__device__ __forceinline__ void rhs_tile(const RhsArgs& a, const RhsTma* tm, const int i0,
                                         const int j0) {
  using T = typename std::conditional<MODE == 1, float, double>::type;
  constexpr bool EX = (MODE == 0) && SWM_EXACT;
  constexpr int TX = RHS_TX, TY = RHS_TY, NT = RHS_NT;
  using SM = RhsSmem<T>;
  constexpr int VX = SM::VX, VY = SM::VY;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sV = reinterpret_cast<double*>(smem_raw);  // [3][VY][VX]
  double* sW = sV + SM::nV;                          // [2][3][4][cells]
  double* sFX = sW + SM::nW;                         // [3][TY][TX+1]
  double* sFY = sFX + SM::nFX;                       // [3][TY+1][TX]
  T* sF1 = reinterpret_cast<T*>(sFY + SM::nFY);      // [2][3][...]
  // split: [3][VY][VX] (hi, lo) pairs, one 8-byte load each
  unsigned long long* sVhl = reinterpret_cast<unsigned long long*>(sF1 + SM::nF1);

  const Grid& gr = a.gr;
  const int nx = gr.nx, ny = gr.ny;
  const int tid = threadIdx.x;

  // ---- load the haloed tile, V = ConsToPrim(U) (equation.f90:778-782) ----
  constexpr int NLD = (VY * VX + NT - 1) / NT;  // cells per thread; all loads issued first
  double lh[NLD], lhu[NLD], lhv[NLD];
  static_assert(kTmaBoxX >= VX + 1 && kTmaBoxY == VY, "TMA box covers the haloed tile");
  static_assert(3 * kTmaBoxX * kTmaBoxY + 16 <= SM::nW, "TMA staging fits the face-value area");
  if (tm != nullptr && tm->enabled && i0 >= 4 && i0 - 4 + kTmaBoxX <= nx && j0 >= 3 &&
      j0 - 3 + kTmaBoxY <= ny) {
    // Interior tile: one thread copies the three 24 x 22 boxes (columns i0-4..i0+19,
    // rows j0-3..j0+18) into the face-value area, unused until the x second sweeps,
    // rounded up to a 128-byte boundary; every thread waits on the barrier.
    __shared__ __align__(8) uint64_t s_bar;
    const unsigned sw0 = smem_u32(sW);
    double* stg = sW + (((sw0 + 127u) & ~127u) - sw0) / sizeof(double);
    if (tid == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (tid == 0) {
      mbar_arrive_expect_tx(&s_bar, 3 * kTmaBoxBytes);
#pragma unroll
      for (int v = 0; v < 3; ++v)
        tma_load_2d(stg + v * kTmaBoxX * kTmaBoxY, &tm->plane[v], i0 - 4, j0 - 3, &s_bar);
    }
    const bool ok = mbar_wait_bounded(&s_bar, 0, kTmaWaitLimit);
    if (__syncthreads_or(!ok)) {  // the copy did not complete: report and give up the tile
      if (tid == 0 && a.status) atomicExch(a.status, -4);
      mbar_wait_bounded(&s_bar, 0, kTmaWaitLimit);  // bounded wait for the copies in flight
      return;
    }
#pragma unroll
    for (int q = 0; q < NLD; ++q) {
      const int it = tid + q * NT;
      if (it < VY * VX) {
        const int k = (it / VX) * kTmaBoxX + it % VX + 1;
        lh[q] = stg[k];
        lhu[q] = stg[kTmaBoxX * kTmaBoxY + k];
        lhv[q] = stg[2 * kTmaBoxX * kTmaBoxY + k];
      }
    }
  } else {
    // Periodic wrap: one conditional add/subtract when the grid is at least one haloed
    // tile wide, the general modulo otherwise.
    const bool wide = nx >= VX && ny >= VY;
#pragma unroll
    for (int q = 0; q < NLD; ++q) {
      const int it = tid + q * NT;
      if (it < VY * VX) {
        int gi = i0 - 3 + it % VX, gj = j0 - 3 + it / VX;
        if (wide) {
          gi += gi < 0 ? nx : (gi >= nx ? -nx : 0);
          gj += gj < 0 ? ny : (gj >= ny ? -ny : 0);
        } else {
          gi = wrap(gi, nx);
          gj = wrap(gj, ny);
        }
        const size_t k = (size_t)gj * nx + gi;
        if (SWM_IN_RANGE(gi, nx, kChkRhsLoad) && SWM_IN_RANGE(gj, ny, kChkRhsLoad)) {
          lh[q] = a.h[k];
          lhu[q] = a.hu[k];
          lhv[q] = a.hv[k];
        } else {
          lh[q] = lhu[q] = lhv[q] = 0.0;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NLD; ++q) {
    const int it = tid + q * NT;
    if (it >= VY * VX) break;
    const int cx = it % VX, cy = it / VX;
    double h = lh[q], hu = lhu[q], hv = lhv[q], u, v;
    cons_to_prim<EX>(h, hu, hv, u, v);
    sV[(0 * VY + cy) * VX + cx] = h;
    sV[(1 * VY + cy) * VX + cx] = u;
    sV[(2 * VY + cy) * VX + cx] = v;
    if constexpr (MODE == 1) {
      const double qv[3] = {h, u, v};
#pragma unroll
      for (int w = 0; w < 3; ++w) {
        const float hi = (float)qv[w];
        sVhl[(w * VY + cy) * VX + cx] = f2_pack(hi, (float)(qv[w] - (double)hi)).v;
      }
    }
  }
  __syncthreads();
#define SV(v, y, x) sV[((v) * VY + (y)) * VX + (x)]
  // split form: V(v,y,x) - V(v,yc,xc) in FP32 from the hi/lo pairs, (hi - hi_c) +
  // (lo - lo_c): exact hi difference for values within a factor 2 (Sterbenz), else
  // one FP32 rounding, the same accuracy as rounding the FP64 difference
  auto dev = [&](int v, int y, int x, int yc, int xc) -> float {
    const int k = (v * VY + y) * VX + x, kc = (v * VY + yc) * VX + xc;
    float dh, dl;
    f2_unpack(sub2(f2{sVhl[k]}, f2{sVhl[kc]}), dh, dl);
    return dh + dl;
  };

  // source term's y sweeps of h at the 4 y Gauss points (split form: own buffer)
  const bool has_src = gr.bathy > 0;
  constexpr int SW_ = TX + 4;  // y-sweep columns i0-2..i0+TX+1
  T* sVt = (MODE == 1) ? reinterpret_cast<T*>(sVhl + SM::nV) : sF1;  // [4][TY][TX+4]
  auto src_sweeps_split = [&]() {
    if constexpr (MODE == 1) {
    static_assert(TY % 2 == 0, "row pairs");
    static_assert(SM::nVt == 4 * TY * SW_, "source sweep buffer");
    for (int it = NT - 1 - tid; it < (TY / 2) * SW_; it += NT) {  // reversed: fills the last round
      int cc = it % SW_, rr = 2 * (it / SW_);
      // U(1) = V(1) = h; rows (j0+rr)-2..+2 -> tile rows rr+1..rr+5; col i0-2+cc -> cc+1
      f2 q[5], w[4];
#pragma unroll
      for (int k = 0; k < 5; ++k)  // k = 2 is each stencil's centre: an exact zero
        if (k != 2)
          q[k] = f2_pack(dev(0, rr + 1 + k, cc + 1, rr + 3, cc + 1),
                         dev(0, rr + 2 + k, cc + 1, rr + 4, cc + 1));
      q[2] = f2_splat(0.f);
      weno5_second_x2<true>(q[0], q[1], q[2], q[3], q[4], w);
#pragma unroll
      for (int g = 0; g < 4; ++g)
        f2_unpack(w[g], sVt[(g * TY + rr) * SW_ + cc], sVt[(g * TY + rr + 1) * SW_ + cc]);
    }
    }
  };

  // ======================= x direction =======================
  {
    constexpr int FW = TX + 2, FH = TY + 4;  // first sweeps: cols i0-1..i0+TX, rows j0-2..j0+TY+1
    T* sTM = sF1;
    T* sTP = sF1 + 3 * FH * FW;
    unsigned long long* sTMP = reinterpret_cast<unsigned long long*>(sF1);  // split: (m, p) pairs
    if constexpr (MODE == 1) {
      // two rows per item (packed pairs), deviations from each stencil's centre
      static_assert(FH % 2 == 0, "row pairs");
      constexpr int FH2 = FH / 2;
      for (int it = tid; it < 3 * FH2 * FW; it += NT) {
        int cc = it % FW, rest = it / FW, rp = rest % FH2, v = rest / FH2;
        const int rr = 2 * rp;
        f2 q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k)  // k = 2 is each stencil's centre: an exact zero
          if (k != 2)
            q[k] = f2_pack(dev(v, rr + 1, cc + k, rr + 1, cc + 2),
                           dev(v, rr + 2, cc + k, rr + 2, cc + 2));
        q[2] = f2_splat(0.f);
        f2 wm, wp;
        weno5_first_x2<true>(q[0], q[1], q[2], q[3], q[4], wm, wp);
        store_mp(sTMP + (v * FH + rr) * FW + cc, FW, wm, wp);
      }
    } else {
      for (int it = tid; it < 3 * FH * FW; it += NT) {
        int cc = it % FW, rest = it / FW, rr = rest % FH, v = rest / FH;
        const double* q = &SV(v, rr + 1, cc);  // V cols (i0-1+cc)-2 .. +2 -> tile cols cc..cc+4
        T wm, wp;
        weno5_first<T, EX>((T)q[0], (T)q[1], (T)q[2], (T)q[3], (T)q[4], wm, wp);
        sTM[(v * FH + rr) * FW + cc] = wm;
        sTP[(v * FH + rr) * FW + cc] = wp;
      }
    }
    __syncthreads();
    // second sweeps along y; cells: cols i0-1..i0+TX (cc), rows j0..j0+TY-1 (rr)
    constexpr int WC = TY * FW;
    for (int it = tid; it < 3 * WC; it += NT) {
      int cc = it % FW, rest = it / FW, rr = rest % TY, v = rest / TY;
      double wmv[4], wpv[4];
      const double Vc = SV(v, rr + 3, cc + 2);
      if constexpr (MODE == 1) {
        float dm[4], dp[4];
        f2 q[5], w[4];
#pragma unroll
        for (int k = 0; k < 5; ++k) {  // k = 2 is the centre row: no offset
          const f2 t = f2{sTMP[(v * FH + rr + k) * FW + cc]};
          q[k] = (k == 2) ? t : add2(f2_splat(dev(v, rr + 1 + k, cc + 2, rr + 3, cc + 2)), t);
        }
        weno5_second_x2(q[0], q[1], q[2], q[3], q[4], w);
#pragma unroll
        for (int g = 0; g < 4; ++g) f2_unpack(w[g], dm[g], dp[g]);
        const int gc = i0 - 1 + cc;
        if (v == 0 && gc != nx) {
          limit_h_dev(gr, Vc, dm, dp, wmv, wpv);
        } else {
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            wmv[g] = Vc + (double)dm[g];
            wpv[g] = Vc + (double)dp[g];
          }
        }
      } else {
        const T* cm = &sTM[(v * FH + rr) * FW + cc];
        const T* cp = &sTP[(v * FH + rr) * FW + cc];
        T tm[4], tp[4];
        weno5_second<T, EX>(cm[0], cm[FW], cm[2 * FW], cm[3 * FW], cm[4 * FW], tm);
        weno5_second<T, EX>(cp[0], cp[FW], cp[2 * FW], cp[3 * FW], cp[4 * FW], tp);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          wmv[g] = tm[g];
          wpv[g] = tp[g];
        }
        const int gc = i0 - 1 + cc;
        if (v == 0 && gc != nx) limit_h(gr, Vc, wmv, wpv);
      }
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        sW[((0 * 3 + v) * 4 + g) * WC + rr * FW + cc] = wmv[g];
        sW[((1 * 3 + v) * 4 + g) * WC + rr * FW + cc] = wpv[g];
      }
    }
    if constexpr (MODE == 1) {  // fills the last, partial round of the second sweeps
      if (has_src) src_sweeps_split();
    }
    __syncthreads();
    // Rusanov at faces f = i0 .. i0+TX (ff), rows rr; left = WP(cell f-1) (cc = ff), right = WM(f)
    auto xface = [&](int f, int g, double& F0, double& F1, double& F2) {
      const int ff = f % (TX + 1), rr = f / (TX + 1);
      const int L = rr * FW + ff, R = rr * FW + ff + 1;
      rusanov<MODE == 1>(gr.g, sW[((1 * 3 + 0) * 4 + g) * WC + L], sW[((1 * 3 + 1) * 4 + g) * WC + L],
              sW[((1 * 3 + 2) * 4 + g) * WC + L], sW[((0 * 3 + 0) * 4 + g) * WC + R],
              sW[((0 * 3 + 1) * 4 + g) * WC + R], sW[((0 * 3 + 2) * 4 + g) * WC + R], F0, F1, F2);
    };
    auto xstore = [&](int f, double s0, double s1, double s2) {
      const int ff = f % (TX + 1), rr = f / (TX + 1);
      sFX[(0 * TY + rr) * (TX + 1) + ff] = s0;
      sFX[(1 * TY + rr) * (TX + 1) + ff] = s1;
      sFX[(2 * TY + rr) * (TX + 1) + ff] = s2;
    };
    face_pass<TY * (TX + 1), NT>(gr, xface, xstore);
    // no barrier: the y first sweeps below share this phase (they write sF1, free since
    // the x second sweeps; this pass reads sW and writes sFX)
  }

  // ======================= y direction =======================
  {
    constexpr int FW = TX + 4, FH = TY + 2;  // first sweeps: cols i0-2..i0+TX+1, rows j0-1..j0+TY
    T* sTM = sF1;
    T* sTP = sF1 + 3 * FH * FW;
    unsigned long long* sTMP = reinterpret_cast<unsigned long long*>(sF1);  // split: (m, p) pairs
    if constexpr (MODE == 1) {
      // two rows per item (packed pairs): the vertical stencils of rows rr and rr+1
      // share four of their six values
      static_assert(FH % 2 == 0, "row pairs");
      constexpr int FH2 = FH / 2;
      for (int it = NT - 1 - tid; it < 3 * FH2 * FW; it += NT) {  // reversed: balances the x faces
        int cc = it % FW, rest = it / FW, rr = 2 * (rest % FH2), v = rest / FH2;
        // V rows (j0-1+rr)-2 .. +2 -> tile rows rr..rr+4; col (i0-2+cc) -> tile col cc+1
        f2 q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k)  // k = 2 is each stencil's centre: an exact zero
          if (k != 2)
            q[k] = f2_pack(dev(v, rr + k, cc + 1, rr + 2, cc + 1),
                           dev(v, rr + k + 1, cc + 1, rr + 3, cc + 1));
        q[2] = f2_splat(0.f);
        f2 wm, wp;
        weno5_first_x2<true>(q[0], q[1], q[2], q[3], q[4], wm, wp);
        store_mp(sTMP + (v * FH + rr) * FW + cc, FW, wm, wp);
      }
    } else {
      for (int it = NT - 1 - tid; it < 3 * FH * FW; it += NT) {  // reversed: balances the x faces
        int cc = it % FW, rest = it / FW, rr = rest % FH, v = rest / FH;
        // V rows (j0-1+rr)-2 .. +2 -> tile rows rr..rr+4; col (i0-2+cc) -> tile col cc+1
        double q0 = SV(v, rr, cc + 1), q1 = SV(v, rr + 1, cc + 1), q2 = SV(v, rr + 2, cc + 1),
               q3 = SV(v, rr + 3, cc + 1), q4 = SV(v, rr + 4, cc + 1);
        T wm, wp;
        weno5_first<T, EX>((T)q0, (T)q1, (T)q2, (T)q3, (T)q4, wm, wp);
        sTM[(v * FH + rr) * FW + cc] = wm;
        sTP[(v * FH + rr) * FW + cc] = wp;
      }
    }
    __syncthreads();
    // second sweeps along x; cells: cols i0..i0+TX-1 (cc), rows j0-1..j0+TY (rr)
    constexpr int WC = FH * TX;
    for (int it = tid; it < 3 * WC; it += NT) {
      int cc = it % TX, rest = it / TX, rr = rest % FH, v = rest / FH;
      double wmv[4], wpv[4];
      const double Vc = SV(v, rr + 2, cc + 3);
      const int gr_row = j0 - 1 + rr;
      if constexpr (MODE == 1) {
        float dm[4], dp[4];
        f2 q[5], w[4];
#pragma unroll
        for (int k = 0; k < 5; ++k) {  // k = 2 is the centre column: no offset
          const f2 t = f2{sTMP[(v * FH + rr) * FW + cc + k]};
          q[k] = (k == 2) ? t : add2(f2_splat(dev(v, rr + 2, cc + 1 + k, rr + 2, cc + 3)), t);
        }
        weno5_second_x2(q[0], q[1], q[2], q[3], q[4], w);
#pragma unroll
        for (int g = 0; g < 4; ++g) f2_unpack(w[g], dm[g], dp[g]);
        if (v == 0 && gr_row != ny) {
          limit_h_dev(gr, Vc, dm, dp, wmv, wpv);
        } else {
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            wmv[g] = Vc + (double)dm[g];
            wpv[g] = Vc + (double)dp[g];
          }
        }
      } else {
        const T* cm = &sTM[(v * FH + rr) * FW + cc];
        const T* cp = &sTP[(v * FH + rr) * FW + cc];
        T tm[4], tp[4];
        weno5_second<T, EX>(cm[0], cm[1], cm[2], cm[3], cm[4], tm);
        weno5_second<T, EX>(cp[0], cp[1], cp[2], cp[3], cp[4], tp);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          wmv[g] = tm[g];
          wpv[g] = tp[g];
        }
        if (v == 0 && gr_row != ny) limit_h(gr, Vc, wmv, wpv);
      }
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        sW[((0 * 3 + v) * 4 + g) * WC + rr * TX + cc] = wmv[g];
        sW[((1 * 3 + v) * 4 + g) * WC + rr * TX + cc] = wpv[g];
      }
    }
    __syncthreads();
    // Rusanov at faces f = j0 .. j0+TY (fr); below = WP(row f-1) (rr = fr), above = WM(f);
    // normal = v (var 2), tangential = u (var 1), so F2 is the hu and F1 the hv component
    auto yface = [&](int f, int g, double& F0, double& F2, double& F1) {
      const int cc = f % TX, fr = f / TX;
      const int L = fr * TX + cc, R = (fr + 1) * TX + cc;
      rusanov<MODE == 1>(gr.g, sW[((1 * 3 + 0) * 4 + g) * WC + L], sW[((1 * 3 + 2) * 4 + g) * WC + L],
              sW[((1 * 3 + 1) * 4 + g) * WC + L], sW[((0 * 3 + 0) * 4 + g) * WC + R],
              sW[((0 * 3 + 2) * 4 + g) * WC + R], sW[((0 * 3 + 1) * 4 + g) * WC + R], F0, F1, F2);
    };
    auto ystore = [&](int f, double s0, double s1, double s2) {
      const int cc = f % TX, fr = f / TX;
      sFY[(0 * (TY + 1) + fr) * TX + cc] = s0;
      sFY[(1 * (TY + 1) + fr) * TX + cc] = s1;
      sFY[(2 * (TY + 1) + fr) * TX + cc] = s2;
    };
    face_pass<(TY + 1) * TX, NT>(gr, yface, ystore);
    // no barrier: the source sweeps below share this phase (they write sF1, whose y
    // first sweeps the y second sweeps have consumed; this pass reads sW, writes sFY)
  }

  // ======================= source term (depth only) =======================
  // (the split form's y sweeps ran in the x second-sweep phase)
  if (has_src) {
    if constexpr (MODE == 0) {
      for (int it = NT - 1 - tid; it < TY * SW_; it += NT) {  // reversed: balances the y faces
        int cc = it % SW_, rr = it / SW_;
        double q0 = SV(0, rr + 1, cc + 1), q1 = SV(0, rr + 2, cc + 1), q2 = SV(0, rr + 3, cc + 1),
               q3 = SV(0, rr + 4, cc + 1), q4 = SV(0, rr + 5, cc + 1);
        T w[4];
        weno5_second<T, EX>((T)q0, (T)q1, (T)q2, (T)q3, (T)q4, w);
#pragma unroll
        for (int g = 0; g < 4; ++g) sVt[(g * TY + rr) * SW_ + cc] = w[g];
      }
    }
  }
  __syncthreads();  // fluxes and source sweeps complete

  // ======================= per-cell epilogue =======================
  for (int it = tid; it < TX * TY; it += NT) {
    int cc = it % TX, rr = it / TX;
    int gi = i0 + cc, gj = j0 + rr;
    if (gi >= nx || gj >= ny) continue;
    double S1 = 0.0, S2 = 0.0;
    if (has_src) {
      double hq[4][4];  // [x-GP a][y-GP b]
      bool done = false;  // split form: S1, S2 already formed from the factor records
      if constexpr (MODE == 1) {
        const double hc = SV(0, rr + 3, cc + 3);
        // depth deviations d_ab = h_ab - hc, y-GP rows b, b+1 packed: wb[b / 2][a]
        f2 wb[2][4];
        T dv[5];
#pragma unroll
        for (int k = 0; k < 5; ++k)  // k = 2 is the centre: an exact zero
          dv[k] = (k == 2) ? 0.f : dev(0, rr + 3, cc + 1 + k, rr + 3, cc + 3);
#pragma unroll
        for (int b = 0; b < 4; b += 2) {
          const T* r0 = &sVt[(b * TY + rr) * SW_ + cc];
          const T* r1 = &sVt[((b + 1) * TY + rr) * SW_ + cc];
          f2 q[5];
#pragma unroll
          for (int k = 0; k < 5; ++k)
            q[k] = (k == 2) ? f2_pack(r0[k], r1[k]) : f2_pack(dv[k] + r0[k], dv[k] + r1[k]);
          weno5_second_x2(q[0], q[1], q[2], q[3], q[4], wb[b / 2]);
        }
        if (a.src_cols) {
          // separable gradient on the deviations, the centre part in FP64:
          //   S_hu = -g (hc sum_a Pw_a sum_b Qw_b + sum_a Pw_a sum_b Qw_b d_ab)
          //   S_hv = -g (hc sum_a Rw_a sum_b Tw_b + sum_b Tw_b sum_a Rw_a d_ab)
          const SrcSplit& C = a.src_cols[gi];
          const SrcSplit& R = a.src_rows[gj];
          const float4 P = __ldg(reinterpret_cast<const float4*>(C.a));
          const ulonglong2 R01 = __ldg(reinterpret_cast<const ulonglong2*>(C.b));
          const ulonglong2 R23 = __ldg(reinterpret_cast<const ulonglong2*>(C.b + 4));
          const ulonglong2 Qp = __ldg(reinterpret_cast<const ulonglong2*>(R.a));
          const ulonglong2 Tp = __ldg(reinterpret_cast<const ulonglong2*>(R.b));
          const double2 cs = __ldg(reinterpret_cast<const double2*>(C.s));
          const double2 rs = __ldg(reinterpret_cast<const double2*>(R.s));
          const float Pa[4] = {P.x, P.y, P.z, P.w};
          const f2 Ra[4] = {f2{R01.x}, f2{R01.y}, f2{R23.x}, f2{R23.y}};  // (R_a, R_a)
          float s1d = 0.f;
#pragma unroll
          for (int aa = 0; aa < 4; ++aa) {
            float x, y;
            f2_unpack(fma2(f2{Qp.y}, wb[1][aa], mul2(f2{Qp.x}, wb[0][aa])), x, y);
            s1d = fmaf(Pa[aa], x + y, s1d);
          }
          f2 r0 = mul2(Ra[0], wb[0][0]), r1 = mul2(Ra[0], wb[1][0]);
#pragma unroll
          for (int aa = 1; aa < 4; ++aa) {
            r0 = fma2(Ra[aa], wb[0][aa], r0);
            r1 = fma2(Ra[aa], wb[1][aa], r1);
          }
          float x, y;
          f2_unpack(fma2(f2{Tp.y}, r1, mul2(f2{Tp.x}, r0)), x, y);
          S1 = -gr.g * fma(hc, cs.x * rs.x, (double)s1d);
          S2 = -gr.g * fma(hc, cs.y * rs.y, (double)(x + y));
          done = true;
        } else {
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int aa = 0; aa < 4; ++aa) {
              float lo, hi;
              f2_unpack(wb[p][aa], lo, hi);
              hq[aa][2 * p] = hc + (double)lo;
              hq[aa][2 * p + 1] = hc + (double)hi;
            }
        }
      } else {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const T* r = &sVt[(b * TY + rr) * SW_ + cc];
          T w[4];
          weno5_second<T, EX>(r[0], r[1], r[2], r[3], r[4], w);
#pragma unroll
          for (int aa = 0; aa < 4; ++aa) hq[aa][b] = (double)w[aa];
        }
      }
      if (!done && a.src_col) {
        // separable gradient: S_hu = -g sum_a Pw_a sum_b Qw_b h_ab,
        //                     S_hv = -g sum_b Tw_b sum_a Rw_a h_ab
        // 16-byte loads of the factor rows (64 bytes per column / row, 16-byte aligned)
        double pc[8], pr[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double2 c2 = __ldg(reinterpret_cast<const double2*>(a.src_col + 8 * (size_t)gi) + q);
          const double2 r2 = __ldg(reinterpret_cast<const double2*>(a.src_row + 8 * (size_t)gj) + q);
          pc[2 * q] = c2.x;
          pc[2 * q + 1] = c2.y;
          pr[2 * q] = r2.x;
          pr[2 * q + 1] = r2.y;
        }
        double s1 = 0.0, s2 = 0.0;
        if constexpr (EX) {
          // FP64 form: every product and sum rounded (the Gauss sums of the reference's
          // source, equation.f90:380-388, regrouped by the separable factors)
#pragma unroll
          for (int aa = 0; aa < 4; ++aa) {
            double in = 0.0;
#pragma unroll
            for (int b = 0; b < 4; ++b) in = __dadd_rn(in, __dmul_rn(pr[b], hq[aa][b]));
            s1 = __dadd_rn(s1, __dmul_rn(pc[aa], in));
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            double in = 0.0;
#pragma unroll
            for (int aa = 0; aa < 4; ++aa) in = __dadd_rn(in, __dmul_rn(pc[4 + aa], hq[aa][b]));
            s2 = __dadd_rn(s2, __dmul_rn(pr[4 + b], in));
          }
        } else {
#pragma unroll
          for (int aa = 0; aa < 4; ++aa) {
            double in = 0.0;
#pragma unroll
            for (int b = 0; b < 4; ++b) in = fma(pr[b], hq[aa][b], in);
            s1 = fma(pc[aa], in, s1);
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            double in = 0.0;
#pragma unroll
            for (int aa = 0; aa < 4; ++aa) in = fma(pc[4 + aa], hq[aa][b], in);
            s2 = fma(pr[4 + b], in, s2);
          }
        }
        S1 = -gr.g * s1;
        S2 = -gr.g * s2;
      } else if (!done) {
        // S = sum_{a (x-GP)} sum_{b (y-GP)} W(a,b) * SourceFunc (equation.f90:380-388,
        // :408-410), gradient from the host table [x-GP][y-GP][comp][cell]
        const size_t nc = (size_t)nx * ny, cell = (size_t)gj * nx + gi;
#pragma unroll
        for (int aa = 0; aa < 4; ++aa) {
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const double bx = a.bgrad[((aa * 4 + b) * 2 + 0) * nc + cell];
            const double by = a.bgrad[((aa * 4 + b) * 2 + 1) * nc + cell];
            double gh = gr.g * hq[aa][b];
            S1 = S1 + gr.wgp[aa][b] * (-(gh * bx));
            S2 = S2 + gr.wgp[aa][b] * (-(gh * by));
          }
        }
      }
    }
    double fxl[3], fxr[3], fyb[3], fyt[3], s[3] = {0.0, S1, S2};
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      fxl[v] = sFX[(v * TY + rr) * (TX + 1) + cc];
      fxr[v] = sFX[(v * TY + rr) * (TX + 1) + cc + 1];
      fyb[v] = sFY[(v * (TY + 1) + rr) * TX + cc];
      fyt[v] = sFY[(v * (TY + 1) + rr + 1) * TX + cc];
    }
    const size_t kx = (size_t)gj * (nx + 1) + gi, ky = (size_t)gj * nx + gi, kc = ky;
    const size_t sfx = (size_t)ny * (nx + 1), sfy = (size_t)(ny + 1) * nx, sc = (size_t)nx * ny;
    if (a.fx_wb) {  // FX = FX - FXWB etc. (finitevolume.f90:485-489)
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        fxl[v] = fxl[v] - a.fx_wb[v * sfx + kx];
        fxr[v] = fxr[v] - a.fx_wb[v * sfx + kx + 1];
        fyb[v] = fyb[v] - a.fy_wb[v * sfy + ky];
        fyt[v] = fyt[v] - a.fy_wb[v * sfy + ky + nx];
        s[v] = s[v] - a.s_wb[v * sc + kc];
      }
    }
    // Ut(2:3) = S - (FX(i)-FX(i-1))/dx - (FY(j)-FY(j-1))/dy (finitevolume.f90:525-527);
    // EXACT rounds the quotients correctly from rdx = RN(1/dx), the others multiply.
    if constexpr (EX) {
      a.ut_hu[kc] = s[1] - div_rn(fxr[1] - fxl[1], gr.dx, gr.rdx) -
                    div_rn(fyt[1] - fyb[1], gr.dy, gr.rdy);
      a.ut_hv[kc] = s[2] - div_rn(fxr[2] - fxl[2], gr.dx, gr.rdx) -
                    div_rn(fyt[2] - fyb[2], gr.dy, gr.rdy);
    } else {
      a.ut_hu[kc] = s[1] - (fxr[1] - fxl[1]) * gr.rdx - (fyt[1] - fyb[1]) * gr.rdy;
      a.ut_hv[kc] = s[2] - (fxr[2] - fxl[2]) * gr.rdx - (fyt[2] - fyb[2]) * gr.rdy;
    }
    if (a.ut_h) {  // Ut(1) = S(1) - dFX(1)/dx - dFY(1)/dy (finitevolume.f90:530-533)
      if constexpr (EX)
        a.ut_h[kc] = s[0] - div_rn(fxr[0] - fxl[0], gr.dx, gr.rdx) -
                     div_rn(fyt[0] - fyb[0], gr.dy, gr.rdy);
      else
        a.ut_h[kc] = s[0] - (fxr[0] - fxl[0]) * gr.rdx - (fyt[0] - fyb[0]) * gr.rdy;
    }
    a.fxm[kx] = fxl[0];
    a.fym[ky] = fyb[0];
    if (gi == nx - 1) a.fxm[kx + 1] = fxr[0];
    if (gj == ny - 1) a.fym[ky + nx] = fyt[0];
    if (a.fx_full) {
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        a.fx_full[v * sfx + kx] = fxl[v];
        a.fy_full[v * sfy + ky] = fyb[v];
        a.s_full[v * sc + kc] = s[v];
        if (gi == nx - 1) a.fx_full[v * sfx + kx + 1] = fxr[v];
        if (gj == ny - 1) a.fy_full[v * sfy + ky + nx] = fyt[v];
      }
    }
  }
#undef SV
}

template <int MODE>
__global__ void __launch_bounds__(RHS_NT, 2)
    rhs_kernel(const RhsArgs a, const __grid_constant__ RhsTma tm) {
  rhs_tile<MODE>(a, &tm, blockIdx.x * RHS_TX, blockIdx.y * RHS_TY);
}

// Ensembles: CTA b computes tile (work[b].y, work[b].z) of problem work[b].x, whose
// descriptor is staged in shared memory; one launch covers every problem's tiles.
template <int MODE>
__global__ void __launch_bounds__(RHS_NT, 2)
    rhs_batch_kernel(const RhsArgs* __restrict__ descs, const int4* __restrict__ work) {
  static_assert(sizeof(RhsArgs) % 8 == 0 && sizeof(RhsArgs) / 8 <= RHS_NT, "descriptor copy");
  __shared__ __align__(16) RhsArgs sa;
  const int4 w = work[blockIdx.x];
  if (threadIdx.x < sizeof(RhsArgs) / 8)
    reinterpret_cast<unsigned long long*>(&sa)[threadIdx.x] =
        reinterpret_cast<const unsigned long long*>(&descs[w.x])[threadIdx.x];
  __syncthreads();
  rhs_tile<MODE>(sa, nullptr, w.y, w.z);
}

}  // namespace SWM_RHS_NS
}  // namespace swm
#endif  // SWM_RHS_NS
