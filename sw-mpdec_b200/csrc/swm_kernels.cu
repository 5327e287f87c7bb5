// swm_kernels.cu -- memory-bound kernels of the mPDeC5 step (sm_100a).
// Built with -fmad=false: every FP64 expression here rounds exactly as the
// reference's source order does (no contraction), which makes the Patankar
// matrix and the Jacobi iterates bit-identical to the CPU restatement given the
// same fluxes, and the CSR and matrix-free solvers bit-identical to each other.
#include <cooperative_groups.h>

#include <cstdio>
#include <cstring>

#include "../../include/swm.h"
#include "swm_kernels.cuh"
#include "swm_solve.cuh"

namespace swm {

SWM_CHECK_READER(check_record_kernels)

void residual_limbs_host(double v, unsigned long long out[3]) {
  unsigned long long a, b, c;
  residual_limbs(v, a, b, c);
  out[0] = a;
  out[1] = b;
  out[2] = c;
}

// ---------------------------------------------------------------------------
// TimeStep (equation.f90:791-837): LambdaMaxX/Y = max |u + sqrt(g h)|, |v + sqrt(g h)|
// ---------------------------------------------------------------------------
__global__ void dt_kernel(const DtArgs a) {
  const int n = a.nx * a.ny;
  double lx = 0.0, ly = 0.0;
  int bad = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double h = a.h[k], hu = a.hu[k], hv = a.hv[k], u, v;
    if (!(h >= 0.0) || !isfinite(h) || !isfinite(hu) || !isfinite(hv)) bad = 1;
    cons_to_prim<true>(h, hu, hv, u, v);
    double c = sqrt(a.g * h);
    lx = dmax(lx, fabs(u + c));
    ly = dmax(ly, fabs(v + c));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lx = dmax(lx, __shfl_down_sync(0xffffffffu, lx, o));
    ly = dmax(ly, __shfl_down_sync(0xffffffffu, ly, o));
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax(&a.lam[0], (unsigned long long)__double_as_longlong(lx));
    atomicMax(&a.lam[1], (unsigned long long)__double_as_longlong(ly));
    if (bad) atomicOr(a.bad, 1);
  }
}

cudaError_t launch_dt(const DtArgs& a, cudaStream_t s) {
  int n = a.nx * a.ny;
  int blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  dt_kernel<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's ghosted array U(1:3,-2:nx+3,-2:ny+3)
// and the device planes [ny][nx].
// ---------------------------------------------------------------------------
__global__ void ghosted_to_planes_kernel(const double* __restrict__ G, int nx, int ny, double* h,
                                         double* hu, double* hv) {
  int n = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int i = k % nx, j = k / nx;
    size_t g = 3 * ((size_t)(i + 3) + (size_t)(nx + 6) * (j + 3));
    h[k] = G[g];
    hu[k] = G[g + 1];
    hv[k] = G[g + 2];
  }
}

// Ghost frame filled periodically (the values BoundaryConditions would write,
// equation.f90:556-776); Vg (nullable) = ConsToPrim on the whole array.
__global__ void planes_to_ghosted_kernel(const double* h, const double* hu, const double* hv,
                                         int nx, int ny, double* G, double* Vg) {
  int W = nx + 6, n = W * (ny + 6);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int gi = k % W - 3, gj = k / W - 3;
    int i = wrap(gi, nx), j = wrap(gj, ny);
    size_t s = (size_t)j * nx + i;
    double a = h[s], b = hu[s], c = hv[s];
    G[3 * (size_t)k] = a;
    G[3 * (size_t)k + 1] = b;
    G[3 * (size_t)k + 2] = c;
    if (Vg) {
      double u, v;
      cons_to_prim<true>(a, b, c, u, v);
      Vg[3 * (size_t)k] = a;
      Vg[3 * (size_t)k + 1] = u;
      Vg[3 * (size_t)k + 2] = v;
    }
  }
}

cudaError_t launch_ghosted_to_planes(const double* G, int nx, int ny, double* h, double* hu,
                                     double* hv, cudaStream_t s) {
  int n = nx * ny, blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  ghosted_to_planes_kernel<<<blocks, 256, 0, s>>>(G, nx, ny, h, hu, hv);
  return cudaGetLastError();
}

cudaError_t launch_planes_to_ghosted(const double* h, const double* hu, const double* hv, int nx,
                                     int ny, double* G, double* Vg, cudaStream_t s) {
  int n = (nx + 6) * (ny + 6), blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  planes_to_ghosted_kernel<<<blocks, 256, 0, s>>>(h, hu, hv, nx, ny, G, Vg);
  return cudaGetLastError();
}

// mass = sum h (per-block partials in fixed order, then one block), min h.
__global__ void summary_kernel(const double* h, int n, double* part_sum, double* part_min) {
  __shared__ double ss[256], sm[256];
  double s = 0.0, m = 1e300;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    s += h[k];
    m = dmin(m, h[k]);
  }
  ss[threadIdx.x] = s;
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      sm[threadIdx.x] = dmin(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part_sum[blockIdx.x] = ss[0];
    part_min[blockIdx.x] = sm[0];
  }
}
__global__ void summary_final_kernel(const double* ps, const double* pm, int nb, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0, m = 1e300;
    for (int b = 0; b < nb; ++b) {
      s += ps[b];
      m = dmin(m, pm[b]);
    }
    out[0] = s;
    out[1] = m;
  }
}
cudaError_t launch_summary(const double* h, int n, double* out, cudaStream_t s) {
  // out must have room for 2 + 2*256 doubles (partials after the result)
  const int nb = 256;
  summary_kernel<<<nb, 256, 0, s>>>(h, n, out + 2, out + 2 + nb);
  summary_final_kernel<<<1, 32, 0, s>>>(out + 2, out + 2 + nb, nb, out);
  return cudaGetLastError();
}

// The three substeps of one mPDeC5 correction iteration in one pass (split and FMA
// forms, stencil layout): the stage RHS planes, face fluxes and U^n momentum are
// read once for all of them; hp(m) and the outputs are per substep.  Every load is
// issued before the arithmetic.  Each substep's arithmetic is that of
// assemble_kernel<true, 4>, so the results are identical.
__global__ void __launch_bounds__(128, 4) assemble_multi_kernel(const AssembleMultiArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= a.base.nx || j >= a.base.ny) return;
  assemble_multi_cell(a, i, j);
}

cudaError_t launch_assemble_multi(const AssembleMultiArgs& a, cudaStream_t s) {
  if (a.nm != kMaxFusedStages || a.base.msteps != 4 || !a.base.fast) return cudaErrorInvalidValue;
  dim3 blk(128), grd((a.base.nx + 127) / 128, a.base.ny);
  assemble_multi_kernel<<<grd, blk, 0, s>>>(a);
  return cudaGetLastError();
}

template <bool FAST, int MS>
__global__ void __launch_bounds__(128) assemble_kernel(const AssembleArgs a, bool csr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= a.nx || j >= a.ny) return;
  assemble_cell<FAST, MS>(a, csr, i, j);
}

// Ensembles: block b covers cells [cell0, cell0+128) of problem blk[b].x, with
// cell0 = blk[b].y; descriptors staged in shared memory (stencil layout only).
template <bool FAST>
__global__ void __launch_bounds__(128)
    assemble_batch_kernel(const AssembleArgs* __restrict__ descs, const int2* __restrict__ blk) {
  static_assert(sizeof(AssembleArgs) % 8 == 0 && sizeof(AssembleArgs) / 8 <= 128, "copy");
  __shared__ __align__(16) AssembleArgs sa;
  const int2 w = blk[blockIdx.x];
  if (threadIdx.x < sizeof(AssembleArgs) / 8)
    reinterpret_cast<unsigned long long*>(&sa)[threadIdx.x] =
        reinterpret_cast<const unsigned long long*>(&descs[w.x])[threadIdx.x];
  __syncthreads();
  const int c = w.y + threadIdx.x;
  if (c >= sa.nx * sa.ny) return;
  if (sa.msteps == 4)
    assemble_cell<FAST, 4>(sa, false, c % sa.nx, c / sa.nx);
  else
    assemble_cell<FAST, 2>(sa, false, c % sa.nx, c / sa.nx);
}

// Ensembles, fast forms: the fused assembly of a correction's three substeps; block b
// covers 128 cells of problem blk[b].x from blk[b].y (descriptor staged in shared memory).
__global__ void __launch_bounds__(128, 4)
    assemble_multi_batch_kernel(const AssembleMultiArgs* __restrict__ descs,
                                const int2* __restrict__ blk) {
  static_assert(sizeof(AssembleMultiArgs) % 8 == 0, "copy");
  __shared__ __align__(16) AssembleMultiArgs sa;
  const int2 w = blk[blockIdx.x];
  for (int q = threadIdx.x; q < (int)(sizeof(AssembleMultiArgs) / 8); q += blockDim.x)
    reinterpret_cast<unsigned long long*>(&sa)[q] =
        reinterpret_cast<const unsigned long long*>(&descs[w.x])[q];
  __syncthreads();
  const int c = w.y + threadIdx.x;
  if (c < sa.base.nx * sa.base.ny) assemble_multi_cell(sa, c % sa.base.nx, c / sa.base.nx);
}

cudaError_t launch_assemble_multi_batch(const AssembleMultiArgs* descs, const int2* blk, int nblk,
                                        cudaStream_t s) {
  if (nblk < 1) return cudaSuccess;
  assemble_multi_batch_kernel<<<nblk, 128, 0, s>>>(descs, blk);
  return cudaGetLastError();
}

cudaError_t launch_assemble_batch(const AssembleArgs* descs, const int2* blk, int nblk, bool fast,
                                  cudaStream_t s) {
  if (nblk < 1) return cudaSuccess;
  if (fast)
    assemble_batch_kernel<true><<<nblk, 128, 0, s>>>(descs, blk);
  else
    assemble_batch_kernel<false><<<nblk, 128, 0, s>>>(descs, blk);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const AssembleArgs& a, bool csr, cudaStream_t s) {
  dim3 blk(128), grd((a.nx + 127) / 128, a.ny);
  const bool fast = a.fast && !csr;
  if (a.msteps == 4) {
    if (fast)
      assemble_kernel<true, 4><<<grd, blk, 0, s>>>(a, csr);
    else
      assemble_kernel<false, 4><<<grd, blk, 0, s>>>(a, csr);
  } else {
    if (fast)
      assemble_kernel<true, 2><<<grd, blk, 0, s>>>(a, csr);
    else
      assemble_kernel<false, 2><<<grd, blk, 0, s>>>(a, csr);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Explicit schemes (timediscretization.f90:104-451): stage combinations.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) combo_kernel(const ComboArgs a) {
  const double dt = *a.dt;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      double acc;
      if (a.form == kComboSsp) {
        acc = a.c[0] * a.X[0][v][k];
        for (int i = 1; i < a.nx; ++i) acc = acc + a.c[i] * a.X[i][v][k];
        for (int j = 0; j < a.ny; ++j) acc = acc + a.d[j] * a.Y[j][v][k] * dt;
      } else if (a.form == kComboRk) {
        double sum = a.d[0] * a.Y[0][v][k];
        for (int j = 1; j < a.ny; ++j) sum = sum + a.d[j] * a.Y[j][v][k];
        acc = a.X[0][v][k] + sum * dt;
      } else {
        acc = a.X[0][v][k];
        for (int j = 0; j < a.ny; ++j) acc = acc + dt * a.d[j] * a.Y[j][v][k];
      }
      a.out[v][k] = acc;
    }
  }
}

cudaError_t launch_combo(const ComboArgs& a, cudaStream_t s) {
  int blocks = (a.n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  combo_kernel<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// One CSR pass (one sweep): sparse_matmul (jacobi_iteration.f90:25-43) + update.
__device__ void csr_pass(const JacobiArgs& a, const double* xin, double* xout, bool first,
                         Acc& acc, unsigned long long (*s_acc)[3]) {
  const int n = a.nx * a.ny;
  const int stride = gridDim.x * blockDim.x;
  // rows per thread between flushes of the part sums (every thread of the block
  // takes part in a flush, so the count is the block's, not the thread's)
  const long long rows_per_flush = (long long)kAccFlushCells * stride;
  for (long long base = blockIdx.x * blockDim.x; base < n; base += rows_per_flush) {
    if (base != blockIdx.x * blockDim.x) acc_reduce<1>(acc, s_acc);
    const int end = (int)((n - base > rows_per_flush) ? base + rows_per_flush : n);
    for (int row = (int)base + threadIdx.x; row < end; row += stride) {
      double prod = 0.;
      for (int sp = a.rowstart[row]; sp <= a.rowstart[row + 1] - 1; ++sp)
        if (SWM_IN_RANGE(sp - 1, 5LL * n, kChkCsr) && SWM_IN_RANGE(a.cols[sp - 1] - 1, n, kChkCsr))
          prod = __dadd_rn(prod, __dmul_rn(a.mass[sp - 1], __ldcg(&xin[a.cols[sp - 1] - 1])));
      const double xv = __ddiv_rn(__dsub_rn(a.b[row], prod), a.diag[row]);
      xout[row] = xv;
      acc_put<1>(acc, fabs(__dsub_rn(xv, __ldcg(&xin[row]))));
      if (first) acc_put<0>(acc, fabs(0. - a.b[row]));
    }
  }
}

template <int TB, bool CSR, bool RECIP>
__global__ void __launch_bounds__(JNT, 2) jacobi_kernel(const JacobiArgs a) {
  extern __shared__ __align__(16) double jsm[];
  __shared__ unsigned long long s_acc[kMaxBlock + 1][3];
  __shared__ unsigned long long s_tot[kMaxBlock + 1][3];
  __shared__ int s_ok;
  JacobiCtl* ctl = a.ctl;
  int p = *((volatile int*)&ctl->pass_next);
  const double* xin = a.b;
  double* xout = a.xa;
  const double* result = nullptr;
  bool first = true, zero_result = false, maxhit = false;
  int k = 0, final_k = 0;
  const int blk = CSR ? 1 : (a.block < 1 ? 1 : (a.block > TB ? TB : a.block));
  int plan = blk;            // sweeps of the next pass (plan_sweeps)
  bool expect_stop = false;  // the residual decay reaches the threshold within it
  double r_prev = -1.0;
  const double thresh_d = limbs_value(a.thresh[0], a.thresh[1], a.thresh[2]);
  Acc acc;
  acc_zero(acc);
  for (;;) {
    int Tp = plan;
    if (a.maxiter - k < Tp) Tp = a.maxiter - k;
    if (Tp < 1) Tp = 1;
    for (int q = threadIdx.x; q < (kMaxBlock + 1) * 3; q += blockDim.x) (&s_acc[0][0])[q] = 0ull;
    __syncthreads();
    if (CSR)
      csr_pass(a, xin, xout, first, acc, s_acc);
    else
      stencil_tiles<TB, RECIP, false>(a, xin, xout, Tp, first, acc, jsm, blockIdx.x, s_acc);
    acc_reduce<TB>(acc, s_acc);
    __syncthreads();
    const int slot = p % kResSlots;
    if (threadIdx.x < (Tp + 1) * 3) {
      int t = threadIdx.x / 3, l = threadIdx.x % 3;
      unsigned long long v = s_acc[t][l];
      if (v) atomicAdd(&ctl->acc[slot][t][l], v);
    }
    if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
    if (threadIdx.x < (Tp + 1) * 3) {
      int t = threadIdx.x / 3, l = threadIdx.x % 3;
      s_tot[t][l] = __ldcg(&ctl->acc[slot][t][l]);
    }
    if (blockIdx.x == 0) {  // recycle the slot of pass p-1 (read by everyone before barrier p)
      const int z = (p + 2) % kResSlots;
      for (int q = threadIdx.x; q < (kMaxBlock + 1) * 3; q += blockDim.x)
        (&ctl->acc[z][0][0])[q] = 0ull;
      __threadfence();
    }
    __syncthreads();
    p++;
    int stop = -1;
    if (first && limbs_le(s_tot[0][0], s_tot[0][1], s_tot[0][2], a.thresh)) {
      stop = 0;
    } else {
      for (int t = 1; t <= Tp; ++t)
        if (limbs_le(s_tot[t][0], s_tot[t][1], s_tot[t][2], a.thresh)) {
          stop = t;
          break;
        }
    }
    first = false;
    if (stop == 0) {
      zero_result = true;
      final_k = 0;
      break;
    }
    if (stop > 0) {
      final_k = k + stop;
      if (stop < Tp && !CSR) {  // the stop falls inside the pass: redo it with `stop` sweeps
        for (int q = threadIdx.x; q < (kMaxBlock + 1) * 3; q += blockDim.x)
          (&s_acc[0][0])[q] = 0ull;
        __syncthreads();
        stencil_tiles<TB, RECIP, false>(a, xin, xout, stop, false, acc, jsm, blockIdx.x, s_acc);
        acc_reduce<TB>(acc, s_acc);
        if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
        if (blockIdx.x == 0) {
          const int z = (p + 2) % kResSlots;
          for (int q = threadIdx.x; q < (kMaxBlock + 1) * 3; q += blockDim.x)
            (&ctl->acc[z][0][0])[q] = 0ull;
          __threadfence();
        }
        p++;
      }
      result = xout;
      break;
    }
    if (!CSR) {
      const double rT = limbs_value(s_tot[Tp][0], s_tot[Tp][1], s_tot[Tp][2]);
      const double rP =
          Tp >= 2 ? limbs_value(s_tot[Tp - 1][0], s_tot[Tp - 1][1], s_tot[Tp - 1][2]) : r_prev;
      r_prev = rT;
      plan = plan_sweeps(rT, rP, thresh_d, blk);
      expect_stop = rP > 0. && rT > 0. && rT < rP && thresh_d > 0. &&
                    log(thresh_d / rT) / log(rT / rP) <= (double)blk;
    }
    k += Tp;
    if (k >= a.maxiter) {
      final_k = k;
      maxhit = true;
      result = xout;
      break;
    }
    // the next pass writes the other ping-pong buffer, or, when it is expected to be
    // the last, the destination itself (unless that is the rhs or holds xin), which
    // saves copying the result there
    xin = xout;
    xout = (xin == a.xa) ? a.xb : a.xa;
    if (expect_stop && a.out != a.b && a.out != xin) xout = a.out;
  }
  // deliver the final iterate (haVec of the reference) to its destination
  const int n = a.nx * a.ny;
  if (zero_result || result != a.out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
      a.out[q] = zero_result ? 0. : __ldcg(&result[q]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->iters[a.solve_idx] = final_k;
    if (maxhit && ctl->status == 0) ctl->status = 1;
    *((volatile int*)&ctl->pass_next) = p;
  }
}

template <int TB, bool CSR, bool RECIP>
static const void* jacobi_fn() {
  return reinterpret_cast<const void*>(&jacobi_kernel<TB, CSR, RECIP>);
}

template <bool RECIP>
static const void* pick_stencil(int block, size_t* smem) {
  if (block <= 1) {
    *smem = JTile<1>::bytes;
    return jacobi_fn<1, false, RECIP>();
  }
  if (block <= 2) {
    *smem = JTile<2>::bytes;
    return jacobi_fn<2, false, RECIP>();
  }
  if (block <= 4) {
    *smem = JTile<4>::bytes;
    return jacobi_fn<4, false, RECIP>();
  }
  *smem = JTile<8>::bytes;
  return jacobi_fn<8, false, RECIP>();
}

static const void* pick_jacobi(bool csr, int block, bool recip, size_t* smem) {
  if (csr) {
    *smem = 0;
    return jacobi_fn<1, true, false>();
  }
  return recip ? pick_stencil<true>(block, smem) : pick_stencil<false>(block, smem);
}

int jacobi_grid_blocks(bool csr, int block, int device, bool recip) {
  size_t smem = 0;
  const void* fn = pick_jacobi(csr, block, recip, &smem);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, JNT, smem) != cudaSuccess)
    return -1;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (per_sm < 1) return -1;
  return per_sm * sms;
}

cudaError_t launch_jacobi(const JacobiArgs& a, bool csr, int grid_blocks, cudaStream_t s) {
  size_t smem = 0;
  const void* fn = pick_jacobi(csr, a.block, a.recip != 0, &smem);
  int n = a.nx * a.ny;
  int blocks = grid_blocks;
  if (csr) {
    int need = (n + JNT - 1) / JNT;
    if (need < blocks) blocks = need;
  } else {
    int tiles = ((a.nx + JBX - 1) / JBX) * ((a.ny + JBY - 1) / JBY);
    if (tiles < blocks) blocks = tiles;
  }
  if (blocks < 1) blocks = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(JNT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {const_cast<JacobiArgs*>(&a)};
  return cudaLaunchKernelExC(&cfg, fn, args);
}

template <int TB, bool RECIP>
__global__ void __launch_bounds__(JNT, 2) jacobi_batch_kernel(const JacobiBatchArgs a) {
  extern __shared__ __align__(16) double jsm[];
  jacobi_batch_solve<TB, RECIP>(a, jsm);
}

template <bool RECIP>
static const void* pick_batch(int block, size_t* smem) {
  if (block <= 1) {
    *smem = JTile<1>::bytes;
    return reinterpret_cast<const void*>(&jacobi_batch_kernel<1, RECIP>);
  }
  if (block <= 2) {
    *smem = JTile<2>::bytes;
    return reinterpret_cast<const void*>(&jacobi_batch_kernel<2, RECIP>);
  }
  if (block <= 4) {
    *smem = JTile<4>::bytes;
    return reinterpret_cast<const void*>(&jacobi_batch_kernel<4, RECIP>);
  }
  *smem = JTile<8>::bytes;
  return reinterpret_cast<const void*>(&jacobi_batch_kernel<8, RECIP>);
}

int jacobi_batch_grid_blocks(int block, int device, bool recip) {
  size_t smem = 0;
  const void* fn = recip ? pick_batch<true>(block, &smem) : pick_batch<false>(block, &smem);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, JNT, smem) != cudaSuccess)
    return -1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm < 1 ? -1 : per_sm * sms;
}

cudaError_t launch_jacobi_batch(const JacobiBatchArgs& a, int grid_blocks, bool recip,
                                cudaStream_t s) {
  size_t smem = 0;
  const void* fn = recip ? pick_batch<true>(a.block, &smem) : pick_batch<false>(a.block, &smem);
  int blocks = grid_blocks < a.ntiles ? grid_blocks : a.ntiles;
  if (blocks < 1) blocks = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(JNT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {const_cast<JacobiBatchArgs*>(&a)};
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// Batched TimeStep: block b covers 128 cells of problem blk[b].x from blk[b].y.
__global__ void __launch_bounds__(128)
    dt_batch_kernel(const DtBatchDesc* __restrict__ d, const int2* __restrict__ blk,
                    unsigned long long* lam, int* bad) {
  const int2 w = blk[blockIdx.x];
  const DtBatchDesc& q = d[w.x];
  const int c = w.y + threadIdx.x;
  double lx = 0.0, ly = 0.0;
  int b = 0;
  if (c < q.nx * q.ny) {
    double h = q.h[c], hu = q.hu[c], hv = q.hv[c], u, v;
    if (!(h >= 0.0) || !isfinite(h) || !isfinite(hu) || !isfinite(hv)) b = 1;
    cons_to_prim<true>(h, hu, hv, u, v);
    double cc = sqrt(q.g * h);
    lx = fabs(u + cc);
    ly = fabs(v + cc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lx = dmax(lx, __shfl_down_sync(0xffffffffu, lx, o));
    ly = dmax(ly, __shfl_down_sync(0xffffffffu, ly, o));
  }
  b = __any_sync(0xffffffffu, b);
  // block maxima first: one pair of atomics per block, not per warp (the atomics of a
  // problem's blocks all go to the same two words)
  __shared__ double s_lx[4], s_ly[4];
  __shared__ int s_b[4];
  static_assert(128 / 32 == 4, "four warps per block");
  if ((threadIdx.x & 31) == 0) {
    s_lx[threadIdx.x >> 5] = lx;
    s_ly[threadIdx.x >> 5] = ly;
    s_b[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < 4; ++q) {
      lx = dmax(lx, s_lx[q]);
      ly = dmax(ly, s_ly[q]);
      b |= s_b[q];
    }
    atomicMax(&lam[2 * w.x], (unsigned long long)__double_as_longlong(lx));
    atomicMax(&lam[2 * w.x + 1], (unsigned long long)__double_as_longlong(ly));
    if (b) atomicOr(&bad[w.x], 1);
  }
}

// dt = CFL * min(HUGE, dx/LambdaMaxX, dy/LambdaMaxY), floored (equation.f90:818-834)
__global__ void dt_finalize_kernel(const DtBatchDesc* d, int nprob, const unsigned long long* lam,
                                   double* dt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  const double LX = __longlong_as_double((long long)lam[2 * p]);
  const double LY = __longlong_as_double((long long)lam[2 * p + 1]);
  double ts = 1.7976931348623157e308;
  const double a1 = d[p].dx / LX, b1 = d[p].dy / LY;
  if (a1 < ts) ts = a1;
  if (b1 < ts) ts = b1;
  ts = d[p].cfl * ts;
  if (ts < 1.0e-30) ts = 1.0e-30;
  dt[p] = ts;
}

size_t ensemble_smem_bytes(int tb, int precision) {
  const size_t rhs = precision == SWM_PREC_SPLIT ? RhsSmem<float>::bytes : RhsSmem<double>::bytes;
  const size_t jac = tb <= 2 ? JTile<2>::bytes : (tb <= 4 ? JTile<4>::bytes : JTile<8>::bytes);
  return rhs > jac ? rhs : jac;
}

cudaError_t launch_dt_batch(const DtBatchDesc* d, const int2* blk, int nblk, int nprob,
                            unsigned long long* lam, int* bad, double* dt, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(lam, 0, sizeof(unsigned long long) * 2 * nprob, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int) * nprob, s);
  if (e != cudaSuccess) return e;
  dt_batch_kernel<<<nblk, 128, 0, s>>>(d, blk, lam, bad);
  dt_finalize_kernel<<<(nprob + 127) / 128, 128, 0, s>>>(d, nprob, lam, dt);
  return cudaGetLastError();
}

}  // namespace swm
