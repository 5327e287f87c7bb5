// swm_ensemble.cuh -- the ensemble step kernel: a whole mPDeC5 step of every problem
// of an ensemble in one cooperative persistent launch.  Included by the RHS units
// (inside their SWM_RHS_NS namespace) so that the RHS phase runs this unit's tile
// code; the assembly and Jacobi phases are the shared device code of swm_solve.cuh.
#pragma once
#include "swm_solve.cuh"

#ifdef SWM_RHS_NS
namespace swm {
namespace SWM_RHS_NS {

// ---------------------------------------------------------------------------
// Ensembles in one persistent launch per mPDeC5 step
// (timediscretization.f90:458-566 for every problem at once).  Phases, each ended by a
// bounded grid barrier that every CTA passes:
//   TimeStep of every problem (per-problem LambdaMax by atomics, then dt);
//   the RHS of U^n for every (problem, tile);
//   for k = 1..5: the combination + Patankar assembly of the correction's substeps
//     (three systems per problem for k < 5, written to separate buffers, so that they
//     are independent), then one batched Jacobi solve of all 3 x nprob systems (each
//     with its own stop rule), then, for k < 5, the RHS of the three new substeps.
// Every member's arithmetic is the single-grid kernels' (the same device code), so a
// member matches the same problem stepped alone bit for bit.
// ---------------------------------------------------------------------------
// TimeStep: LambdaMax of one block of kEnsCells cells (one cell per thread).
__device__ __forceinline__ void ens_dt_block(const EnsembleArgs& a, const int2 w) {
  const DtBatchDesc& q = a.dtd[w.x];
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
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&a.lam[2 * w.x], (unsigned long long)__double_as_longlong(lx));
    atomicMax(&a.lam[2 * w.x + 1], (unsigned long long)__double_as_longlong(ly));
    if (b) atomicOr(&a.bad[w.x], 1);
  }
}

// dt = CFL * min(HUGE, dx/LambdaMaxX, dy/LambdaMaxY), floored (equation.f90:818-834)
__device__ __forceinline__ double ens_dt_of(const DtBatchDesc& d, unsigned long long lx,
                                            unsigned long long ly) {
  const double LX = __longlong_as_double((long long)lx), LY = __longlong_as_double((long long)ly);
  double ts = 1.7976931348623157e308;
  const double a1 = d.dx / LX, b1 = d.dy / LY;
  if (a1 < ts) ts = a1;
  if (b1 < ts) ts = b1;
  ts = d.cfl * ts;
  if (ts < 1.0e-30) ts = 1.0e-30;
  return ts;
}

// One RHS tile of this unit's form MODE, kept out of line: the step kernel's other
// phases and the tile code get their registers allocated separately.
template <int MODE>
static __device__ __noinline__ void ens_tile(const RhsArgs& a, int i0, int j0) {
  rhs_tile<MODE>(a, nullptr, i0, j0);
}

// The RHS of descriptor sets set0 .. set0 + nsets - 1 for every (problem, tile).  CTAs
// take chunks of kRhsChunk consecutive tiles from the counter *ctr (the next chunk
// fetched while this one runs), which balances the phase across SMs; a chunk's items
// come in one round trip, and a problem's descriptor is staged again only when the
// problem changes (consecutive tiles mostly share it), so no tile waits on dependent
// global loads before it starts.
constexpr int kRhsChunk = 4;
template <int MODE>
__device__ __forceinline__ void ens_rhs(const EnsembleArgs& a, int set0, int nsets,
                                        unsigned int* ctr) {
  __shared__ __align__(16) RhsArgs sr;
  __shared__ int4 s_items[kRhsChunk];
  __shared__ int s_next;
  static_assert(sizeof(RhsArgs) % 8 == 0 && sizeof(RhsArgs) / 8 <= JNT, "descriptor copy");
  const int total = nsets * a.nrtiles;
  int staged = -1;  // (set0 + set) * nprob + problem of the descriptor in sr
  if (threadIdx.x == 0) s_next = (int)atomicAdd(ctr, 1u) * kRhsChunk;
  __syncthreads();
  for (int w0 = s_next; w0 < total; w0 = s_next) {
    if (threadIdx.x < kRhsChunk) {
      const int w = w0 + threadIdx.x;
      int4 t = make_int4(-1, 0, 0, 0);
      if (w < total) {
        const int set = w / a.nrtiles;
        t = a.rtiles[w - set * a.nrtiles];
        t.w = set;
      }
      s_items[threadIdx.x] = t;
    }
    __syncthreads();  // the chunk's items staged; every thread has read s_next
    // the next chunk, fetched now and published at the chunk's end, so that no thread
    // waits for the atomic before the chunk's work
    int nxt = 0;
    if (threadIdx.x == 0) nxt = (int)atomicAdd(ctr, 1u) * kRhsChunk;
    for (int q = 0; q < kRhsChunk; ++q) {
      const int4 t = s_items[q];
      if (t.x < 0) break;
      if (!SWM_IN_RANGE(t.x, a.nprob, kChkEnsItem)) continue;
      const int key = (set0 + t.w) * a.nprob + t.x;
      if (key != staged) {
        if (threadIdx.x < sizeof(RhsArgs) / 8)
          reinterpret_cast<unsigned long long*>(&sr)[threadIdx.x] =
              reinterpret_cast<const unsigned long long*>(&a.rhs[key])[threadIdx.x];
        __syncthreads();
        staged = key;
      }
      ens_tile<MODE>(sr, t.y, t.z);
      __syncthreads();  // the tile is done with sr and the dynamic shared memory
    }
    if (threadIdx.x == 0) s_next = nxt;
    __syncthreads();
  }
}

// Combination + assembly of the nsub substeps of correction k (solves solve0 ..
// solve0 + nsub - 1) for every cell of every problem: the fast forms' three substeps
// fused per cell (assemble_multi_kernel's arithmetic), otherwise one substep at a time
// (assemble_kernel's).
template <bool FAST>
static __device__ __forceinline__ void ens_assemble(const EnsembleArgs& a, int k, int solve0,
                                                 int nsub) {
  constexpr int kWords = (sizeof(AssembleArgs) * kMaxFusedStages > sizeof(AssembleMultiArgs)
                              ? sizeof(AssembleArgs) * kMaxFusedStages
                              : sizeof(AssembleMultiArgs)) / 8;
  static_assert(sizeof(AssembleArgs) % 8 == 0 && sizeof(AssembleMultiArgs) % 8 == 0, "copy");
  // blocks in chunks of kChunk taken from the phase's counter, the next chunk fetched
  // while the current one runs (consecutive blocks mostly share a problem's
  // descriptors, which stay staged)
  constexpr int kChunk = 8;
  __shared__ __align__(16) unsigned long long sdesc[kWords];
  __shared__ int2 s_cells[kChunk];
  __shared__ int s_next;
  const bool fused = FAST && nsub == kMaxFusedStages;
  unsigned int* ctr = a.work + 5 + (k - 1);
  int staged = -1;
  if (threadIdx.x == 0) s_next = (int)atomicAdd(ctr, 1u) * kChunk;
  __syncthreads();
  for (int b0 = s_next; b0 < a.ncells; b0 = s_next) {
    if (threadIdx.x < kChunk && b0 + (int)threadIdx.x < a.ncells)
      s_cells[threadIdx.x] = a.cells[b0 + threadIdx.x];  // the chunk's blocks at once
    __syncthreads();  // every thread has read s_next; the blocks are staged
    int nxt = 0;  // the next chunk, published at this chunk's end
    if (threadIdx.x == 0) nxt = (int)atomicAdd(ctr, 1u) * kChunk;
    const int b1 = b0 + kChunk < a.ncells ? b0 + kChunk : a.ncells;
    for (int b = b0; b < b1; ++b) {
      const int2 w = s_cells[b - b0];
      if (w.x != staged) {  // stage this problem's descriptors
        __syncthreads();
        if (fused) {
          const unsigned long long* src = reinterpret_cast<const unsigned long long*>(
              &a.asmm[(size_t)(k - 1) * a.nprob + w.x]);
          for (int q = threadIdx.x; q < (int)(sizeof(AssembleMultiArgs) / 8); q += blockDim.x)
            sdesc[q] = src[q];
        } else {
          constexpr int n1 = sizeof(AssembleArgs) / 8;
          for (int q = threadIdx.x; q < nsub * n1; q += blockDim.x)
            sdesc[q] = reinterpret_cast<const unsigned long long*>(
                &a.asmd[(size_t)(solve0 + q / n1) * a.nprob + w.x])[q % n1];
        }
        __syncthreads();
        staged = w.x;
      }
      const int c = w.y + threadIdx.x;
      if (fused) {
        const AssembleMultiArgs& am = *reinterpret_cast<const AssembleMultiArgs*>(sdesc);
        if (c < am.base.nx * am.base.ny) assemble_multi_cell(am, c % am.base.nx, c / am.base.nx);
      } else {
        const AssembleArgs* ad = reinterpret_cast<const AssembleArgs*>(sdesc);
        if (c < ad[0].nx * ad[0].ny)
          for (int q = 0; q < nsub; ++q)
            assemble_cell<FAST, 4>(ad[q], false, c % ad[q].nx, c / ad[q].nx);
      }
    }
    if (threadIdx.x == 0) s_next = nxt;
    __syncthreads();  // the chunk is done; s_next is visible
  }
}

// One batched solve of the correction's systems, out of line like the RHS tile (the
// assembly is inlined: out of line it spilled more and ran 9% slower).
template <int TB, bool FAST>
static __device__ __noinline__ bool ens_jacobi(const JacobiBatchArgs& ja, double* esm) {
  return jacobi_batch_solve<TB, FAST>(ja, esm);
}

// MODE 1: split form; MODE 0: this unit's FP64 form (FMA contraction in
// swm_rhs_fast.cu, the reference's order in swm_rhs_exact.cu).  The fast forms use the
// fused reciprocal assembly and the reciprocal Jacobi, as their single grids do.
__device__ __forceinline__ void ens_mark(const EnsembleArgs& a, int i) {
  if (a.clock && blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    a.clock[i] = t;
  }
}

template <int TB, int MODE>
__global__ void __launch_bounds__(JNT, 2) ensemble_step_kernel(const EnsembleArgs a) {
  constexpr bool FAST = (MODE == 1) || !SWM_EXACT;
  extern __shared__ __align__(128) double esm[];
  __shared__ int s_ok;
  JacBatchCtl* ctl = a.ctl;
  int mark = 0;
  ens_mark(a, mark++);
  // ---- TimeStep of every problem ----
  for (int b = blockIdx.x; b < a.ncells; b += gridDim.x) ens_dt_block(a, a.cells[b]);
  if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
  if (blockIdx.x == 0)
    for (int p = threadIdx.x; p < a.nprob; p += blockDim.x)
      a.dt[p] = ens_dt_of(a.dtd[p], __ldcg(&a.lam[2 * p]), __ldcg(&a.lam[2 * p + 1]));
  if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
  ens_mark(a, mark++);
  // ---- RHS of U^n (FUp(1..4) alias it at k = 1) ----
  ens_rhs<MODE>(a, 0, 1, a.work + 0);
  if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
  ens_mark(a, mark++);
  int solve = 0;
  for (int k = 1; k <= 5; ++k) {
    const int nsub = (k == 5) ? 1 : kMaxFusedStages;
    ens_assemble<FAST>(a, k, solve, nsub);
    if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
    ens_mark(a, mark++);
    JacobiBatchArgs ja;
    ja.descs = a.jac + (size_t)(k - 1) * kMaxFusedStages * a.nprob;
    ja.tiles = a.jtiles;
    ja.ntiles = a.njtiles;
    ja.nprob = a.nprob;
    ja.nsets = nsub;
    ja.st = a.st;
    ja.ctl = ctl;
    ja.iters = a.iters + (size_t)solve * a.nprob;
    ja.block = a.block;
    ja.spin_limit = a.spin_limit;
    ja.work = a.work + 10;
    if (!ens_jacobi<TB, FAST>(ja, esm)) return;
    if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;  // the solutions are delivered
    ens_mark(a, mark++);
    solve += nsub;
    if (k < 5) {
      ens_rhs<MODE>(a, 1 + (k & 1) * kMaxFusedStages, kMaxFusedStages, a.work + k);
      if (!grid_barrier(ctl, a.spin_limit, &s_ok)) return;
      ens_mark(a, mark++);
    }
  }
}

// The step kernel of form MODE for Jacobi temporal block tb (2, 4 or 8).
template <int MODE>
static const void* ensemble_kernel(int tb) {
  if (tb <= 2) return reinterpret_cast<const void*>(&ensemble_step_kernel<2, MODE>);
  if (tb <= 4) return reinterpret_cast<const void*>(&ensemble_step_kernel<4, MODE>);
  return reinterpret_cast<const void*>(&ensemble_step_kernel<8, MODE>);
}

}  // namespace SWM_RHS_NS
}  // namespace swm
#endif  // SWM_RHS_NS
