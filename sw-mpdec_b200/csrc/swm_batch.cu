// swm_batch.cu -- ensembles of independent problems on uneven grids.
//
// A whole mPDeC5 step of every problem is one cooperative persistent launch (the
// ensemble step kernel, swm_ensemble.cuh): per-problem TimeStep, the RHS of every
// (problem, tile), and per correction the assembly of its three substeps into three
// independent Patankar systems per problem and one batched Jacobi solve of all of
// them, each system with its own stop rule, phases separated by bounded grid
// barriers.  The step (three memsets and that launch) is captured once into a CUDA
// graph.  jacobi_block = 0 lets the first step time the candidate schedules -- Jacobi
// temporal block (sweeps per pass, which sets the haloed tile shape 64+2T x 16+2T)
// and CTAs per SM -- on the initial state and keep the fastest (results do not depend
// on it: every candidate produces the same iterates).  The earlier form, one launch
// per phase (40 per step), stays selectable for comparison
// (swm_batch_debug_set_launches).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/swm.h"
#include "swm_host.h"
#include "swm_kernels.cuh"

using namespace swm;

namespace swm {
void set_last_error(const char* msg);
}

namespace {

int bfail(int code, const std::string& msg) {
  swm::set_last_error(msg.c_str());
  return code;
}

#define BCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return bfail(SWM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

const int kSolves = 13;    // mPDeC5: 3 substeps x 4 corrections + 1
const int kRhsSets = 7;    // U^n, and Ua(m) for m = 2..4 at both correction parities
const int kCandidates[3] = {2, 4, 8};
const int kSubsteps = 3;   // systems per problem solved together (substeps m = 2..4)

struct BProblem {
  swm_params p{};
  int nx = 0, ny = 0;
  size_t N = 0;
  Grid gr{};
  double *h = nullptr, *hu = nullptr, *hv = nullptr;
  double* hbuf[4][2] = {};
  double* hum[4] = {};
  double* hvm[4] = {};
  double* fu[4] = {};
  double* fv[4] = {};
  double* fxm[4] = {};
  double* fym[4] = {};
  // Patankar systems: one per substep m = 2..4 (set q = m - 2; the single-launch-per-
  // phase path and the last correction use set 0), planes S, W, E, N, D and the two
  // Jacobi iterate buffers, rows padded to the even pitch jp (16-byte aligned rows for
  // the Jacobi tile copies); for odd nx also the rhs h^n in that layout (bp, written
  // by the step's first assembly)
  int jp = 0;
  double* sys[kSubsteps][5] = {};
  double* xa[kSubsteps] = {};
  double* xb[kSubsteps] = {};
  double* bp = nullptr;
  double *src_col = nullptr, *src_row = nullptr, *bgrad = nullptr;
  SrcSplit *src_cols = nullptr, *src_rows = nullptr;
  double* save[3] = {};  // state copy used while tuning
};

}  // namespace

struct swm_batch {
  std::vector<BProblem> pr;
  int n = 0, device = 0, precision = 0, block = 4;
  bool autotune = false, fast = false;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  RhsArgs* d_rhs = nullptr;        // [kRhsSets][n]
  // per-substep systems (both step forms)
  AssembleArgs* d_asm3 = nullptr;        // [kSolves][n], outputs in the substep's set
  AssembleMultiArgs* d_asmm = nullptr;   // [4][n] fused substeps of corrections 1..4
  JacobiArgs* d_jac5 = nullptr;          // [5][kSubsteps n] systems of each correction
  int2* d_cells256 = nullptr;            // kEnsCells-cell blocks (problem, first cell)
  int ncell256 = 0;
  bool persistent = true;                // one launch per step (else a kernel per phase)
  bool mode_fixed = false;               // the caller chose the step form (no tuning of it)
  long long spin_limit = kDefaultSpinLimit;  // polls of a grid-barrier wait
  int ens_grid = 0;                      // CTAs of the step kernel (autotuned)
  int ens_max[9] = {};                   // co-resident CTAs of the step kernel, per block
  unsigned long long* d_clock = nullptr; // phase timestamps (swm_batch_debug_phase_times)
  unsigned int* d_work = nullptr;        // work-item counters of the step kernel's phases
  bool clocked = false;
  int4* d_rhs_work = nullptr;            // RHS tiles (problem, i0, j0, 0)
  int4* d_rhs_work3 = nullptr;           // the same for three consecutive sets (q n + problem, ...)
  int nrhs = 0;
  int2* d_cells = nullptr;         // 128-cell blocks (problem, first cell)
  int ncellblk = 0;
  int2* d_tiles = nullptr;         // Jacobi tiles (problem, tile)
  int ntiles = 0;
  DtBatchDesc* d_dtd = nullptr;
  double* d_dt = nullptr;
  unsigned long long* d_lam = nullptr;
  int* d_bad = nullptr;
  JacBatchState* d_st = nullptr;
  JacBatchCtl* d_ctl = nullptr;
  int* d_iters = nullptr;          // [kSolves][n]
  int jac_blocks[9] = {};
  cudaGraphExec_t graph = nullptr;
  // host mirrors
  std::vector<double> h_dt;
  std::vector<int> h_iters, h_bad;
  long long cells = 0;
  long long iters_total = 0;
  bool have_state = false;

  template <typename T>
  int alloc(T** ptr, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 256);
    if (e != cudaSuccess) return bfail(SWM_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    cudaMemset(q, 0, count * sizeof(T) + 256);
    allocs.push_back(q);
    *ptr = static_cast<T*>(q);
    return SWM_OK;
  }
};

static int batch_valid(int n, const swm_params* p) {
  if (n < 1 || !p) return bfail(SWM_ERR_PARAM, "n >= 1 problems required");
  for (int i = 0; i < n; ++i) {
    const swm_params& q = p[i];
    if (q.nx < 3 || q.ny < 3) return bfail(SWM_ERR_PARAM, "nx, ny must be >= 3");
    if (q.timescheme != 5) return bfail(SWM_ERR_PARAM, "ensembles run mPDeC5 (timescheme 5)");
    if (q.well_balanced) return bfail(SWM_ERR_PARAM, "ensembles take no well-balanced reference");
    if (q.precision != p[0].precision) return bfail(SWM_ERR_PARAM, "one precision per ensemble");
    if (q.precision < 0 || q.precision > 2) return bfail(SWM_ERR_PARAM, "unknown precision");
    if (q.bathy_flag < 0 || q.bathy_flag > 3) return bfail(SWM_ERR_PARAM, "unknown bathymetry");
    if (q.jacobi_maxiter < 1 || !(q.jacobi_tol >= 0.0)) return bfail(SWM_ERR_PARAM, "Jacobi limits");
    if (!(q.g > 0.0) || !(q.cfl > 0.0) || q.x1[0] == q.x0[0] || q.x1[1] == q.x0[1])
      return bfail(SWM_ERR_PARAM, "invalid domain, g or cfl");
  }
  if (p[0].jacobi_block < 0 || p[0].jacobi_block > kMaxBlock)
    return bfail(SWM_ERR_PARAM, "jacobi_block must be in 0..8");
  return SWM_OK;
}

// Per-problem arrays (same roles as in the single-grid handle).
static int batch_alloc_problem(swm_batch* b, BProblem& q) {
  const size_t N = q.N, nfx = (size_t)(q.nx + 1) * q.ny, nfy = (size_t)q.nx * (q.ny + 1);
  int rc = 0;
#define BA(ptr, cnt) \
  if (!rc) rc = b->alloc(&(ptr), (cnt))
  BA(q.h, N);
  BA(q.hu, N);
  BA(q.hv, N);
  for (int m = 1; m < 4; ++m) {
    BA(q.hbuf[m][0], N);
    BA(q.hbuf[m][1], N);
    BA(q.hum[m], N);
    BA(q.hvm[m], N);
  }
  for (int r = 0; r < 4; ++r) {
    BA(q.fu[r], N);
    BA(q.fv[r], N);
    BA(q.fxm[r], nfx);
    BA(q.fym[r], nfy);
  }
  const size_t NP = (size_t)q.jp * q.ny;
  for (int q3 = 0; q3 < kSubsteps; ++q3) {
    for (int c = 0; c < 5; ++c) BA(q.sys[q3][c], NP);
    BA(q.xa[q3], NP);
    BA(q.xb[q3], NP);
  }
  if (q.jp != q.nx) BA(q.bp, NP);
#undef BA
  if (rc) return rc;
  const Grid& gr = q.gr;
  if (separable_source(q.p)) {
    std::vector<double> col, row;
    host_source_factors(q.p, gr, col, row);
    if ((rc = b->alloc(&q.src_col, col.size())) || (rc = b->alloc(&q.src_row, row.size())))
      return rc;
    BCK(cudaMemcpy(q.src_col, col.data(), sizeof(double) * col.size(), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(q.src_row, row.data(), sizeof(double) * row.size(), cudaMemcpyHostToDevice));
    std::vector<SrcSplit> cols, rows;
    host_source_split(col, row, cols, rows);
    if ((rc = b->alloc(&q.src_cols, cols.size())) || (rc = b->alloc(&q.src_rows, rows.size())))
      return rc;
    BCK(cudaMemcpy(q.src_cols, cols.data(), sizeof(SrcSplit) * cols.size(), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(q.src_rows, rows.data(), sizeof(SrcSplit) * rows.size(), cudaMemcpyHostToDevice));
  } else if (full_source_table(q.p)) {
    std::vector<double> tab;
    host_bgrad_table(q.p, gr, tab);
    if ((rc = b->alloc(&q.bgrad, tab.size()))) return rc;
    BCK(cudaMemcpy(q.bgrad, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
  }
  return SWM_OK;
}

// RHS descriptor: input state (h, hu, hv) -> stage slot `slot`.
static RhsArgs batch_rhs_desc(const BProblem& q, const double* h, const double* hu,
                              const double* hv, int slot) {
  RhsArgs a{};
  a.gr = q.gr;
  a.h = h;
  a.hu = hu;
  a.hv = hv;
  a.ut_hu = q.fu[slot];
  a.ut_hv = q.fv[slot];
  a.fxm = q.fxm[slot];
  a.fym = q.fym[slot];
  a.src_col = q.src_col;
  a.src_row = q.src_row;
  a.src_cols = q.src_cols;
  a.src_rows = q.src_rows;
  a.bgrad = q.bgrad;
  return a;
}

// Assembly descriptor of solve (k, m) of problem q with its outputs in system set qs.
static AssembleArgs batch_asm_desc(const swm_batch* b, const BProblem& q, int i, int k, int m,
                                   int qs) {
  const bool last = (k == 5);
  AssembleArgs aa{};
  aa.nx = q.nx;
  aa.ny = q.ny;
  aa.dx = q.gr.dx;
  aa.dy = q.gr.dy;
  aa.m = m;
  aa.msteps = 4;
  for (int r = 0; r < 4; ++r) aa.theta[r] = kTheta5[m - 1][r];
  aa.dt = b->d_dt + i;
  aa.hu_n = q.hu;
  aa.hv_n = q.hv;
  for (int r = 0; r < 4; ++r) {
    const int slot = (k == 1) ? 0 : r;
    aa.fu[r] = q.fu[slot];
    aa.fv[r] = q.fv[slot];
    aa.fxm[r] = q.fxm[slot];
    aa.fym[r] = q.fym[slot];
    aa.hp[r] = (r == 0 || k == 1) ? q.h : q.hbuf[r][(k - 1) & 1];
  }
  aa.hu_out = last ? q.hu : q.hum[m - 1];
  aa.hv_out = last ? q.hv : q.hvm[m - 1];
  aa.cS = q.sys[qs][0];
  aa.cW = q.sys[qs][1];
  aa.cE = q.sys[qs][2];
  aa.cN = q.sys[qs][3];
  aa.cD = q.sys[qs][4];
  aa.jpitch = q.jp;
  aa.rhs_out = (k == 1 && m == 2) ? q.bp : nullptr;  // padded rhs, once per step
  aa.fast = b->fast ? 1 : 0;
  aa.inv_dx = 1.0 / q.gr.dx;
  aa.inv_dy = 1.0 / q.gr.dy;
  return aa;
}

// Jacobi descriptor of solve (k, m) of problem q on system set qs.
static JacobiArgs batch_jac_desc(const swm_batch* b, const BProblem& q, int k, int m, int qs) {
  JacobiArgs jj{};
  jj.nx = q.nx;
  jj.ny = q.ny;
  jj.maxiter = q.p.jacobi_maxiter;
  residual_limbs_host(q.p.jacobi_tol * (double)q.N, jj.thresh);
  jj.b = q.bp ? q.bp : q.h;
  jj.pitch = q.jp;
  jj.cS = q.sys[qs][0];
  jj.cW = q.sys[qs][1];
  jj.cE = q.sys[qs][2];
  jj.cN = q.sys[qs][3];
  jj.cD = q.sys[qs][4];
  jj.xa = q.xa[qs];
  jj.xb = q.xb[qs];
  jj.out = (k == 5) ? q.h : q.hbuf[m - 1][k & 1];
  jj.recip = b->fast ? 1 : 0;
  return jj;
}

// Descriptor tables of the fixed step sequence (the same sequence enqueue_step issues):
// each substep m of a correction in its own system set m - 2 (the last correction's
// single solve in set 0), the fused substeps of corrections 1..4 (fast forms), and the
// Jacobi systems of each correction.
static int batch_tables(swm_batch* b) {
  const int n = b->n;
  std::vector<RhsArgs> rhs((size_t)kRhsSets * n);
  std::vector<AssembleArgs> as3((size_t)kSolves * n);
  std::vector<AssembleMultiArgs> am((size_t)4 * n);
  std::vector<JacobiArgs> ja5((size_t)5 * kSubsteps * n);
  for (int i = 0; i < n; ++i) {
    const BProblem& q = b->pr[i];
    rhs[i] = batch_rhs_desc(q, q.h, q.hu, q.hv, 0);
    for (int par = 0; par < 2; ++par)
      for (int m = 2; m <= 4; ++m)
        rhs[(size_t)(1 + par * 3 + (m - 2)) * n + i] =
            batch_rhs_desc(q, q.hbuf[m - 1][par], q.hum[m - 1], q.hvm[m - 1], m - 1);
    int solve = 0;
    for (int k = 1; k <= 5; ++k) {
      const int mlo = (k == 5) ? 4 : 2;
      for (int m = mlo; m <= 4; ++m, ++solve) {
        const int qs = (k == 5) ? 0 : m - 2;
        as3[(size_t)solve * n + i] = batch_asm_desc(b, q, i, k, m, qs);
        ja5[((size_t)(k - 1) * kSubsteps + qs) * n + i] = batch_jac_desc(b, q, k, m, qs);
      }
      if (k < 5) {  // the three substeps of this correction fused per cell
        AssembleMultiArgs& ma = am[(size_t)(k - 1) * n + i];
        ma.base = as3[(size_t)(solve - kSubsteps) * n + i];
        ma.nm = kSubsteps;
        for (int qq = 0; qq < kSubsteps; ++qq) {
          const AssembleArgs& s3 = as3[(size_t)(solve - kSubsteps + qq) * n + i];
          ma.m[qq] = s3.m;
          for (int r = 0; r < 4; ++r) ma.theta[qq][r] = s3.theta[r];
          ma.hu_out[qq] = s3.hu_out;
          ma.hv_out[qq] = s3.hv_out;
          ma.cS[qq] = s3.cS;
          ma.cW[qq] = s3.cW;
          ma.cE[qq] = s3.cE;
          ma.cN[qq] = s3.cN;
          ma.cD[qq] = s3.cD;
        }
      }
    }
  }
  BCK(cudaMemcpy(b->d_rhs, rhs.data(), sizeof(RhsArgs) * rhs.size(), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_asm3, as3.data(), sizeof(AssembleArgs) * as3.size(), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_asmm, am.data(), sizeof(AssembleMultiArgs) * am.size(),
                 cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_jac5, ja5.data(), sizeof(JacobiArgs) * ja5.size(), cudaMemcpyHostToDevice));
  return SWM_OK;
}

// RHS of descriptor set `set` (nsets = 1: the tile list of one set) or of the three
// consecutive sets set .. set + 2 (nsets = 3) for every problem, in one launch.
static cudaError_t batch_rhs(swm_batch* b, int set, int nsets) {
  const RhsArgs* d = b->d_rhs + (size_t)set * b->n;
  const int4* work = nsets == 1 ? b->d_rhs_work : b->d_rhs_work3;
  const int nw = nsets * b->nrhs;
  if (b->precision == SWM_PREC_FP64) return launch_rhs_batch_exact(d, work, nw, b->stream);
  return launch_rhs_batch_fast(b->precision == SWM_PREC_SPLIT ? 1 : 0, d, work, nw, b->stream);
}

// One mPDeC5 step of every problem (timediscretization.f90:458-566) as a sequence of
// kernels, dt per problem from the batched TimeStep, all on b->stream: per correction
// the assembly of its substeps into their own systems (fast forms: the three fused per
// cell), one batched Jacobi solve of all of them, and one RHS launch over the three new
// substeps -- the persistent step's phases and descriptors, phase by phase.
// marks (measurement, uncaptured): an event recorded before the step and after each
// phase, the persistent step's phase boundaries (kEnsMarks events).
static int batch_enqueue_phases(swm_batch* b, int block, cudaEvent_t* marks = nullptr) {
  int mk = 0;
  auto mark = [&]() -> cudaError_t {
    return marks ? cudaEventRecord(marks[mk++], b->stream) : cudaSuccess;
  };
  BCK(mark());
  BCK(cudaMemsetAsync(b->d_ctl, 0, sizeof(JacBatchCtl), b->stream));
  BCK(launch_dt_batch(b->d_dtd, b->d_cells, b->ncellblk, b->n, b->d_lam, b->d_bad, b->d_dt,
                      b->stream));
  BCK(mark());
  BCK(batch_rhs(b, 0, 1));
  BCK(mark());
  int solve = 0;
  for (int k = 1; k <= 5; ++k) {
    const int nsub = (k == 5) ? 1 : kSubsteps;
    if (b->fast && nsub == kSubsteps) {
      BCK(launch_assemble_multi_batch(b->d_asmm + (size_t)(k - 1) * b->n, b->d_cells,
                                      b->ncellblk, b->stream));
    } else {
      for (int q = 0; q < nsub; ++q)
        BCK(launch_assemble_batch(b->d_asm3 + (size_t)(solve + q) * b->n, b->d_cells,
                                  b->ncellblk, b->fast, b->stream));
    }
    BCK(mark());
    JacobiBatchArgs ja{};
    ja.descs = b->d_jac5 + (size_t)(k - 1) * kSubsteps * b->n;
    ja.tiles = b->d_tiles;
    ja.ntiles = b->ntiles;
    ja.nprob = b->n;
    ja.nsets = nsub;
    ja.st = b->d_st;
    ja.ctl = b->d_ctl;
    ja.iters = b->d_iters + (size_t)solve * b->n;
    ja.block = block;
    ja.spin_limit = b->spin_limit;
    ja.work = b->d_work + 10;  // reset by the solve itself
    BCK(launch_jacobi_batch(ja, b->jac_blocks[block], b->fast, b->stream));
    BCK(mark());
    solve += nsub;
    if (k < 5) {
      BCK(batch_rhs(b, 1 + (k & 1) * kSubsteps, kSubsteps));
      BCK(mark());
    }
  }
  return SWM_OK;
}

// The ensemble step kernel of this batch's form for Jacobi temporal block tb.
static const void* ens_kernel(const swm_batch* b, int tb) {
  const int t = tb <= 2 ? 2 : (tb <= 4 ? 4 : 8);
  return b->precision == SWM_PREC_FP64
             ? ensemble_kernel_exact(t)
             : ensemble_kernel_fast(b->precision == SWM_PREC_SPLIT ? 1 : 0, t);
}

// One mPDeC5 step of every problem in one cooperative launch of `grid` CTAs (at most
// the co-resident count), `block` Jacobi sweeps per pass.
static int batch_enqueue_persistent(swm_batch* b, int block, int grid) {
  BCK(cudaMemsetAsync(b->d_lam, 0, sizeof(unsigned long long) * 2 * b->n, b->stream));
  BCK(cudaMemsetAsync(b->d_bad, 0, sizeof(int) * b->n, b->stream));
  BCK(cudaMemsetAsync(b->d_ctl, 0, sizeof(JacBatchCtl), b->stream));
  BCK(cudaMemsetAsync(b->d_work, 0, sizeof(unsigned int) * kEnsCounters, b->stream));
  EnsembleArgs a{};
  a.nprob = b->n;
  a.precision = b->precision;
  a.dtd = b->d_dtd;
  a.cells = b->d_cells256;
  a.ncells = b->ncell256;
  a.lam = b->d_lam;
  a.bad = b->d_bad;
  a.dt = b->d_dt;
  a.rhs = b->d_rhs;
  a.rtiles = b->d_rhs_work;
  a.nrtiles = b->nrhs;
  a.asmd = b->d_asm3;
  a.asmm = b->d_asmm;
  a.jac = b->d_jac5;
  a.jtiles = b->d_tiles;
  a.njtiles = b->ntiles;
  a.st = b->d_st;
  a.ctl = b->d_ctl;
  a.iters = b->d_iters;
  a.block = block;
  a.spin_limit = b->spin_limit;
  a.clock = b->clocked ? b->d_clock : nullptr;
  a.work = b->d_work;
  const int tb = block <= 2 ? 2 : (block <= 4 ? 4 : 8);
  const int gmax = b->ens_max[tb];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid < 1 || grid > gmax ? gmax : grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = ensemble_smem_bytes(tb, b->precision);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[] = {&a};
  BCK(cudaLaunchKernelExC(&cfg, ens_kernel(b, tb), args));
  return SWM_OK;
}

static int batch_enqueue(swm_batch* b, bool persistent, int block, int grid) {
  return persistent ? batch_enqueue_persistent(b, block, grid) : batch_enqueue_phases(b, block);
}

static int batch_graph(swm_batch* b) {
  if (b->graph) return SWM_OK;
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = batch_enqueue(b, b->persistent, b->block, b->ens_grid);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return bfail(SWM_ERR_CUDA, cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->graph = nullptr;
    return bfail(SWM_ERR_CUDA, cudaGetErrorString(e));
  }
  return SWM_OK;
}

static int batch_copy_state(swm_batch* b, bool to_save) {
  for (auto& q : b->pr) {
    double* live[3] = {q.h, q.hu, q.hv};
    for (int v = 0; v < 3; ++v) {
      double* dst = to_save ? q.save[v] : live[v];
      double* src = to_save ? live[v] : q.save[v];
      BCK(cudaMemcpyAsync(dst, src, sizeof(double) * q.N, cudaMemcpyDeviceToDevice, b->stream));
    }
  }
  return SWM_OK;
}

// Autotuner: time one step per candidate schedule on the initial state, restore the
// state after each, keep the fastest.  Candidates: the step form (the persistent launch,
// or a kernel per phase, unless the caller fixed it), the Jacobi temporal block 2, 4, 8
// (the haloed tile of a pass is 64+2T x 16+2T cells) and, for the persistent step, the
// co-resident grid or half of it (one CTA per SM instead of two).  Every schedule gives
// the same results.
static int batch_tune(swm_batch* b) {
  NvtxRange range("ensemble autotune");
  for (auto& q : b->pr)
    for (int v = 0; v < 3; ++v)
      if (!q.save[v]) {
        int rc = b->alloc(&q.save[v], q.N);
        if (rc) return rc;
      }
  int rc = batch_copy_state(b, true);
  if (rc) return rc;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  struct Cand {
    bool persistent;
    int block, grid;
  };
  std::vector<Cand> cands;
  for (int form = 0; form < 2; ++form) {
    const bool pers = form == 0;
    if (b->mode_fixed && pers != b->persistent) continue;
    for (int c : kCandidates) {
      if (!pers) {
        cands.push_back({false, c, 0});
        continue;
      }
      cands.push_back({true, c, b->ens_max[c]});
      if (b->ens_max[c] >= 2 * sms) cands.push_back({true, c, b->ens_max[c] / 2});
    }
  }
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  float best = 1e30f;
  Cand pick = cands[0];
  for (const auto& c : cands) {
    for (int rep = 0; rep < 2; ++rep) {  // first repetition warms the kernels
      BCK(cudaEventRecord(e0, b->stream));
      if ((rc = batch_enqueue(b, c.persistent, c.block, c.grid))) return rc;
      BCK(cudaEventRecord(e1, b->stream));
      BCK(cudaStreamSynchronize(b->stream));
      if ((rc = batch_copy_state(b, false))) return rc;
    }
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      pick = c;
    }
  }
  BCK(cudaStreamSynchronize(b->stream));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->persistent = pick.persistent;
  b->block = pick.block;
  b->ens_grid = pick.grid;
  b->autotune = false;
  return SWM_OK;
}

extern "C" {

int swm_batch_destroy(swm_batch_handle b) {
  if (!b) return SWM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (void* q : b->allocs) cudaFree(q);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return SWM_OK;
}

int swm_batch_create(int n, const swm_params* p, swm_batch_handle* out) {
  if (!out) return bfail(SWM_ERR_PARAM, "null handle pointer");
  *out = nullptr;
  int rc = batch_valid(n, p);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return bfail(SWM_ERR_CUDA, "no CUDA device available");
  if (p[0].device < 0 || p[0].device >= ndev) return bfail(SWM_ERR_PARAM, "invalid device ordinal");
  BCK(cudaSetDevice(p[0].device));
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, p[0].device);
  if (major != 10) return bfail(SWM_ERR_UNSUPPORTED, "this build targets sm_100a (B200) only");
  swm_batch* b = new swm_batch();
  auto cleanup = [&](int code) {
    swm_batch_destroy(b);
    return code;
  };
  b->n = n;
  b->device = p[0].device;
  b->precision = p[0].precision;
  b->fast = b->precision != SWM_PREC_FP64;
  b->autotune = p[0].jacobi_block == 0;
  b->block = b->autotune ? 4 : p[0].jacobi_block;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(bfail(SWM_ERR_CUDA, "cudaStreamCreate failed"));
  b->pr.resize(n);
  std::vector<int4> rw;
  std::vector<int2> cb, cb256, tl;
  std::vector<DtBatchDesc> dd(n);
  for (int i = 0; i < n; ++i) {
    BProblem& q = b->pr[i];
    q.p = p[i];
    q.nx = p[i].nx;
    q.ny = p[i].ny;
    q.N = (size_t)q.nx * q.ny;
    q.jp = q.nx + (q.nx & 1);
    q.gr = host_grid(p[i]);
    const Grid& gr = q.gr;
    if ((rc = batch_alloc_problem(b, q))) return cleanup(rc);
    for (int ty = 0; ty < (q.ny + RHS_TY - 1) / RHS_TY; ++ty)
      for (int tx = 0; tx < (q.nx + RHS_TX - 1) / RHS_TX; ++tx)
        rw.push_back(make_int4(i, tx * RHS_TX, ty * RHS_TY, 0));
    for (size_t c0 = 0; c0 < q.N; c0 += 128) cb.push_back(make_int2(i, (int)c0));
    for (size_t c0 = 0; c0 < q.N; c0 += kEnsCells) cb256.push_back(make_int2(i, (int)c0));
    const int jt = ((q.nx + 63) / 64) * ((q.ny + 15) / 16);  // Jacobi tiles (64 x 16)
    for (int t = 0; t < jt; ++t) tl.push_back(make_int2(i, t));
    dd[i] = DtBatchDesc{q.nx, q.ny, gr.g, p[i].cfl, gr.dx, gr.dy, q.h, q.hu, q.hv};
    b->cells += (long long)q.N;
  }
  b->nrhs = (int)rw.size();
  b->ncellblk = (int)cb.size();
  b->ncell256 = (int)cb256.size();
  b->ntiles = (int)tl.size();
  std::vector<int4> rw3;  // the tile list of three consecutive descriptor sets
  for (int q3 = 0; q3 < kSubsteps; ++q3)
    for (const int4& t : rw) rw3.push_back(make_int4(q3 * n + t.x, t.y, t.z, 0));
  if ((rc = b->alloc(&b->d_rhs, (size_t)kRhsSets * n)) || (rc = b->alloc(&b->d_rhs_work, rw.size())) ||
      (rc = b->alloc(&b->d_rhs_work3, rw3.size())) ||
      (rc = b->alloc(&b->d_cells, cb.size())) || (rc = b->alloc(&b->d_tiles, tl.size())) ||
      (rc = b->alloc(&b->d_dtd, (size_t)n)) || (rc = b->alloc(&b->d_dt, (size_t)n)) ||
      (rc = b->alloc(&b->d_lam, 2 * (size_t)n)) || (rc = b->alloc(&b->d_bad, (size_t)n)) ||
      (rc = b->alloc(&b->d_st, (size_t)kSubsteps * n)) || (rc = b->alloc(&b->d_ctl, 1)) ||
      (rc = b->alloc(&b->d_asm3, (size_t)kSolves * n)) ||
      (rc = b->alloc(&b->d_asmm, (size_t)4 * n)) ||
      (rc = b->alloc(&b->d_jac5, (size_t)5 * kSubsteps * n)) ||
      (rc = b->alloc(&b->d_cells256, cb256.size())) ||
      (rc = b->alloc(&b->d_work, (size_t)kEnsCounters)) ||
      (rc = b->alloc(&b->d_iters, (size_t)kSolves * n)))
    return cleanup(rc);
  if (cudaMemcpy(b->d_rhs_work, rw.data(), sizeof(int4) * rw.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_rhs_work3, rw3.data(), sizeof(int4) * rw3.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_cells, cb.data(), sizeof(int2) * cb.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_tiles, tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_cells256, cb256.data(), sizeof(int2) * cb256.size(),
                 cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_dtd, dd.data(), sizeof(DtBatchDesc) * n, cudaMemcpyHostToDevice))
    return cleanup(bfail(SWM_ERR_CUDA, "table upload failed"));
  if ((rc = batch_tables(b))) return cleanup(rc);
  for (int c = 1; c <= kMaxBlock; c *= 2) {
    b->jac_blocks[c] = jacobi_batch_grid_blocks(c, b->device, b->fast);
    if (b->jac_blocks[c] < 1) return cleanup(bfail(SWM_ERR_CUDA, "Jacobi kernel cannot be resident"));
  }
  // co-resident CTAs of the ensemble step kernel per temporal block (cooperative launch)
  for (int c = 2; c <= kMaxBlock; c *= 2) {
    const void* fn = ens_kernel(b, c);
    const size_t smem = ensemble_smem_bytes(c, b->precision);
    int per_sm = 0, sms = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess ||
        per_sm < 1)
      return cleanup(bfail(SWM_ERR_CUDA, "ensemble step kernel cannot be resident"));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    b->ens_max[c] = per_sm * sms;
  }
  b->ens_max[1] = b->ens_max[2];
  if (b->block != 1 && b->block != 2 && b->block != 4 && b->block != 8)
    b->block = b->block < 2 ? 1 : (b->block < 4 ? 2 : (b->block < 8 ? 4 : 8));
  b->h_dt.assign(n, 0.0);
  b->h_iters.assign((size_t)kSolves * n, 0);
  b->h_bad.assign(n, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(bfail(SWM_ERR_CUDA, "initialisation failed"));
  *out = b;
  return SWM_OK;
}

int swm_batch_set_planes(swm_batch_handle b, int i, const double* planes) {
  if (!b || !planes || i < 0 || i >= b->n) return bfail(SWM_ERR_PARAM, "invalid argument");
  BCK(cudaSetDevice(b->device));
  const BProblem& q = b->pr[i];
  BCK(cudaMemcpyAsync(q.h, planes, sizeof(double) * q.N, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(q.hu, planes + q.N, sizeof(double) * q.N, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(q.hv, planes + 2 * q.N, sizeof(double) * q.N, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  b->have_state = true;
  return SWM_OK;
}

int swm_batch_get_planes(swm_batch_handle b, int i, double* planes) {
  if (!b || !planes || i < 0 || i >= b->n) return bfail(SWM_ERR_PARAM, "invalid argument");
  BCK(cudaSetDevice(b->device));
  const BProblem& q = b->pr[i];
  BCK(cudaMemcpyAsync(planes, q.h, sizeof(double) * q.N, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(planes + q.N, q.hu, sizeof(double) * q.N, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(planes + 2 * q.N, q.hv, sizeof(double) * q.N, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return SWM_OK;
}

int swm_batch_step(swm_batch_handle b, double* dt_out) {
  NvtxRange range("swm_batch_step");
  if (!b) return bfail(SWM_ERR_PARAM, "null handle");
  if (!b->have_state) return bfail(SWM_ERR_STATE, "no state set");
  BCK(cudaSetDevice(b->device));
  int rc;
  if (b->autotune && (rc = batch_tune(b))) return rc;
  if ((rc = batch_graph(b))) return rc;
  BCK(cudaGraphLaunch(b->graph, b->stream));
  JacBatchCtl ctl;
  BCK(cudaMemcpyAsync(b->h_dt.data(), b->d_dt, sizeof(double) * b->n, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(b->h_iters.data(), b->d_iters, sizeof(int) * b->h_iters.size(),
                      cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(b->h_bad.data(), b->d_bad, sizeof(int) * b->n, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(&ctl, b->d_ctl, sizeof(JacBatchCtl), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  if (dt_out)
    for (int i = 0; i < b->n; ++i) dt_out[i] = b->h_dt[i];
  for (int v : b->h_iters) b->iters_total += v;
  for (int v : b->h_bad)
    if (v) return bfail(SWM_ERR_NAN, "non-finite or negative depth in an ensemble member");
  if (ctl.status < 0) return bfail(SWM_ERR_WATCHDOG, "Jacobi grid barrier watchdog expired");
  if (ctl.status == 1) return SWM_WARN_JACOBI_MAXITER;
  return SWM_OK;
}

int swm_batch_cells(swm_batch_handle b, long long* cells) {
  if (!b || !cells) return bfail(SWM_ERR_PARAM, "invalid argument");
  *cells = b->cells;
  return SWM_OK;
}

int swm_batch_get_stats(swm_batch_handle b, int* jacobi_block, long long* iters_total,
                        int* last_iters) {
  if (!b) return bfail(SWM_ERR_PARAM, "null handle");
  if (jacobi_block) *jacobi_block = b->block;
  if (iters_total) *iters_total = b->iters_total;
  if (last_iters)
    for (size_t k = 0; k < b->h_iters.size(); ++k) last_iters[k] = b->h_iters[k];
  return SWM_OK;
}

int swm_batch_get_stream(swm_batch_handle b, void** stream) {
  if (!b || !stream) return bfail(SWM_ERR_PARAM, "invalid argument");
  *stream = (void*)b->stream;
  return SWM_OK;
}

int swm_batch_debug_set_launches(swm_batch_handle b, int per_phase) {
  if (!b) return bfail(SWM_ERR_PARAM, "null handle");
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  if (per_phase < 0) {  // the autotuner's choice (on the first step, if it has not run)
    b->mode_fixed = false;
    return SWM_OK;
  }
  b->mode_fixed = true;
  b->persistent = per_phase == 0;
  if (!b->persistent && b->block > kMaxBlock) b->block = kMaxBlock;
  return SWM_OK;
}

int swm_batch_debug_phase_times(swm_batch_handle b, double* ms, int cap, int* n) {
  NvtxRange range("swm_batch_debug_phase_times");
  if (!b || !ms || cap < kEnsMarks - 1) return bfail(SWM_ERR_PARAM, "invalid argument");
  if (!b->have_state) return bfail(SWM_ERR_STATE, "no state set");
  BCK(cudaSetDevice(b->device));
  int rc;
  if (b->autotune && (rc = batch_tune(b))) return rc;
  if (!b->persistent) {  // per-phase form: CUDA events between its kernels
    cudaEvent_t ev[kEnsMarks] = {};
    for (auto& e : ev) BCK(cudaEventCreate(&e));
    rc = batch_enqueue_phases(b, b->block, ev);
    if (!rc) {
      BCK(cudaStreamSynchronize(b->stream));
      for (int i = 0; i + 1 < kEnsMarks; ++i) {
        float f = 0.f;
        BCK(cudaEventElapsedTime(&f, ev[i], ev[i + 1]));
        ms[i] = f;
      }
      if (n) *n = kEnsMarks - 1;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
  }
  if (!b->d_clock && (rc = b->alloc(&b->d_clock, kEnsMarks))) return rc;
  BCK(cudaMemsetAsync(b->d_clock, 0, sizeof(unsigned long long) * kEnsMarks, b->stream));
  b->clocked = true;
  rc = batch_enqueue_persistent(b, b->block, b->ens_grid);
  b->clocked = false;
  if (rc) return rc;
  unsigned long long t[kEnsMarks];
  BCK(cudaMemcpyAsync(t, b->d_clock, sizeof(t), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i + 1 < kEnsMarks; ++i) ms[i] = (double)(t[i + 1] - t[i]) * 1e-6;
  if (n) *n = kEnsMarks - 1;
  return SWM_OK;
}

int swm_batch_debug_set_spin_limit(swm_batch_handle b, long long limit) {
  if (!b) return bfail(SWM_ERR_PARAM, "null handle");
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  if (b->graph) cudaGraphExecDestroy(b->graph);  // the limit is a kernel parameter
  b->graph = nullptr;
  b->spin_limit = limit;
  return SWM_OK;
}

int swm_batch_get_launch_info(swm_batch_handle b, int* launches_per_step, int* ctas) {
  if (!b) return bfail(SWM_ERR_PARAM, "null handle");
  const int tb = b->block <= 2 ? 2 : (b->block <= 4 ? 4 : 8);
  const int gmax = b->ens_max[tb];
  // per phase: TimeStep (2), RHS of U^n, per correction 1..4 the assembly (fast forms
  // fused, else one per substep), the batched solve and the substeps' RHS, then the last
  // correction's assembly and solve
  if (launches_per_step)
    *launches_per_step = b->persistent ? 1 : 2 + 1 + 4 * ((b->fast ? 1 : kSubsteps) + 2) + 2;
  if (ctas)
    *ctas = !b->persistent ? 0 : (b->ens_grid < 1 || b->ens_grid > gmax ? gmax : b->ens_grid);
  return SWM_OK;
}

}  // extern "C"
