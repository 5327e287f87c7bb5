// swm_batch.cu -- ensembles of independent problems on uneven grids.
//
// Every phase of an mPDeC5 step is one launch covering all problems: the batched
// dt reduction (per-problem TimeStep, computed on the device), 13 batched RHS
// launches (one CTA per (problem, tile)), 13 batched assemblies and 13 cooperative
// Jacobi launches in which each problem keeps its own stop rule.  The whole step
// is captured once into a CUDA graph.  jacobi_block = 0 lets the first step try
// the candidate sweeps-per-pass on the initial state and keep the fastest
// (results do not depend on it: every candidate produces the same iterates).
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

// thetaDeC (timediscretization.f90:491-506), rows m = 1..4
const double kTh5[4][4] = {
    {0.0000000000000000000, 0.0000000000000000000, 0.0000000000000000000, 0.0000000000000000000},
    {0.1103005664791649049, 0.1896994335208351257, -0.0339073642291439076, 0.0103005664791649201},
    {0.0730327668541684294, 0.4505740308958107176, 0.2269672331458314485, -0.0269672331458315692},
    {0.0833333333333333287, 0.4166666666666666852, 0.4166666666666666852, 0.0833333333333333287}};
const int kSolves = 13;    // mPDeC5: 3 substeps x 4 corrections + 1
const int kRhsSets = 7;    // U^n, and Ua(m) for m = 2..4 at both correction parities
const int kCandidates[3] = {2, 4, 8};

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
  double *cS = nullptr, *cW = nullptr, *cE = nullptr, *cN = nullptr, *cD = nullptr;
  double *xa = nullptr, *xb = nullptr;
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
  AssembleArgs* d_asm = nullptr;   // [kSolves][n]
  JacobiArgs* d_jac = nullptr;     // [kSolves][n]
  int4* d_rhs_work = nullptr;
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
  BA(q.cS, N);
  BA(q.cW, N);
  BA(q.cE, N);
  BA(q.cN, N);
  BA(q.cD, N);
  BA(q.xa, N);
  BA(q.xb, N);
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

// Descriptor tables of the fixed step sequence (the same sequence enqueue_step issues).
static int batch_tables(swm_batch* b) {
  const int n = b->n;
  std::vector<RhsArgs> rhs((size_t)kRhsSets * n);
  std::vector<AssembleArgs> as((size_t)kSolves * n);
  std::vector<JacobiArgs> ja((size_t)kSolves * n);
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
        const bool last = (k == 5);
        AssembleArgs& aa = as[(size_t)solve * n + i];
        aa.nx = q.nx;
        aa.ny = q.ny;
        aa.dx = q.gr.dx;
        aa.dy = q.gr.dy;
        aa.m = m;
        aa.msteps = 4;
        for (int r = 0; r < 4; ++r) aa.theta[r] = kTh5[m - 1][r];
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
        aa.cS = q.cS;
        aa.cW = q.cW;
        aa.cE = q.cE;
        aa.cN = q.cN;
        aa.cD = q.cD;
        aa.fast = b->fast ? 1 : 0;
        aa.inv_dx = 1.0 / q.gr.dx;
        aa.inv_dy = 1.0 / q.gr.dy;
        JacobiArgs& jj = ja[(size_t)solve * n + i];
        jj.nx = q.nx;
        jj.ny = q.ny;
        jj.maxiter = q.p.jacobi_maxiter;
        residual_limbs_host(q.p.jacobi_tol * (double)q.N, jj.thresh);
        jj.b = q.h;
        jj.cS = q.cS;
        jj.cW = q.cW;
        jj.cE = q.cE;
        jj.cN = q.cN;
        jj.cD = q.cD;
        jj.xa = q.xa;
        jj.xb = q.xb;
        jj.out = last ? q.h : q.hbuf[m - 1][k & 1];
        jj.recip = b->fast ? 1 : 0;
      }
    }
  }
  BCK(cudaMemcpy(b->d_rhs, rhs.data(), sizeof(RhsArgs) * rhs.size(), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_asm, as.data(), sizeof(AssembleArgs) * as.size(), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_jac, ja.data(), sizeof(JacobiArgs) * ja.size(), cudaMemcpyHostToDevice));
  return SWM_OK;
}

static cudaError_t batch_rhs(swm_batch* b, int set) {
  const RhsArgs* d = b->d_rhs + (size_t)set * b->n;
  if (b->precision == SWM_PREC_FP64) return launch_rhs_batch_exact(d, b->d_rhs_work, b->nrhs, b->stream);
  return launch_rhs_batch_fast(b->precision == SWM_PREC_SPLIT ? 1 : 0, d, b->d_rhs_work, b->nrhs,
                               b->stream);
}

// One mPDeC5 step of every problem (timediscretization.f90:458-566), dt per problem
// from the batched TimeStep, all on b->stream.
static int batch_enqueue(swm_batch* b, int block) {
  BCK(cudaMemsetAsync(b->d_ctl, 0, sizeof(JacBatchCtl), b->stream));
  BCK(launch_dt_batch(b->d_dtd, b->d_cells, b->ncellblk, b->n, b->d_lam, b->d_bad, b->d_dt,
                      b->stream));
  BCK(batch_rhs(b, 0));
  int solve = 0;
  for (int k = 1; k <= 5; ++k) {
    const int mlo = (k == 5) ? 4 : 2;
    for (int m = mlo; m <= 4; ++m, ++solve) {
      BCK(launch_assemble_batch(b->d_asm + (size_t)solve * b->n, b->d_cells, b->ncellblk, b->fast,
                                b->stream));
      JacobiBatchArgs ja{};
      ja.descs = b->d_jac + (size_t)solve * b->n;
      ja.tiles = b->d_tiles;
      ja.ntiles = b->ntiles;
      ja.nprob = b->n;
      ja.st = b->d_st;
      ja.ctl = b->d_ctl;
      ja.iters = b->d_iters + (size_t)solve * b->n;
      ja.block = block;
      ja.spin_limit = kDefaultSpinLimit;
      BCK(launch_jacobi_batch(ja, b->jac_blocks[block], b->fast, b->stream));
    }
    if (k < 5)
      for (int m = 2; m <= 4; ++m) BCK(batch_rhs(b, 1 + (k & 1) * 3 + (m - 2)));
  }
  return SWM_OK;
}

static int batch_graph(swm_batch* b) {
  if (b->graph) return SWM_OK;
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = batch_enqueue(b, b->block);
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

// Autotuner: time one step per candidate sweeps-per-pass on the initial state,
// restore the state after each, keep the fastest.
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
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_block = 4;
  for (int c : kCandidates) {
    for (int rep = 0; rep < 2; ++rep) {  // first repetition warms the kernels
      BCK(cudaEventRecord(e0, b->stream));
      if ((rc = batch_enqueue(b, c))) return rc;
      BCK(cudaEventRecord(e1, b->stream));
      BCK(cudaStreamSynchronize(b->stream));
      if ((rc = batch_copy_state(b, false))) return rc;
    }
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_block = c;
    }
  }
  BCK(cudaStreamSynchronize(b->stream));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->block = best_block;
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
  std::vector<int2> cb, tl;
  std::vector<DtBatchDesc> dd(n);
  for (int i = 0; i < n; ++i) {
    BProblem& q = b->pr[i];
    q.p = p[i];
    q.nx = p[i].nx;
    q.ny = p[i].ny;
    q.N = (size_t)q.nx * q.ny;
    q.gr = host_grid(p[i]);
    const Grid& gr = q.gr;
    if ((rc = batch_alloc_problem(b, q))) return cleanup(rc);
    for (int ty = 0; ty < (q.ny + RHS_TY - 1) / RHS_TY; ++ty)
      for (int tx = 0; tx < (q.nx + RHS_TX - 1) / RHS_TX; ++tx)
        rw.push_back(make_int4(i, tx * RHS_TX, ty * RHS_TY, 0));
    for (size_t c0 = 0; c0 < q.N; c0 += 128) cb.push_back(make_int2(i, (int)c0));
    const int jt = ((q.nx + 63) / 64) * ((q.ny + 15) / 16);  // Jacobi tiles (64 x 16)
    for (int t = 0; t < jt; ++t) tl.push_back(make_int2(i, t));
    dd[i] = DtBatchDesc{q.nx, q.ny, gr.g, p[i].cfl, gr.dx, gr.dy, q.h, q.hu, q.hv};
    b->cells += (long long)q.N;
  }
  b->nrhs = (int)rw.size();
  b->ncellblk = (int)cb.size();
  b->ntiles = (int)tl.size();
  if ((rc = b->alloc(&b->d_rhs, (size_t)kRhsSets * n)) || (rc = b->alloc(&b->d_asm, (size_t)kSolves * n)) ||
      (rc = b->alloc(&b->d_jac, (size_t)kSolves * n)) || (rc = b->alloc(&b->d_rhs_work, rw.size())) ||
      (rc = b->alloc(&b->d_cells, cb.size())) || (rc = b->alloc(&b->d_tiles, tl.size())) ||
      (rc = b->alloc(&b->d_dtd, (size_t)n)) || (rc = b->alloc(&b->d_dt, (size_t)n)) ||
      (rc = b->alloc(&b->d_lam, 2 * (size_t)n)) || (rc = b->alloc(&b->d_bad, (size_t)n)) ||
      (rc = b->alloc(&b->d_st, (size_t)n)) || (rc = b->alloc(&b->d_ctl, 1)) ||
      (rc = b->alloc(&b->d_iters, (size_t)kSolves * n)))
    return cleanup(rc);
  if (cudaMemcpy(b->d_rhs_work, rw.data(), sizeof(int4) * rw.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_cells, cb.data(), sizeof(int2) * cb.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_tiles, tl.data(), sizeof(int2) * tl.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_dtd, dd.data(), sizeof(DtBatchDesc) * n, cudaMemcpyHostToDevice))
    return cleanup(bfail(SWM_ERR_CUDA, "table upload failed"));
  if ((rc = batch_tables(b))) return cleanup(rc);
  for (int c = 1; c <= kMaxBlock; c *= 2) {
    b->jac_blocks[c] = jacobi_batch_grid_blocks(c, b->device, b->fast);
    if (b->jac_blocks[c] < 1) return cleanup(bfail(SWM_ERR_CUDA, "Jacobi kernel cannot be resident"));
  }
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

}  // extern "C"
