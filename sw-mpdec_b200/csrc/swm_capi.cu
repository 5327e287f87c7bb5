// swm_capi.cu -- C ABI (include/swm.h) and host orchestration of one mPDeC step.
//
// Replaces the reference's module procedures TimeStep() (equation.f90:791-837)
// and TimeDiscretizationByMPDeC5/2(t) (timediscretization.f90:458-664).  The
// state lives on the device as three planes [ny][nx]; one step is the fixed
// sequence of kernels below, captured once into a CUDA graph (dt is read from
// device memory, so the graph is replayed unchanged every step).
#include <array>
#include <atomic>
#include <cmath>
#include <initializer_list>
#include <utility>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/swm.h"
#include "swm_host.h"
#include "swm_kernels.cuh"

using namespace swm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// Host-side allocation-failure injection (swm_debug_inject_alloc_failure): the
// library's device and pinned-host allocations are counted, and the one whose
// number equals g_alloc_fail_at is refused as if the allocator had failed.
std::atomic<long long> g_alloc_count{0};
std::atomic<long long> g_alloc_fail_at{0};

bool injected_alloc_failure() {
  const long long n = ++g_alloc_count;
  const long long at = g_alloc_fail_at.load();
  return at > 0 && n == at;
}

cudaError_t lib_malloc(void** p, size_t bytes) {
  if (injected_alloc_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

cudaError_t lib_malloc_host(void** p, size_t bytes) {
  if (injected_alloc_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(SWM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// mPDeC2 (timediscretization.f90:604)
const double kTheta2[2][2] = {{0.0, 0.0}, {0.5, 0.5}};

}  // namespace

namespace swm {
// Lets other translation units report through swm_last_error().
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace swm

struct swm_solver {
  swm_params p{};
  int nx = 0, ny = 0;
  size_t N = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  Grid gr{};
  std::vector<void*> allocs;
  // state U^n
  double *h = nullptr, *hu = nullptr, *hv = nullptr;
  // substep states Ua(m) for m = 2..4 (index m-1); depth double-buffered by correction parity
  double* hbuf[4][2] = {};
  double* hum[4] = {};
  double* hvm[4] = {};
  // stage RHS slots r = 1..4 (index r-1)
  double* fu[4] = {};
  double* fv[4] = {};
  double* fxm[4] = {};
  double* fym[4] = {};
  // Patankar system
  double *cS = nullptr, *cW = nullptr, *cE = nullptr, *cN = nullptr, *cD = nullptr;
  // stencil mPDeC5: the systems of substeps 3 and 4 when a correction iteration's
  // three substeps are assembled in one launch ([q][S, W, E, N, D], q = m - 3)
  double* cset[2][5] = {};
  double *csr_mass = nullptr, *csr_diag = nullptr;
  int *rowstart = nullptr, *cols = nullptr;
  double *xa = nullptr, *xb = nullptr, *rhs_compat = nullptr;
  // well-balanced reference
  double *fxwb = nullptr, *fywb = nullptr, *swb = nullptr;
  bool have_wb = false;
  // bathymetry source tables: separable factors [nx][2][4], [ny][2][4] or the full
  // gradient [4][4][2][N] at the interior Gauss points
  double *src_col = nullptr, *src_row = nullptr;
  SrcSplit *src_cols = nullptr, *src_rows = nullptr;
  double* bgrad = nullptr;
  // scalars
  double* dt_dev = nullptr;
  unsigned long long* lam = nullptr;  // [2] LambdaMax bit patterns, then the flag
  int* bad = nullptr;                 // inside the same allocation as lam
  JacobiCtl* ctl = nullptr;
  double* summary = nullptr;
  double* l1_scratch = nullptr;  // L1 error: 3 * kIcMaxBlocks partials + 3 results
  double* ex[7][3] = {};          // explicit schemes: 7 stage slots of (h, hu, hv) planes
  // formatted output: value planes (V, Bath, Error) and line buffers
  double* out_planes = nullptr;  // 5 planes: u, v, Bath, error h, error hu (+ error hv below)
  double* out_err_hv = nullptr;
  bool have_bath = false;
  char* out_dev = nullptr;
  char* out_host = nullptr;  // pinned
  size_t out_cap = 0;
  double* stage = nullptr;  // ghosted staging (3*(nx+6)*(ny+6))
  double* stage2 = nullptr;
  // pinned host mirrors
  double* h_dt = nullptr;
  JacobiCtl* h_ctl = nullptr;
  unsigned long long* h_lam = nullptr;  // pinned mirror of lam and bad (3 words)
  int* h_bad = nullptr;
  // graph
  cudaGraphExec_t graph = nullptr;
  bool graph_failed = false;
  int jac_blocks = 0;
  int n_solves = 0;
  // grid-barrier watchdog of the Jacobi launches (polls before giving up)
  long long spin_limit = kDefaultSpinLimit;
  // the step's last launch computes LambdaMax and the non-finite/negative-depth flag
  // of the new state; swm_timestep uses them while the state is unchanged
  bool lam_fresh = false;
  // TMA staging of the RHS tiles: tensor maps of every plane an RHS reads, by address
  bool tma = true;
  std::vector<std::pair<const double*, CUtensorMap>> tmaps;
  // per-launch event profiling (swm_profile_step)
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_cls;
  // stats
  swm_stats stats{};
  bool have_state = false;

  template <typename T>
  int dalloc(T** ptr, size_t count) {
    void* p_ = nullptr;
    cudaError_t e = lib_malloc(&p_, count * sizeof(T) + 64);
    if (e != cudaSuccess) return fail(SWM_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    cudaMemset(p_, 0, count * sizeof(T) + 64);
    allocs.push_back(p_);
    *ptr = static_cast<T*>(p_);
    return SWM_OK;
  }
};

static int valid_params(const swm_params* p) {
  if (!p) return fail(SWM_ERR_PARAM, "null params");
  if (p->nx < 3 || p->ny < 3) return fail(SWM_ERR_PARAM, "nx, ny must be >= 3");
  if ((long long)p->nx * p->ny > (1LL << 28)) return fail(SWM_ERR_PARAM, "grid too large");
  if (p->timescheme < 1 || p->timescheme > 7)
    return fail(SWM_ERR_PARAM,
                "timescheme must be 1 (Euler), 2 (SSPRK4), 3 (RK65), 4 (DeC5), 5 (mPDeC5), "
                "6 (mPEuler) or 7 (mPDeC2)");
  if (p->precision < 0 || p->precision > 2) return fail(SWM_ERR_PARAM, "unknown precision");
  if (p->solver != SWM_SOLVER_CSR && p->solver != SWM_SOLVER_STENCIL)
    return fail(SWM_ERR_PARAM, "unknown solver");
  if (p->bathy_flag < 0 || p->bathy_flag > 3) return fail(SWM_ERR_PARAM, "unknown bathymetry");
  if (p->jacobi_maxiter < 1) return fail(SWM_ERR_PARAM, "jacobi_maxiter must be >= 1");
  if (!(p->jacobi_tol >= 0.0)) return fail(SWM_ERR_PARAM, "jacobi_tol must be >= 0");
  if (p->jacobi_block < 0 || p->jacobi_block > kMaxBlock)
    return fail(SWM_ERR_PARAM, "jacobi_block must be in 0..8");
  if (!(p->x1[0] != p->x0[0]) || !(p->x1[1] != p->x0[1]))
    return fail(SWM_ERR_PARAM, "empty domain");
  if (!(p->g > 0.0) || !(p->cfl > 0.0)) return fail(SWM_ERR_PARAM, "g and cfl must be > 0");
  if (p->source_table != 0 && p->source_table != 1)
    return fail(SWM_ERR_PARAM, "source_table must be 0 or 1");
  return SWM_OK;
}

// The split and FMA forms use the reciprocal Patankar weights and the 1/Diagonal
// stencil Jacobi; the FP64 form keeps every division of the reference.
static bool fast_patankar(const swm_params& p) {
  return p.precision != SWM_PREC_FP64 && p.solver == SWM_SOLVER_STENCIL;
}

static int jacobi_block_of(const swm_params& p) {
  if (p.solver == SWM_SOLVER_CSR) return 1;
  return p.jacobi_block > 0 ? p.jacobi_block : 4;
}

static RhsArgs make_rhs_args(swm_solver* s, const double* h, const double* hu, const double* hv,
                             int slot) {
  RhsArgs a{};
  a.gr = s->gr;
  a.h = h;
  a.hu = hu;
  a.hv = hv;
  a.ut_hu = s->fu[slot];
  a.ut_hv = s->fv[slot];
  a.fxm = s->fxm[slot];
  a.fym = s->fym[slot];
  if (s->have_wb && s->p.well_balanced) {
    a.fx_wb = s->fxwb;
    a.fy_wb = s->fywb;
    a.s_wb = s->swb;
  }
  a.src_col = s->src_col;
  a.src_row = s->src_row;
  a.src_cols = s->src_cols;
  a.src_rows = s->src_rows;
  a.bgrad = s->bgrad;
  a.status = &s->ctl->status;
  return a;
}

// cuTensorMapEncodeTiled from the driver, looked up once (no link against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  }
  return fn;
}

// Tensor map of one [ny][nx] FP64 plane for the RHS tile box (kTmaBoxX x kTmaBoxY);
// false when the plane cannot be described (row pitch not a multiple of 16 bytes,
// base not 16-byte aligned, grid smaller than the box, no encoder).
static bool plane_map(swm_solver* s, const double* base, CUtensorMap* out) {
  for (const auto& e : s->tmaps)
    if (e.first == base) {
      *out = e.second;
      return true;
    }
  auto enc = tensor_map_encoder();
  if (!enc || (s->nx % 2) != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0 ||
      s->nx < kTmaBoxX || s->ny < kTmaBoxY)
    return false;
  const cuuint64_t dims[2] = {(cuuint64_t)s->nx, (cuuint64_t)s->ny};
  const cuuint64_t strides[1] = {(cuuint64_t)s->nx * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)kTmaBoxX, (cuuint32_t)kTmaBoxY};
  const cuuint32_t estr[2] = {1, 1};
  CUtensorMap m;
  if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  s->tmaps.emplace_back(base, m);
  *out = m;
  return true;
}

static cudaError_t launch_rhs(swm_solver* s, const RhsArgs& a) {
  RhsTma tm;
  std::memset(&tm, 0, sizeof(tm));
  tm.enabled = s->tma && plane_map(s, a.h, &tm.plane[0]) && plane_map(s, a.hu, &tm.plane[1]) &&
               plane_map(s, a.hv, &tm.plane[2]);
  if (s->p.precision == SWM_PREC_FP64) return launch_rhs_exact(a, tm, s->stream);
  return launch_rhs_fast(s->p.precision == SWM_PREC_SPLIT ? 1 : 0, a, tm, s->stream);
}

// One RHS outside a step, waited for: a tile whose TMA load gave up is reported.
static int run_rhs_sync(swm_solver* s, const RhsArgs& a) {
  CK(cudaMemsetAsync(&s->ctl->status, 0, sizeof(int), s->stream));
  CK(launch_rhs(s, a));
  int st = 0;
  CK(cudaMemcpyAsync(&st, &s->ctl->status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (st < 0) return fail(SWM_ERR_WATCHDOG, "an RHS tile load did not complete");
  return SWM_OK;
}

static void fill_thresh(const swm_solver* s, unsigned long long t[3]) {
  // stop when sum|dx| <= tol * n  (jacobi_iteration.f90:71,77)
  residual_limbs_host(s->p.jacobi_tol * (double)s->N, t);
}

// Event pair around one launch when profiling (class 0 RHS, 1 assembly, 2 Jacobi).
static void prof_mark(swm_solver* s, int cls) {
  if (!s->profiling) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, s->stream);
  s->prof_ev.push_back(e);
  s->prof_cls.push_back(cls);
}

// Enqueue one complete mPDeC step on s->stream (dt read from s->dt_dev).
// Patankar solves per step: mPDeC5 13, mPDeC2 2, mPEuler 1, explicit schemes none.
static int solves_per_step(int timescheme) {
  return timescheme == 5 ? 13 : (timescheme == 7 ? 2 : (timescheme == 6 ? 1 : 0));
}

// ---- explicit schemes (timediscretization.f90:104-451; build without PATANKAR) ----
using Planes = std::array<double*, 3>;

static Planes state_planes(swm_solver* s) { return {s->h, s->hu, s->hv}; }
static Planes slot(swm_solver* s, int k) { return {s->ex[k][0], s->ex[k][1], s->ex[k][2]}; }

// RHS of state X into R (all three components), mass fluxes to the slot-0 scratch.
static int explicit_rhs(swm_solver* s, const Planes& X, const Planes& R) {
  RhsArgs a = make_rhs_args(s, X[0], X[1], X[2], 0);
  a.ut_h = R[0];
  a.ut_hu = R[1];
  a.ut_hv = R[2];
  prof_mark(s, 0);
  CK(launch_rhs(s, a));
  prof_mark(s, -1);
  return SWM_OK;
}

static int combo(swm_solver* s, int form, std::initializer_list<std::pair<double, Planes>> xs,
                 std::initializer_list<std::pair<double, Planes>> ys, const Planes& out) {
  ComboArgs c{};
  c.n = (int)s->N;
  c.form = form;
  c.dt = s->dt_dev;
  for (const auto& x : xs) {
    c.c[c.nx] = x.first;
    for (int v = 0; v < 3; ++v) c.X[c.nx][v] = x.second[v];
    ++c.nx;
  }
  for (const auto& y : ys) {
    c.d[c.ny] = y.first;
    for (int v = 0; v < 3; ++v) c.Y[c.ny][v] = y.second[v];
    ++c.ny;
  }
  for (int v = 0; v < 3; ++v) c.out[v] = out[v];
  CK(launch_combo(c, s->stream));
  return SWM_OK;
}

#define XCK(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_) return rc_;       \
  } while (0)

static int enqueue_explicit(swm_solver* s) {
  const Planes U = state_planes(s);
  switch (s->p.timescheme) {
    case 1: {  // forward Euler: U = K0 + Ut dt
      const Planes R = slot(s, 0);
      XCK(explicit_rhs(s, U, R));
      XCK(combo(s, kComboSsp, {{1.0, U}}, {{1.0, R}}, U));
    } break;
    case 2: {  // SSPRK(5,4) (timediscretization.f90:128-189)
      const Planes K0 = slot(s, 0), K1 = slot(s, 1), K2 = slot(s, 2), K3 = slot(s, 3),
                   K4 = slot(s, 4), R = slot(s, 5), R2 = slot(s, 6);
      for (int v = 0; v < 3; ++v)
        CK(cudaMemcpyAsync(K0[v], U[v], sizeof(double) * s->N, cudaMemcpyDeviceToDevice,
                           s->stream));
      XCK(explicit_rhs(s, K0, R));
      XCK(combo(s, kComboSsp, {{1.00000000000000, K0}}, {{0.39175222700392, R}}, K1));
      XCK(explicit_rhs(s, K1, R));
      XCK(combo(s, kComboSsp, {{0.44437049406734, K0}, {0.55562950593266, K1}},
                {{0.36841059262959, R}}, K2));
      XCK(explicit_rhs(s, K2, R));
      XCK(combo(s, kComboSsp, {{0.62010185138540, K0}, {0.37989814861460, K2}},
                {{0.25189177424738, R}}, K3));
      XCK(explicit_rhs(s, K3, R));
      XCK(combo(s, kComboSsp, {{0.17807995410773, K0}, {0.82192004589227, K3}},
                {{0.54497475021237, R}}, K4));
      XCK(explicit_rhs(s, K4, R2));  // K5 = R (the fourth stage's Ut), R2 the fifth's
      XCK(combo(s, kComboSsp,
                {{0.00683325884039, K0}, {0.51723167208978, K2}, {0.12759831133288, K3},
                 {0.34833675773694, K4}},
                {{0.08460416338212, R}, {0.22600748319395, R2}}, U));
    } break;
    case 3: {  // RK65 (timediscretization.f90:247-348); UN0 is U until the final update
      static const double A[6][5] = {{0., 0., 0., 0., 0.},
                                     {0.25, 0., 0., 0., 0.},
                                     {0.125, 0.125, 0., 0., 0.},
                                     {0., 0., 0.5, 0., 0.},
                                     {0.1875, -0.375, 0.375, 0.5625, 0.},
                                     {-0.42857142857142855, 1.1428571428571428, 0.8571428571428571,
                                      -1.7142857142857142, 1.1428571428571428}};
      static const double b[6] = {0.077777777777777778, 0., 0.35555555555555556,
                                  0.13333333333333333, 0.35555555555555556, 0.077777777777777778};
      const Planes St = slot(s, 6);
      XCK(explicit_rhs(s, U, slot(s, 0)));
      for (int st = 1; st <= 5; ++st) {
        ComboArgs c{};
        c.n = (int)s->N;
        c.form = kComboRk;
        c.dt = s->dt_dev;
        c.nx = 1;
        for (int v = 0; v < 3; ++v) c.X[0][v] = U[v];
        c.ny = st;
        for (int j = 0; j < st; ++j) {
          c.d[j] = A[st][j];
          for (int v = 0; v < 3; ++v) c.Y[j][v] = s->ex[j][v];
        }
        for (int v = 0; v < 3; ++v) c.out[v] = St[v];
        CK(launch_combo(c, s->stream));
        XCK(explicit_rhs(s, St, slot(s, st)));
      }
      ComboArgs c{};
      c.n = (int)s->N;
      c.form = kComboRk;
      c.dt = s->dt_dev;
      c.nx = 1;
      c.ny = 6;
      for (int v = 0; v < 3; ++v) {
        c.X[0][v] = U[v];
        c.out[v] = U[v];
      }
      for (int j = 0; j < 6; ++j) {
        c.d[j] = b[j];
        for (int v = 0; v < 3; ++v) c.Y[j][v] = s->ex[j][v];
      }
      CK(launch_combo(c, s->stream));
    } break;
    case 4: {  // DeC5 (timediscretization.f90:353-451): Ua(1) = U, Ua(2..4), FUp(1..4)
      const Planes Ua[5] = {Planes{}, U, slot(s, 0), slot(s, 1), slot(s, 2)};
      Planes F[5] = {Planes{}, slot(s, 3), slot(s, 3), slot(s, 3), slot(s, 3)};
      XCK(explicit_rhs(s, U, F[1]));  // FUp(1..4) = F(U^n), one copy
      for (int kk = 1; kk <= 5; ++kk) {
        const int mlo = (kk == 5) ? 4 : 2;
        for (int ii = mlo; ii <= 4; ++ii) {
          ComboArgs c{};
          c.n = (int)s->N;
          c.form = kComboDec;
          c.dt = s->dt_dev;
          c.nx = 1;
          c.ny = 4;
          for (int v = 0; v < 3; ++v) {
            c.X[0][v] = U[v];  // Ua(1)
            c.out[v] = (kk == 5) ? U[v] : Ua[ii][v];  // the last correction is the new U
          }
          for (int jj = 1; jj <= 4; ++jj) {
            c.d[jj - 1] = kTheta5[ii - 1][jj - 1];
            for (int v = 0; v < 3; ++v) c.Y[jj - 1][v] = F[jj][v];
          }
          CK(launch_combo(c, s->stream));
        }
        if (kk != 5)
          for (int ii = 2; ii <= 4; ++ii) {
            F[ii] = slot(s, 2 + ii);  // FUp(2..4) in slots 4..6
            XCK(explicit_rhs(s, Ua[ii], F[ii]));
          }
      }
    } break;
    default:
      return fail(SWM_ERR_PARAM, "not an explicit scheme");
  }
  return SWM_OK;
}

// LambdaMax and the non-finite/negative-depth flag of the state (TimeStep's
// reduction, equation.f90:791-837), into s->lam / s->bad.
static int enqueue_dt(swm_solver* s) {
  CK(cudaMemsetAsync(s->lam, 0, 3 * sizeof(unsigned long long), s->stream));
  DtArgs a{s->nx, s->ny, s->p.g, s->h, s->hu, s->hv, s->lam, s->bad};
  CK(launch_dt(a, s->stream));
  return SWM_OK;
}

static int enqueue_patankar(swm_solver* s);

// One step: the scheme's launches, then the reduction of the new state, so that a
// non-finite value born inside the step is reported by the step itself and the next
// TimeStep() needs no launch of its own.  The Jacobi control block is cleared first:
// every step starts from a clean barrier and residual state, also after a solve
// that gave up on its grid barrier.
static int enqueue_step(swm_solver* s) {
  CK(cudaMemsetAsync(s->ctl, 0, sizeof(JacobiCtl), s->stream));
  int rc;
  if (s->p.timescheme <= 4) {
    s->n_solves = 0;
    rc = enqueue_explicit(s);
  } else {
    rc = enqueue_patankar(s);
  }
  if (rc) return rc;
  return enqueue_dt(s);
}

static int enqueue_patankar(swm_solver* s) {
  const bool two = (s->p.timescheme != 5);  // mPDeC2 or mPEuler: MSteps = 2
  const int ms = two ? 2 : 4, kc = two ? (s->p.timescheme == 7 ? 2 : 1) : 5;
  const bool csr = (s->p.solver == SWM_SOLVER_CSR);
  const bool compat = two && s->p.mpdec2_compat;
  // RHS at U^n (timediscretization.f90:519), stored in slot 1 and used for all r at k=1
  {
    NvtxRange r("rhs");
    prof_mark(s, 0);
    CK(launch_rhs(s, make_rhs_args(s, s->h, s->hu, s->hv, 0)));
    prof_mark(s, -1);
  }
  int solve = 0;
  // the three substeps of an mPDeC5 correction iteration depend only on the previous
  // iteration, so (split and FMA forms, stencil layout) they are assembled in one
  // launch into three systems, then solved one after another
  const bool fused = !csr && ms == 4 && fast_patankar(s->p) && s->cset[1][4] != nullptr;
  for (int k = 1; k <= kc; ++k) {
    const int mlo = (k == kc) ? ms : 2;
    const bool fuse_k = fused && k < kc;
    for (int m = mlo; m <= ms; ++m) {
      AssembleArgs aa{};
      aa.nx = s->nx;
      aa.ny = s->ny;
      aa.dx = s->gr.dx;
      aa.dy = s->gr.dy;
      aa.m = m;
      aa.msteps = ms;
      aa.compat2 = compat ? 1 : 0;
      for (int r = 0; r < 4; ++r) aa.theta[r] = two ? (r < 2 ? kTheta2[m - 1][r] : 0.0) : kTheta5[m - 1][r];
      aa.dt = s->dt_dev;
      aa.hu_n = s->hu;
      aa.hv_n = s->hv;
      for (int r = 0; r < ms; ++r) {
        const int slot = (k == 1) ? 0 : r;
        aa.fu[r] = s->fu[slot];
        aa.fv[r] = s->fv[slot];
        aa.fxm[r] = s->fxm[slot];
        aa.fym[r] = s->fym[slot];
        aa.hp[r] = (r == 0 || k == 1) ? s->h : s->hbuf[r][(k - 1) & 1];
      }
      const bool last = (k == kc);
      aa.hu_out = last ? s->hu : s->hum[m - 1];
      aa.hv_out = last ? s->hv : s->hvm[m - 1];
      aa.cS = s->cS;
      aa.cW = s->cW;
      aa.cE = s->cE;
      aa.cN = s->cN;
      aa.cD = s->cD;
      aa.csr_mass = s->csr_mass;
      aa.csr_diag = s->csr_diag;
      aa.rhs_out = compat ? s->rhs_compat : nullptr;
      aa.fast = fast_patankar(s->p) ? 1 : 0;
      aa.inv_dx = 1.0 / s->gr.dx;
      aa.inv_dy = 1.0 / s->gr.dy;
      // substep m's system: the first set, or for a fused iteration the m-th
      double* sys[5] = {s->cS, s->cW, s->cE, s->cN, s->cD};
      if (fuse_k && m > 2)
        for (int c = 0; c < 5; ++c) sys[c] = s->cset[m - 3][c];
      if (!fuse_k) {
        NvtxRange r("patankar assembly");
        prof_mark(s, 1);
        CK(launch_assemble(aa, csr, s->stream));
        prof_mark(s, -1);
      } else if (m == 2) {
        NvtxRange r("patankar assembly (3 substeps)");
        AssembleMultiArgs ma{};
        ma.base = aa;
        ma.nm = 3;
        for (int q = 0; q < 3; ++q) {
          const int mq = 2 + q;
          ma.m[q] = mq;
          for (int r = 0; r < 4; ++r) ma.theta[q][r] = kTheta5[mq - 1][r];
          ma.hu_out[q] = s->hum[mq - 1];
          ma.hv_out[q] = s->hvm[mq - 1];
          double* const* set = q == 0 ? nullptr : s->cset[q - 1];
          ma.cS[q] = q == 0 ? s->cS : set[0];
          ma.cW[q] = q == 0 ? s->cW : set[1];
          ma.cE[q] = q == 0 ? s->cE : set[2];
          ma.cN[q] = q == 0 ? s->cN : set[3];
          ma.cD[q] = q == 0 ? s->cD : set[4];
        }
        prof_mark(s, 1);
        CK(launch_assemble_multi(ma, s->stream));
        prof_mark(s, -1);
      }
      JacobiArgs ja{};
      ja.nx = s->nx;
      ja.ny = s->ny;
      ja.solve_idx = solve < kMaxSolves ? solve : kMaxSolves - 1;
      ja.maxiter = s->p.jacobi_maxiter;
      fill_thresh(s, ja.thresh);
      ja.b = compat ? s->rhs_compat : s->h;
      ja.cS = sys[0];
      ja.cW = sys[1];
      ja.cE = sys[2];
      ja.cN = sys[3];
      ja.cD = sys[4];
      ja.rowstart = s->rowstart;
      ja.cols = s->cols;
      ja.mass = s->csr_mass;
      ja.diag = s->csr_diag;
      ja.xa = s->xa;
      ja.xb = s->xb;
      ja.out = last ? s->h : s->hbuf[m - 1][k & 1];
      ja.ctl = s->ctl;
      ja.block = jacobi_block_of(s->p);
      ja.recip = fast_patankar(s->p) ? 1 : 0;
      ja.spin_limit = s->spin_limit;
      {
        NvtxRange r("jacobi");
        prof_mark(s, 2);
        CK(launch_jacobi(ja, csr, s->jac_blocks, s->stream));
        prof_mark(s, -1);
      }
      solve++;
    }
    if (k < kc) {  // RHS at Ua(m) (timediscretization.f90:550-557)
      for (int m = 2; m <= ms; ++m) {
        NvtxRange r("rhs");
        prof_mark(s, 0);
        CK(launch_rhs(s, make_rhs_args(s, s->hbuf[m - 1][k & 1], s->hum[m - 1], s->hvm[m - 1],
                                       m - 1)));
        prof_mark(s, -1);
      }
    }
  }
  s->n_solves = solve;
  return SWM_OK;
}

static int build_graph(swm_solver* s) {
  if (s->graph || s->graph_failed || !s->p.use_graph) return SWM_OK;
  NvtxRange range("capture step graph");
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    s->graph_failed = true;
    return SWM_OK;
  }
  int rc = enqueue_step(s);
  cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (rc != SWM_OK || e != cudaSuccess || !g) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    s->graph_failed = true;
    return SWM_OK;
  }
  e = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    s->graph = nullptr;
    s->graph_failed = true;
  }
  return SWM_OK;
}

static void drop_graph(swm_solver* s) {
  if (s->graph) cudaGraphExecDestroy(s->graph);
  s->graph = nullptr;
  s->graph_failed = false;
}

extern "C" {

int swm_params_default(swm_params* p, int nx, int ny, double x00, double x01, double x10,
                       double x11) {
  if (!p) return fail(SWM_ERR_PARAM, "null params");
  std::memset(p, 0, sizeof(*p));
  p->nx = nx;
  p->ny = ny;
  p->x0[0] = x00;
  p->x0[1] = x01;
  p->x1[0] = x10;
  p->x1[1] = x11;
  p->g = 9.81;
  p->cfl = 1.0;
  p->timescheme = 5;
  p->bathy_flag = 0;
  p->well_balanced = 0;
  p->precision = SWM_PREC_FP64;
  p->solver = SWM_SOLVER_CSR;
  p->jacobi_maxiter = 1000;
  p->jacobi_tol = 1.0e-16;
  p->jacobi_block = 0;
  p->mpdec2_compat = 0;
  p->use_graph = 1;
  p->device = 0;
  p->source_table = 1;
  return SWM_OK;
}

int swm_create(const swm_params* p, swm_handle* out) {
  if (!out) return fail(SWM_ERR_PARAM, "null handle pointer");
  *out = nullptr;
  int rc = valid_params(p);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SWM_ERR_CUDA, "no CUDA device available");
  if (p->device < 0 || p->device >= ndev) return fail(SWM_ERR_PARAM, "invalid device ordinal");
  CK(cudaSetDevice(p->device));
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, p->device);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, p->device);
  if (major != 10 || minor != 0)
    return fail(SWM_ERR_UNSUPPORTED, "this build targets sm_100a (B200) only");
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, p->device);
  if (!coop) return fail(SWM_ERR_UNSUPPORTED, "cooperative launch not supported");

  swm_solver* s = new swm_solver();
  s->p = *p;
  s->device = p->device;
  s->nx = p->nx;
  s->ny = p->ny;
  s->N = (size_t)p->nx * p->ny;
  // mesh.f90:58-60 and quadrature
  s->gr = host_grid(*p);
  const Grid& gr = s->gr;

  auto cleanup = [&](int code) {
    swm_destroy(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(SWM_ERR_CUDA, "cudaStreamCreate failed"));
  const size_t N = s->N, nx = s->nx, ny = s->ny;
  const size_t nfx = (nx + 1) * ny, nfy = nx * (ny + 1);
  const bool csr = p->solver == SWM_SOLVER_CSR;
#define AL(ptr, cnt)                          \
  do {                                        \
    int rc_ = s->dalloc(&(ptr), (cnt));       \
    if (rc_) return cleanup(rc_);             \
  } while (0)
  AL(s->h, N);
  AL(s->hu, N);
  AL(s->hv, N);
  for (int m = 1; m < 4; ++m) {
    AL(s->hbuf[m][0], N);
    AL(s->hbuf[m][1], N);
    AL(s->hum[m], N);
    AL(s->hvm[m], N);
  }
  for (int r = 0; r < 4; ++r) {
    AL(s->fu[r], N);
    AL(s->fv[r], N);
    AL(s->fxm[r], nfx);
    AL(s->fym[r], nfy);
  }
  if (csr) {
    AL(s->csr_mass, 5 * N);
    AL(s->csr_diag, N);
    AL(s->rowstart, N + 1);
    AL(s->cols, 5 * N);
  } else {
    AL(s->cS, N);
    AL(s->cW, N);
    AL(s->cE, N);
    AL(s->cN, N);
    AL(s->cD, N);
    if (p->timescheme == 5 && fast_patankar(*p))
      for (int q = 0; q < 2; ++q)
        for (int c = 0; c < 5; ++c) AL(s->cset[q][c], N);
  }
  AL(s->xa, N);
  AL(s->xb, N);
  if ((p->timescheme == 7 || p->timescheme == 6) && p->mpdec2_compat) AL(s->rhs_compat, N);
  if (p->timescheme <= 4)
    for (int k = 0; k < 7; ++k)
      for (int v = 0; v < 3; ++v) AL(s->ex[k][v], N);
  if (p->well_balanced) {
    AL(s->fxwb, 3 * nfx);
    AL(s->fywb, 3 * nfy);
    AL(s->swb, 3 * N);
  }
  AL(s->dt_dev, 1);
  AL(s->lam, 3);
  s->bad = reinterpret_cast<int*>(s->lam + 2);
  AL(s->ctl, 1);
  AL(s->summary, 2 + 512);
  AL(s->stage, 3 * (nx + 6) * (ny + 6));
  AL(s->stage2, 3 * (nx + 6) * (ny + 6));
#undef AL
  if (lib_malloc_host((void**)&s->h_dt, sizeof(double)) != cudaSuccess ||
      lib_malloc_host((void**)&s->h_ctl, sizeof(JacobiCtl)) != cudaSuccess ||
      lib_malloc_host((void**)&s->h_lam, 3 * sizeof(unsigned long long)) != cudaSuccess)
    return cleanup(fail(SWM_ERR_ALLOC, "cudaMallocHost failed"));
  s->h_bad = reinterpret_cast<int*>(s->h_lam + 2);

  if (csr) {  // finitevolume.f90:219-267 CSR pattern, 1-based, slot order S, W, C, E, N
    std::vector<int> rs(N + 1), cl(5 * N);
    auto ge = [&](int ii, int jj) {  // mesh.f90:168 GlobalElem
      int a = (jj - 1) % (int)ny;
      if (a < 0) a += ny;
      int b = (ii - 1) % (int)nx;
      if (b < 0) b += nx;
      return a * (int)nx + b + 1;
    };
    int isv = 0, irs = 0;
    for (int jj = 1; jj <= (int)ny; ++jj)
      for (int ii = 1; ii <= (int)nx; ++ii) {
        isv++;
        irs++;
        rs[irs - 1] = isv;
        cl[isv - 1] = ge(ii, jj - 1);
        isv++;
        cl[isv - 1] = ge(ii - 1, jj);
        isv++;
        cl[isv - 1] = ge(ii, jj);
        isv++;
        cl[isv - 1] = ge(ii + 1, jj);
        isv++;
        cl[isv - 1] = ge(ii, jj + 1);
      }
    rs[N] = rs[N - 1] + 5;
    if (cudaMemcpy(s->rowstart, rs.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(s->cols, cl.data(), sizeof(int) * 5 * N, cudaMemcpyHostToDevice) != cudaSuccess)
      return cleanup(fail(SWM_ERR_CUDA, "CSR upload failed"));
  }
  if (separable_source(*p)) {
    std::vector<double> col, row;
    host_source_factors(*p, gr, col, row);
    int rc2 = s->dalloc(&s->src_col, col.size());
    if (!rc2) rc2 = s->dalloc(&s->src_row, row.size());
    if (rc2) return cleanup(rc2);
    std::vector<SrcSplit> cols, rows;
    host_source_split(col, row, cols, rows);
    if (!rc2) rc2 = s->dalloc(&s->src_cols, cols.size());
    if (!rc2) rc2 = s->dalloc(&s->src_rows, rows.size());
    if (rc2) return cleanup(rc2);
    if (cudaMemcpy(s->src_col, col.data(), sizeof(double) * col.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(s->src_row, row.data(), sizeof(double) * row.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(s->src_cols, cols.data(), sizeof(SrcSplit) * cols.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->src_rows, rows.data(), sizeof(SrcSplit) * rows.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return cleanup(fail(SWM_ERR_CUDA, "bathymetry factor upload failed"));
  } else if (full_source_table(*p)) {  // host libm (equation.f90:451-509)
    std::vector<double> tab;
    host_bgrad_table(*p, gr, tab);
    int rc2 = s->dalloc(&s->bgrad, tab.size());
    if (rc2) return cleanup(rc2);
    if (cudaMemcpy(s->bgrad, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return cleanup(fail(SWM_ERR_CUDA, "bathymetry table upload failed"));
  }
  s->jac_blocks = jacobi_grid_blocks(csr, jacobi_block_of(s->p), s->device, fast_patankar(s->p));
  if (s->jac_blocks < 1) return cleanup(fail(SWM_ERR_CUDA, "Jacobi kernel cannot be resident"));
  // the RHS kernels' shared-memory attribute is set on first launch
  if (cudaDeviceSynchronize() != cudaSuccess)
    return cleanup(fail(SWM_ERR_CUDA, "initialisation failed"));
  s->stats.jacobi_iters_min = 0;
  *out = s;
  return SWM_OK;
}

int swm_destroy(swm_handle s) {
  if (!s) return SWM_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  for (void* ptr : s->allocs) cudaFree(ptr);
  if (s->h_dt) cudaFreeHost(s->h_dt);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_lam) cudaFreeHost(s->h_lam);
  if (s->out_dev) cudaFree(s->out_dev);
  if (s->out_host) cudaFreeHost(s->out_host);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return SWM_OK;
}

static int upload_ghosted(swm_solver* s, const double* U, double* h, double* hu, double* hv) {
  const size_t cnt = 3 * (size_t)(s->nx + 6) * (s->ny + 6);
  CK(cudaMemcpyAsync(s->stage, U, cnt * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(launch_ghosted_to_planes(s->stage, s->nx, s->ny, h, hu, hv, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return SWM_OK;
}

int swm_set_state(swm_handle s, const double* U) {
  NvtxRange range("swm_set_state");
  if (!s || !U) return fail(SWM_ERR_PARAM, "null argument");
  CK(cudaSetDevice(s->device));
  int rc = upload_ghosted(s, U, s->h, s->hu, s->hv);
  if (rc) return rc;
  s->have_state = true;
  s->lam_fresh = false;
  return SWM_OK;
}

int swm_get_state(swm_handle s, double* U, double* V) {
  NvtxRange range("swm_get_state");
  if (!s || !U) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  CK(cudaSetDevice(s->device));
  const size_t cnt = 3 * (size_t)(s->nx + 6) * (s->ny + 6);
  CK(launch_planes_to_ghosted(s->h, s->hu, s->hv, s->nx, s->ny, s->stage, V ? s->stage2 : nullptr,
                              s->stream));
  CK(cudaMemcpyAsync(U, s->stage, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (V) CK(cudaMemcpyAsync(V, s->stage2, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return SWM_OK;
}

int swm_set_planes(swm_handle s, const double* P) {
  if (!s || !P) return fail(SWM_ERR_PARAM, "null argument");
  CK(cudaSetDevice(s->device));
  CK(cudaMemcpyAsync(s->h, P, s->N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->hu, P + s->N, s->N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->hv, P + 2 * s->N, s->N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->have_state = true;
  s->lam_fresh = false;
  return SWM_OK;
}

int swm_get_planes(swm_handle s, double* P) {
  if (!s || !P) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  CK(cudaSetDevice(s->device));
  CK(cudaMemcpyAsync(P, s->h, s->N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(P + s->N, s->hu, s->N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(P + 2 * s->N, s->hv, s->N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return SWM_OK;
}

// Initial condition / exact solution arguments for planes (h, hu, hv).
static int make_ic_args(swm_solver* s, int ic, const double* par, int npar, double t, double* h,
                        double* hu, double* hv, IcArgs* a) {
  if (!ic_supported(ic)) return fail(SWM_ERR_PARAM, "unknown initial condition");
  if (npar < 0 || npar > 8 || (npar > 0 && !par))
    return fail(SWM_ERR_PARAM, "npar must be 0..8 with a parameter array");
  *a = IcArgs{};
  a->gr = s->gr;
  a->ic = ic;
  for (int k = 0; k < npar; ++k) a->par[k] = par[k];
  a->t = t;
  a->sx[0] = fabs(s->p.x1[0] - s->p.x0[0]);
  a->sx[1] = fabs(s->p.x1[1] - s->p.x0[1]);
  a->h = h;
  a->hu = hu;
  a->hv = hv;
  return SWM_OK;
}

int swm_fill_ic(swm_handle s, int ic, const double* par, int npar) {
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  IcArgs a;
  int rc = make_ic_args(s, ic, par, npar, 0.0, s->h, s->hu, s->hv, &a);
  if (rc) return rc;
  CK(cudaSetDevice(s->device));
  CK(launch_ic_fill(a, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->have_state = true;
  s->lam_fresh = false;
  return SWM_OK;
}

int swm_init_wb_ic(swm_handle s, int ic, const double* par, int npar) {
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  if (!s->p.well_balanced) return fail(SWM_ERR_STATE, "handle created without well_balanced");
  // scratch planes: substep-2 buffers are free between steps
  double *h = s->hbuf[1][0], *hu = s->hum[1], *hv = s->hvm[1];
  IcArgs ia;
  int rc = make_ic_args(s, ic, par, npar, 0.0, h, hu, hv, &ia);
  if (rc) return rc;
  CK(cudaSetDevice(s->device));
  CK(launch_ic_fill(ia, s->stream));
  RhsArgs a = make_rhs_args(s, h, hu, hv, 1);
  a.fx_wb = a.fy_wb = a.s_wb = nullptr;  // FXWB = 0 during InitializeWBVariables
  a.fx_full = s->fxwb;
  a.fy_full = s->fywb;
  a.s_full = s->swb;
  rc = run_rhs_sync(s, a);
  if (rc) return rc;
  s->have_wb = true;
  drop_graph(s);  // the step graph bakes the WB pointers in
  return SWM_OK;
}

int swm_l1_error(swm_handle s, int ic, const double* par, int npar, double t, double l1[3]) {
  if (!s || !l1) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  IcArgs a;
  int rc = make_ic_args(s, ic, par, npar, t, s->h, s->hu, s->hv, &a);
  if (rc) return rc;
  CK(cudaSetDevice(s->device));
  if (!s->l1_scratch && (rc = s->dalloc(&s->l1_scratch, 3 * (size_t)kIcMaxBlocks + 3))) return rc;
  double* out = s->l1_scratch + 3 * kIcMaxBlocks;
  CK(launch_l1_error(a, s->l1_scratch, out, s->stream));
  CK(cudaMemcpyAsync(l1, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return SWM_OK;
}

// ---- formatted output (output.f90) ----
static int out_buffers(swm_solver* s, size_t bytes) {
  if (bytes <= s->out_cap) return SWM_OK;
  if (s->out_dev) cudaFree(s->out_dev);
  if (s->out_host) cudaFreeHost(s->out_host);
  s->out_dev = nullptr;
  s->out_host = nullptr;
  s->out_cap = 0;
  if (lib_malloc((void**)&s->out_dev, bytes) != cudaSuccess ||
      lib_malloc_host((void**)&s->out_host, bytes) != cudaSuccess)
    return fail(SWM_ERR_ALLOC, "output line buffers");
  s->out_cap = bytes;
  return SWM_OK;
}

// TIMESTAMP (output.f90:375-395): F15.7 of the time with blanks as zeros
static std::string timestamp(const char* name, double t) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%15.7f", t);
  for (char* c = buf; *c; ++c)
    if (*c == ' ') *c = '0';
  return std::string(name) + "_" + buf;
}

static std::string trimmed(const char* fmt, double v) {
  char buf[64];
  snprintf(buf, sizeof(buf), fmt, v);
  const char* p = buf;
  while (*p == ' ') ++p;
  return p;
}

// Formats the lines on the device, copies them back and writes header + lines.
static int write_lines(swm_solver* s, const std::string& path, const std::string& header,
                       OutLines ol) {
  const size_t lw = out_line_width(ol), bytes = lw * s->N;
  int rc = out_buffers(s, bytes);
  if (rc) return rc;
  ol.out = s->out_dev;
  CK(launch_out_lines(ol, s->stream));
  CK(cudaMemcpyAsync(s->out_host, s->out_dev, bytes, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return fail(SWM_ERR_PARAM, ("cannot open " + path).c_str());
  const bool ok = fwrite(header.data(), 1, header.size(), f) == header.size() &&
                  fwrite(s->out_host, 1, bytes, f) == bytes;
  if (fclose(f) != 0 || !ok) return fail(SWM_ERR_PARAM, ("cannot write " + path).c_str());
  return SWM_OK;
}

static const char* const kVarNames[4] = {"Depth", "VelocityX", "VelocityY", "Bathymetry"};

// WriteDataToDisk_TECPLOT (output.f90:236-305) header
static std::string tecplot_header(const swm_solver* s, double t) {
  std::string h = "VARIABLES=\"CoordinateX\",\"CoordinateY\"";
  for (const char* v : kVarNames) h += std::string(",\"") + v + "\"";
  h += "\nZONE T=\"FV2D\",STRANDID=1,SOLUTIONTIME=" + trimmed("%15.8f", t) +
       ", DATAPACKING=POINT, ZONETYPE=ORDERED, I=" + std::to_string(s->nx) +
       ", J=" + std::to_string(s->ny) + "\n";
  return h;
}

// WriteDataToDisk_OCTAVE (output.f90:310-370) header: names left-justified in 23
static std::string octave_header() {
  std::string h;
  for (const char* v : kVarNames) {
    std::string f(v);
    f.resize(23, ' ');
    h += f;
  }
  return h + "\n";
}

int swm_write_output(swm_handle s, double t, int which_output, int ic, const double* par,
                     int npar, const char* directory, int flags) {
  if (!s || !directory) return fail(SWM_ERR_PARAM, "null argument");
  if (which_output < 1 || which_output > 3) return fail(SWM_ERR_PARAM, "which_output must be 1..3");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  IcArgs ia;
  int rc = make_ic_args(s, ic, par, npar, t, s->h, s->hu, s->hv, &ia);
  if (rc) return rc;
  CK(cudaSetDevice(s->device));
  const size_t N = s->N;
  if (!s->out_planes) {
    if ((rc = s->dalloc(&s->out_planes, 5 * N))) return rc;
    if ((rc = s->dalloc(&s->out_err_hv, N))) return rc;
  }
  double *pu = s->out_planes, *pv = pu + N, *pb = pv + N, *e0 = pb + N, *e1 = e0 + N;
  if (!s->have_bath) {  // Bath: cell averages of the bathymetry (finitevolume.f90:323-325)
    CK(launch_bath_average(ia, pb, s->stream));
    s->have_bath = true;
  }
  // U_NVisu(1:3) = V: ConsToPrim of the state, or of the last RHS input of the step
  // (the reference's V after BoundaryConditions; mPDeC5: Ua(4) of correction 4)
  const double *vh = s->h, *vhu = s->hu, *vhv = s->hv;
  if ((flags & SWM_OUT_V_LAST_RHS) && s->p.timescheme == 5 && s->stats.steps > 0) {
    vh = s->hbuf[3][0];
    vhu = s->hum[3];
    vhv = s->hvm[3];
  }
  CK(launch_prim(vh, vhu, vhv, pu, pv, (int)N, s->stream));
  double* const ep[3] = {e0, e1, s->out_err_hv};
  CK(launch_error_planes(ia, ep, s->stream));
  const std::string dir = std::string(directory) + "/";
  OutLines ol{};
  ol.nx = s->nx;
  ol.ny = s->ny;
  ol.sep = 2;
  ol.zero_small = 1;
  ol.x0 = s->gr.x0;
  ol.y0 = s->gr.y0;
  ol.dx = s->gr.dx;
  ol.dy = s->gr.dy;
  ol.nval = 4;
  for (int pass = 0; pass < 2; ++pass) {  // SOLUTION, then ERROR (output.f90:86-184)
    const char* kind = pass == 0 ? "SOLUTION" : "ERROR";
    if (pass == 0) {
      ol.val[0] = vh;
      ol.val[1] = pu;
      ol.val[2] = pv;
      ol.val[3] = pb;
    } else {
      ol.val[0] = e0;
      ol.val[1] = e1;
      ol.val[2] = s->out_err_hv;
      ol.val[3] = nullptr;  // Error(nVar+1) = 0
    }
    if (which_output == 2 || which_output == 3) {
      ol.ncoord = 2;
      rc = write_lines(s, dir + timestamp((std::string(kind) + "_TEC").c_str(), t) + ".dat",
                       tecplot_header(s, t), ol);
      if (rc) return rc;
    }
    if (which_output == 1 || which_output == 3) {
      ol.ncoord = 0;
      rc = write_lines(s, dir + timestamp((std::string(kind) + "_OCT").c_str(), t) + ".dat",
                       octave_header(), ol);
      if (rc) return rc;
    }
  }
  return SWM_OK;
}

// WriteMeshToDisk (output.f90:190-231): barycentre coordinates, one (SP,ES21.14E2) a line
int swm_write_mesh(swm_handle s, const char* directory) {
  if (!s || !directory) return fail(SWM_ERR_PARAM, "null argument");
  CK(cudaSetDevice(s->device));
  const int n[2] = {s->nx, s->ny};
  const double x0[2] = {s->gr.x0, s->gr.y0}, dx[2] = {s->gr.dx, s->gr.dy};
  for (int d = 0; d < 2; ++d) {
    std::vector<double> c(n[d]);
    for (int i = 0; i < n[d]; ++i) c[i] = (x0[d] + ((double)i) * dx[d]) + 0.5 * dx[d];
    std::vector<char> txt(21 * (size_t)n[d]);
    int rc = swm_debug_format(s, c.data(), n[d], txt.data());
    if (rc) return rc;
    const std::string path = std::string(directory) + (d ? "/MESH_CoordinateY.dat" : "/MESH_CoordinateX.dat");
    FILE* f = fopen(path.c_str(), "w");
    if (!f) return fail(SWM_ERR_PARAM, ("cannot open " + path).c_str());
    fputs(d ? "CoordinateY\n" : "CoordinateX\n", f);
    for (int i = 0; i < n[d]; ++i) {
      fwrite(&txt[21 * (size_t)i], 1, 21, f);
      fputc('\n', f);
    }
    if (fclose(f) != 0) return fail(SWM_ERR_PARAM, ("cannot write " + path).c_str());
  }
  return SWM_OK;
}

int swm_debug_format(swm_handle s, const double* x, int n, char* out) {
  if (!s || (n > 0 && (!x || !out)) || n < 0) return fail(SWM_ERR_PARAM, "bad argument");
  if (n == 0) return SWM_OK;
  CK(cudaSetDevice(s->device));
  double* dx = nullptr;
  char* dout = nullptr;
  CK(cudaMalloc(&dx, sizeof(double) * n));
  cudaError_t e = cudaMalloc(&dout, 21 * (size_t)n);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_format_values(dx, n, dout, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, 21 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  if (e != cudaSuccess) return fail(SWM_ERR_CUDA, cudaGetErrorString(e));
  return SWM_OK;
}

int swm_set_wb_state(swm_handle s, const double* Uwb) {
  if (!s || !Uwb) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->p.well_balanced) return fail(SWM_ERR_STATE, "handle created without well_balanced");
  CK(cudaSetDevice(s->device));
  // scratch planes: substep-2 buffers are free between steps
  double *h = s->hbuf[1][0], *hu = s->hum[1], *hv = s->hvm[1];
  int rc = upload_ghosted(s, Uwb, h, hu, hv);
  if (rc) return rc;
  RhsArgs a = make_rhs_args(s, h, hu, hv, 1);
  a.fx_wb = a.fy_wb = a.s_wb = nullptr;  // FXWB = 0 during InitializeWBVariables
  a.fx_full = s->fxwb;
  a.fy_full = s->fywb;
  a.s_full = s->swb;
  rc = run_rhs_sync(s, a);
  if (rc) return rc;
  s->have_wb = true;
  drop_graph(s);  // the step graph bakes the WB pointers in
  return SWM_OK;
}

int swm_timestep(swm_handle s, double* dt_min) {
  NvtxRange range("swm_timestep");
  if (!s || !dt_min) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  CK(cudaSetDevice(s->device));
  if (!s->lam_fresh) {  // the state changed since the last step's reduction
    int rc = enqueue_dt(s);
    if (rc) return rc;
    CK(cudaMemcpyAsync(s->h_lam, s->lam, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->lam_fresh = true;
  }
  double LX, LY;
  std::memcpy(&LX, &s->h_lam[0], sizeof(double));
  std::memcpy(&LY, &s->h_lam[1], sizeof(double));
  s->stats.lambda_max[0] = LX;
  s->stats.lambda_max[1] = LY;
  // equation.f90:818-834
  double ts = 1.7976931348623157e308;  // HUGE(1.0)
  double a1 = s->gr.dx / LX, b1 = s->gr.dy / LY;
  if (a1 < ts) ts = a1;
  if (b1 < ts) ts = b1;
  ts = s->p.cfl * ts;
  if (ts < 1.0e-30) ts = 1.0e-30;
  *dt_min = ts;
  if (*s->h_bad) return fail(SWM_ERR_NAN, "non-finite or negative depth in the state");
  return SWM_OK;
}

int swm_step(swm_handle s, double t, double dt) {
  (void)t;  // stage times are not read by the periodic BC or the source (equation.f90:515,284)
  NvtxRange range("swm_step");
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(SWM_ERR_PARAM, "dt must be finite and > 0");
  if (s->p.well_balanced && !s->have_wb)
    return fail(SWM_ERR_STATE, "well_balanced handle without swm_set_wb_state");
  CK(cudaSetDevice(s->device));
  *s->h_dt = dt;
  CK(cudaMemcpyAsync(s->dt_dev, s->h_dt, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  int rc = build_graph(s);
  if (rc) return rc;
  if (s->graph) {
    CK(cudaGraphLaunch(s->graph, s->stream));
  } else {
    rc = enqueue_step(s);
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(JacobiCtl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(s->h_lam, s->lam, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->lam_fresh = true;
  if (s->n_solves == 0) {  // graph built without a host pass: count solves
    s->n_solves = solves_per_step(s->p.timescheme);
  }
  const JacobiCtl& c = *s->h_ctl;
  swm_stats& st = s->stats;
  st.n_solves = s->n_solves;
  st.jacobi_iters_min = 1 << 30;
  st.jacobi_iters_max = 0;
  for (int k = 0; k < s->n_solves && k < kMaxSolves; ++k) {
    st.jacobi_iters[k] = c.iters[k];
    st.jacobi_iters_total += c.iters[k];
    if (c.iters[k] < st.jacobi_iters_min) st.jacobi_iters_min = c.iters[k];
    if (c.iters[k] > st.jacobi_iters_max) st.jacobi_iters_max = c.iters[k];
  }
  st.steps++;
  st.status = c.status;
  if (c.status < 0) return fail(SWM_ERR_WATCHDOG, "Jacobi grid barrier watchdog expired");
  if (*s->h_bad) {
    st.status = SWM_ERR_NAN;
    return fail(SWM_ERR_NAN, "the step produced a non-finite value or a negative depth");
  }
  if (c.status == 1) {
    g_last_error = "Jacobi not converged (maxIter reached)";
    return SWM_WARN_JACOBI_MAXITER;
  }
  return SWM_OK;
}

int swm_get_stream(swm_handle s, void** stream) {
  if (!s || !stream) return fail(SWM_ERR_PARAM, "null argument");
  *stream = (void*)s->stream;
  return SWM_OK;
}

int swm_profile_step(swm_handle s, double t, double dt, float* ms, int* launches) {
  if (!s || !ms) return fail(SWM_ERR_PARAM, "null argument");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  CK(cudaSetDevice(s->device));
  *s->h_dt = dt;
  CK(cudaMemcpyAsync(s->dt_dev, s->h_dt, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  s->profiling = true;
  CK(cudaEventRecord(e0, s->stream));
  int rc = enqueue_step(s);
  CK(cudaEventRecord(e1, s->stream));
  s->profiling = false;
  CK(cudaStreamSynchronize(s->stream));
  float acc[3] = {0.f, 0.f, 0.f};
  int cnt[3] = {0, 0, 0};
  for (size_t k = 0; k + 1 < s->prof_ev.size(); k += 2) {
    float x = 0.f;
    cudaEventElapsedTime(&x, s->prof_ev[k], s->prof_ev[k + 1]);
    int c = s->prof_cls[k];
    if (c >= 0 && c < 3) {
      acc[c] += x;
      cnt[c]++;
    }
  }
  float tot = 0.f;
  cudaEventElapsedTime(&tot, e0, e1);
  for (auto e : s->prof_ev) cudaEventDestroy(e);
  s->prof_ev.clear();
  s->prof_cls.clear();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  for (int c = 0; c < 3; ++c) {
    ms[c] = acc[c];
    if (launches) launches[c] = cnt[c];
  }
  ms[3] = tot;
  CK(cudaMemcpy(s->h_ctl, s->ctl, sizeof(JacobiCtl), cudaMemcpyDeviceToHost));
  s->lam_fresh = false;
  for (int k = 0; k < s->n_solves && k < kMaxSolves; ++k) s->stats.jacobi_iters[k] = s->h_ctl->iters[k];
  s->stats.n_solves = s->n_solves;
  return s->h_ctl->status < 0 ? fail(SWM_ERR_WATCHDOG, "watchdog") : SWM_OK;
}

int swm_run(swm_handle s, double t_end, int n_outputs, int* n_steps, double* t_reached) {
  if (!s || n_outputs < 1) return fail(SWM_ERR_PARAM, "invalid argument");
  // timediscretization.f90:46-95 (I/O omitted)
  double t = 0.0, dt_an = t_end / (double)n_outputs, t_an = t + dt_an;
  int steps = 0, warn = 0;
  if (t != t_end) {
    for (;;) {
      double dt_min;
      int rc = swm_timestep(s, &dt_min);
      if (rc < 0) return rc;
      double a = dt_min < (t_an - t) ? dt_min : (t_an - t);
      double b = dt_min < (t_end - t) ? dt_min : (t_end - t);
      double dt = a < b ? a : b;
      rc = swm_step(s, t, dt);
      if (rc < 0) return rc;
      if (rc > 0) warn = rc;
      steps++;
      t = t + dt;
      if (fabs(t_an - t) < 1.0e-10) {
        t_an = t_an + dt_an;
        if (t_an > t_end) t_an = t_end;
      }
      if (fabs(t - t_end) < 1.0e-10) break;
    }
  }
  if (n_steps) *n_steps = steps;
  if (t_reached) *t_reached = t;
  return warn;
}

int swm_get_stats(swm_handle s, swm_stats* out) {
  if (!s || !out) return fail(SWM_ERR_PARAM, "null argument");
  *out = s->stats;
  return SWM_OK;
}

int swm_state_summary(swm_handle s, double* mass, double* min_h) {
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  if (!s->have_state) return fail(SWM_ERR_STATE, "no state set");
  CK(cudaSetDevice(s->device));
  CK(launch_summary(s->h, (int)s->N, s->summary, s->stream));
  double res[2];
  CK(cudaMemcpyAsync(res, s->summary, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (mass) *mass = res[0];
  if (min_h) *min_h = res[1];
  return SWM_OK;
}

const char* swm_last_error(void) { return g_last_error.c_str(); }

const char* swm_strerror(int status) {
  switch (status) {
    case SWM_OK: return "ok";
    case SWM_WARN_JACOBI_MAXITER: return "Jacobi not converged (maxIter reached)";
    case SWM_ERR_PARAM: return "invalid parameter";
    case SWM_ERR_CUDA: return "CUDA error";
    case SWM_ERR_NAN: return "non-finite state";
    case SWM_ERR_WATCHDOG: return "device watchdog expired";
    case SWM_ERR_ALLOC: return "allocation failed";
    case SWM_ERR_STATE: return "call out of order";
    case SWM_ERR_UNSUPPORTED: return "unsupported on this device";
    default: return "unknown status";
  }
}

int swm_debug_rhs(swm_handle s, const double* U, double* Ut, double* FX, double* FY, double* S) {
  if (!s || !U) return fail(SWM_ERR_PARAM, "null argument");
  if (s->p.well_balanced && !s->have_wb) return fail(SWM_ERR_STATE, "WB state not set");
  CK(cudaSetDevice(s->device));
  const size_t nx = s->nx, ny = s->ny, N = s->N;
  const size_t nfx = (nx + 1) * ny, nfy = nx * (ny + 1);
  double *h = s->hbuf[1][0], *hu = s->hum[1], *hv = s->hvm[1];
  int rc = upload_ghosted(s, U, h, hu, hv);
  if (rc) return rc;
  double *dfx = nullptr, *dfy = nullptr, *ds = nullptr, *dh = nullptr;
  CK(cudaMalloc(&dfx, 3 * nfx * sizeof(double)));
  CK(cudaMalloc(&dfy, 3 * nfy * sizeof(double)));
  CK(cudaMalloc(&ds, 3 * N * sizeof(double)));
  CK(cudaMalloc(&dh, N * sizeof(double)));
  RhsArgs a = make_rhs_args(s, h, hu, hv, 1);
  a.fx_full = dfx;
  a.fy_full = dfy;
  a.s_full = ds;
  a.ut_h = dh;  // Ut(1), as the build without PATANKAR computes it
  rc = run_rhs_sync(s, a);
  cudaError_t e = rc ? cudaErrorUnknown : cudaSuccess;
  std::vector<double> hfx(3 * nfx), hfy(3 * nfy), hs(3 * N), hht(N), hut(N), hvt(N);
  if (e == cudaSuccess) e = cudaMemcpy(hht.data(), dh, N * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hfx.data(), dfx, 3 * nfx * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hfy.data(), dfy, 3 * nfy * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hs.data(), ds, 3 * N * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hut.data(), s->fu[1], N * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hvt.data(), s->fv[1], N * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dfx);
  cudaFree(dfy);
  cudaFree(ds);
  cudaFree(dh);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(SWM_ERR_CUDA, cudaGetErrorString(e));
  // to the reference's column-major (3, ., .) layouts
  for (size_t j = 0; j < ny; ++j)
    for (size_t i = 0; i < nx; ++i) {
      size_t c = j * nx + i;
      if (Ut) {
        Ut[3 * c] = hht[c];
        Ut[3 * c + 1] = hut[c];
        Ut[3 * c + 2] = hvt[c];
      }
      if (S)
        for (int v = 0; v < 3; ++v) S[3 * c + v] = hs[v * N + c];
    }
  if (FX)
    for (size_t j = 0; j < ny; ++j)
      for (size_t f = 0; f <= nx; ++f)
        for (int v = 0; v < 3; ++v) FX[3 * (j * (nx + 1) + f) + v] = hfx[v * nfx + j * (nx + 1) + f];
  if (FY)
    for (size_t f = 0; f <= ny; ++f)
      for (size_t i = 0; i < nx; ++i)
        for (int v = 0; v < 3; ++v) FY[3 * (f * nx + i) + v] = hfy[v * nfy + f * nx + i];
  return SWM_OK;
}

int swm_debug_jacobi(swm_handle s, const double* mass, const double* diag, const double* rhs,
                     double* sol, int* iters) {
  if (!s || !mass || !diag || !rhs || !sol) return fail(SWM_ERR_PARAM, "null argument");
  CK(cudaSetDevice(s->device));
  const size_t N = s->N;
  const bool csr = s->p.solver == SWM_SOLVER_CSR;
  double* b = s->hbuf[1][0];
  double* out = s->hbuf[1][1];
  CK(cudaMemcpy(b, rhs, N * sizeof(double), cudaMemcpyHostToDevice));
  if (csr) {
    CK(cudaMemcpy(s->csr_mass, mass, 5 * N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->csr_diag, diag, N * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    // the fast solver's planes hold the row divided by its Diagonal and rhs/Diagonal
    // (the fast assembly writes the same: products with RN(1/D))
    const bool fast = fast_patankar(s->p);
    std::vector<double> pl(5 * N);
    for (size_t k = 0; k < N; ++k) {
      const double r = fast ? 1.0 / diag[k] : 1.0;
      pl[k] = fast ? mass[5 * k + 0] * r : mass[5 * k + 0];
      pl[N + k] = fast ? mass[5 * k + 1] * r : mass[5 * k + 1];
      pl[2 * N + k] = fast ? mass[5 * k + 3] * r : mass[5 * k + 3];
      pl[3 * N + k] = fast ? mass[5 * k + 4] * r : mass[5 * k + 4];
      pl[4 * N + k] = fast ? rhs[k] * r : diag[k];
    }
    CK(cudaMemcpy(s->cS, pl.data(), N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->cW, pl.data() + N, N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->cE, pl.data() + 2 * N, N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->cN, pl.data() + 3 * N, N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->cD, pl.data() + 4 * N, N * sizeof(double), cudaMemcpyHostToDevice));
  }
  CK(cudaMemset(s->ctl, 0, sizeof(JacobiCtl)));
  JacobiArgs ja{};
  ja.nx = s->nx;
  ja.ny = s->ny;
  ja.solve_idx = 0;
  ja.maxiter = s->p.jacobi_maxiter;
  fill_thresh(s, ja.thresh);
  ja.b = b;
  ja.cS = s->cS;
  ja.cW = s->cW;
  ja.cE = s->cE;
  ja.cN = s->cN;
  ja.cD = s->cD;
  ja.rowstart = s->rowstart;
  ja.cols = s->cols;
  ja.mass = s->csr_mass;
  ja.diag = s->csr_diag;
  ja.xa = s->xa;
  ja.xb = s->xb;
  ja.out = out;
  ja.ctl = s->ctl;
  ja.block = jacobi_block_of(s->p);
  ja.recip = fast_patankar(s->p) ? 1 : 0;
  ja.spin_limit = s->spin_limit;
  CK(launch_jacobi(ja, csr, s->jac_blocks, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(sol, out, N * sizeof(double), cudaMemcpyDeviceToHost));
  JacobiCtl c;
  CK(cudaMemcpy(&c, s->ctl, sizeof(JacobiCtl), cudaMemcpyDeviceToHost));
  if (iters) *iters = c.iters[0];
  if (c.status < 0) return fail(SWM_ERR_WATCHDOG, "Jacobi grid barrier watchdog expired");
  return c.status == 1 ? SWM_WARN_JACOBI_MAXITER : SWM_OK;
}

int swm_debug_checked_status(int* site, unsigned long long* count) {
  if (!site || !count) return fail(SWM_ERR_PARAM, "null argument");
  int sites[3] = {0, 0, 0};
  unsigned long long counts[3] = {0, 0, 0};
  if (check_record_kernels(&sites[0], &counts[0]) || check_record_rhs_fast(&sites[1], &counts[1]) ||
      check_record_rhs_exact(&sites[2], &counts[2]))
    return fail(SWM_ERR_CUDA, "reading the checked-build records failed");
  if (sites[0] < 0) return fail(SWM_ERR_UNSUPPORTED, "not a checked build (-DSWM_CHECKED)");
  *site = sites[0] ? sites[0] : (sites[1] ? sites[1] : sites[2]);
  *count = counts[0] + counts[1] + counts[2];
  return SWM_OK;
}

int swm_debug_set_tma(swm_handle s, int enable) {
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  s->tma = enable != 0;
  drop_graph(s);
  return SWM_OK;
}

int swm_debug_set_spin_limit(swm_handle s, long long limit) {
  if (!s) return fail(SWM_ERR_PARAM, "null handle");
  s->spin_limit = limit;
  drop_graph(s);  // the step graph bakes the limit into its Jacobi launches
  return SWM_OK;
}

int swm_debug_inject_alloc_failure(long long nth, long long* counted) {
  if (nth < 0) return fail(SWM_ERR_PARAM, "nth must be >= 0");
  const long long n = g_alloc_count.exchange(0);
  if (counted) *counted = n;
  g_alloc_fail_at.store(nth);
  return SWM_OK;
}

}  // extern "C"
