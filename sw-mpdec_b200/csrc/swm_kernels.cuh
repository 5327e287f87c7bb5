// swm_kernels.cuh -- declarations shared by the host orchestration and the
// memory-bound kernels (dt, layouts, Patankar assembly, Jacobi).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "swm_device.cuh"
#include "swm_rhs.cuh"

namespace swm {

// Residual accumulator: |dx| in units of 2^-100 split into three 40-bit limbs.
// Integer addition is associative, so the residual sum (and with it the Jacobi
// stop index) does not depend on tiling, launch shape or atomic ordering.
constexpr int kResSlots = 3;    // ring of pass slots (see jacobi kernels)
constexpr int kMaxBlock = 8;    // max Jacobi sweeps per stencil pass
constexpr int kMaxSolves = 16;  // solves recorded per step
// Polls of a grid-barrier wait before it gives up (status -4); ~1 s at 40 ns a poll.
// A limit <= 0 makes every wait that is not already open give up at once.
constexpr long long kDefaultSpinLimit = 1LL << 26;

struct JacobiCtl {
  unsigned long long acc[kResSlots][kMaxBlock + 1][3];  // [slot][0 = initial, 1..T sweeps][limb]
  unsigned int bar_count;
  unsigned int bar_gen;
  int iters[kMaxSolves];  // iterations of each solve of the current step
  int status;             // 0 ok, 1 maxiter, -4 watchdog
  int pass_next;          // pass counter carried across solves (slot ring position)
};

struct AssembleArgs {
  int nx, ny;
  double dx, dy;
  int m;                  // substep 2..4 (1-based, as in the reference)
  int msteps;             // 4 (mPDeC5) or 2 (mPDeC2)
  int compat2;            // mPDeC2 sequence-association read of hp
  int jpitch;             // row pitch of the stencil planes and rhs_out (<= 0: nx)
  double theta[4];        // thetaDeC(m, 1:4)
  const double* dt;       // device scalar
  const double* hu_n;     // Ua(1, 2:3) = U^n momentum
  const double* hv_n;
  const double* fu[4];    // FUp(r, 2) planes
  const double* fv[4];    // FUp(r, 3)
  const double* fxm[4];   // mass fluxes of stage r: [ny][nx+1]
  const double* fym[4];   // [ny+1][nx]
  const double* hp[4];    // Up(r, 1) for r = 1..msteps (hp(m,.) is hp[m-1])
  double* hu_out;         // Ua(m, 2:3)
  double* hv_out;
  // stencil layout: 5 planes (S, W, E, N, Diag); CSR layout: mass[5N], diag[N]
  double* cS;
  double* cW;
  double* cE;
  double* cN;
  double* cD;
  double* csr_mass;
  double* csr_diag;
  double* rhs_out;        // nullable: rhs = hp(1,.) (needed when hp is read through compat2)
  // split form: PATANKAR_DIV from one reciprocal per depth, P/D by 1/dx, and the
  // stencil planes holding the row divided by its Diagonal, the D plane b/Diagonal
  // (not bit-identical to the reference order)
  int fast;
  double inv_dx, inv_dy;
};

// Substeps m of one mPDeC5 correction iteration assembled in one launch (stencil
// layout): `base` carries the shared inputs (stage RHS slots, face fluxes, hp, U^n
// momentum, dt, grid); per substep its number, weights and output planes.
constexpr int kMaxFusedStages = 3;
struct AssembleMultiArgs {
  AssembleArgs base;
  int nm;
  int m[kMaxFusedStages];  // 1-based substeps
  double theta[kMaxFusedStages][4];
  double* hu_out[kMaxFusedStages];
  double* hv_out[kMaxFusedStages];
  double* cS[kMaxFusedStages];
  double* cW[kMaxFusedStages];
  double* cE[kMaxFusedStages];
  double* cN[kMaxFusedStages];
  double* cD[kMaxFusedStages];
};

struct JacobiArgs {
  int nx, ny;
  int solve_idx;          // slot in ctl->iters
  int maxiter;
  int pitch;              // stencil: row pitch of b, the coefficient planes and xa/xb
                          // (<= 0: nx); out is unpadded
  unsigned long long thresh[3];  // tol * n in residual units (limbs)
  const double* b;        // rhs (= hp(1) = h^n)
  // stencil coefficients
  const double* cS;
  const double* cW;
  const double* cE;
  const double* cN;
  const double* cD;
  // CSR
  const int* rowstart;    // 1-based (finitevolume.f90:230,267)
  const int* cols;        // 1-based
  const double* mass;
  const double* diag;
  double* xa;             // ping-pong buffers
  double* xb;
  double* out;            // final iterate destination
  JacobiCtl* ctl;
  int block;              // sweeps per pass (stencil)
  int recip;              // stencil (split form): S..N hold Mass/Diagonal, cD holds b/Diagonal
  long long spin_limit;   // grid-barrier watchdog
};

struct DtArgs {
  int nx, ny;
  double g;
  const double* h;
  const double* hu;
  const double* hv;
  unsigned long long* lam;  // [2] bit patterns of LambdaMaxX/Y (non-negative doubles)
  int* bad;                 // non-finite or negative depth seen
};

// ---- ensembles: one launch covers every problem ----
// Jacobi state of one problem during a batched solve (global memory).
struct JacBatchState {
  int active;    // still iterating
  int k;         // sweeps done
  int Tp;        // sweeps of the coming pass
  int rollback;  // the coming pass redoes the last one with Tp sweeps
  int first;     // the coming pass is the first (initial residual checked)
  int cur;       // buffer holding x^k: 0 = b, 1 = xa, 2 = xb, 3 = the destination
  int result;    // final iterate: 0 = zero vector, 1 = xa, 2 = xb, 3 = the destination
  int final_k;
  int maxhit;
  int xnext;     // buffer the coming pass writes: 1 = xa, 2 = xb, 3 = the destination
  double r_prev;  // residual sum of the last sweep of the previous pass (pass planning)
  unsigned long long acc[kMaxBlock + 1][3];
};
struct JacBatchCtl {
  unsigned int bar_count, bar_gen;
  int n_active;
  int status;  // 0 ok, 1 some problem hit maxIter, -4 watchdog
};
struct JacobiBatchArgs {
  // per system (set q, problem p -> q * nprob + p): nx, ny, b, stencil planes, xa, xb,
  // out, thresh, maxiter
  const JacobiArgs* descs;
  const int2* tiles;        // (problem, tile index) of every tile of every problem
  int ntiles, nprob;
  int nsets;                // independent systems per problem solved together (>= 1)
  JacBatchState* st;        // [nsets * nprob]
  JacBatchCtl* ctl;
  int* iters;               // [nsets * nprob] sweeps of each system's solve
  int block;
  long long spin_limit;
  // nullable: work-item counter; when set, CTAs take a pass's tiles one at a time from
  // it (reset to 0 before every pass) instead of striding by CTA
  unsigned int* work;
};
struct DtBatchDesc {
  int nx, ny;
  double g, cfl, dx, dy;
  const double* h;
  const double* hu;
  const double* hv;
};

// ---- ensembles in one persistent launch per mPDeC5 step ----
constexpr int kEnsCells = 256;  // cells of one TimeStep / assembly work item (= CTA size)

struct EnsembleArgs {
  int nprob;
  int precision;             // SWM_PREC_*: which RHS tile function runs
  // TimeStep (equation.f90:791-837) of every problem
  const DtBatchDesc* dtd;
  const int2* cells;         // (problem, first cell) of every kEnsCells-cell block
  int ncells;
  unsigned long long* lam;   // [2 nprob] LambdaMax bit patterns, zeroed before the launch
  int* bad;                  // [nprob] non-finite / negative depth, zeroed before the launch
  double* dt;                // [nprob]
  // RHS: descriptors [set][nprob] (set 0: U^n; 1 + 3 par + m - 2: Ua(m) of correction
  // parity par) and the (problem, i0, j0) tiles of one set
  const RhsArgs* rhs;
  const int4* rtiles;
  int nrtiles;
  // combination + assembly: per (solve, problem) [13][nprob]; the fast forms' three
  // substeps of corrections 1..4 fused per cell [4][nprob]
  const AssembleArgs* asmd;
  const AssembleMultiArgs* asmm;
  // Jacobi: the systems of correction k = 1..5, [5][3 nprob]: set q = substep m - 2
  // (the last correction's one system is set 0)
  const JacobiArgs* jac;
  const int2* jtiles;        // (problem, tile) of every problem's Jacobi tiles
  int njtiles;
  JacBatchState* st;         // [3 nprob]
  JacBatchCtl* ctl;          // grid barrier and status, zeroed before the launch
  int* iters;                // [13][nprob] sweeps of every solve
  int block;                 // Jacobi sweeps per pass
  long long spin_limit;      // grid-barrier watchdog
  // nullable: the global timer (ns) when CTA 0 starts and leaves each phase's
  // closing barrier, kEnsMarks entries (measurement only)
  unsigned long long* clock;
  // work-item counters, zeroed before the launch: [0..4] RHS phases (U^n, k = 1..4),
  // [5..9] assembly phases (k = 1..5), [10] the Jacobi passes
  unsigned int* work;
};
constexpr int kEnsCounters = 11;
// start, TimeStep, RHS of U^n, then per correction assembly, Jacobi and (k < 5) RHS
constexpr int kEnsMarks = 3 + 5 * 3 - 1;
// The ensemble step kernel (swm_ensemble.cuh) of a precision form and a Jacobi
// temporal block tb (2, 4 or 8), as instantiated in the RHS units: split and FP64-FMA
// forms in swm_rhs_fast.cu, the FP64 form in swm_rhs_exact.cu.
const void* ensemble_kernel_fast(int mode, int tb);  // mode 1 split, 0 FP64-FMA
const void* ensemble_kernel_exact(int tb);
// dynamic shared memory of that kernel: the larger of the RHS tile's and the Jacobi
// tile's (swm_kernels.cu)
size_t ensemble_smem_bytes(int tb, int precision);

// Checked-build records of the three units with device-side index checks (see
// SWM_IN_RANGE): read and cleared; site -1 when the unit was built without them.
int check_record_kernels(int* site, unsigned long long* count);
int check_record_rhs_fast(int* site, unsigned long long* count);
int check_record_rhs_exact(int* site, unsigned long long* count);

// Host launchers (swm_kernels.cu, swm_rhs_*.cu)
cudaError_t launch_rhs_batch_fast(int mode, const RhsArgs* descs, const int4* work, int nwork,
                                  cudaStream_t s);
cudaError_t launch_rhs_batch_exact(const RhsArgs* descs, const int4* work, int nwork,
                                   cudaStream_t s);
cudaError_t launch_assemble_multi_batch(const AssembleMultiArgs* descs, const int2* blk, int nblk,
                                        cudaStream_t s);
cudaError_t launch_assemble_batch(const AssembleArgs* descs, const int2* blk, int nblk, bool fast,
                                  cudaStream_t s);
cudaError_t launch_jacobi_batch(const JacobiBatchArgs& a, int grid_blocks, bool recip,
                                cudaStream_t s);
int jacobi_batch_grid_blocks(int block, int device, bool recip);
cudaError_t launch_dt_batch(const DtBatchDesc* d, const int2* blk, int nblk, int nprob,
                            unsigned long long* lam, int* bad, double* dt, cudaStream_t s);
cudaError_t launch_rhs_fast(int mode, const RhsArgs& a, const RhsTma& tm, cudaStream_t s);
cudaError_t launch_rhs_exact(const RhsArgs& a, const RhsTma& tm, cudaStream_t s);
size_t rhs_smem_bytes(int mode);

cudaError_t launch_dt(const DtArgs& a, cudaStream_t s);
cudaError_t launch_assemble(const AssembleArgs& a, bool csr, cudaStream_t s);
cudaError_t launch_assemble_multi(const AssembleMultiArgs& a, cudaStream_t s);
cudaError_t launch_jacobi(const JacobiArgs& a, bool csr, int grid_blocks, cudaStream_t s);
int jacobi_grid_blocks(bool csr, int block, int device, bool recip = false);
cudaError_t launch_ghosted_to_planes(const double* G, int nx, int ny, double* h, double* hu,
                                     double* hv, cudaStream_t s);
cudaError_t launch_planes_to_ghosted(const double* h, const double* hu, const double* hv, int nx,
                                     int ny, double* G, double* Vg, cudaStream_t s);
cudaError_t launch_summary(const double* h, int n, double* out /*[2]*/, cudaStream_t s);

// Stage combinations of the explicit schemes, out[v] for v = h, hu, hv (FP64, each
// product and sum rounded in the reference's order; out may alias X[0]):
//  kComboSsp  sum_i c_i X_i + sum_j (d_j Y_j) dt      SSPRK(5,4), forward Euler
//  kComboRk   X_0 + (sum_j d_j Y_j) dt                RK65
//  kComboDec  X_0 + sum_j (dt d_j) Y_j                DeC5
enum { kComboSsp = 0, kComboRk = 1, kComboDec = 2 };
constexpr int kComboMax = 6;
struct ComboArgs {
  int n;        // cells
  int form;
  int nx, ny;   // terms in X and Y
  double c[kComboMax], d[kComboMax];
  const double* dt;  // device scalar
  const double* X[kComboMax][3];
  const double* Y[kComboMax][3];
  double* out[3];
};
cudaError_t launch_combo(const ComboArgs& a, cudaStream_t s);

// Formatted output (swm_output.cu): one fixed-width line per cell.
struct OutLines {
  int nx, ny;
  int ncoord;      // 0 or 2: the barycentre coordinates first
  int nval;        // values per line after the coordinates (<= 4)
  int sep;         // spaces after every field (2X)
  int zero_small;  // print |v| < 1e-70 as 0
  double x0, y0, dx, dy;
  const double* val[4];  // planes [ny][nx]; null prints 0
  char* out;             // nx*ny lines of out_line_width() bytes
};
size_t out_line_width(const OutLines& a);
cudaError_t launch_out_lines(const OutLines& a, cudaStream_t s);
cudaError_t launch_prim(const double* h, const double* hu, const double* hv, double* u, double* v,
                        int n, cudaStream_t s);
// n values as 21-character (SP,ES21.14E2) fields, back to back
cudaError_t launch_format_values(const double* x, int n, char* out, cudaStream_t s);

// Initial conditions and the L1 error on the device (swm_ic.cu).
struct IcArgs {
  Grid gr;
  int ic;            // ExactFunction case: 1..6 (equation.f90:109-206), 101..105
  double par[8];     // parameters of cases 101..105
  double t;          // time of the exact solution (case 1 is advected)
  double sx[2];      // domain extents |x1 - x0| (MESH_SX)
  double* h;         // planes [ny][nx]: written by the fill, read by the L1 error
  double* hu;
  double* hv;
};
constexpr int kIcMaxBlocks = 148 * 8;
bool ic_supported(int ic);
int ic_blocks(int ncells);
cudaError_t launch_ic_fill(const IcArgs& a, cudaStream_t s);
// partial: 3 * ic_blocks(nx*ny) doubles of scratch; out: 3 doubles (device)
cudaError_t launch_l1_error(const IcArgs& a, double* partial, double* out, cudaStream_t s);
// Error(1:3) = U - Uexact(ic, t) into e[3] planes (output.f90:76-85; U read from a.h/hu/hv)
cudaError_t launch_error_planes(const IcArgs& a, double* const e[3], cudaStream_t s);
// Bath = 4x4 Gauss average of Bathymetry (finitevolume.f90:323-325) into b[N]
cudaError_t launch_bath_average(const IcArgs& a, double* b, cudaStream_t s);
void residual_limbs_host(double v, unsigned long long out[3]);

}  // namespace swm
