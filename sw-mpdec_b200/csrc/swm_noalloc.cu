// swm_noalloc.cu -- a Jacobi solve of one Patankar system that allocates nothing.
//
// The handle API allocates all its device memory in swm_create.  Some callers
// cannot let a library allocate: drivers that own every byte of device memory
// through their own pool (or share a hard memory cap between several solvers),
// and callers that must not pay the device-wide synchronisation of a
// cudaMalloc/cudaFree pair inside their loop.  For them, swm_jacobi_noalloc
// runs the matrix-free stencil Jacobi kernel on caller-owned device arrays and
// keeps its only scratch -- one iterate buffer and the solver's control block --
// in the file-scope array below, which every GPU that loads this library holds
// until the process exits.
#include <cstdint>
#include <mutex>

#include "../../include/swm.h"
#include "swm_kernels.cuh"

namespace {

using swm::JacobiArgs;
using swm::JacobiCtl;

constexpr size_t kNoAllocMaxCells = size_t(1) << 20;  // 1,048,576 cells, e.g. 1024 x 1024
constexpr size_t kCtlDoubles = (sizeof(JacobiCtl) + sizeof(double) - 1) / sizeof(double);
constexpr int kMaxDevices = 64;

// [0, kNoAllocMaxCells): the second Jacobi iterate buffer (8 MiB);
// [kNoAllocMaxCells, +kCtlDoubles): the residual accumulators, grid-barrier
// counters and iteration count of the solve.
static __device__ __align__(256) double g_jacobi_scratch[kNoAllocMaxCells + kCtlDoubles];

struct DeviceSetup {
  bool ready = false;
  double* scratch = nullptr;  // device address of g_jacobi_scratch on that device
  int blocks[swm::kMaxBlock + 1] = {};
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

}  // namespace

namespace swm {
void set_last_error(const char* msg);  // swm_capi.cu: the text swm_last_error() returns
}

namespace {
int noalloc_fail(int code, const char* msg) {
  swm::set_last_error(msg);
  return code;
}
}  // namespace

extern "C" {

int swm_jacobi_noalloc(int nx, int ny, const double* cS, const double* cW, const double* cE,
                       const double* cN, const double* cD, const double* rhs, double* sol,
                       int maxiter, double tol, int block, int* iters, void* stream) {
  if (nx < 3 || ny < 3) return noalloc_fail(SWM_ERR_PARAM, "nx, ny must be >= 3");
  if ((size_t)nx * (size_t)ny > kNoAllocMaxCells)
    return noalloc_fail(SWM_ERR_PARAM,
                        "nx*ny exceeds the 1048576-cell scratch of swm_jacobi_noalloc");
  if (!cS || !cW || !cE || !cN || !cD || !rhs || !sol)
    return noalloc_fail(SWM_ERR_PARAM, "null device array");
  // sol is written during the solve (it doubles as an iterate buffer) while the six
  // inputs are read, so its byte range must not intersect any of theirs.
  {
    const size_t bytes = (size_t)nx * (size_t)ny * sizeof(double);
    const uintptr_t s0 = reinterpret_cast<uintptr_t>(sol), s1 = s0 + bytes;
    const double* in[6] = {cS, cW, cE, cN, cD, rhs};
    for (const double* q : in) {
      const uintptr_t q0 = reinterpret_cast<uintptr_t>(q), q1 = q0 + bytes;
      if (q0 < s1 && s0 < q1)
        return noalloc_fail(SWM_ERR_PARAM, "sol must not overlap rhs or a coefficient plane");
    }
  }
  if (maxiter < 1 || !(tol >= 0.0)) return noalloc_fail(SWM_ERR_PARAM, "maxiter >= 1, tol >= 0");
  if (block < 1 || block > swm::kMaxBlock) return noalloc_fail(SWM_ERR_PARAM, "block in 1..8");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(SWM_ERR_CUDA, "no current CUDA device");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The call ends by synchronising `st` to read the iteration count, which a stream
  // under capture cannot do (and doing it would invalidate the caller's capture).
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return noalloc_fail(SWM_ERR_STATE,
                          "swm_jacobi_noalloc synchronises its stream: not callable during capture");
    }
  }

  // Once per device, with that device current: the device address of the scratch
  // array (its host-side name is only a stand-in) and the persistent grid size.
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& ds = g_setup[dev];
    if (!ds.ready) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_jacobi_scratch);
      if (e != cudaSuccess || !p) return noalloc_fail(SWM_ERR_CUDA, cudaGetErrorString(e));
      ds.scratch = static_cast<double*>(p);
      ds.ready = true;
    }
    if (ds.blocks[block] == 0) {
      int nb = swm::jacobi_grid_blocks(false, block, dev);
      if (nb < 1) return noalloc_fail(SWM_ERR_CUDA, "Jacobi kernel cannot be resident");
      ds.blocks[block] = nb;
    }
  }
  const DeviceSetup& ds = g_setup[dev];
  JacobiCtl* ctl = reinterpret_cast<JacobiCtl*>(ds.scratch + kNoAllocMaxCells);

  // The control block keeps the previous call's contents: clear accumulators,
  // barrier counters, status and iteration count before every solve.
  cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(JacobiCtl), st);
  if (e != cudaSuccess) return noalloc_fail(SWM_ERR_CUDA, cudaGetErrorString(e));

  JacobiArgs ja{};
  ja.nx = nx;
  ja.ny = ny;
  ja.solve_idx = 0;
  ja.maxiter = maxiter;
  swm::residual_limbs_host(tol * (double)nx * (double)ny, ja.thresh);
  ja.b = rhs;
  ja.cS = cS;
  ja.cW = cW;
  ja.cE = cE;
  ja.cN = cN;
  ja.cD = cD;
  ja.xa = ds.scratch;  // second iterate buffer from the static scratch
  ja.xb = sol;         // the caller's output doubles as the first
  ja.out = sol;
  ja.ctl = ctl;
  ja.block = block;
  ja.spin_limit = swm::kDefaultSpinLimit;
  e = swm::launch_jacobi(ja, false, ds.blocks[block], st);
  if (e != cudaSuccess) return noalloc_fail(SWM_ERR_CUDA, cudaGetErrorString(e));
  int res[2] = {0, 0};  // iters[0], status
  e = cudaMemcpyAsync(&res[0], &ctl->iters[0], sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&res[1], &ctl->status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_fail(SWM_ERR_CUDA, cudaGetErrorString(e));
  if (iters) *iters = res[0];
  if (res[1] < 0) return noalloc_fail(SWM_ERR_WATCHDOG, "Jacobi grid barrier watchdog expired");
  return res[1] == 1 ? SWM_WARN_JACOBI_MAXITER : SWM_OK;
}

}  // extern "C"
