// swm_rhs_exact.cu -- RHS kernel instance for the EXACT FP64 form.  Built with
// -fmad=false so that every expression rounds as the reference's source order
// does; with IEEE division and square root this reproduces the CPU restatement
// bit for bit except where a libm function (exp, sin, cos) is evaluated.
#define SWM_EXACT 1
#define SWM_RHS_NS rhs_exact
#include "swm_kernels.cuh"
#include "swm_ensemble.cuh"

namespace swm {

SWM_CHECK_READER(check_record_rhs_exact)

const void* ensemble_kernel_exact(int tb) { return rhs_exact::ensemble_kernel<0>(tb); }

cudaError_t launch_rhs_exact(const RhsArgs& a, const RhsTma& tm, cudaStream_t s) {
  dim3 grd((a.gr.nx + RHS_TX - 1) / RHS_TX, (a.gr.ny + RHS_TY - 1) / RHS_TY);
  size_t sm = RhsSmem<double>::bytes;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(rhs_exact::rhs_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    attr = true;
  }
  rhs_exact::rhs_kernel<0><<<grd, RHS_NT, sm, s>>>(a, tm);
  return cudaGetLastError();
}

cudaError_t launch_rhs_batch_exact(const RhsArgs* descs, const int4* work, int nwork,
                                   cudaStream_t s) {
  if (nwork < 1) return cudaSuccess;
  size_t sm = RhsSmem<double>::bytes;
  cudaFuncSetAttribute(rhs_exact::rhs_batch_kernel<0>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  rhs_exact::rhs_batch_kernel<0><<<nwork, RHS_NT, sm, s>>>(descs, work);
  return cudaGetLastError();
}

}  // namespace swm
