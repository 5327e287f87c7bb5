// swm_rhs_fast.cu -- RHS kernel instances for the FP64 form (FMA contraction,
// shared reciprocals) and the split FP32/FP64 form.
#define SWM_EXACT 0
#define SWM_RHS_NS rhs_fast
#include "swm_kernels.cuh"
#include "swm_ensemble.cuh"

namespace swm {

SWM_CHECK_READER(check_record_rhs_fast)

const void* ensemble_kernel_fast(int mode, int tb) {
  return mode == 1 ? rhs_fast::ensemble_kernel<1>(tb) : rhs_fast::ensemble_kernel<0>(tb);
}

size_t rhs_smem_bytes(int mode) {
  return mode == 1 ? RhsSmem<float>::bytes : RhsSmem<double>::bytes;
}

cudaError_t launch_rhs_fast(int mode, const RhsArgs& a, const RhsTma& tm, cudaStream_t s) {
  dim3 grd((a.gr.nx + RHS_TX - 1) / RHS_TX, (a.gr.ny + RHS_TY - 1) / RHS_TY);
  if (mode == 1) {
    size_t sm = RhsSmem<float>::bytes;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(rhs_fast::rhs_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
      attr = true;
    }
    rhs_fast::rhs_kernel<1><<<grd, RHS_NT, sm, s>>>(a, tm);
  } else {
    size_t sm = RhsSmem<double>::bytes;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(rhs_fast::rhs_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
      attr = true;
    }
    rhs_fast::rhs_kernel<0><<<grd, RHS_NT, sm, s>>>(a, tm);
  }
  return cudaGetLastError();
}

cudaError_t launch_rhs_batch_fast(int mode, const RhsArgs* descs, const int4* work, int nwork,
                                  cudaStream_t s) {
  if (nwork < 1) return cudaSuccess;
  if (mode == 1) {
    size_t sm = RhsSmem<float>::bytes;
    cudaFuncSetAttribute(rhs_fast::rhs_batch_kernel<1>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    rhs_fast::rhs_batch_kernel<1><<<nwork, RHS_NT, sm, s>>>(descs, work);
  } else {
    size_t sm = RhsSmem<double>::bytes;
    cudaFuncSetAttribute(rhs_fast::rhs_batch_kernel<0>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    rhs_fast::rhs_batch_kernel<0><<<nwork, RHS_NT, sm, s>>>(descs, work);
  }
  return cudaGetLastError();
}

}  // namespace swm
