// swm_tma.cuh -- tensor-memory-accelerator (TMA) tile loads into shared memory,
// completed on an mbarrier (sm_90+ PTX, used here on sm_100a).
//
// One elected thread issues cp.async.bulk.tensor copies of 2D boxes of a row-major
// FP64 plane into this CTA's shared memory and announces their bytes on an
// mbarrier; every thread then waits on the barrier's phase.  The waits are bounded:
// a wait that runs out reports failure to the caller, which records an error status
// and gives up the tile instead of spinning for ever.  No multicast: every copy reads
// this GPU's own memory into this CTA alone.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace swm {

// Tensor maps of the three state planes (h, hu, hv) an RHS launch reads, as a
// __grid_constant__ kernel parameter.  `enabled` is 0 when the planes cannot be
// described (odd row pitch, grid smaller than a haloed tile).
struct alignas(64) RhsTma {
  CUtensorMap plane[3];
  int enabled;
};

// The box every map copies: 24 x 22 doubles.  Its x origin is the tile origin
// minus 4 (a multiple of 4, so x * 8 bytes is 16-byte aligned); rows start 3 above.
constexpr int kTmaBoxX = 24;
constexpr int kTmaBoxY = 22;
constexpr unsigned kTmaBoxBytes = kTmaBoxX * kTmaBoxY * sizeof(double);

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  // make the initialised barrier visible to the asynchronous (TMA) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Waits for the barrier's phase `parity` to complete; false when `limit` polls
// (each a hardware-suspended try_wait) ran out first.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit) {
  const unsigned b = smem_u32(bar);
  for (long long k = 0; k < limit; ++k) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2D tiled copy of the box at element coordinates (x, y) of `map` into `dst`
// (128-byte aligned shared memory), counted on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Polls of a TMA completion wait before the tile is given up (status -4).
constexpr long long kTmaWaitLimit = 1LL << 24;

}  // namespace swm
