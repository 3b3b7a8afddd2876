// lcs_tma.cuh -- TMA tile loads and bounded mbarrier waits for the sweep
// kernels: the tensor maps of the velocity buffers and of P (kernel
// parameters), 3-D tiled loads into shared memory completing on an mbarrier
// (no multicast: every CTA loads its own tiles from this GPU's memory), and
// waits that give up after a bound instead of hanging.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "lcs_common.cuh"

namespace lcs {
namespace {

constexpr int kVelMaps = 9;

// Kernel parameter (__grid_constant__): tensor maps of the 9 physical
// velocity buffers (box TX+4 x TY+4 x 1) and of P (box TX x TY x 1).
struct TensorMaps {
  CUtensorMap vel[kVelMaps];
  CUtensorMap P;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3-D tiled TMA load into shared memory, completion counted on `bar`.  No
// multicast: every CTA loads its own tiles from this GPU's memory.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait: true when the phase completed, false after 2^22 polls or
// about 0.25 s (5e8 SM cycles), whichever comes first.  A try_wait may itself
// suspend the thread for a while, so the poll count alone does not bound the
// time.  The clock is read only once the first poll has failed.
constexpr long long kMbarWaitCycles = 500000000;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 0; it < (1 << 22); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > kMbarWaitCycles) break;
  }
  return false;
}

}  // namespace
}  // namespace lcs
