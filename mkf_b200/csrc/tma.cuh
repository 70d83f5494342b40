// tma.cuh - tile copies by the tensor memory accelerator (cp.async.bulk.tensor) into a warp's ring
// of shared-memory stages, completed through mbarriers; shared by the TMA-staged kernels. Every
// tensor map covers this GPU's own memory, and no copy uses cluster multicast.
#pragma once
#include <cuda.h>
#include "mkf_common.cuh"

namespace mkf {

static constexpr long kTmaWaitLimit = 1L << 22;  // mbarrier polls before a wait gives up

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Announce the bytes of the barrier's next phase and start the copy of one 3D tile (one lane).
__device__ __forceinline__ void tmaTile3D(const CUtensorMap *tm, uint32_t dst, uint32_t bar, int x, int y, int z,
                                          uint32_t bytes)
{
   // the stage was last read through the generic proxy; order those reads before the async write
   asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
   asm volatile(
       "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
       "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(bar)
       : "memory");
}

// Wait for phase `parity` of a barrier; false after kTmaWaitLimit polls.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity)
{
   for (long i = 0; i < kTmaWaitLimit; i++) {
      uint32_t done;
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
          : "=r"(done)
          : "r"(bar), "r"(parity)
          : "memory");
      if (done) { return true; }
   }
   return false;
}

// Tensor map of a 3D field (X fastest, element strides 1, sy, sz; FP32 or FP64) with boxes of
// boxX x boxY x 1 elements, zero fill out of bounds. false when the driver lacks the call or the
// layout is not one a tensor map can describe (base or strides off 16-byte boundaries).
bool encodeField3D(CUtensorMap *tm, const void *base, int enc, int X, int Y, int Z, int64_t sy, int64_t sz, int boxX, int boxY,
                   bool promote256 = true);

// Fault flags of the kernels whose waits gave up (per translation unit); clear when asked.
unsigned thermoTmaFaults(bool clear);

}  // namespace mkf
