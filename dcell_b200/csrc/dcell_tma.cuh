// Shared-memory staging primitives of the TMA-fed kernels (sm_100a):
// mbarriers with bounded waits and 3-D tiled bulk-tensor loads (no
// multicast).  Every wait gives up after a bounded number of polls and
// reports it, so a kernel never hangs on a phase that does not complete.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace dcell {

constexpr unsigned kWaitLimit = 1u << 20;  // bounded mbarrier polls (a normal phase completes in microseconds)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for phase `parity` of the mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Bounded wait that lets the hardware suspend the thread until the phase
// completes (or `kSleepNs` pass) instead of spinning: pipeline waits where
// warps routinely wait a few hundred cycles.  At most kSleepLimit rounds
// (well under a second in all).
constexpr uint32_t kSleepNs = 20000;
constexpr unsigned kSleepLimit = 1u << 15;
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kSleepLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(kSleepNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (TMA) writes into it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 3-D tiled TMA load (no multicast) of the box at (c0, c1, c2) into shared
// memory, completing `bytes` of the mbarrier's transaction count.  c0 times
// the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace dcell
