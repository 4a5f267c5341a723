// Bulk global -> shared copies (the Hopper/Blackwell TMA unit, untiled form)
// completed through shared-memory mbarriers, as inline PTX for sm_100a.
//
// A copy moves a contiguous byte range whose global start, shared
// destination and size are multiples of 16 bytes; the mbarrier's transaction
// count is raised by the expected bytes first (arrive.expect_tx) and each
// copy lowers it as its bytes land, completing the barrier's current phase.
// Waiters poll try_wait.parity with an iteration bound, so a copy that never
// lands turns into an error status instead of a hang.
#pragma once

#include <stdint.h>

namespace ilbm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals)
               : "memory");
}

// makes barrier initialisation visible to the async (copy) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of incoming copies
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the phase with the given parity (about two seconds and
// at most 2^26 polls, whichever ends first; a single poll may itself suspend
// for a while); false if the phase never came
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (int it = 0; it < (1 << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 2000000000ull) break;
  }
  return false;
}

// a plain arrival (no transaction bytes)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same shared memory
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// bulk copy of `bytes` (multiple of 16) from global `src` (16-byte aligned)
// to shared `dst` (16-byte aligned), completing on `bar`
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace ilbm
