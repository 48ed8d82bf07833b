// tma.cuh -- 1-D bulk copies (cp.async.bulk, no multicast) into shared memory, completed
// on an mbarrier, with bounded waits.
//
// Rules kept here: every source and destination address and every size is a multiple of
// 16 bytes (callers stage whole 32- or 64-byte records from cudaMalloc'd arrays); no
// cluster-multicast form is used; every wait gives up after a fixed number of
// polls and reports it, so a lost completion cannot hang the GPU.
#pragma once

#include <cstdint>

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Poll the barrier phase a bounded number of times (each try_wait itself blocks for a
// short hardware-defined interval).  Returns false on give-up.
constexpr int kMbarPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase) {
  for (int it = 0; it < kMbarPolls; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}
