// bulk_copy.cuh -- shared-memory staging with the bulk-copy (TMA) engine:
// one-dimensional cp.async.bulk global -> shared copies into the issuing
// block's own shared memory that complete on an mbarrier, and a bounded wait
// on that mbarrier.
#pragma once
#include <cuda_runtime.h>

namespace spect {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one thread: copy `bytes` from src0 (and src1 when given) into dst0 (dst1),
// completing on bar.  bytes and the addresses are multiples of 16.
__device__ __forceinline__ void tma_planes(unsigned long long* bar, float* dst0, const float* src0, float* dst1,
                                           const float* src1, unsigned bytes) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  const unsigned total = src1 ? 2u * bytes : bytes;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(total) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst0)),
               "l"(src0), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
  if (src1)
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst1)),
                 "l"(src1), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// bounded wait for the phase with the given parity; false when it gave up
// after `limit` polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit = 1 << 22) {
  for (int it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}


// one thread: expect `bytes` more on bar (call before the copies it covers)
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// copy `bytes` (a multiple of 16, 16-byte aligned ends) completing on bar
__device__ __forceinline__ void bulk_copy(unsigned long long* bar, void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace spect
