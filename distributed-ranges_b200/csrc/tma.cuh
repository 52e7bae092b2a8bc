// tma.cuh -- mbarrier and bulk-copy (TMA, non-tensor) helpers for sm_100a.
//
// Every wait is bounded: mbar_wait() gives up after kWaitNs nanoseconds of
// %globaltimer and returns false; kernels then record DRB_ERR_TIMEOUT in a
// device error word and leave their loops instead of hanging the GPU.
// Every copy here lands in the issuing CTA's own shared memory only (no
// cluster-wide delivery).
#pragma once

#include <cstdint>

namespace drb::tma {

constexpr uint64_t kWaitNs = 1000000000ull; // 1 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

// Makes the initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity to complete; false once
// `limit_ns` nanoseconds have passed without it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          uint64_t limit_ns = kWaitNs) {
  if (mbar_try_wait(bar, parity))
    return true;
  const uint64_t t0 = globaltimer();
  for (;;) {
    for (int i = 0; i < 64; i++)
      if (mbar_try_wait(bar, parity))
        return true;
    if (globaltimer() - t0 > limit_ns)
      return false;
  }
}

// As mbar_wait, but also gives up (returning 1) as soon as *stop or *stop2
// becomes non-zero; 0 = the phase completed, 2 = the limit ran out.
__device__ __forceinline__ int mbar_wait_or_stop(uint64_t *bar, uint32_t parity,
                                                 uint64_t limit_ns,
                                                 const volatile int *stop,
                                                 const volatile int *stop2) {
  if (mbar_try_wait(bar, parity))
    return 0;
  const uint64_t t0 = globaltimer();
  for (;;) {
    for (int i = 0; i < 64; i++)
      if (mbar_try_wait(bar, parity))
        return 0;
    if (*stop || *stop2)
      return 1;
    if (globaltimer() - t0 > limit_ns)
      return 2;
  }
}

// Bulk copy global -> shared (this CTA), completion counted in bytes on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar,
                                         uint64_t policy) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::"
               "bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
               : "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) writes to the same addresses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Named barrier over `nthreads` threads (a multiple of 32), id 1..15.
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Named barrier that also ORs a predicate across the participants.
__device__ __forceinline__ bool named_sync_or(int id, int nthreads, bool pred) {
  uint32_t out;
  asm volatile("{\n\t.reg .pred p, q;\n\t"
               "setp.ne.u32 p, %1, 0;\n\t"
               "bar.red.or.pred q, %2, %3, p;\n\t"
               "selp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(out)
               : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
               : "memory");
  return out != 0;
}

} // namespace drb::tma
