// Bulk asynchronous global -> shared copies (cp.async.bulk, sm_90+) completed
// through an mbarrier transaction count. No cluster multicast is used.
#pragma once

#include <cstdint>

namespace mpmb200 {

constexpr int kErrWaitTimeout = 4;  // device error flag: a bounded wait gave up

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the barrier initialisation visible to the async proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders earlier generic-proxy accesses to shared memory before later
// async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// bytes: multiple of 16; src and dst 16-byte aligned.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Per-thread prefetch of one line of global memory into L2.
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Default poll limit of a bounded wait (a bulk copy lands within a few
// microseconds; 2^24 polls are far longer).
constexpr uint32_t kWaitPolls = 1u << 24;

// Waits for the barrier phase with an iteration limit; on timeout sets
// kErrWaitTimeout in *err and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  uint32_t limit = kWaitPolls) {
  for (uint32_t it = 0; it < limit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, kErrWaitTimeout);
  return false;
}

}  // namespace mpmb200
