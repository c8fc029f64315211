// Bulk asynchronous global -> shared copies completing on an mbarrier
// (sm_90+ cp.async.bulk), with a bounded wait.
//
// Every copy must start and end on 16-byte boundaries (addresses and size).
// A wait gives up after a bounded number of polls (kMaxWaitTries unless the
// caller passes fewer) and returns false, so the caller can record the
// failure; nothing here spins without limit.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qpb {

inline constexpr int kMaxWaitTries = 1 << 22;

__device__ __forceinline__ std::uint32_t smem_addr(const void* p) {
  return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(std::uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  // make the initialised barrier visible to the asynchronous (bulk copy) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives once on the barrier and raises its expected transaction bytes.
__device__ __forceinline__ void mbar_arrive_expect_tx(std::uint64_t* bar, unsigned bytes) {
  asm volatile(
      "{\n\t.reg .b64 state;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// Copies `bytes` (a multiple of 16) from global `src` to shared `dst`; both
// 16-byte aligned. Completion is signalled on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         std::uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Copies `bytes` (a multiple of 16) from shared `src` to global `dst`, both
// 16-byte aligned, as part of this thread's current bulk group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Blocks until this thread's committed bulk stores have finished reading
// shared memory (after which it may be reused or the CTA may exit).
__device__ __forceinline__ void bulk_wait_reads() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later
// asynchronous-proxy (bulk copy) reads of them.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, unsigned parity) {
  std::uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity` of `bar` to complete; false after `tries`
// unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(std::uint64_t* bar, unsigned parity,
                                          int tries = kMaxWaitTries) {
  for (int i = 0; i < tries; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  return false;
}

}  // namespace qpb
