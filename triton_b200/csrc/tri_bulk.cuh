// tri_bulk.cuh -- bulk asynchronous copies (the TMA engine's untiled form,
// cp.async.bulk) from global into shared memory, completing on an mbarrier.
// No cluster multicast: every copy lands in the issuing CTA's own memory.
#pragma once

#include <stdint.h>

namespace tri {

// Iterations of mbarrier.try_wait before a wait gives up (each try may
// suspend the thread for a while; the limit bounds a wait to well under a
// minute even if a copy never completed).
constexpr uint32_t kSpinLimit = 1u << 24;
// Device-side status codes (DevClock::status).
constexpr int32_t kStatusStageTimeout = 1;
constexpr int32_t kStatusTestWait = 2;  // the wait of the test hook gave up (tri_domain_set_wait_test)
constexpr int32_t kStatusStepWait = 3;  // a wait of the single-launch batch kernel gave up (k_batch_steps)
// Polls of one dependency wait of k_batch_steps (with 128 ns sleeps: about
// 2 s, where the dependencies it waits for take micro- to milliseconds).
constexpr uint32_t kStepWaitPolls = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Adds 'bytes' to the transaction count the current phase waits for.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
      : "memory");
}

// One bounded wait for the phase with the given parity: at most 'limit'
// polls; true once complete, false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kSpinLimit) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < limit; ++it) {
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

// Arrives on 'bar' and adds 'bytes' to the transaction count of its phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// Invalidates an mbarrier whose phases are all complete, so its shared
// memory can hold a new one (a block that stages several tiles in turn).
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Orders this thread's view of global memory (writes other blocks made
// visible to it by an acquire) before its later bulk copies, which read
// through the async proxy.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Acquire load of a counter other blocks increment (gpu scope).
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Copies 'bytes' (a multiple of 16) from global 'src' (16-byte aligned) to
// shared 'dst' (16-byte aligned); completion is counted on 'bar'.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace tri
