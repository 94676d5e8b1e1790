// ffvgpu_async.cuh -- shared-memory mbarriers and bulk copies (global ->
// shared, and global -> L2 prefetch) for the persistent kernels, sm_100a.
//
// Every wait is bounded in time: mbar_wait gives up after the caller's limit
// (a pool setting, DEFAULT_WAIT_NS unless changed), records the caller's role
// in an abort word and returns false, so a kernel whose copy never lands
// reports an error instead of spinning.  After an abort, mbar_drain waits for
// copies already issued into the CTA's shared memory; its bound (DRAIN_NS)
// does not depend on the pool setting, so a short wait limit never lets a
// CTA exit while a copy is still landing in its shared memory.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ffvgpu_layout.h"

namespace ffvgpu {
namespace async {

constexpr uint64_t DRAIN_NS = 2000000000ull;         // a post-abort drain gives up after 2 s
// SolveState::timeout_where bit of a drain that gave up: a copy was still in
// flight when the CTA left (never seen: copies from device memory complete
// in microseconds)
constexpr int ROLE_DRAIN = 16;

__device__ __forceinline__ uint32_t sa(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa(b)), "r"(count) : "memory");
}
// Makes initialised mbarriers visible to the async proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait; false when it gave up (recording its role) or another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag,
                                          int role, uint64_t limit_ns) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = now_ns();
  for (;;) {
    if (mbar_try_wait(b, parity)) return true;
    if (*abort_flag) return false;
    if (now_ns() - t0 > limit_ns) {
      atomicOr((int*)abort_flag, role);
      return false;
    }
  }
}
// Waits, bounded by DRAIN_NS and regardless of any abort, until the phase
// with the given parity has completed (every copy armed on it has landed);
// false if it gave up.
__device__ __forceinline__ bool mbar_drain(uint64_t* b, uint32_t parity) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = now_ns();
  for (;;) {
    if (mbar_try_wait(b, parity)) return true;
    if (now_ns() - t0 > DRAIN_NS) return false;
  }
}
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          sa(dst)),
      "l"(src), "r"(bytes), "r"(sa(bar))
      : "memory");
}
// Hint: bring [src, src + bytes) into L2 (16-byte aligned, multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// Orders this thread's reads of shared memory before later async-proxy
// (TMA) writes to it.  Buffers refilled by TMA must be released only after
// it: without it a refill can overwrite data a lane is still reading.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace async
}  // namespace ffvgpu
