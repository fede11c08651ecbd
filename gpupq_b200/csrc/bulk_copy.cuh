// One-dimensional TMA bulk copies (cp.async.bulk, sm_90+) from this GPU's global memory
// into the issuing CTA's shared memory, completed through an mbarrier.
//
// A CTA stages an input tile with one instruction from one thread instead of a load per
// thread: the copy engine moves the bytes while the threads do other work (digit scans,
// split reads), and the threads wait on the mbarrier's phase.  Rules kept here: source and
// destination 16-byte aligned, sizes multiples of 16 bytes (queue items are 16 bytes), at
// most 1 MiB of transactions per phase; no cluster multicast (every source is this GPU's
// own memory and every copy lands in the issuing CTA only).  Every wait is bounded: a
// wait that runs out records GPQ_ERR_TIMEOUT, waits once more (bounded) for the copies in
// flight so that none still writes the CTA's shared memory when it returns, and reports
// failure so that the caller skips the tile.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initializes an mbarrier expecting one arrival (one thread), visible to the async proxy.
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The issuing thread's arrival, announcing `bytes` of transactions for this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Copies `bytes` (a multiple of 16, > 0) from global `src` to shared `dst` (both 16-byte
// aligned); completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return done != 0u;
}

static constexpr uint32_t kBulkWaitLimit = 1u << 24;  // try_wait polls (each may suspend briefly)

// All threads of the CTA: waits for phase `phase` of `bar`.  Returns false after recording
// GPQ_ERR_TIMEOUT in *err (if given) when the copies did not complete within the limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t* err) {
  for (uint32_t i = 0; i < kBulkWaitLimit; ++i)
    if (mbar_try_wait(bar, phase)) return true;
  if (err) gpq_set_error(err, GPQ_ERR_TIMEOUT);
  for (uint32_t i = 0; i < kBulkWaitLimit; ++i)  // let copies in flight land before the CTA moves on
    if (mbar_try_wait(bar, phase)) break;
  return false;
}
