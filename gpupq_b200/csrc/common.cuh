// Device-side helpers shared by the gpupq_b200 kernels: error words, warp
// reductions, and a bounded grid barrier for persistent launches.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gpq.h"

#define GPQ_FULL_MASK 0xffffffffu

static constexpr uint32_t kInfBits = 0x7f800000u;  // +inf as float bits

// The first error code wins; later ones are dropped.
__device__ __forceinline__ void gpq_set_error(uint32_t* err, uint32_t code) {
  atomicCAS(err, 0u, code);
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GPQ_FULL_MASK, v, o);
  return v;
}

__device__ __forceinline__ uint32_t warp_min_u32(uint32_t v) {
  return __reduce_min_sync(GPQ_FULL_MASK, v);
}

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
  return __reduce_add_sync(GPQ_FULL_MASK, v);
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a cooperative (co-resident) launch.  `ctr` counts arrivals
// and is never reset during a launch: barrier number b completes when the counter
// reaches nblocks * (b + 1).  Thread 0 arrives with a release reduction (the CTA's
// writes, ordered before it by the block barrier, become visible at GPU scope before the
// arrival; no wait for a returned value) and polls with acquire loads; the block barrier
// after the poll orders every thread's later reads after the other CTAs' writes.  The wait
// is bounded by `spin_limit` polls; on timeout the error word gets GPQ_ERR_TIMEOUT and the
// function returns false, so no block ever spins forever.
__device__ __forceinline__ bool grid_barrier(unsigned long long* ctr, unsigned long long target,
                                             uint64_t spin_limit, uint32_t* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(ctr) : "memory");
    uint64_t it = 0;
    while (ld_acquire_u64(ctr) < target) {
      if (++it > spin_limit) {
        gpq_set_error(err, GPQ_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
  return ok != 0;
}

// grid_barrier whose arrival also publishes a CTA-wide minimum: the CTA's threads min'ed
// their values into the shared word *smin before the call; thread 0 folds it into *gmin
// with one atomicMin (released with the arrival) and resets *smin to all ones.
__device__ __forceinline__ bool grid_barrier_min(unsigned long long* ctr, unsigned long long target,
                                                 uint64_t spin_limit, uint32_t* err, uint32_t* smin, uint32_t* gmin) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const uint32_t v = *smin;
    *smin = 0xffffffffu;
    if (v != 0xffffffffu) atomicMin(gmin, v);
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(ctr) : "memory");
    uint64_t it = 0;
    while (ld_acquire_u64(ctr) < target) {
      if (++it > spin_limit) {
        gpq_set_error(err, GPQ_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
  return ok != 0;
}

// Block-wide min of a u32 (all threads call; result valid in all threads).
__device__ __forceinline__ uint32_t block_min_u32(uint32_t v, uint32_t* scratch /* >= 32 */) {
  v = warp_min_u32(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  uint32_t r = (lane < nw) ? scratch[lane] : kInfBits;
  if (warp == 0) {
    r = warp_min_u32(r);
    if (lane == 0) scratch[0] = r;
  }
  __syncthreads();
  r = scratch[0];
  __syncthreads();
  return r;
}
