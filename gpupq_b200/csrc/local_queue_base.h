// Shared host/device plumbing of the per-LP queue objects (LAQ, LHQ, LSQ): an
// insert buffer per LP filled by queue_insert and drained by queue_post, device
// counters for get_enqueue_count / get_dequeue_count, and a sticky error word.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "host_common.h"
#include "queue_impl.h"

namespace gpq {

struct LocalQueueCounters {
  unsigned long long enqueued;
  unsigned long long dequeued;
  uint32_t err;
  uint32_t min_bits;
};

// queue_insert for a batch (src/local_array_queue.cu:486-513): reserve a slot in the
// item's LP buffer with atomicAdd; a full buffer records GPQ_ERR_INSERT_FULL.
__global__ void lq_insert_kernel(const gpq_item* __restrict__ items, uint64_t n, uint32_t L, gpq_item* ibuf,
                                 uint32_t* icnt, uint32_t ibc, LocalQueueCounters* ctr);

// Per-LP exclusive prefix sum of counts (single block; used by the dequeue paths).
__global__ void lq_exclusive_scan_kernel(const uint32_t* __restrict__ cnt, uint32_t L, unsigned long long* offs);

class LocalQueueBase : public QueueImpl {
 public:
  ~LocalQueueBase() override;
  uint32_t num_lps() const override { return L_; }
  cudaStream_t stream() const override { return own_; }
  gpq_status insert(const gpq_item* items, uint64_t n, bool on_device, cudaStream_t st) override;
  gpq_status counts(uint64_t* enqueued, uint64_t* dequeued, cudaStream_t st) override;

 protected:
  gpq_status init_base(uint32_t L, uint32_t ibc);
  // Reads and clears the sticky error word; returns it as a status.
  gpq_status take_error(cudaStream_t st);
  // Device exclusive scan of per-LP counts into offs_ (L+1 entries; offs_[L] = total).
  gpq_status scan_counts(const uint32_t* cnt, uint64_t* total, cudaStream_t st);

  uint32_t L_ = 0;
  uint32_t ibc_ = 0;
  cudaStream_t own_ = nullptr;
  gpq_item* ibuf_ = nullptr;  // [L][ibc]
  uint32_t* icnt_ = nullptr;  // [L]
  LocalQueueCounters* ctr_ = nullptr;
  LocalQueueCounters* h_ctr_ = nullptr;  // pinned
  gpq_item* staging_ = nullptr;
  uint64_t staging_n_ = 0;
  uint32_t* dq_cnt_ = nullptr;             // [L] per-LP dequeue counts
  unsigned long long* dq_off_ = nullptr;   // [L + 1]
  gpq_item* dq_out_ = nullptr;
  uint64_t dq_out_n_ = 0;
};

}  // namespace gpq
