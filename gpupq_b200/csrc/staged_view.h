// Device-side access (include/gpq/queue.cuh) to the queue kinds whose items do not sit in
// per-LP arrays: the global array queue, the heap queue and the local splay queue.
//
// The reference's model kernels see one item per LP per step through queue_peek: the
// global array queue marks the earliest safe item of every LP (mark_safe_events,
// src/global_array_queue.cu:147-179), the heap queue hands out its root's safe items.
// Here gpq_queue_set_bound stages, for every LP, its earliest item below the bound in a
// per-LP head slot (the kind's own dequeue with at most one item per LP); queue_peek
// returns that slot and queue_set_done marks it taken.  gpq_queue_post then gives back
// the heads the model did not take, together with the items the model inserted (per-LP
// insert buffers, as for the per-LP kinds), before the kind's own post.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "gpq.h"

namespace gpq {

class QueueImpl;

class StagedView {
 public:
  ~StagedView();
  gpq_status init(uint32_t num_lps, uint32_t insert_capacity, cudaStream_t st);
  void fill(gpq_device_queue* v, uint32_t kind) const;
  // Stages each LP's earliest item with ts < bound (and sets the bound queue_peek uses).
  gpq_status set_bound(QueueImpl* q, float bound, cudaStream_t st);
  // Returns untaken heads and the inserted items to the queue (before its post); reports
  // an insert-buffer overflow or an unsupported device call made since the last flush.
  gpq_status flush(QueueImpl* q, cudaStream_t st);
  // Heads staged and given back unchanged: removed from the queue's counts.
  uint64_t restaged() const { return restaged_; }

 private:
  uint32_t L_ = 0, ibc_ = 0;
  gpq_item* head_ = nullptr;      // [L] ts = +inf: no head
  uint32_t* taken_ = nullptr;     // [L]
  gpq_item* ibuf_ = nullptr;      // [L][ibc]
  uint32_t* icnt_ = nullptr;      // [L]
  float* bound_ = nullptr;
  unsigned long long* ctr_ = nullptr;  // [0] enqueued [1] dequeued (device-side tallies)
  uint32_t* words_ = nullptr;     // [0] error word [1] items to flush [2] heads given back
  gpq_item* out_ = nullptr;       // [L * ibc + L] flush buffer
  std::vector<gpq_item> h_out_, h_head_;
  uint32_t* h_words_ = nullptr;   // pinned
  uint64_t restaged_ = 0;
};

}  // namespace gpq
