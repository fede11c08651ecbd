// Internal interface of the queue objects behind the gpq_queue handle.  One class per
// queue kind implements the reference's host queue functions (src/queue.h:86-115);
// the device-side operations are kernels over the kind's own layout.
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "gpq.h"
#include "staged_view.h"

namespace gpq {

class QueueImpl {
 public:
  virtual ~QueueImpl() = default;
  virtual uint32_t num_lps() const = 0;
  virtual cudaStream_t stream() const = 0;
  virtual gpq_status insert(const gpq_item* items, uint64_t n, bool on_device, cudaStream_t st) = 0;
  virtual gpq_status pre(cudaStream_t) { return GPQ_OK; }
  virtual gpq_status post(cudaStream_t st) = 0;
  virtual gpq_status get_min(float* min_ts, cudaStream_t st) = 0;
  virtual gpq_status dequeue(float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                             cudaStream_t st) = 0;
  virtual gpq_status length(uint32_t lp, uint32_t* len, cudaStream_t st) = 0;
  virtual gpq_status clear(uint32_t lp, cudaStream_t st) = 0;
  virtual gpq_status dump(uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out, cudaStream_t st) = 0;
  virtual gpq_status counts(uint64_t* enqueued, uint64_t* dequeued, cudaStream_t st) = 0;
  // Device-side access for model kernels (include/gpq/queue.cuh) over the kind's own
  // per-LP arrays (local array and local heap queues); the other kinds are reached through
  // staged per-LP heads (staged_view.h).
  virtual gpq_status device_view(gpq_device_queue*) { return GPQ_ERR_UNSUPPORTED; }
  virtual gpq_status set_bound(float, cudaStream_t) { return GPQ_ERR_UNSUPPORTED; }
};

gpq_status make_laq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out);
gpq_status make_lpq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out);
gpq_status make_gaq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out);
gpq_status make_hq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out);
gpq_status make_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out);

}  // namespace gpq

struct gpq_queue {
  std::unique_ptr<gpq::QueueImpl> impl;
  gpq_queue_config cfg{};
  std::unique_ptr<gpq::StagedView> staged;  // device-side access for GAQ, HQ and LSQ
};
