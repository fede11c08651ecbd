// Queue objects: the reference's host queue API (src/queue.h:86-115) over the rebuilt
// queue kinds, one C++ class per kind behind the opaque gpq_queue handle.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "host_common.h"
#include "queue_impl.h"

extern "C" {

gpq_status gpq_queue_create(const gpq_queue_config* cfg, gpq_queue** out) {
  GPQ_CHECK_ARG(cfg && out, "NULL argument");
  *out = nullptr;
  GPQ_CHECK_ARG(cfg->num_lps > 0 && cfg->num_lps <= (1u << 24), "num_lps must be in [1, 2^24]");
  std::unique_ptr<gpq::QueueImpl> impl;
  gpq_status st = gpq::make_queue(*cfg, impl);
  if (st != GPQ_OK) return st;
  gpq_queue* q = new (std::nothrow) gpq_queue();
  if (!q) return GPQ_ERR_NOMEM;
  q->impl = std::move(impl);
  q->cfg = *cfg;
  *out = q;
  return GPQ_OK;
}

gpq_status gpq_queue_destroy(gpq_queue* q) {
  if (!q) return GPQ_ERR_INVALID;
  delete q;
  return GPQ_OK;
}

gpq_status gpq_queue_insert(gpq_queue* q, const gpq_item* items, uint64_t n, int items_on_device, void* stream) {
  GPQ_CHECK_ARG(q && (items || n == 0), "NULL argument");
  if (n == 0) return GPQ_OK;
  return q->impl->insert(items, n, items_on_device != 0, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_pre(gpq_queue* q, void* stream) {
  GPQ_CHECK_ARG(q, "NULL queue");
  return q->impl->pre(gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_post(gpq_queue* q, void* stream) {
  GPQ_CHECK_ARG(q, "NULL queue");
  const cudaStream_t st = gpq::as_stream(stream, q->impl->stream());
  if (q->staged) {
    const gpq_status s = q->staged->flush(q->impl.get(), st);
    if (s != GPQ_OK) return s;
  }
  return q->impl->post(st);
}

gpq_status gpq_queue_post_init(gpq_queue* q, void* stream) { return gpq_queue_post(q, stream); }

gpq_status gpq_queue_get_min(gpq_queue* q, float* min_ts, void* stream) {
  GPQ_CHECK_ARG(q && min_ts, "NULL argument");
  return q->impl->get_min(min_ts, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_dequeue(gpq_queue* q, float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity,
                             uint64_t* n_out, void* stream) {
  GPQ_CHECK_ARG(q && n_out && (out || out_capacity == 0), "NULL argument");
  return q->impl->dequeue(bound, max_per_lp, out, out_capacity, n_out, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_length(gpq_queue* q, uint32_t lp, uint32_t* length, void* stream) {
  GPQ_CHECK_ARG(q && length, "NULL argument");
  GPQ_CHECK_ARG(lp < q->impl->num_lps(), "lp out of range");
  return q->impl->length(lp, length, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_clear(gpq_queue* q, uint32_t lp, void* stream) {
  GPQ_CHECK_ARG(q, "NULL queue");
  GPQ_CHECK_ARG(lp < q->impl->num_lps(), "lp out of range");
  return q->impl->clear(lp, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_dump(gpq_queue* q, uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                          void* stream) {
  GPQ_CHECK_ARG(q && n_out && (out || out_capacity == 0), "NULL argument");
  GPQ_CHECK_ARG(lp < q->impl->num_lps(), "lp out of range");
  return q->impl->dump(lp, out, out_capacity, n_out, gpq::as_stream(stream, q->impl->stream()));
}

gpq_status gpq_queue_counts(gpq_queue* q, uint64_t* enqueued, uint64_t* dequeued, void* stream) {
  GPQ_CHECK_ARG(q && enqueued && dequeued, "NULL argument");
  const gpq_status s = q->impl->counts(enqueued, dequeued, gpq::as_stream(stream, q->impl->stream()));
  if (s == GPQ_OK && q->staged) {  // heads staged and given back untouched are neither
    *enqueued -= q->staged->restaged();
    *dequeued -= q->staged->restaged();
  }
  return s;
}

gpq_status gpq_queue_device_view(gpq_queue* q, gpq_device_queue* out) {
  GPQ_CHECK_ARG(q && out, "NULL argument");
  if (q->staged) {
    q->staged->fill(out, q->cfg.kind);
    return GPQ_OK;
  }
  const gpq_status s = q->impl->device_view(out);
  if (s != GPQ_ERR_UNSUPPORTED) return s;
  std::unique_ptr<gpq::StagedView> v(new (std::nothrow) gpq::StagedView());
  if (!v) return GPQ_ERR_NOMEM;
  const gpq_status si = v->init(q->impl->num_lps(), q->cfg.insert_capacity, q->impl->stream());
  if (si != GPQ_OK) return si;
  q->staged = std::move(v);
  q->staged->fill(out, q->cfg.kind);
  return GPQ_OK;
}

gpq_status gpq_queue_set_bound(gpq_queue* q, float bound, void* stream) {
  GPQ_CHECK_ARG(q, "NULL argument");
  const cudaStream_t st = gpq::as_stream(stream, q->impl->stream());
  if (q->staged) return q->staged->set_bound(q->impl.get(), bound, st);
  const gpq_status s = q->impl->set_bound(bound, st);
  if (s == GPQ_ERR_UNSUPPORTED)
    gpq::set_last_error("gpq_queue_set_bound: take the device view (gpq_queue_device_view) of this queue first");
  return s;
}

}  // extern "C"
