// The reference's host queue API over one library-owned queue (include/gpq/legacy.h).
//
// The reference's host code drives one global queue chosen at compile time
// (src/queue.h:86-115: queue_init, queue_post_init, queue_pre, queue_post,
// queue_get_min_ts, queue_finish, get_enqueue_count, get_dequeue_count); these functions
// keep that shape over a gpq_queue created from the configuration set by
// gpq_legacy_configure.  The window bound of queue_peek is set by queue_pre from the last
// minimum read by queue_get_min_ts plus the configured lookahead, in the order des_run
// calls them (src/des.cu:179-214: get_min, pre, model step, post).
#include <mutex>

#include "host_common.h"
#include "queue_impl.h"

namespace {

struct Legacy {
  std::mutex m;
  gpq_queue_config cfg{};
  bool configured = false;
  float lookahead = 1.0f;
  float end_time = 0.f;
  float last_min = 0.f;
  bool have_min = false;
  gpq_queue* q = nullptr;
  gpq_status sticky = GPQ_OK;
};

Legacy& state() {
  static Legacy s;
  return s;
}

gpq_status keep(Legacy& s, gpq_status st) {
  if (st != GPQ_OK && s.sticky == GPQ_OK) s.sticky = st;
  return st;
}

}  // namespace

extern "C" {

gpq_status gpq_legacy_configure(const gpq_queue_config* cfg, float lookahead, float end_time) {
  GPQ_CHECK_ARG(cfg, "NULL config");
  GPQ_CHECK_ARG(lookahead > 0.f, "lookahead must be positive");
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  s.cfg = *cfg;
  s.lookahead = lookahead;
  s.end_time = end_time;
  s.configured = true;
  return GPQ_OK;
}

gpq_status gpq_legacy_init(gpq_queue** out) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  if (!s.configured) {
    gpq::set_last_error("queue_init: call gpq_legacy_configure first");
    return keep(s, GPQ_ERR_INVALID);
  }
  if (s.q) gpq_queue_destroy(s.q);
  s.q = nullptr;
  s.sticky = GPQ_OK;
  s.have_min = false;
  const gpq_status st = gpq_queue_create(&s.cfg, &s.q);
  if (out) *out = s.q;
  return keep(s, st);
}

gpq_queue* gpq_legacy_queue(void) { return state().q; }

gpq_status gpq_legacy_post(void) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  if (!s.q) return keep(s, GPQ_ERR_NOT_READY);
  s.have_min = false;
  return keep(s, gpq_queue_post(s.q, nullptr));
}

gpq_status gpq_legacy_pre(void) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  if (!s.q) return keep(s, GPQ_ERR_NOT_READY);
  gpq_status st = gpq_queue_pre(s.q, nullptr);
  if (st != GPQ_OK) return keep(s, st);
  float m = s.last_min;
  if (!s.have_min) {
    st = gpq_queue_get_min(s.q, &m, nullptr);
    if (st != GPQ_OK) return keep(s, st);
  }
  float bound = m + s.lookahead;                            // global_min + LOOKAHEAD
  if (s.end_time > 0.f && s.end_time < bound) bound = s.end_time;  // and ts < end time
  return keep(s, gpq_queue_set_bound(s.q, bound, nullptr));
}

float gpq_legacy_get_min_ts(void) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  float m = __builtin_inff();
  if (!s.q) {
    keep(s, GPQ_ERR_NOT_READY);
    return m;
  }
  if (s.have_min) return s.last_min;  // cached until the next post (src/local_array_queue.cu:453-478)
  if (keep(s, gpq_queue_get_min(s.q, &m, nullptr)) == GPQ_OK) {
    s.last_min = m;
    s.have_min = true;
  }
  return m;
}

gpq_status gpq_legacy_counts(uint64_t* enqueued, uint64_t* dequeued) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  if (!s.q) return keep(s, GPQ_ERR_NOT_READY);
  return keep(s, gpq_queue_counts(s.q, enqueued, dequeued, nullptr));
}

gpq_status gpq_legacy_finish(void) {
  Legacy& s = state();
  std::lock_guard<std::mutex> lk(s.m);
  if (s.q) gpq_queue_destroy(s.q);
  s.q = nullptr;
  s.have_min = false;
  return GPQ_OK;
}

gpq_status gpq_legacy_status(void) { return state().sticky; }

}  // extern "C"
