/*
 * gpq/legacy.h -- the reference's host queue API (src/queue.h:86-115) over one queue
 * owned by the library, for host code written against the reference:
 *
 *   queue_init()        create the queue configured by gpq_legacy_configure (the
 *                       reference sizes it from config.h) and bind it for this
 *                       translation unit's model kernels (include/gpq/queue.cuh);
 *   queue_post_init()   merge the initial events (after each populate chunk);
 *   queue_pre()         set the window bound: last queue_get_min_ts() + lookahead, capped
 *                       at the end time (the reference's peek compares with
 *                       global_min + LOOKAHEAD, src/local_array_queue.cu:760-779);
 *   queue_post()        merge the items the model inserted;
 *   queue_get_min_ts()  smallest pending timestamp (+inf when empty), cached until the
 *                       next queue_post as in src/local_array_queue.cu:453-478;
 *   queue_finish()      destroy the queue;
 *   get_enqueue_count() / get_dequeue_count()   items inserted / removed since queue_init;
 *   queue_check_phold() nothing to check (the reference's local array queue does none).
 *
 * The reference exits on errors; these functions record the first failing status,
 * readable with gpq_legacy_status() (and gpq_last_error()).  Timestamps are float32
 * (the reference's PHOLD uses integer timestamps).  A translation unit with model
 * kernels other than the one that called queue_init binds the queue itself with
 * gpq_queue_bind(gpq_legacy_queue()).  CUDA translation units only.
 */
#ifndef GPQ_LEGACY_H
#define GPQ_LEGACY_H

#include "gpq.h"
#include "gpq/queue.cuh"

static inline void queue_init(void) {
  gpq_queue* q = NULL;
  if (gpq_legacy_init(&q) == GPQ_OK) gpq_queue_bind(q);
}
static inline void queue_post_init(void) { gpq_legacy_post(); }
static inline void queue_pre(void) { gpq_legacy_pre(); }
static inline void queue_post(void) { gpq_legacy_post(); }
static inline float queue_get_min_ts(void) { return gpq_legacy_get_min_ts(); }
static inline void queue_finish(void) { gpq_legacy_finish(); }
static inline int get_enqueue_count(void) {
  uint64_t e = 0, d = 0;
  gpq_legacy_counts(&e, &d);
  return (int)e;
}
static inline int get_dequeue_count(void) {
  uint64_t e = 0, d = 0;
  gpq_legacy_counts(&e, &d);
  return (int)d;
}
static inline void queue_check_phold(void) {}

#endif /* GPQ_LEGACY_H */
