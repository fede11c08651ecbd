// TEST INFRASTRUCTURE: the PHOLD handler of the drop-in models, written like the
// reference's handle_next_event (src/phold.cu:81-117): peek one event per LP, count it,
// set it done, insert its child.  Included by phold_model.cu and phold_legacy.cu.
#pragma once
#include "gpq.h"
#include "gpq/queue.cuh"

static __global__ void handle_next_event(gpq_phold_params p, uint32_t L, uint32_t* num_events, unsigned long long* csum,
                                         unsigned long long* ohash) {
  for (uint32_t idx = threadIdx.x + blockDim.x * blockIdx.x; idx < L; idx += blockDim.x * gridDim.x) {
    queue_item* ev = NULL;
    const int event_index = queue_peek(&ev, (int)idx);
    if (event_index != -1) {
      const gpq_item e = *ev;
      const uint32_t lp = e.lp;
      const uint64_t h = gpq_ev_hash(e.id, gpq_f2u(e.ts));
      csum[lp] += h;
      ohash[lp] += gpq_seq_hash(h, num_events[lp]);
      num_events[lp]++;
      const gpq_item child = gpq_phold_child(p, e);
      queue_set_done(event_index);
      const bool result = queue_insert(child);
      (void)result;  // a full buffer is reported by the next gpq_queue_post
    }
  }
}

static inline gpq_phold_params dropin_params(const gpq_phold_config* cfg) {
  gpq_phold_params p = {};
  p.seed = cfg->seed;
  p.num_lps = cfg->num_lps;
  p.dest_mode = cfg->dest_mode;
  p.ring_width = cfg->ring_width;
  p.ring_threshold = cfg->ring_threshold;
  p.lookahead = cfg->lookahead;
  p.end_time = cfg->end_time;
  return p;
}
