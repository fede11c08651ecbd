// Host-side PHOLD configuration helpers shared by the engine entry points.
#pragma once

#include <algorithm>
#include <cmath>

#include "host_common.h"

namespace gpq {

inline gpq_phold_params phold_params_of(const gpq_phold_config& c) {
  gpq_phold_params p;
  p.seed = c.seed;
  p.num_lps = c.num_lps;
  p.dest_mode = c.dest_mode;
  p.ring_width = c.ring_width;
  p.ring_threshold = c.ring_threshold;
  p.lookahead = c.lookahead;
  p.end_time = c.end_time;
  return p;
}

inline bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }
inline uint32_t ilog2_ceil(uint32_t x) { uint32_t r = 0; while ((1u << r) < x) ++r; return r; }

// Checks that hold for every queue kind and loop mode.
inline gpq_status validate_phold_config(const gpq_phold_config* c) {
  GPQ_CHECK_ARG(c, "config is NULL");
  GPQ_CHECK_ARG(c->num_lps > 0 && c->num_lps <= (1u << 24), "num_lps must be in [1, 2^24]");
  GPQ_CHECK_ARG(c->events_per_lp > 0, "events_per_lp must be > 0");
  GPQ_CHECK_ARG((uint64_t)c->num_lps * c->events_per_lp <= 0xFFFFFFFFull, "num_lps * events_per_lp must fit 32-bit ids");
  GPQ_CHECK_ARG(c->lookahead > 0.f && c->lookahead < 1e30f, "lookahead must be positive and finite");
  GPQ_CHECK_ARG(c->end_time >= 0.f && c->end_time < 1e30f, "end_time must be finite and >= 0");
  GPQ_CHECK_ARG(c->dest_mode == GPQ_DEST_UNIFORM || c->dest_mode == GPQ_DEST_RING, "dest_mode");
  if (c->dest_mode == GPQ_DEST_RING)
    GPQ_CHECK_ARG(c->ring_width >= 1 && 2ull * c->ring_width < c->num_lps, "ring_width must satisfy 1 <= 2w < num_lps");
  GPQ_CHECK_ARG(c->loop_mode == GPQ_LOOP_PLAIN || c->loop_mode == GPQ_LOOP_PERSISTENT, "loop_mode");
  GPQ_CHECK_ARG(c->queue_kind <= GPQ_QUEUE_LSQ, "queue_kind");
  GPQ_CHECK_ARG(c->laq_mode <= 2 && (c->laq_mode == 0 || c->queue_kind == GPQ_QUEUE_LAQ),
                "laq_mode must be 0, or 1 or 2 with the local array queue");
  return GPQ_OK;
}

// Geometry of the bucketed local array queue (laq_mode 2): bucket width w chosen so that
// about 6 events sit in the front bucket of an LP (the pending events of an LP spread over
// about lookahead + 1 time units, the mean increment), but at least lookahead / 2.5 so
// that a window spans at most 4 buckets; NB buckets (a power of two) covering
// lookahead + 7 time units ahead of the window minimum (an increment beyond lookahead + 7
// has probability e^-7) and at least lookahead / w + 4 buckets, so that one window's
// bucket range never wraps; C slots per bucket, twice the expected front occupancy plus
// 4; spill lists of max(64, C) events.
struct LabGeometry {
  uint32_t nb_log2, c_log2, spill;
  float inv_w;
};

inline uint32_t next_pow2(double x) {
  uint32_t p = 1;
  while ((double)p < x && p < (1u << 30)) p <<= 1;
  return p;
}

inline gpq_status lab_geometry(const gpq_phold_config& c, LabGeometry* g) {
  const double la = c.lookahead, E = c.events_per_lp;
  double w = std::max(6.0 * (la + 1.0) / E, la / 2.5);
  double need = std::max(std::ceil((la + 7.0) / w), std::ceil(la / w) + 4.0);
  if (need > 1024.0) {
    w = std::max((la + 7.0) / 1024.0, la / 1020.0);
    need = 1024.0;
  }
  const uint32_t nb = std::max(16u, next_pow2(need));
  const double occ = E * w / (la + 1.0);
  const uint32_t cs = std::min(1024u, std::max(16u, next_pow2(std::ceil(2.0 * occ + 4.0))));
  g->nb_log2 = ilog2_ceil(nb);
  g->c_log2 = ilog2_ceil(cs);
  g->spill = std::max(64u, cs);
  g->inv_w = (float)(1.0 / w);
  GPQ_CHECK_ARG((double)c.lookahead * g->inv_w + 3.0 <= (double)nb,
                "bucketed local array queue: lookahead too wide for the bucket ring");
  GPQ_CHECK_ARG(((double)c.end_time + la + 20.0) * g->inv_w < 2147483648.0,
                "bucketed local array queue: end_time too large for the bucket width");
  return GPQ_OK;
}

// Fills the per-kind defaults (capacity 256, insert capacity 64, 256-thread CTAs,
// 8 lanes per LP; one lane for the splay queue) and checks them.
inline gpq_status normalize_queue_config(gpq_phold_config* c) {
  if (c->capacity == 0) c->capacity = 256;
  if (c->insert_capacity == 0) c->insert_capacity = 64;
  GPQ_CHECK_ARG(is_pow2(c->capacity) && c->capacity >= 32 && c->capacity <= (1u << 16),
                "capacity must be a power of two in [32, 65536]");
  if (c->queue_kind == GPQ_QUEUE_LSQ)
    GPQ_CHECK_ARG(c->capacity <= 32768, "splay queue capacity must be <= 32768");
  GPQ_CHECK_ARG(c->insert_capacity >= 1 && c->insert_capacity <= 1024, "insert_capacity must be in [1, 1024]");
  GPQ_CHECK_ARG(c->events_per_lp <= c->capacity, "events_per_lp must not exceed capacity");
  GPQ_CHECK_ARG(c->events_per_lp <= 8192, "events_per_lp must be <= 8192");
  if (c->block_threads == 0) c->block_threads = 256;
  GPQ_CHECK_ARG(c->block_threads % 32 == 0 && c->block_threads >= 32 && c->block_threads <= 1024,
                "block_threads must be a multiple of 32 in [32, 1024]");
  if (c->queue_kind == GPQ_QUEUE_LSQ) c->lanes_per_lp = 1;
  if (c->lanes_per_lp == 0) c->lanes_per_lp = 8;
  if (c->queue_kind == GPQ_QUEUE_LAQ)
    GPQ_CHECK_ARG(c->lanes_per_lp == 4 || c->lanes_per_lp == 8 || c->lanes_per_lp == 16 || c->lanes_per_lp == 32,
                  "lanes_per_lp must be 4, 8, 16 or 32 for the local array queue");
  if (c->queue_kind == GPQ_QUEUE_LHQ)
    GPQ_CHECK_ARG(c->lanes_per_lp == 1 || c->lanes_per_lp == 4 || c->lanes_per_lp == 8 || c->lanes_per_lp == 16 ||
                      c->lanes_per_lp == 32,
                  "lanes_per_lp must be 1, 4, 8, 16 or 32 for the local heap queue");
  return GPQ_OK;
}

// The LAQ entry points call this name.
inline gpq_status normalize_laq_config(gpq_phold_config* c) { return normalize_queue_config(c); }

// Halves the CTA size until the per-CTA merge scratch (one slice per lane group) fits
// `limit` bytes of shared memory.  Returns false if even one warp does not fit.
inline bool fit_block_to_smem(uint32_t* block, uint32_t group, size_t group_bytes, size_t limit) {
  while ((size_t)(*block / group) * group_bytes > limit && *block > 32) *block /= 2;
  if (*block < 32) *block = 32;
  return (size_t)(*block / group) * group_bytes <= limit;
}

}  // namespace gpq
