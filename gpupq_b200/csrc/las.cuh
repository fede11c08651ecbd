// Local array queue, selection form.
//
// Reference: src/local_array_queue.cu keeps each LP's events in a ring and orders them on
// queue_post, by insertion sort (d_insertion_sort, :254-299, the default
// _LAQ_INSERTION_SORT of src/config.h:96) or by appending and sorting the LP's run
// (d_sort + quicksort_seq, :300-319).  Both order every event at every post although a
// window only dequeues the events below its bound.
//
// This form orders only what a window dequeues: an LP's array is unordered; per window a
// group of G lanes streams through the array and the children of the previous window
// (independent, coalesced loads), keeps the keys of the safe events in shared memory,
// ranks them by key (their positions in the LP's sequence), stages them for the CTA-wide
// event pass, fills the holes they leave with the children that stay, appends the rest,
// and moves tail items into holes only when fewer children than holes remain.  The
// array uses the LAQ storage with the read counter fixed at 0 (wr = number of items), so
// population, results and the pending count are shared with the sorted form.
#pragma once

#include "laq.cuh"

static constexpr uint32_t kLasSafeCap = 64;  // safe events of one LP per window kept in shared memory

struct LasGroupSmem {
  uint64_t* key;   // [kLasSafeCap] keys of the LP's safe events
  uint32_t* src;   // [kLasSafeCap] where each is: array position (< n) or n + insert-buffer index
  uint32_t* hole;  // [kLasSafeCap] array positions to refill
};

__host__ __device__ inline size_t las_group_smem_bytes() {
  return ((size_t)kLasSafeCap * (8 + 4 + 4) + 15) & ~(size_t)15;
}

__device__ __forceinline__ LasGroupSmem las_group_smem(unsigned char* base) {
  LasGroupSmem s;
  s.key = reinterpret_cast<uint64_t*>(base);
  s.src = reinterpret_cast<uint32_t*>(s.key + kLasSafeCap);
  s.hole = s.src + kLasSafeCap;
  return s;
}

struct LasMeta {
  uint32_t k, n, count;
  unsigned long long csum, ohash;
};

__device__ __forceinline__ LasMeta las_load_meta(const PholdDev& d, const LaqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t prevb) {
  LasMeta m;
  m.k = ib.cnt[(size_t)prevb * d.L + lp];
  m.n = q.wr[lp];
  m.count = d.count[lp];
  m.csum = d.csum[lp];
  m.ohash = d.ohash[lp];
  return m;
}

__device__ __forceinline__ bool las_safe(const gpq_item& e, float bound, float T) { return e.ts < bound && e.ts < T; }

// One LP, one window s: select, rank and stage the safe events among the LP's array and
// the previous window's children, and rebuild the array from the rest.  Returns the
// minimum timestamp bits of what stays, min'ed with any child processed here.  All lanes
// of the group, convergent.
template <int G>
__device__ uint32_t las_lp_stage(const PholdDev& d, const LaqDev& q, const InsDev& ib, uint32_t lp, uint32_t slot,
                                 uint32_t s, float bound, const LasGroupSmem& sm, const PholdStage& st,
                                 const LaneGroup<G>& g, uint32_t* err_slot, const LasMeta& mt) {
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const uint32_t cap = 1u << q.cap_log2;
  gpq_item* arr = q.ring + ((size_t)lp << q.cap_log2);
  const float T = d.p.end_time;
  const uint32_t n = mt.n;
  const uint32_t k = mt.k < ib.ibc ? mt.k : ib.ibc;  // an overflow was flagged by the inserter
  const gpq_item* src = ib.buf + ((size_t)prevb * d.L + lp) * ib.ibc;
  const uint32_t lt = (1u << g.gl) - 1u;
  const uint32_t m = n + k;

  // 1. scan: safe keys into shared memory, the minimum of what stays
  uint32_t sc = 0, sb = 0, umin = kInfBits;
  for (uint32_t c0 = 0; c0 < m; c0 += G) {
    const uint32_t i = c0 + g.gl;
    const bool valid = i < m;
    gpq_item e;
    if (valid) e = i < n ? arr[i] : src[i - n];
    const bool safe = valid && las_safe(e, bound, T);
    const uint32_t b = g.ballot(safe);
    if (safe) {
      const uint32_t pos = sc + __popc(b & lt);
      if (pos < kLasSafeCap) {
        sm.key[pos] = gpq_lp_key(e);
        sm.src[pos] = i;
      }
    }
    sc += __popc(b);
    sb += __popc(g.ballot(safe && i < n));
    if (valid && !safe) umin = min(umin, gpq_f2u(e.ts));
  }
  umin = g.umin(umin);
  if (g.gl == 0) phold_stage_slot_init(st, slot, mt.count, mt.csum, mt.ohash);
  g.sync();
  const uint32_t ku = k - (sc - sb);  // children that stay
  uint32_t n2 = n - sb + ku;
  if (n2 > cap) {
    if (g.gl == 0) {
      gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL);
      atomicOr(err_slot, 1u);
    }
    n2 = cap;
  }
  uint32_t cmin = kInfBits;

  if (sc <= kLasSafeCap) {
    // 2. rank (position in the LP's sequence = number of smaller safe keys) and stage
    for (uint32_t j0 = 0; j0 < sc; j0 += G) {
      const uint32_t j = j0 + g.gl;
      const bool have = j < sc;
      gpq_item e;
      uint32_t r = 0;
      if (have) {
        const uint64_t kj = sm.key[j];
        for (uint32_t t = 0; t < sc; ++t) r += sm.key[t] < kj ? 1u : 0u;
        const uint32_t i = sm.src[j];
        e = i < n ? arr[i] : src[i - n];
      }
      const uint32_t c = sc - j0 < (uint32_t)G ? sc - j0 : (uint32_t)G;
      cmin = min(cmin, phold_stage_batch<G>(d, ib, st, g, e, have, r, c, slot, curb, err_slot));
    }
    g.sync();
    // 3. holes below the new end, in the order of the safe list
    uint32_t hl = 0;
    for (uint32_t j0 = 0; j0 < sc; j0 += G) {
      const uint32_t j = j0 + g.gl;
      const uint32_t p = j < sc ? sm.src[j] : ~0u;
      const bool low = p < n && p < n2;
      const uint32_t b = g.ballot(low);
      if (low) sm.hole[hl + __popc(b & lt)] = p;
      hl += __popc(b);
    }
    g.sync();
    // 4. children that stay: into the holes, then appended after the old end
    uint32_t ord = 0;
    for (uint32_t c0 = 0; c0 < k; c0 += G) {
      const uint32_t j = c0 + g.gl;
      gpq_item e;
      bool stay = false;
      if (j < k) {
        e = src[j];
        stay = !las_safe(e, bound, T);
      }
      const uint32_t b = g.ballot(stay);
      if (stay) {
        const uint32_t o = ord + __popc(b & lt);
        const uint32_t dst = o < hl ? sm.hole[o] : n + (o - hl);
        if (dst < cap) arr[dst] = e;
      }
      ord += __popc(b);
    }
    // 5. fewer children than holes: the tail's remaining items fill the other holes
    if (ord < hl) {
      uint32_t t = ord;
      for (uint32_t c0 = n2; c0 < n; c0 += G) {
        const uint32_t p = c0 + g.gl;
        gpq_item e;
        bool stay = false;
        if (p < n) {
          e = arr[p];
          stay = !las_safe(e, bound, T);
        }
        const uint32_t b = g.ballot(stay);
        if (stay) arr[sm.hole[t + __popc(b & lt)]] = e;
        t += __popc(b);
      }
    }
  } else {
    // rare: more safe events than the shared list holds -- rank by scanning, then rebuild
    // the array by a stable in-place compaction
    for (uint32_t c0 = 0; c0 < m; c0 += G) {
      const uint32_t i = c0 + g.gl;
      gpq_item e;
      bool safe = false;
      if (i < m) {
        e = i < n ? arr[i] : src[i - n];
        safe = las_safe(e, bound, T);
      }
      uint32_t r = 0;
      if (safe) {
        const uint64_t kj = gpq_lp_key(e);
        for (uint32_t t = 0; t < m; ++t) {
          const gpq_item o = t < n ? arr[t] : src[t - n];
          if (las_safe(o, bound, T) && gpq_lp_key(o) < kj) ++r;
        }
      }
      // stage the safe lanes of this chunk: compact them to lanes 0..c-1 by shuffles
      const uint32_t b = g.ballot(safe);
      const uint32_t c = __popc(b);
      gpq_item e2 = e;
      uint32_t r2 = r;
      {
        // the lane holding the c-th safe item of the chunk for destination lane gl
        uint32_t srcl = 0, seen = 0;
        for (uint32_t l = 0; l < (uint32_t)G; ++l)
          if ((b >> l) & 1u) {
            if (seen == g.gl) srcl = l;
            ++seen;
          }
        const uint32_t* w = reinterpret_cast<const uint32_t*>(&e);
        uint32_t v[4];
        for (int x = 0; x < 4; ++x) v[x] = g.shfl(w[x], srcl);
        e2.ts = gpq_u2f(v[0]);
        e2.lp = v[1];
        e2.id = v[2];
        e2.aux = v[3];
        r2 = g.shfl(r, srcl);
      }
      g.sync();
      cmin = min(cmin, phold_stage_batch<G>(d, ib, st, g, e2, g.gl < c, r2, c, slot, curb, err_slot));
    }
    g.sync();
    uint32_t kept = 0;
    for (uint32_t c0 = 0; c0 < n; c0 += G) {
      const uint32_t p = c0 + g.gl;
      gpq_item e;
      bool stay = false;
      if (p < n) {
        e = arr[p];
        stay = !las_safe(e, bound, T);
      }
      const uint32_t b = g.ballot(stay);
      g.sync();  // the chunk is read before any of it is written
      if (stay) arr[kept + __popc(b & lt)] = e;
      kept += __popc(b);
    }
    for (uint32_t c0 = 0; c0 < k; c0 += G) {
      const uint32_t j = c0 + g.gl;
      gpq_item e;
      bool stay = false;
      if (j < k) {
        e = src[j];
        stay = !las_safe(e, bound, T);
      }
      const uint32_t b = g.ballot(stay);
      const uint32_t dst = kept + __popc(b & lt);
      if (stay && dst < cap) arr[dst] = e;
      kept += __popc(b);
    }
  }
  g.sync();
  if (g.gl == 0) {
    st.lp[slot] = sc > 0 ? lp : ~0u;
    if (sc > 0) d.count[lp] = mt.count + sc;
    q.wr[lp] = n2;
    if (k) ib.cnt[(size_t)prevb * d.L + lp] = 0;
  }
  return min(umin, g.umin(cmin));
}

// The selection form as a PHOLD engine policy.
template <int G_>
struct LasPolicy {
  static constexpr int G = G_;
  using Dev = LaqDev;
  using Meta = LasMeta;
  using Smem = LasGroupSmem;
  __host__ __device__ static size_t group_smem_bytes(uint32_t) { return las_group_smem_bytes(); }
  __device__ static Smem smem(unsigned char* base, uint32_t) { return las_group_smem(base); }
  __device__ static Meta load_meta(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t prevb) {
    return las_load_meta(d, q, ib, lp, prevb);
  }
  __device__ static uint32_t stage_lp(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t slot,
                                      uint32_t s, float bound, const Smem& sm, const PholdStage& st,
                                      const LaneGroup<G>& g, uint32_t* err_slot, const Meta& mt) {
    return las_lp_stage<G>(d, q, ib, lp, slot, s, bound, sm, st, g, err_slot, mt);
  }
};
