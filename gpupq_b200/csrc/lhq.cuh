// Local heap queue (LHQ), B200 form.
//
// Reference: src/local_heap_queue.cu.  Each LP owns a binary heap in an array of
// FEL_SIZE items (fel[lp * FEL_SIZE + i], item_count[lp]); queue_insert appends behind
// the heap with atomicAdd (:398-419), queue_post restores the heap with copy_last
// (move the last item to the root after a dequeue, :128-145), heapify_down (:249-267)
// and heapify_up for the new items (:216-233), one thread per LP; queue_peek returns
// the root inside the window (:430-447).
//
// Here the heap is D-ary with D = max(G, 4) children per node stored contiguously, so
// a lane group reads all children of a node with one coalesced access and picks the
// smallest with a shuffle reduction; sift-down therefore takes log_D(n) group steps.
// Children of window s-1 are pushed (sift-up) before the window's safe events are
// popped in key order and staged for the CTA-wide event pass.
#pragma once

#include "phold_common.cuh"

static constexpr uint32_t kLhqNil = 0xffffffffu;

struct LhqDev {
  gpq_item* items;  // num_lps << cap_log2 items; heap of LP l at items[l << cap_log2]
  uint32_t* size;   // per-LP heap size
  uint32_t cap_log2;
};

struct LhqMeta {
  uint32_t k, n, count;
  unsigned long long csum, ohash;
};

__device__ __forceinline__ LhqMeta lhq_load_meta(const PholdDev& d, const LhqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t prevb) {
  LhqMeta m;
  m.k = ib.cnt[(size_t)prevb * d.L + lp];
  m.n = q.size[lp];
  m.count = d.count[lp];
  m.csum = d.csum[lp];
  m.ohash = d.ohash[lp];
  return m;
}

// Push x into the heap h of n items (sift-up; one lane).
template <int D>
__device__ __forceinline__ void lhq_push(gpq_item* h, uint32_t n, const gpq_item x) {
  const uint64_t kx = gpq_lp_key(x);
  uint32_t pos = n;
  while (pos > 0) {
    const uint32_t parent = (pos - 1) / D;
    const gpq_item p = h[parent];
    if (gpq_lp_key(p) <= kx) break;
    h[pos] = p;
    pos = parent;
  }
  h[pos] = x;
}

// Remove the root of the heap h of n > 0 items (sift-down of the last item with the
// group reading the D children of a node together).  All lanes of the group.
template <int G, int D>
__device__ __forceinline__ void lhq_pop(gpq_item* h, uint32_t n, const LaneGroup<G>& g) {
  const uint32_t last = n - 1;
  if (last == 0) return;
  const gpq_item x = h[last];
  const uint64_t kx = gpq_lp_key(x);
  uint32_t pos = 0;
  for (;;) {
    const uint32_t fc = pos * D + 1;
    if (fc >= last) break;
    uint64_t best = ~0ull;
    uint32_t bidx = kLhqNil;
    gpq_item bit;
#pragma unroll
    for (int j = 0; j < D / G; ++j) {
      const uint32_t c = fc + g.gl + (uint32_t)j * G;
      if (c < last) {
        const gpq_item it = h[c];
        const uint64_t kc = gpq_lp_key(it);
        if (kc < best) { best = kc; bidx = c; bit = it; }
      }
    }
    uint32_t who;
    const uint64_t kmin = g.kmin(best, &who);
    if (kmin >= kx) break;
    const uint32_t cidx = g.shfl(bidx, who);
    if (g.gl == who) h[pos] = bit;
    pos = cidx;
    g.sync();
  }
  if (g.gl == 0) h[pos] = x;
  g.sync();
}

// One LP, one window s, first pass: push the children of window s-1, then pop every
// event with ts < bound and ts < end_time in key order and stage it.  Returns the new
// root's timestamp bits, min'ed with any child processed here.
template <int G>
__device__ __forceinline__ uint32_t lhq_lp_stage(const PholdDev& d, const LhqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t slot, uint32_t s, float bound, const PholdStage& st,
                                                 const LaneGroup<G>& g, uint32_t* err_slot, const LhqMeta& mt) {
  constexpr int D = G >= 4 ? G : 4;
  const uint32_t L = d.L;
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const uint32_t cap = 1u << q.cap_log2;
  gpq_item* h = q.items + ((size_t)lp << q.cap_log2);
  const float T = d.p.end_time;
  uint32_t n = mt.n;
  uint32_t k = mt.k;
  if (k > 0) {
    if (k > ib.ibc) k = ib.ibc;
    if (n + k > cap) {
      if (g.gl == 0) { gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL); atomicOr(err_slot, 1u); }
      k = cap - n;
    }
    const gpq_item* src = ib.buf + ((size_t)prevb * L + lp) * ib.ibc;
    if (g.gl == 0) {
      for (uint32_t j = 0; j < k; ++j) lhq_push<D>(h, n + j, src[j]);
      ib.cnt[(size_t)prevb * L + lp] = 0;
    }
    n += k;
    g.sync();
  }
  if (g.gl == 0) phold_stage_slot_init(st, slot, mt.count, mt.csum, mt.ohash);
  g.sync();
  uint32_t done = 0, cmin = kInfBits, head = kInfBits;
  gpq_item mine;
  bool have = false;
  while (n > 0) {
    const gpq_item top = h[0];
    if (!((top.ts < bound) && (top.ts < T))) { head = gpq_f2u(top.ts); break; }
    if (g.gl == done % G) { mine = top; have = true; }
    lhq_pop<G, D>(h, n, g);
    --n;
    ++done;
    if (done % G == 0) {  // a full batch of G events
      cmin = min(cmin, phold_stage_batch<G>(d, ib, st, g, mine, true, done - G + g.gl, G, slot, curb, err_slot));
      have = false;
    }
  }
  const uint32_t rem = done % G;
  if (rem) cmin = min(cmin, phold_stage_batch<G>(d, ib, st, g, mine, have, done - rem + g.gl, rem, slot, curb, err_slot));
  if (g.gl == 0) {
    q.size[lp] = n;
    st.lp[slot] = done > 0 ? lp : ~0u;
    if (done > 0) d.count[lp] = mt.count + done;
  }
  return min(head, g.umin(cmin));
}

template <int G_>
struct LhqPolicy {
  static constexpr int G = G_;
  using Dev = LhqDev;
  using Meta = LhqMeta;
  struct Smem {};
  __host__ __device__ static size_t group_smem_bytes(uint32_t) { return 0; }
  __device__ static Smem smem(unsigned char*, uint32_t) { return Smem{}; }
  __device__ static Meta load_meta(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t prevb) {
    return lhq_load_meta(d, q, ib, lp, prevb);
  }
  __device__ static uint32_t stage_lp(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t slot,
                                      uint32_t s, float bound, const Smem&, const PholdStage& st,
                                      const LaneGroup<G>& g, uint32_t* err_slot, const Meta& mt) {
    return lhq_lp_stage<G>(d, q, ib, lp, slot, s, bound, st, g, err_slot, mt);
  }
};
