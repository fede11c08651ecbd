// Local array queue (LAQ), B200 form.
//
// Reference: src/local_array_queue.cu.  Each LP owns a ring buffer of FEL_SIZE items
// holding its events sorted by timestamp in [fel_read, fel_write)
// (src/local_array_queue.cu:38-45).  queue_insert reserves a slot behind fel_write with
// atomicAdd and writes the item there (:486-513); queue_post then insertion-sorts every
// new item into the ring, one thread per LP, shifting one 16-byte item per step
// (:254-299, src/sort.cu:329-353); queue_peek returns the head if it lies inside the
// window (:760-779) and queue_set_done advances fel_read (:710-728).
//
// Here each LP is handled by a group of G lanes (G = 4, 8, 16 or 32; 32/G LPs per warp):
//   * inserts land in a per-LP insert buffer (double-buffered by window parity, so the
//     children of window s can be written while window s-1's children are merged);
//   * the merge ranks the k new items among themselves in shared memory, then walks the
//     sorted ring backwards in chunks of 4G items with 16-byte loads, moves every old
//     item up by the number of new items below it (binary search in the sorted new keys)
//     and drops the new items into the gaps -- one pass over the part of the ring that
//     moves, instead of one pass per inserted item; the merged head is kept in shared
//     memory for the drain;
//   * the drain finds the safe prefix with a ballot and stages those events in shared
//     memory; the whole CTA then processes the staged events one per thread (hashes,
//     child, insert), so the event arithmetic runs on full warps.
#pragma once

#include "phold_common.cuh"

struct LaqDev {
  gpq_item* ring;  // num_lps << cap_log2 items
  uint32_t* rd;    // per-LP read counter (fel_read); slot = counter & (cap - 1)
  uint32_t* wr;    // per-LP write counter (fel_write)
  uint32_t cap_log2;
};

// Per-group shared memory: the merge's new-key arrays and a copy of the merged head.
struct LaqGroupSmem {
  gpq_item* head;  // [G] first G items of the merged run (valid when the merge saw them all)
  uint64_t* ku;    // [ibc] new keys, arrival order
  uint64_t* ks;    // [ibc] new keys, sorted
  uint32_t* rk;    // [ibc] rank of the j-th new item
  uint32_t* hist;  // [ibc + 1] number of moved old items per shift
};

__host__ __device__ inline size_t laq_group_smem_bytes(uint32_t ibc, uint32_t group) {
  size_t b = (size_t)group * 16 + (size_t)ibc * 8 * 2 + (size_t)ibc * 4 + (size_t)(ibc + 1) * 4;
  return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ LaqGroupSmem laq_group_smem(unsigned char* base, uint32_t ibc, uint32_t group) {
  LaqGroupSmem s;
  s.head = reinterpret_cast<gpq_item*>(base);
  s.ku = reinterpret_cast<uint64_t*>(base + (size_t)group * 16);
  s.ks = s.ku + ibc;
  s.rk = reinterpret_cast<uint32_t*>(s.ks + ibc);
  s.hist = s.rk + ibc;
  return s;
}

// Ranks the k new items (keys -> smem ks in order, rk[j] = rank of item j); clears hist.
template <int G>
__device__ __forceinline__ void laq_rank_new(const gpq_item* __restrict__ src, uint32_t k, const LaqGroupSmem& sm,
                                             const LaneGroup<G>& g) {
  for (uint32_t j = g.gl; j < k; j += G) sm.ku[j] = gpq_lp_key(src[j]);
  g.sync();
  for (uint32_t j = g.gl; j < k; j += G) {
    const uint64_t kj = sm.ku[j];
    uint32_t r = 0;
    for (uint32_t i = 0; i < k; ++i) r += (sm.ku[i] < kj) ? 1u : 0u;
    sm.ks[r] = kj;
    sm.rk[j] = r;
  }
  for (uint32_t h = g.gl; h <= k; h += G) sm.hist[h] = 0;
  g.sync();
}

__device__ __forceinline__ uint32_t laq_count_below(const uint64_t* ks, uint32_t k, uint64_t key) {
  uint32_t a = 0, b = k;
  while (a < b) {
    const uint32_t mid = (a + b) >> 1;
    if (ks[mid] < key) a = mid + 1; else b = mid;
  }
  return a;
}

// Merge the k unsorted items at `src` into the sorted ring run [rd, rd + n) (n + k <=
// capacity).  Old items are visited backwards in chunks of 4G (lane-strided); an item
// moves up by the number of new items below it (binary search in the sorted new keys),
// and the new items then drop into the gaps.  Items whose merged position is below G are also copied to
// sm.head.  Returns true when sm.head holds the complete merged head (every item that
// ends below position G was visited).  All lanes of the group, convergent.
template <int G>
__device__ __forceinline__ bool laq_merge(gpq_item* ring, uint32_t mask, uint32_t rd, uint32_t n,
                                          const gpq_item* __restrict__ src, uint32_t k, const LaqGroupSmem& sm,
                                          const LaneGroup<G>& g) {
  constexpr int U = 4;  // consecutive items per lane per chunk
  int32_t hi = (int32_t)n;
  int32_t lo = hi > U * G ? hi - U * G : 0;
  gpq_item o[U];
  // The first (topmost) chunk is loaded before the new items are ranked so that both
  // loads are in flight together.
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int32_t i = lo + u * G + (int32_t)g.gl;
    if (i < hi) o[u] = ring[(rd + (uint32_t)i) & mask];
  }
  laq_rank_new<G>(src, k, sm, g);
  bool complete = true;
  while (hi > 0) {
    uint32_t sh[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t i = lo + u * G + (int32_t)g.gl;
      sh[u] = (i < hi) ? laq_count_below(sm.ks, k, gpq_lp_key(o[u])) : 0u;
    }
    const uint32_t sh_lo = g.shfl(sh[0], 0);  // shift of item `lo`, the chunk's smallest
    g.sync();                                 // every load of the chunk precedes every store
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t i = lo + u * G + (int32_t)g.gl;
      if (i < hi) {
        const uint32_t pos = (uint32_t)i + sh[u];
        if (sh[u] > 0) {
          ring[(rd + pos) & mask] = o[u];
          atomicAdd(&sm.hist[sh[u]], 1u);
        }
        if (pos < (uint32_t)G) sm.head[pos] = o[u];
      }
    }
    if (sh_lo == 0) {  // shifts are non-decreasing: nothing below `lo` moves
      complete = (lo == 0);  // unvisited items [0, lo) keep positions below lo
      break;
    }
    hi = lo;
    lo = hi > U * G ? hi - U * G : 0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t i = lo + u * G + (int32_t)g.gl;
      if (i < hi) o[u] = ring[(rd + (uint32_t)i) & mask];
    }
  }
  g.sync();
  // New item of rank r lands after the n - (#old items with shift > r) old items below it.
  for (uint32_t j = g.gl; j < k; j += G) {
    const uint32_t r = sm.rk[j];
    uint32_t gt = 0;
    for (uint32_t h = r + 1; h <= k; ++h) gt += sm.hist[h];
    const uint32_t pos = r + n - gt;
    const gpq_item it = src[j];
    ring[(rd + pos) & mask] = it;
    if (pos < (uint32_t)G) sm.head[pos] = it;
  }
  g.sync();
  return complete;
}

// Per-LP state read at the start of its window (prefetched one LP ahead).
struct LaqMeta {
  uint32_t k, rd, wr, count;
  unsigned long long csum, ohash;
};

__device__ __forceinline__ LaqMeta laq_load_meta(const PholdDev& d, const LaqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t prevb) {
  LaqMeta m;
  m.k = ib.cnt[(size_t)prevb * d.L + lp];
  m.rd = q.rd[lp];
  m.wr = q.wr[lp];
  m.count = d.count[lp];
  m.csum = d.csum[lp];
  m.ohash = d.ohash[lp];
  return m;
}

// One LP, one window s, first pass: merge the children of window s-1, then find the
// safe prefix (ts < bound = m_s + lookahead and ts < end_time) and stage it for the
// CTA-wide event pass; advance fel_read past it.  Returns the new head's timestamp
// bits, min'ed with any child processed here.  All lanes of the group, convergent.
template <int G>
__device__ __forceinline__ uint32_t laq_lp_stage(const PholdDev& d, const LaqDev& q, const InsDev& ib,
                                                 uint32_t lp, uint32_t slot, uint32_t s, float bound,
                                                 const LaqGroupSmem& sm, const PholdStage& st, const LaneGroup<G>& g,
                                                 uint32_t* err_slot, const LaqMeta& mt) {
  const uint32_t L = d.L;
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const uint32_t cap = 1u << q.cap_log2, mask = cap - 1u;
  gpq_item* ring = q.ring + ((size_t)lp << q.cap_log2);
  const float T = d.p.end_time;

  uint32_t k = mt.k;
  const uint32_t rd = mt.rd;
  uint32_t n = mt.wr - rd;
  bool head_in_smem = false;
  if (k > 0) {
    if (k > ib.ibc) k = ib.ibc;  // overflow was flagged by the inserter
    if (n + k > cap) {
      if (g.gl == 0) { gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL); atomicOr(err_slot, 1u); }
      k = cap - n;
    }
    const gpq_item* src = ib.buf + ((size_t)prevb * L + lp) * ib.ibc;
    head_in_smem = laq_merge<G>(ring, mask, rd, n, src, k, sm, g);
    n += k;
    if (g.gl == 0) {
      q.wr[lp] = mt.wr + k;
      ib.cnt[(size_t)prevb * L + lp] = 0;
    }
  }

  if (g.gl == 0) phold_stage_slot_init(st, slot, mt.count, mt.csum, mt.ohash);
  g.sync();
  uint32_t done = 0, head = kInfBits, cmin = kInfBits;
  while (done < n) {
    const uint32_t i = done + g.gl;
    gpq_item e;
    bool safe = false;
    if (i < n) {
      e = (head_in_smem && i < (uint32_t)G) ? sm.head[i] : ring[(rd + i) & mask];
      safe = (e.ts < bound) && (e.ts < T);
    }
    const uint32_t c = __popc(g.ballot(safe));  // the run is sorted: safe items form a prefix
    cmin = min(cmin, phold_stage_batch<G>(d, ib, st, g, e, safe, i, c, slot, curb, err_slot));
    if (c < (uint32_t)G) {
      head = g.shfl((i < n) ? gpq_f2u(e.ts) : kInfBits, c);
      done += c;
      break;
    }
    done += G;
  }
  if (g.gl == 0) {
    st.lp[slot] = done > 0 ? lp : ~0u;  // the event pass writes the checksums back
    if (done > 0) {
      d.count[lp] = mt.count + done;
      q.rd[lp] = rd + done;
    }
  }
  return min(head, g.umin(cmin));
}

// Local array queue as a PHOLD engine policy.
template <int G_>
struct LaqPolicy {
  static constexpr int G = G_;
  using Dev = LaqDev;
  using Meta = LaqMeta;
  using Smem = LaqGroupSmem;
  __host__ __device__ static size_t group_smem_bytes(uint32_t ibc) { return laq_group_smem_bytes(ibc, G); }
  __device__ static Smem smem(unsigned char* base, uint32_t ibc) { return laq_group_smem(base, ibc, G); }
  __device__ static Meta load_meta(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t prevb) {
    return laq_load_meta(d, q, ib, lp, prevb);
  }
  __device__ static uint32_t stage_lp(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t slot,
                                      uint32_t s, float bound, const Smem& sm, const PholdStage& st,
                                      const LaneGroup<G>& g, uint32_t* err_slot, const Meta& mt) {
    return laq_lp_stage<G>(d, q, ib, lp, slot, s, bound, sm, st, g, err_slot, mt);
  }
};
