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
//     moves, instead of one pass per inserted item;
//   * the drain reads the head G items at a time; a ballot finds the safe prefix and each
//     lane handles one event (hashes, child, insert) in parallel.
#pragma once

#include "common.cuh"
#include "gpq/model.h"

struct LaqDev {
  gpq_item* ring;  // num_lps << cap_log2 items
  uint32_t* rd;    // per-LP read counter (fel_read); slot = counter & (cap - 1)
  uint32_t* wr;    // per-LP write counter (fel_write)
  uint32_t cap_log2;
};

struct InsDev {
  gpq_item* buf;  // [2][num_lps][ibc]
  uint32_t* cnt;  // [2][num_lps]
  uint32_t ibc;
};

// Control words of one PHOLD instance (device memory).
struct PholdCtrl {
  uint32_t mins[3];  // window minimum slots (float bits), rotating by window index
  uint32_t errs[3];  // per-window error slots, rotating like mins
  uint32_t err;      // sticky error word reported to the host
  uint32_t phase;    // index of the next window to run
  unsigned long long bar;    // grid-barrier arrival counter (persistent launch)
  unsigned long long steps;  // windows executed
};

struct PholdDev {
  gpq_phold_params p;
  uint32_t L;
  uint32_t* count;
  unsigned long long* csum;
  unsigned long long* ohash;
  PholdCtrl* ctrl;
  uint64_t spin_limit;
};

// A group of G consecutive lanes of one warp working on one LP.
template <int G>
struct LaneGroup {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
  uint32_t gl;    // lane within the group
  uint32_t base;  // first lane of the group
  uint32_t mask;  // the group's lanes
  __device__ __forceinline__ LaneGroup() {
    const uint32_t lane = threadIdx.x & 31u;
    gl = lane & (G - 1);
    base = lane & ~(uint32_t)(G - 1);
    mask = (G == 32) ? GPQ_FULL_MASK : (((1u << G) - 1u) << base);
  }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ uint32_t ballot(bool p) const {
    const uint32_t b = __ballot_sync(mask, p);
    return (G == 32) ? b : ((b >> base) & ((1u << G) - 1u));
  }
  __device__ __forceinline__ uint32_t shfl(uint32_t v, uint32_t src) const { return __shfl_sync(mask, v, src, G); }
  __device__ __forceinline__ uint64_t sum(uint64_t v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
  }
  __device__ __forceinline__ uint32_t umin(uint32_t v) const { return __reduce_min_sync(mask, v); }
};

// Per-group shared memory used by the merge.
struct LaqGroupSmem {
  uint64_t* ku;    // [ibc] new keys, arrival order
  uint64_t* ks;    // [ibc] new keys, sorted
  uint32_t* rk;    // [ibc] rank of the j-th new item
  uint32_t* hist;  // [ibc + 1] number of moved old items per shift
};

__host__ __device__ inline size_t laq_group_smem_bytes(uint32_t ibc) {
  size_t b = (size_t)ibc * 8 * 2 + (size_t)ibc * 4 + (size_t)(ibc + 1) * 4;
  return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ LaqGroupSmem laq_group_smem(unsigned char* base, uint32_t ibc) {
  LaqGroupSmem s;
  s.ku = reinterpret_cast<uint64_t*>(base);
  s.ks = s.ku + ibc;
  s.rk = reinterpret_cast<uint32_t*>(s.ks + ibc);
  s.hist = s.rk + ibc;
  return s;
}

// Merge the k unsorted items at `src` into the sorted ring run [rd, rd + n).
// The caller guarantees n + k <= capacity.  All lanes of the group, convergent.
template <int G>
__device__ __forceinline__ void laq_merge(gpq_item* ring, uint32_t mask, uint32_t rd, uint32_t n,
                                          const gpq_item* __restrict__ src, uint32_t k, const LaqGroupSmem& sm,
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

  constexpr int U = 4;  // items per lane per chunk
  int32_t hi = (int32_t)n;
  while (hi > 0) {
    const int32_t lo = hi > U * G ? hi - U * G : 0;
    gpq_item o[U];
    uint32_t sh[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t i = lo + u * G + (int32_t)g.gl;
      sh[u] = 0;
      if (i < hi) {
        o[u] = ring[(rd + (uint32_t)i) & mask];
        const uint64_t key = gpq_lp_key(o[u]);
        uint32_t a = 0, b = k;
        while (a < b) {
          const uint32_t mid = (a + b) >> 1;
          if (sm.ks[mid] < key) a = mid + 1; else b = mid;
        }
        sh[u] = a;  // number of new items below this old item
      }
    }
    const uint32_t sh_lo = g.shfl(sh[0], 0);  // shift of item `lo`, the chunk's smallest
    g.sync();                                 // every load of the chunk precedes every store
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t i = lo + u * G + (int32_t)g.gl;
      if (i < hi && sh[u] > 0) {
        ring[(rd + (uint32_t)i + sh[u]) & mask] = o[u];
        atomicAdd(&sm.hist[sh[u]], 1u);
      }
    }
    if (sh_lo == 0) break;  // shifts are non-decreasing: nothing below `lo` moves
    hi = lo;
  }
  g.sync();
  // New item of rank r lands after the n - (#old items with shift > r) old items below it.
  for (uint32_t j = g.gl; j < k; j += G) {
    const uint32_t r = sm.rk[j];
    uint32_t gt = 0;
    for (uint32_t h = r + 1; h <= k; ++h) gt += sm.hist[h];
    ring[(rd + r + n - gt) & mask] = src[j];
  }
  g.sync();
}

// Result of one LP's window.
struct LaqWindowOut {
  uint32_t committed;
  uint32_t min_bits;  // min over the LP's new head and the children's timestamps
};

// One LP, one window s: merge the children of window s-1, then drain every event with
// ts < bound (= m_s + lookahead) and ts < end_time, in key order, inserting the children
// into the window-s insert buffers.  All lanes of the group, convergent.
template <int G>
__device__ __forceinline__ LaqWindowOut laq_lp_window(const PholdDev& d, const LaqDev& q, const InsDev& ib,
                                                      uint32_t lp, uint32_t s, float bound, const LaqGroupSmem& sm,
                                                      const LaneGroup<G>& g, uint32_t* err_slot) {
  const uint32_t L = d.L;
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const uint32_t cap = 1u << q.cap_log2, mask = cap - 1u;
  gpq_item* ring = q.ring + ((size_t)lp << q.cap_log2);
  const float T = d.p.end_time;

  uint32_t k = ib.cnt[(size_t)prevb * L + lp];
  const uint32_t rd = q.rd[lp];
  uint32_t wr = q.wr[lp];
  const uint32_t seq0 = d.count[lp];
  uint32_t n = wr - rd;

  if (k > 0) {
    if (k > ib.ibc) k = ib.ibc;  // overflow was flagged by the inserter
    if (n + k > cap) {
      if (g.gl == 0) { gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL); atomicOr(err_slot, 1u); }
      k = cap - n;
    }
    const gpq_item* src = ib.buf + ((size_t)prevb * L + lp) * ib.ibc;
    laq_merge<G>(ring, mask, rd, n, src, k, sm, g);
    n += k;
    wr += k;
    if (g.gl == 0) {
      q.wr[lp] = wr;
      ib.cnt[(size_t)prevb * L + lp] = 0;
    }
  }

  // Drain the safe prefix.
  uint32_t done = 0;
  uint64_t acc_cs = 0, acc_oh = 0;
  uint32_t cmin = kInfBits, head = kInfBits;
  gpq_item* const ins_base = ib.buf + (size_t)curb * L * ib.ibc;
  uint32_t* const ins_cnt = ib.cnt + (size_t)curb * L;
  while (done < n) {
    const uint32_t i = done + g.gl;
    gpq_item e;
    bool safe = false;
    if (i < n) {
      e = ring[(rd + i) & mask];
      safe = (e.ts < bound) && (e.ts < T);
    }
    const uint32_t c = __popc(g.ballot(safe));  // ring is sorted: the safe items form a prefix
    if (safe) {
      const uint32_t tb = gpq_f2u(e.ts);
      const uint64_t h = gpq_ev_hash(e.id, tb);
      acc_cs += h;
      acc_oh += gpq_seq_hash(h, (uint64_t)seq0 + i);
      const gpq_item ch = gpq_phold_child(d.p, e);
      const uint32_t slot = atomicAdd(&ins_cnt[ch.lp], 1u);
      if (slot < ib.ibc) {
        ins_base[(size_t)ch.lp * ib.ibc + slot] = ch;
      } else {
        gpq_set_error(&d.ctrl->err, GPQ_ERR_INSERT_FULL);
        atomicOr(err_slot, 1u);
      }
      cmin = min(cmin, gpq_f2u(ch.ts));
    }
    if (c < (uint32_t)G) {
      head = g.shfl((i < n) ? gpq_f2u(e.ts) : kInfBits, c);
      done += c;
      break;
    }
    done += G;
  }
  acc_cs = g.sum(acc_cs);
  acc_oh = g.sum(acc_oh);
  cmin = g.umin(cmin);
  if (g.gl == 0 && done > 0) {
    d.count[lp] = seq0 + done;
    d.csum[lp] += acc_cs;
    d.ohash[lp] += acc_oh;
    q.rd[lp] = rd + done;
  }
  LaqWindowOut out;
  out.committed = done;
  out.min_bits = min(cmin, head);
  return out;
}
