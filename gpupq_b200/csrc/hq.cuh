// Parallel heap queue (HQ), B200 form.
//
// Reference: src/heap_queue.cu.  A heap of nodes, each a sorted array of HQ_NODE_SIZE (r)
// items, with max(node) <= min(child) (HeapQueueData, :17-88).  Each step merges the
// enqueue buffer with the root (merge_fel_enqueue + mgpu mergesort, :1541-1553,
// :1448-1470), takes the safe items from the merged buffer (partition_merged_parallel_*,
// :478-547), refills the root from the last nodes (copy_last, :975-1094) and restores
// the order with delete-update processes (:631-784) while insert-update processes carry
// the remaining new items down to their target nodes (:817-960, :1097-1249), one
// mergesort per node on its own stream, driven by host threads.
//
// Here one CTA owns one heap and runs all of its windows itself; every node merge is a
// shared-memory merge-path over the CTA's threads:
//   * insert-update: the window's new items are sorted (bitonic, shared memory) and cut
//     into pieces that fill the last node and then new nodes; each piece walks the
//     root-to-target path, every node on the path keeping the smallest r of
//     (node + piece) and passing the rest down;
//   * the root then holds the r smallest items; the safe items are its prefix below
//     min(m + lookahead, end time);
//   * copy-last: the taken items are replaced by the largest items of the last nodes;
//   * delete-update: walking down one path, a node merged with its two children keeps
//     the smallest r, the child with the larger old maximum takes the middle items (they
//     stay below its own children) and the other child the largest ones; the walk
//     continues at that other child (delete_update_post, src/heap_queue.cu:728-784).
#pragma once

#include "phold_common.cuh"

static constexpr uint32_t kHqMaxR = 1024;  // node size limit (8 r items of shared memory)

struct HqDev {
  gpq_item* nodes;   // [maxnodes][r]
  uint32_t* cnt;     // [maxnodes] items per node
  uint32_t* meta;    // [0] last non-empty node, [1] windows executed
  gpq_item* ch;      // children of the current window (PHOLD engine; population-sized)
  uint32_t r;
  uint32_t maxnodes;
};

__device__ __forceinline__ gpq_item hq_max_item() {
  gpq_item e;
  e.ts = gpq_u2f(0xffffffffu);
  e.lp = 0xffffffffu;
  e.id = 0xffffffffu;
  e.aux = 0;
  return e;
}

__device__ __forceinline__ bool hq_less(const gpq_item& a, const gpq_item& b) { return gpq_item_less(a, b); }

// Bitonic sort of a[0, n) in shared memory; a has room for P = next power of two >= n.
static __device__ void hq_cta_sort(gpq_item* a, uint32_t n) {
  uint32_t P = 1;
  while (P < n) P <<= 1;
  for (uint32_t i = n + threadIdx.x; i < P; i += blockDim.x) a[i] = hq_max_item();
  __syncthreads();
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const gpq_item x = a[i], y = a[ixj];
          const bool up = (i & k) == 0;
          if (up ? hq_less(y, x) : hq_less(x, y)) { a[i] = y; a[ixj] = x; }
        }
      }
      __syncthreads();
    }
  }
}

__device__ __forceinline__ uint32_t hq_path_split(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb,
                                                  uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0u, hi = min(diag, na);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (!hq_less(B[diag - 1 - mid], A[mid])) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// out[0, na+nb) = merge of sorted A and B (all in shared memory, out distinct).
static __device__ void hq_cta_merge(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb, gpq_item* out) {
  const uint32_t total = na + nb;
  const uint32_t per = (total + blockDim.x - 1) / blockDim.x;
  const uint32_t d0 = threadIdx.x * per;
  if (d0 < total) {
    uint32_t ia = hq_path_split(A, na, B, nb, d0);
    uint32_t ib = d0 - ia;
    const uint32_t lim = min(d0 + per, total);
    for (uint32_t o = d0; o < lim; ++o) {
      const bool take_a = ib >= nb || (ia < na && !hq_less(B[ib], A[ia]));
      out[o] = take_a ? A[ia++] : B[ib++];
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void hq_load(gpq_item* dst, const gpq_item* src, uint32_t n) {
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

__device__ __forceinline__ void hq_store(gpq_item* dst, const gpq_item* src, uint32_t n) {
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// Shared-memory work areas of one heap (8 r items).
struct HqSmem {
  gpq_item* a;  // [r]
  gpq_item* b;  // [r]
  gpq_item* c;  // [r]
  gpq_item* t;  // [2r]
  gpq_item* m;  // [3r]
};

// Insert the sorted piece x[0, px) (x = sm.b) into target node tgt (which has room).
static __device__ void hq_insert_piece(const HqDev& h, const HqSmem& sm, uint32_t px, uint32_t tgt) {
  const uint32_t r = h.r;
  uint32_t depth = 0;
  while (((tgt + 1) >> (depth + 1)) != 0) ++depth;
  for (uint32_t l = 0; l < depth; ++l) {
    const uint32_t p = ((tgt + 1) >> (depth - l)) - 1;  // full ancestor on the path
    hq_load(sm.a, h.nodes + (size_t)p * r, r);
    hq_cta_merge(sm.a, r, sm.b, px, sm.t);
    hq_store(h.nodes + (size_t)p * r, sm.t, r);
    hq_store(sm.b, sm.t + r, px);
  }
  const uint32_t nt = h.cnt[tgt];
  hq_load(sm.a, h.nodes + (size_t)tgt * r, nt);
  hq_cta_merge(sm.a, nt, sm.b, px, sm.t);
  hq_store(h.nodes + (size_t)tgt * r, sm.t, nt + px);
  if (threadIdx.x == 0) h.cnt[tgt] = nt + px;
  __syncthreads();
}

// Insert the unsorted items e[0, ke) (in shared memory, room for the next power of two)
// into the heap.  Returns false if the heap runs out of nodes.
static __device__ bool hq_insert(const HqDev& h, const HqSmem& sm, gpq_item* e, uint32_t ke, uint32_t* s_last) {
  if (ke == 0) return true;
  hq_cta_sort(e, ke);
  const uint32_t r = h.r;
  uint32_t off = 0;
  while (off < ke) {
    uint32_t last = *s_last;
    uint32_t tgt = last;
    if (h.cnt[last] == r) {
      tgt = last + 1;
      if (tgt >= h.maxnodes) return false;
      __syncthreads();
      if (threadIdx.x == 0) { h.cnt[tgt] = 0; *s_last = tgt; }
      __syncthreads();
    }
    const uint32_t px = min(ke - off, r - h.cnt[tgt]);
    hq_store(sm.b, e + off, px);
    hq_insert_piece(h, sm, px, tgt);
    off += px;
  }
  return true;
}

// Bitonic sort of 32-bit keys k[0, n) in shared memory (room for the next power of two).
static __device__ void hq_cta_sort_u32(uint32_t* k, uint32_t n) {
  uint32_t P = 1;
  while (P < n) P <<= 1;
  for (uint32_t i = n + threadIdx.x; i < P; i += blockDim.x) k[i] = 0xffffffffu;
  __syncthreads();
  for (uint32_t q = 2; q <= P; q <<= 1) {
    for (uint32_t j = q >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const uint32_t x = k[i], y = k[ixj];
          const bool up = (i & q) == 0;
          if (up ? (y < x) : (x < y)) { k[i] = y; k[ixj] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// The root now holds sm.a[0, keep) (sorted, a remainder of the old root).  Refill it from
// the largest items of the last nodes (copy-last), then restore the heap order along one
// path (delete-update).
static __device__ void hq_refill_root(const HqDev& h, const HqSmem& sm, uint32_t keep, uint32_t* s_last) {
  const uint32_t r = h.r;
  const uint32_t want = r - keep;
  uint32_t got = 0;
  __syncthreads();
  while (got < want && *s_last > 0) {
    const uint32_t last = *s_last;
    const uint32_t nl = h.cnt[last];
    const uint32_t t = min(want - got, nl);
    hq_store(sm.b + got, h.nodes + (size_t)last * r + (nl - t), t);
    got += t;
    if (threadIdx.x == 0) {
      h.cnt[last] = nl - t;
      if (nl - t == 0) *s_last = last - 1;
    }
    __syncthreads();
  }
  if (got > 0) {
    hq_cta_sort(sm.b, got);
    hq_cta_merge(sm.a, keep, sm.b, got, sm.t);
    hq_store(h.nodes, sm.t, keep + got);
  } else {
    hq_store(h.nodes, sm.a, keep);
  }
  if (threadIdx.x == 0) h.cnt[0] = keep + got;
  __syncthreads();
  // delete-update
  uint32_t p = 0;
  for (;;) {
    const uint32_t c1 = 2 * p + 1, c2 = 2 * p + 2;
    const uint32_t np = h.cnt[p];
    const uint32_t n1 = (c1 <= *s_last) ? h.cnt[c1] : 0u;
    const uint32_t n2 = (c2 <= *s_last) ? h.cnt[c2] : 0u;
    if (np == 0 || (n1 == 0 && n2 == 0)) break;
    const gpq_item pmax = h.nodes[(size_t)p * r + np - 1];
    const bool ok1 = n1 == 0 || hq_less(pmax, h.nodes[(size_t)c1 * r]);
    const bool ok2 = n2 == 0 || hq_less(pmax, h.nodes[(size_t)c2 * r]);
    if (ok1 && ok2) break;
    hq_load(sm.a, h.nodes + (size_t)p * r, np);
    hq_load(sm.b, h.nodes + (size_t)c1 * r, n1);
    hq_load(sm.c, h.nodes + (size_t)c2 * r, n2);
    hq_cta_merge(sm.a, np, sm.b, n1, sm.t);
    hq_cta_merge(sm.t, np + n1, sm.c, n2, sm.m);
    hq_store(h.nodes + (size_t)p * r, sm.m, np);
    if (n2 == 0) {
      hq_store(h.nodes + (size_t)c1 * r, sm.m + np, n1);
      p = c1;
      continue;
    }
    if (n1 == 0) {
      hq_store(h.nodes + (size_t)c2 * r, sm.m + np, n2);
      p = c2;
      continue;
    }
    // The middle items go to the child with the larger old maximum: all of them are at
    // most that maximum, hence below that child's own children.  A partial c2 is the
    // last node and has no children, so it takes the middle items too.  The largest
    // items go to the other child, where the walk continues.
    const bool mid2 = n2 < r || hq_less(sm.b[n1 - 1], sm.c[n2 - 1]);
    const uint32_t mid = mid2 ? c2 : c1, lrg = mid2 ? c1 : c2;
    const uint32_t nmid = mid2 ? n2 : n1, nlrg = mid2 ? n1 : n2;
    hq_store(h.nodes + (size_t)mid * r, sm.m + np, nmid);
    hq_store(h.nodes + (size_t)lrg * r, sm.m + np + nmid, nlrg);
    p = lrg;
  }
}

// Ranks of the root's first c items within their LPs (c <= 2048): keys[p] sorted by
// (lp, position); seg[p] = first sorted position of the same LP.
static __device__ void hq_lp_ranks(const gpq_item* s, uint32_t c, uint32_t* keys, uint32_t* seg) {
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) keys[i] = (s[i].lp << 11) | i;
  __syncthreads();
  hq_cta_sort_u32(keys, c);
  for (uint32_t p = threadIdx.x; p < c; p += blockDim.x) {
    uint32_t q = p;
    const uint32_t lp = keys[p] >> 11;
    while (q > 0 && (keys[q - 1] >> 11) == lp) --q;
    seg[p] = q;
  }
  __syncthreads();
}
