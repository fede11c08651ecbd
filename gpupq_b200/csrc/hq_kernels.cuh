// Parallel heap queue kernels: the whole PHOLD window loop of one heap in one CTA, and
// the single-CTA operations of the HQ queue object.
#pragma once

#include "hq.cuh"

__host__ __device__ inline size_t hq_smem_bytes(uint32_t r) {
  return (size_t)r * 9 * sizeof(gpq_item) + (size_t)r * 2 * sizeof(uint32_t);
}

struct HqWork {
  HqSmem sm;
  gpq_item* e;     // [r] the window's new items
  uint32_t* keys;  // [r]
  uint32_t* seg;   // [r]
};

__device__ __forceinline__ HqWork hq_work(unsigned char* raw, uint32_t r) {
  HqWork w;
  gpq_item* it = reinterpret_cast<gpq_item*>(raw);
  w.sm.a = it;
  w.sm.b = it + r;
  w.sm.c = it + 2 * r;
  w.sm.t = it + 3 * r;
  w.sm.m = it + 5 * r;
  w.e = it + 8 * r;
  w.keys = reinterpret_cast<uint32_t*>(it + 9 * r);
  w.seg = w.keys + r;
  return w;
}

// One heap, all windows (des_run over the parallel heap).  Per window: insert the
// previous window's children (from h.ch, r at a time), fix the window bound from the
// root's head, then repeatedly take the root's prefix below the bound S, fold S into
// the per-LP outputs in key order per LP (ranks from a sort by (lp, position)), append
// S's children to h.ch, remove S from the root and refill it -- until the root's head
// reaches the bound.  The root always holds the r smallest items, so the batches come
// in global key order; a child is never safe in its parent's window, so the children
// wait for the next window.  One CTA; blockDim a multiple of 32.
static __device__ void hq_phold_run(const PholdDev& d, const HqDev& h, uint32_t max_steps, unsigned char* raw) {
  const uint32_t r = h.r;
  const HqWork w = hq_work(raw, r);
  __shared__ uint32_t s_last, s_nch, s_c, s_n0, s_stop, s_steps, s_lim;
  if (threadIdx.x == 0) {
    s_last = h.meta[0];
    s_nch = 0;
    s_steps = 0;
  }
  __syncthreads();
  for (;;) {
    // the previous window's children
    const uint32_t nch = s_nch;
    bool full = false;
    for (uint32_t off = 0; off < nch && !full; off += r) {
      const uint32_t k = min(r, nch - off);
      hq_load(w.e, h.ch + off, k);
      full = !hq_insert(h, w.sm, w.e, k, &s_last);
    }
    if (full) {
      if (threadIdx.x == 0) gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL);
      break;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_nch = 0;
      const uint32_t n0 = h.cnt[0];
      uint32_t stop = (n0 == 0) || (max_steps != 0 && s_steps >= max_steps);
      if (!stop) {
        const float m = h.nodes[0].ts;
        stop = !(m < d.p.end_time);
        if (!stop) {
          s_lim = min(gpq_f2u(GPQ_FADD(m, d.p.lookahead)), gpq_f2u(d.p.end_time));
          ++s_steps;
        }
      }
      s_stop = stop;
    }
    __syncthreads();
    if (s_stop) break;
    for (;;) {  // batches of the window
      if (threadIdx.x == 0) {
        const uint32_t n0 = h.cnt[0];
        uint32_t lo = 0, hi = n0;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (gpq_f2u(h.nodes[mid].ts) < s_lim) lo = mid + 1; else hi = mid;
        }
        s_c = lo;
        s_n0 = n0;
      }
      __syncthreads();
      const uint32_t c = s_c, n0 = s_n0, base = s_nch;
      if (c == 0) break;
      hq_load(w.sm.a, h.nodes, c);
      hq_lp_ranks(w.sm.a, c, w.keys, w.seg);
      for (uint32_t p = threadIdx.x; p < c; p += blockDim.x) {
        const uint32_t key = w.keys[p];
        const uint32_t i = key & 0x7ffu, lp = key >> 11;
        const gpq_item e = w.sm.a[i];
        const uint64_t hh = gpq_ev_hash(e.id, gpq_f2u(e.ts));
        atomicAdd(&d.csum[lp], (unsigned long long)hh);
        atomicAdd(&d.ohash[lp], (unsigned long long)gpq_seq_hash(hh, (uint64_t)d.count[lp] + (p - w.seg[p])));
        h.ch[base + i] = gpq_phold_child(d.p, e);
      }
      __syncthreads();
      for (uint32_t p = threadIdx.x; p < c; p += blockDim.x) {
        const uint32_t lp = w.keys[p] >> 11;
        if (p + 1 == c || (w.keys[p + 1] >> 11) != lp) d.count[lp] += p - w.seg[p] + 1;
      }
      hq_load(w.sm.a, h.nodes + c, n0 - c);
      hq_refill_root(h, w.sm, n0 - c, &s_last);
      if (threadIdx.x == 0) s_nch = base + c;
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    h.meta[0] = s_last;
    h.meta[1] = s_steps;
    d.ctrl->steps = s_steps;
  }
}

static __global__ void __launch_bounds__(512) hq_phold_kernel(PholdDev d, HqDev h, uint32_t max_steps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  hq_phold_run(d, h, max_steps, smem_raw);
}

// Pending events of the heap and the per-LP digest (one CTA per node range, grid-stride).
static __global__ void hq_finalize_kernel(PholdDev d, HqDev h, unsigned long long* acc, uint32_t* pmin) {
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t mn = kInfBits;
  const uint32_t last = h.meta[0];
  const uint64_t total = (uint64_t)(last + 1) * h.r;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint32_t node = (uint32_t)(i / h.r), j = (uint32_t)(i % h.r);
    if (j >= h.cnt[node]) continue;
    const gpq_item e = h.nodes[i];
    pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
    pend += 1;
    mn = min(mn, gpq_f2u(e.ts));
  }
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < d.L; lp += (uint32_t)stride) {
    const uint32_t c = d.count[lp];
    com += c;
    const uint64_t lph = gpq_mix64(gpq_mix64(((uint64_t)lp << 32) | c) ^ d.csum[lp]) + d.ohash[lp];
    dig += gpq_mix64(lph);
  }
  pend = warp_sum_u64(pend);
  pcs = warp_sum_u64(pcs);
  dig = warp_sum_u64(dig);
  com = warp_sum_u64(com);
  mn = warp_min_u32(mn);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[0], (unsigned long long)com);
    atomicAdd(&acc[1], (unsigned long long)pend);
    atomicAdd(&acc[2], (unsigned long long)pcs);
    atomicAdd(&acc[3], (unsigned long long)dig);
    atomicMin(pmin, mn);
  }
}

// Queue object: insert the n buffered items (in global memory) into the heap.
static __global__ void __launch_bounds__(512) hq_post_kernel(HqDev h, const gpq_item* pend, uint32_t n, uint32_t* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HqWork w = hq_work(smem_raw, h.r);
  __shared__ uint32_t s_last;
  if (threadIdx.x == 0) s_last = h.meta[0];
  __syncthreads();
  for (uint32_t off = 0; off < n; off += h.r) {
    const uint32_t k = min(h.r, n - off);
    hq_load(w.e, pend + off, k);
    if (!hq_insert(h, w.sm, w.e, k, &s_last)) {
      if (threadIdx.x == 0) gpq_set_error(err, GPQ_ERR_QUEUE_FULL);
      break;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) h.meta[0] = s_last;
}

// Queue object: from the root's items below `bound` take, per LP, the first max_per_lp
// (0 = all) in key order (the reference's partition takes one per LP from the merged
// root buffer, src/heap_queue.cu:478-547); out receives them grouped by LP; the rest of
// the root stays and the root is refilled.  out_n[0] = number taken.
static __global__ void __launch_bounds__(512) hq_dequeue_kernel(HqDev h, float bound, uint32_t max_per_lp,
                                                                  gpq_item* out, uint32_t* out_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HqWork w = hq_work(smem_raw, h.r);
  __shared__ uint32_t s_last, s_c, s_n0, s_keep;
  if (threadIdx.x == 0) {
    s_last = h.meta[0];
    const uint32_t n0 = h.cnt[0];
    uint32_t lo = 0, hi = n0;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (h.nodes[mid].ts < bound) lo = mid + 1; else hi = mid;
    }
    s_c = lo;
    s_n0 = n0;
  }
  __syncthreads();
  const uint32_t c = s_c, n0 = s_n0;
  if (c == 0) {
    if (threadIdx.x == 0) out_n[0] = 0;
    return;
  }
  hq_load(w.sm.a, h.nodes, n0);
  hq_lp_ranks(w.sm.a, c, w.keys, w.seg);
  // taken flags in w.e[i].aux (scratch), output in sorted (lp, position) order
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) w.e[i].aux = 0;
  __syncthreads();
  for (uint32_t p = threadIdx.x; p < c; p += blockDim.x) {
    const uint32_t rank = p - w.seg[p];
    if (max_per_lp == 0 || rank < max_per_lp) w.e[w.keys[p] & 0x7ffu].aux = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0, k = 0;
    for (uint32_t p = 0; p < c; ++p) {
      const uint32_t i = w.keys[p] & 0x7ffu;
      if (w.e[i].aux) out[t++] = w.sm.a[i];
    }
    for (uint32_t i = 0; i < n0; ++i)
      if (i >= c || !w.e[i].aux) w.sm.b[k++] = w.sm.a[i];
    s_keep = k;
    out_n[0] = t;
  }
  __syncthreads();
  hq_load(w.sm.a, w.sm.b, s_keep);
  hq_refill_root(h, w.sm, s_keep, &s_last);
  if (threadIdx.x == 0) h.meta[0] = s_last;
}
