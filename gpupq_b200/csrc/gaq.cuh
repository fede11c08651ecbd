// Global array queue (GAQ), B200 form: device kernels.
//
// Reference: src/global_array_queue.cu.  All events live in one array `fel` of
// (item, done) pairs; each step appends the per-thread insert buffers
// (calc_offsets + copy_insert_buffers, :84-108), mergesorts the whole array with
// moderngpu (sort_fel, :62-74; done items sort to the back and are trimmed, :139-142),
// and a single thread walks the sorted array to give each LP its first safe event
// (mark_safe_events, :147-179).
//
// Here the array is kept sorted by timestamp bits at all times:
//   * the window's safe events are the array's prefix below the bound (one binary
//     search, gaq_split_kernel) and are staged per LP (gaq_stage_kernel);
//   * each LP's staged events are ranked by (ts bits, id) in shared memory and handled
//     in that order (gaq_process_kernel); their children go to one buffer, reserved
//     with one atomic per CTA;
//   * the children are sorted with our own stable LSD radix sort on the timestamp bits
//     minus the window's smallest child (8-bit digits, only as many passes as the key
//     range needs: rs_hist / rs_scan / rs_scatter), then merged with the rest of the
//     array by merge path into the other buffer (mp_merge_kernel).
// Ties in timestamp between different LPs may sit in any order in the array; the
// per-LP ranking restores the (ts bits, LP, id) order where it is observable.
#pragma once

#include "phold_common.cuh"

static constexpr uint32_t kRsThreads = 256;  // = number of 8-bit digits
static constexpr uint32_t kRsPer = 16;
static constexpr uint32_t kRsTile = kRsThreads * kRsPer;
static constexpr uint32_t kMpThreads = 256;
static constexpr uint32_t kMpPer = 8;
static constexpr uint32_t kMpTile = kMpThreads * kMpPer;

__device__ __forceinline__ uint32_t rs_digit(const gpq_item& e, uint32_t kmin, uint32_t shift) {
  return ((gpq_f2u(e.ts) - kmin) >> shift) & 0xffu;
}

// Per-tile digit counts: hist[digit * ntiles + tile].
static __global__ void rs_hist_kernel(const gpq_item* __restrict__ in, uint32_t n, uint32_t kmin, uint32_t shift,
                                      uint32_t* hist, uint32_t ntiles) {
  __shared__ uint32_t cnt[256];
  const uint32_t tile = blockIdx.x;
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = tile * kRsTile;
  for (uint32_t j = 0; j < kRsPer; ++j) {
    const uint32_t i = base + j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[rs_digit(in[i], kmin, shift)], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + tile] = cnt[threadIdx.x];
}

// In-place exclusive scan of `total` counts (one CTA of 1024 threads).
static __global__ void rs_scan_kernel(uint32_t* a, uint32_t total) {
  __shared__ uint32_t part[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < total; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = (i < total) ? a[i] : 0u;
    part[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
      const uint32_t t = (threadIdx.x >= o) ? part[threadIdx.x - o] : 0u;
      __syncthreads();
      part[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < total) a[i] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += part[threadIdx.x];
    __syncthreads();
  }
}

// Stable scatter of one tile: items are taken in tile order (round j holds items
// j*256 + t); an item's rank among same-digit items of the tile is the count in earlier
// rounds + earlier warps of this round + lower lanes of its warp (warp match).
static __global__ void rs_scatter_kernel(const gpq_item* __restrict__ in, gpq_item* out, uint32_t n, uint32_t kmin,
                                         uint32_t shift, const uint32_t* __restrict__ off, uint32_t ntiles) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t wc[kRsThreads / 32][256];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t tile = blockIdx.x;
  run[t] = 0;
  const uint32_t base = tile * kRsTile;
  for (uint32_t j = 0; j < kRsPer; ++j) {
    for (uint32_t x = t; x < (kRsThreads / 32) * 256; x += kRsThreads) (&wc[0][0])[x] = 0;
    __syncthreads();
    const uint32_t i = base + j * kRsThreads + t;
    const bool valid = i < n;
    gpq_item e;
    uint32_t dgt = 0;
    if (valid) {
      e = in[i];
      dgt = rs_digit(e, kmin, shift);
    }
    const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, valid ? dgt : (0x100u + lane));
    if (valid && lane == (uint32_t)(__ffs(peers) - 1)) wc[warp][dgt] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (uint32_t w = 0; w < warp; ++w) pre += wc[w][dgt];
      const uint32_t below = __popc(peers & ((1u << lane) - 1u));
      out[off[dgt * ntiles + tile] + run[dgt] + pre + below] = e;
    }
    __syncthreads();
    uint32_t sum = 0;
    for (uint32_t w = 0; w < kRsThreads / 32; ++w) sum += wc[w][t];
    run[t] += sum;
    __syncthreads();
  }
}

// Number of A items among the first `diag` outputs of the stable merge (A first on ties).
__device__ __forceinline__ uint32_t mp_search(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb,
                                              uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0u, hi = min(diag, na);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (gpq_f2u(A[mid].ts) <= gpq_f2u(B[diag - 1 - mid].ts)) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Merge path: CTA b writes outputs [b*kMpTile, (b+1)*kMpTile) of merge(A, B).
static __global__ void mp_merge_kernel(const gpq_item* __restrict__ A, uint32_t na, const gpq_item* __restrict__ B,
                                       uint32_t nb, gpq_item* out) {
  __shared__ gpq_item s[kMpTile];
  __shared__ uint32_t sa[2];
  const uint32_t total = na + nb;
  const uint32_t d0 = blockIdx.x * kMpTile;
  const uint32_t d1 = min(d0 + kMpTile, total);
  if (threadIdx.x < 2) sa[threadIdx.x] = mp_search(A, na, B, nb, threadIdx.x == 0 ? d0 : d1);
  __syncthreads();
  const uint32_t a0 = sa[0], a1 = sa[1];
  const uint32_t b0 = d0 - a0, b1 = d1 - a1;
  const uint32_t la = a1 - a0, lb = b1 - b0;
  for (uint32_t x = threadIdx.x; x < la; x += kMpThreads) s[x] = A[a0 + x];
  for (uint32_t x = threadIdx.x; x < lb; x += kMpThreads) s[la + x] = B[b0 + x];
  __syncthreads();
  const uint32_t my0 = threadIdx.x * kMpPer;
  if (my0 < la + lb) {
    uint32_t ia = mp_search(s, la, s + la, lb, my0);
    uint32_t ib = my0 - ia;
    const uint32_t lim = min(my0 + kMpPer, la + lb);
    for (uint32_t o = my0; o < lim; ++o) {
      const bool take_a = ib >= lb || (ia < la && gpq_f2u(s[ia].ts) <= gpq_f2u(s[la + ib].ts));
      out[d0 + o] = take_a ? s[ia++] : s[la + ib++];
    }
  }
}

// GAQ engine state visible to kernels.
struct GaqDev {
  gpq_item* stg;        // [L][ibc] per-LP staging of the window's safe prefix
  uint32_t* stg_cnt;    // [L]
  gpq_item* ch;         // children of the window (unsorted)
  uint32_t* info;       // [0] prefix length c, [1] children count, [2] child key min, [3] child key max
  uint32_t ibc;
  uint32_t ch_cap;
};

// Length of the safe prefix of arr[0, n): items with ts < bound and ts < end_time.
static __global__ void gaq_split_kernel(const gpq_item* __restrict__ arr, uint32_t n, float bound, float T,
                                        uint32_t* info) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t lim = min(gpq_f2u(bound), gpq_f2u(T));
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (gpq_f2u(arr[mid].ts) < lim) lo = mid + 1; else hi = mid;
  }
  info[0] = lo;
  info[1] = 0;
  info[2] = 0xffffffffu;
  info[3] = 0;
}

static __global__ void gaq_stage_kernel(const gpq_item* __restrict__ arr, const uint32_t* info, GaqDev g, uint32_t L,
                                        uint32_t* err) {
  const uint32_t c = info[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const gpq_item e = arr[i];
    if (e.lp >= L) { gpq_set_error(err, GPQ_ERR_INVALID); continue; }
    const uint32_t slot = atomicAdd(&g.stg_cnt[e.lp], 1u);
    if (slot < g.ibc) g.stg[(size_t)e.lp * g.ibc + slot] = e;
    else gpq_set_error(err, GPQ_ERR_INSERT_FULL);
  }
}

// One lane group of G lanes per LP: rank the LP's staged events by (ts bits, id), fold
// them into the LP's outputs in that order, and write their children to the window's
// child buffer (one global reservation per CTA and round).
template <int G>
static __global__ void gaq_process_kernel(PholdDev d, GaqDev g, uint32_t* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t cta_n, cta_base, kmin_s, kmax_s;
  const LaneGroup<G> grp;
  const uint32_t gib = threadIdx.x / G, gpb = blockDim.x / G;
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem_raw) + (size_t)gib * g.ibc;
  const uint32_t ngroups = gridDim.x * gpb;
  for (uint32_t r0 = blockIdx.x * gpb; r0 < d.L; r0 += ngroups) {
    const uint32_t lp = r0 + gib;
    if (threadIdx.x == 0) { cta_n = 0; kmin_s = 0xffffffffu; kmax_s = 0; }
    __syncthreads();
    uint32_t k = 0, local = 0;
    const gpq_item* src = nullptr;
    if (lp < d.L) {
      k = min(g.stg_cnt[lp], g.ibc);
      src = g.stg + (size_t)lp * g.ibc;
      for (uint32_t j = grp.gl; j < k; j += G) keys[j] = gpq_lp_key(src[j]);
      if (grp.gl == 0 && k) local = atomicAdd(&cta_n, k);
    }
    __syncthreads();
    if (threadIdx.x == 0 && cta_n) {
      cta_base = atomicAdd(&g.info[1], cta_n);
      if (cta_base + cta_n > g.ch_cap) gpq_set_error(err, GPQ_ERR_INSERT_FULL);
    }
    __syncthreads();
    if (lp < d.L && k) {
      local = grp.shfl(local, 0);
      const uint32_t seq0 = d.count[lp];
      uint64_t cs = 0, oh = 0;
      uint32_t kmn = 0xffffffffu, kmx = 0;
      for (uint32_t j = grp.gl; j < k; j += G) {
        const uint64_t kj = keys[j];
        uint32_t rnk = 0;
        for (uint32_t i = 0; i < k; ++i) rnk += (keys[i] < kj) ? 1u : 0u;
        const gpq_item e = src[j];
        const uint64_t h = gpq_ev_hash(e.id, gpq_f2u(e.ts));
        cs += h;
        oh += gpq_seq_hash(h, (uint64_t)seq0 + rnk);
        const gpq_item chd = gpq_phold_child(d.p, e);
        const uint32_t pos = cta_base + local + j;
        if (pos < g.ch_cap) g.ch[pos] = chd;
        kmn = min(kmn, gpq_f2u(chd.ts));
        kmx = max(kmx, gpq_f2u(chd.ts));
      }
      cs = grp.sum(cs);
      oh = grp.sum(oh);
      kmn = grp.umin(kmn);
      kmx = __reduce_max_sync(grp.mask, kmx);
      if (grp.gl == 0) {
        d.count[lp] = seq0 + k;
        d.csum[lp] += cs;
        d.ohash[lp] += oh;
        g.stg_cnt[lp] = 0;
        atomicMin(&kmin_s, kmn);
        atomicMax(&kmax_s, kmx);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && cta_n) {
      atomicMin(&g.info[2], kmin_s);
      atomicMax(&g.info[3], kmax_s);
    }
  }
}

// End of run: pending events (the array) and per-LP digest.
static __global__ void gaq_finalize_kernel(PholdDev d, const gpq_item* __restrict__ arr, uint32_t n,
                                           unsigned long long* acc /* committed, pending, pending_csum, digest */,
                                           uint32_t* pmin) {
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t mn = kInfBits;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const gpq_item e = arr[i];
    pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
    pend += 1;
    mn = min(mn, gpq_f2u(e.ts));
  }
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < d.L; lp += stride) {
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

static __global__ void gaq_initial_kernel(gpq_phold_params p, uint32_t L, uint32_t per_lp, const gpq_item* src,
                                          gpq_item* out, uint32_t* kminmax) {
  uint32_t mn = 0xffffffffu, mx = 0;
  const uint64_t n = (uint64_t)L * per_lp;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t lp = (uint32_t)(i / per_lp), k = (uint32_t)(i % per_lp);
    gpq_item e = src ? src[i] : gpq_phold_initial(p, lp, k, per_lp);
    out[i] = e;
    mn = min(mn, gpq_f2u(e.ts));
    mx = max(mx, gpq_f2u(e.ts));
  }
  mn = warp_min_u32(mn);
  mx = __reduce_max_sync(GPQ_FULL_MASK, mx);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&kminmax[0], mn);
    atomicMax(&kminmax[1], mx);
  }
}

static __global__ void gaq_zero_stats_kernel(PholdDev d) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < d.L; lp += gridDim.x * blockDim.x) {
    d.count[lp] = 0;
    d.csum[lp] = 0;
    d.ohash[lp] = 0;
  }
}
