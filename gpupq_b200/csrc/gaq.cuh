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

#include "bulk_copy.cuh"
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

// Exclusive scan of `total` counts from `in` into `out` plus `add` (in == out allowed), by
// one CTA: each thread owns a contiguous run of ceil(total / blockDim) entries, sums it,
// the CTA scans the per-thread sums (warp shuffles + one round over the warp totals), and
// each thread writes its run.  Returns the total (without `add`).
__device__ __forceinline__ uint32_t rs_scan_into(const uint32_t* in, uint32_t* out, uint32_t total, uint32_t add) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t s_all;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t per = (total + blockDim.x - 1) / blockDim.x;
  const uint32_t b0 = min(t * per, total), b1 = min(b0 + per, total);
  uint32_t sum = 0;
  for (uint32_t i = b0; i < b1; ++i) sum += in[i];
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(GPQ_FULL_MASK, incl, o);
    if (lane >= (uint32_t)o) incl += u;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = blockDim.x >> 5;
    const uint32_t v = lane < nw ? wsum[lane] : 0u;
    uint32_t wi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(GPQ_FULL_MASK, wi, o);
      if (lane >= (uint32_t)o) wi += u;
    }
    if (lane < nw) wsum[lane] = wi - v;
    if (lane == nw - 1) s_all = wi;
  }
  __syncthreads();
  uint32_t run = add + wsum[warp] + incl - sum;
  for (uint32_t i = b0; i < b1; ++i) {
    const uint32_t v = in[i];
    out[i] = run;
    run += v;
  }
  const uint32_t all = s_all;
  __syncthreads();
  return all;
}

__device__ __forceinline__ uint32_t rs_scan_block(uint32_t* a, uint32_t total) { return rs_scan_into(a, a, total, 0u); }

static __global__ void rs_scan_kernel(uint32_t* a, uint32_t total) { rs_scan_block(a, total); }

// Device-wide exclusive scan in three kernels (gpq::scan_exclusive): chunk sums, one CTA
// over the sums, then every chunk scanned from its base.
static constexpr uint32_t kScanChunk = 4096;

static __global__ void __launch_bounds__(1024) rs_chunk_sum_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                                   uint32_t* sums) {
  __shared__ uint32_t wsum[32];
  const uint64_t c0 = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t s = 0;
  for (uint32_t k = threadIdx.x; k < kScanChunk; k += blockDim.x)
    if (c0 + k < n) s += in[c0 + k];
  s = __reduce_add_sync(GPQ_FULL_MASK, s);
  if ((threadIdx.x & 31u) == 0) wsum[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < (blockDim.x >> 5) ? wsum[threadIdx.x] : 0u;
    v = __reduce_add_sync(GPQ_FULL_MASK, v);
    if (threadIdx.x == 0) sums[blockIdx.x] = v;
  }
}

static __global__ void __launch_bounds__(1024) rs_chunk_scan_kernel(const uint32_t* in, uint32_t* out, uint32_t n,
                                                                    const uint32_t* __restrict__ base) {
  const uint64_t c0 = (uint64_t)blockIdx.x * kScanChunk;
  const uint64_t rest = (uint64_t)n - c0;
  rs_scan_into(in + c0, out + c0, (uint32_t)(rest < kScanChunk ? rest : kScanChunk), base[blockIdx.x]);
}

// Stable scatter of one tile through shared memory.  Warp w owns the tile's items
// [w * 512, (w + 1) * 512); they arrive in shared memory with one TMA bulk copy per warp
// (issued by its lane 0, completed on the warp's own mbarrier, while the CTA scans the
// tile's digit counts), so each warp starts ranking as soon as its own 8 KB land.  It
// ranks them without block barriers: an item's rank among the same-digit items of its warp
// is the warp's running count for the digit (warp-private counters, one leader lane per
// group of equal digits updates it) plus the lower lanes of its round with that digit.
// After one barrier, a digit's items of warp w start at the tile's start for the digit
// (exclusive scan of the tile's counts) plus the counts of warps 0..w-1, which keeps the
// tile order.  The tile is laid out in digit order in shared memory and written so that
// consecutive threads write consecutive addresses of each digit's run: an item at shared
// position k with digit d goes to off[d][tile] + k - (start of d in the tile).
static constexpr uint32_t kRsWarps = kRsThreads / 32;
static constexpr uint32_t kRsWarpItems = kRsTile / kRsWarps;

static __global__ void __launch_bounds__(kRsThreads) rs_scatter_kernel(const gpq_item* __restrict__ in, gpq_item* out,
                                                                       uint32_t n, uint32_t kmin, uint32_t shift,
                                                                       const uint32_t* __restrict__ cnt,
                                                                       const uint32_t* __restrict__ off, uint32_t ntiles,
                                                                       uint32_t* err) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  gpq_item* s_it = reinterpret_cast<gpq_item*>(rs_smem);  // [kRsTile]: the input tile, then the output layout
  __shared__ uint32_t gpos[256], wtot[kRsWarps];
  __shared__ uint32_t wc[kRsWarps][256];  // per-warp digit counts, then the warp's start per digit
  __shared__ __align__(8) uint64_t bar[kRsWarps];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t tile = blockIdx.x;
  const uint32_t t0 = tile * kRsTile;
  const uint32_t tn = min(kRsTile, n - t0);
  const uint32_t w0 = min(warp * kRsWarpItems, tn), wn = min(tn - w0, kRsWarpItems);  // this warp's items
  if (lane == 0) {
    mbar_init(&bar[warp]);
    mbar_arrive_expect_tx(&bar[warp], wn * (uint32_t)sizeof(gpq_item));
    if (wn) bulk_g2s(s_it + w0, in + t0 + w0, wn * (uint32_t)sizeof(gpq_item), &bar[warp]);
  }
  const uint32_t base = t0 + warp * kRsWarpItems;
  for (uint32_t d = lane; d < 256; d += 32) wc[warp][d] = 0;
  // the tile's digit runs: exclusive scan of its counts (thread t = digit t)
  const uint32_t c = cnt[(size_t)t * ntiles + tile];
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(GPQ_FULL_MASK, incl, o);
    if (lane >= (uint32_t)o) incl += u;
  }
  if (lane == 31) wtot[warp] = incl;
  __syncwarp();
  const bool arrived = mbar_wait_bounded(&bar[warp], 0, err);
  gpq_item ev[kRsPer];
#pragma unroll
  for (uint32_t j = 0; j < kRsPer; ++j) {
    const uint32_t k = warp * kRsWarpItems + j * 32 + lane;
    if (k < tn) ev[j] = s_it[k];
  }
  // warp-private ranks
  uint32_t rk[kRsPer];
#pragma unroll
  for (uint32_t j = 0; j < kRsPer; ++j) {
    const bool valid = base + j * 32 + lane < n;
    const uint32_t dgt = valid ? rs_digit(ev[j], kmin, shift) : 0u;
    const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, valid ? dgt : (0x100u + lane));
    const uint32_t before = valid ? wc[warp][dgt] : 0u;
    rk[j] = before + __popc(peers & ((1u << lane) - 1u));
    __syncwarp();
    if (valid && lane == (uint32_t)(__ffs(peers) - 1)) wc[warp][dgt] = before + __popc(peers);
    __syncwarp();
  }
  if (!__syncthreads_and(arrived)) return;  // a staging copy did not complete: skip the tile (error recorded)
  // thread t = digit t: the tile's start for t, then each warp's start
  uint32_t wbase = 0;
  for (uint32_t w = 0; w < warp; ++w) wbase += wtot[w];
  uint32_t pos = wbase + incl - c;
  gpos[t] = off[(size_t)t * ntiles + tile] - pos;  // modulo 2^32; + k gives the output index
#pragma unroll
  for (uint32_t w = 0; w < kRsWarps; ++w) {
    const uint32_t k = wc[w][t];
    wc[w][t] = pos;
    pos += k;
  }
  __syncthreads();
#pragma unroll
  for (uint32_t j = 0; j < kRsPer; ++j)
    if (base + j * 32 + lane < n) s_it[wc[warp][rs_digit(ev[j], kmin, shift)] + rk[j]] = ev[j];
  __syncthreads();
  for (uint32_t k = t; k < tn; k += kRsThreads) {
    const gpq_item e = s_it[k];
    out[gpos[rs_digit(e, kmin, shift)] + k] = e;
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

// Merge-path splits of merge(A, B): split[b] = A items among the first b * kMpTile outputs,
// one thread per tile boundary (all searches at once, in their own pass).
static __global__ void mp_splits_kernel(const gpq_item* __restrict__ A, uint32_t na, const gpq_item* __restrict__ B,
                                        uint32_t nb, uint32_t* split) {
  const uint32_t total = na + nb;
  const uint32_t tiles = (total + kMpTile - 1) / kMpTile;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= tiles; b += gridDim.x * blockDim.x)
    split[b] = mp_search(A, na, B, nb, min(b * kMpTile, total));
}

// Stages A[a0, a0 + la) and B[b0, b0 + lb) at s[0, la) and s[la, la + lb) with TMA bulk
// copies issued by thread 0; all threads.  Returns false (for every thread) if the copies
// did not complete within the bound.
__device__ __forceinline__ bool mp_stage_inputs(gpq_item* s, const gpq_item* A, uint32_t a0, uint32_t la,
                                                const gpq_item* B, uint32_t b0, uint32_t lb, uint64_t* bar,
                                                uint32_t* err) {
  if (threadIdx.x == 0) mbar_init(bar);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(bar, (la + lb) * (uint32_t)sizeof(gpq_item));
    if (la) bulk_g2s(s, A + a0, la * (uint32_t)sizeof(gpq_item), bar);
    if (lb) bulk_g2s(s + la, B + b0, lb * (uint32_t)sizeof(gpq_item), bar);
  }
  return __syncthreads_and(mbar_wait_bounded(bar, 0, err)) != 0;
}

// Shared-memory slot of key j in the merge's key array: one pad word per 32 keys, so that
// the lanes of a warp, kMpPer keys apart, read 32 different banks.
__device__ __forceinline__ uint32_t mp_kp(uint32_t j) { return j + (j >> 5); }

// mp_search over the padded keys k (A = keys [0, na), B = keys [na, na + nb)).
__device__ __forceinline__ uint32_t mp_search_keys(const uint32_t* k, uint32_t na, uint32_t nb, uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0u, hi = min(diag, na);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (k[mp_kp(mid)] <= k[mp_kp(na + diag - 1 - mid)]) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Merges the staged s[0, la) and s[la, la + lb) (A first on ties) into out[0, la + lb).
// The merge runs on the timestamp keys, copied into a padded array (each thread's kMpPer
// outputs are consecutive, so the lanes' positions are kMpPer keys apart; items read at
// that stride would all fall in one bank group), and produces only the source slot of
// each output; the CTA then writes the tile in output order, each thread gathering its
// items from the staged inputs.  All threads (kMpThreads).
__device__ __forceinline__ void mp_merge_tile(const gpq_item* s, uint32_t la, uint32_t lb, uint32_t* kp, uint16_t* src,
                                              gpq_item* out) {
  const uint32_t len = la + lb;
  for (uint32_t j = threadIdx.x; j < len; j += kMpThreads) kp[mp_kp(j)] = gpq_f2u(s[j].ts);
  __syncthreads();
  const uint32_t my0 = threadIdx.x * kMpPer;
  if (my0 < len) {
    uint32_t ia = mp_search_keys(kp, la, lb, my0);
    uint32_t ib = my0 - ia;
    uint32_t ka = ia < la ? kp[mp_kp(ia)] : 0u, kb = ib < lb ? kp[mp_kp(la + ib)] : 0u;
#pragma unroll
    for (uint32_t k = 0; k < kMpPer; ++k) {
      if (my0 + k < len) {
        if (ib >= lb || (ia < la && ka <= kb)) {
          src[my0 + k] = (uint16_t)ia;
          if (++ia < la) ka = kp[mp_kp(ia)];
        } else {
          src[my0 + k] = (uint16_t)(la + ib);
          if (++ib < lb) kb = kp[mp_kp(la + ib)];
        }
      }
    }
  }
  __syncthreads();
  for (uint32_t x = threadIdx.x; x < len; x += kMpThreads) out[x] = s[src[x]];
}

// Merge path: CTA b writes outputs [b*kMpTile, (b+1)*kMpTile) of merge(A, B), its inputs
// located by the precomputed splits and staged by TMA.
static __global__ void mp_merge_kernel(const gpq_item* __restrict__ A, uint32_t na, const gpq_item* __restrict__ B,
                                       uint32_t nb, gpq_item* out, const uint32_t* __restrict__ split, uint32_t* err) {
  __shared__ __align__(16) gpq_item s[kMpTile];
  __shared__ uint32_t kp[kMpTile + kMpTile / 32];
  __shared__ uint16_t src[kMpTile];
  __shared__ __align__(8) uint64_t bar;
  static_assert(kMpTile <= 65536, "source slots are 16 bits wide");
  const uint32_t total = na + nb;
  const uint32_t d0 = blockIdx.x * kMpTile;
  const uint32_t d1 = min(d0 + kMpTile, total);
  const uint32_t a0 = split[blockIdx.x], a1 = split[blockIdx.x + 1];
  const uint32_t b0 = d0 - a0, b1 = d1 - a1;
  const uint32_t la = a1 - a0, lb = b1 - b0;
  if (!mp_stage_inputs(s, A, a0, la, B, b0, lb, &bar, err)) return;
  mp_merge_tile(s, la, lb, kp, src, out + d0);
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
                                        uint32_t* err, const uint32_t* gate = nullptr) {
  if (gate && !*gate) return;
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
static __global__ void gaq_process_kernel(PholdDev d, GaqDev g, uint32_t* err, const uint32_t* gate = nullptr) {
  if (gate && !*gate) return;
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

// ---- the window loop as a replayable sequence (CUDA graph) ----
//
// The host-driven loop reads the head and the child key range back every window.  Here
// every size lives in device memory (GaqWin): the first kernel of a window decides
// whether it runs (gate), finds the safe prefix, and the later kernels -- launched with
// grids sized for the largest array -- read their sizes and exit early.  One window is
// captured once into a CUDA graph and replayed many times between host checks; windows
// replayed after the end are no-ops.

// The window loop sorts each window's children with smaller radix tiles than the bulk
// sort (more CTAs for a few hundred thousand items).
static constexpr uint32_t kWinRsPer = 4;
static constexpr uint32_t kWinRsTile = kRsThreads * kWinRsPer;

struct GaqWin {
  uint32_t c, nc, kmin, kmax;   // as GaqDev::info: prefix length, children, child key range
  uint32_t n, cur, passes, ntiles;
  uint32_t gate;                // this window runs
  uint32_t done;                // the minimum reached the end time (or an error stopped the run)
  uint32_t windows;             // windows executed
  uint32_t stop_at;             // do not start window number stop_at (pause)
  uint32_t total, pad[3];
};

// One CTA: the safe prefix by a multi-way search -- the answer lies in [lo, hi] (items
// before lo are below the limit, items from hi on are not); every round each thread
// probes one position of [lo, hi), probes below the limit raise lo past them, the others
// lower hi to them, so the range shrinks by about blockDim each round.
static __global__ void gaq_win_begin_kernel(const gpq_item* arr0, const gpq_item* arr1, GaqWin* w, float la, float T,
                                            const uint32_t* err) {
  __shared__ uint32_t s_run, s_lo, s_hi, s_lim;
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    if (!w->done) {
      if (*err) w->done = 1;
      else if (w->windows < w->stop_at) {
        const gpq_item* a = w->cur ? arr1 : arr0;
        if (w->n == 0 || !(a[0].ts < T)) w->done = 1;
        else {
          run = 1;
          s_lim = min(gpq_f2u(GPQ_FADD(a[0].ts, la)), gpq_f2u(T));
        }
      }
    }
    s_run = run;
    s_lo = 0;
    s_hi = w->n;
  }
  __syncthreads();
  if (!s_run) {
    if (threadIdx.x == 0) w->gate = 0;
    return;
  }
  const gpq_item* a = w->cur ? arr1 : arr0;
  const uint32_t lim = s_lim;
  for (;;) {
    const uint32_t lo = s_lo, hi = s_hi;
    __syncthreads();  // everyone has read the range before it changes
    if (lo >= hi) break;
    const uint32_t pos = lo + (uint32_t)(((uint64_t)(hi - lo) * threadIdx.x) / blockDim.x);
    if (gpq_f2u(a[pos].ts) < lim) atomicMax(&s_lo, pos + 1);
    else atomicMin(&s_hi, pos);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    w->c = s_lo;
    w->nc = 0;
    w->kmin = 0xffffffffu;
    w->kmax = 0;
    w->gate = 1;
    w->windows += 1;
  }
}

// The stage kernel takes the array through a pointer chosen by the window's buffer.
static __global__ void gaq_win_stage_kernel(const gpq_item* arr0, const gpq_item* arr1, GaqWin* w, GaqDev g,
                                            uint32_t L, uint32_t* err) {
  if (!w->gate) return;
  const gpq_item* a = w->cur ? arr1 : arr0;
  const uint32_t c = w->c;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const gpq_item e = a[i];
    if (e.lp >= L) { gpq_set_error(err, GPQ_ERR_INVALID); continue; }
    const uint32_t slot = atomicAdd(&g.stg_cnt[e.lp], 1u);
    if (slot < g.ibc) g.stg[(size_t)e.lp * g.ibc + slot] = e;
    else gpq_set_error(err, GPQ_ERR_INSERT_FULL);
  }
}

static __global__ void gaq_win_sort_setup_kernel(GaqWin* w, uint32_t cap, uint32_t ch_cap, uint32_t* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || !w->gate) return;
  const uint32_t nc = min(w->nc, ch_cap);
  w->nc = nc;
  uint32_t passes = 0;
  if (nc > 1 && w->kmax > w->kmin) passes = (32u - __clz(w->kmax - w->kmin) + 7u) / 8u;
  w->passes = passes;
  w->ntiles = (nc + kWinRsTile - 1) / kWinRsTile;
  const uint64_t total = (uint64_t)w->n - w->c + nc;
  if (total > cap) {
    gpq_set_error(err, GPQ_ERR_QUEUE_FULL);
    w->gate = 0;
    w->done = 1;
    return;
  }
  w->total = (uint32_t)total;
}

__device__ __forceinline__ bool gaq_win_pass(const GaqWin* w, uint32_t p) { return w->gate && p < w->passes; }

static __global__ void gaq_win_hist_kernel(const gpq_item* ch, const gpq_item* ch_tmp, const GaqWin* w, uint32_t p,
                                           uint32_t* hist) {
  if (!gaq_win_pass(w, p) || blockIdx.x >= w->ntiles) return;
  __shared__ uint32_t cnt[256];
  const gpq_item* in = (p & 1u) ? ch_tmp : ch;
  const uint32_t tile = blockIdx.x, ntiles = w->ntiles, n = w->nc, kmin = w->kmin, shift = 8u * p;
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = tile * kWinRsTile;
  for (uint32_t j = 0; j < kWinRsPer; ++j) {
    const uint32_t i = base + j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[rs_digit(in[i], kmin, shift)], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + tile] = cnt[threadIdx.x];
}

// The digit offsets of a pass on many CTAs: block d scans digit d's counts across the
// tiles (hist[d * ntiles + tile], exclusive) and leaves the digit's total in dig[d]; then
// one CTA turns dig into exclusive digit offsets.  The scatter adds both.
static __global__ void gaq_win_rowscan_kernel(const GaqWin* w, uint32_t p, uint32_t* hist, uint32_t* dig) {
  if (!gaq_win_pass(w, p)) return;
  const uint32_t ntiles = w->ntiles;
  const uint32_t tot = rs_scan_block(hist + (size_t)blockIdx.x * ntiles, ntiles);
  if (threadIdx.x == 0) dig[blockIdx.x] = tot;
}

static __global__ void gaq_win_digscan_kernel(const GaqWin* w, uint32_t p, uint32_t* dig) {
  if (!gaq_win_pass(w, p)) return;
  rs_scan_block(dig, 256u);
}

static __global__ void gaq_win_scatter_kernel(gpq_item* ch, gpq_item* ch_tmp, const GaqWin* w, uint32_t p,
                                              const uint32_t* __restrict__ off, const uint32_t* __restrict__ dig) {
  if (!gaq_win_pass(w, p) || blockIdx.x >= w->ntiles) return;
  __shared__ uint32_t run[256];
  __shared__ uint32_t wc[kRsThreads / 32][256];
  const gpq_item* in = (p & 1u) ? ch_tmp : ch;
  gpq_item* out = (p & 1u) ? ch : ch_tmp;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t tile = blockIdx.x, ntiles = w->ntiles, n = w->nc, kmin = w->kmin, shift = 8u * p;
  run[t] = 0;
  const uint32_t base = tile * kWinRsTile;
  for (uint32_t j = 0; j < kWinRsPer; ++j) {
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
      for (uint32_t q = 0; q < warp; ++q) pre += wc[q][dgt];
      const uint32_t below = __popc(peers & ((1u << lane) - 1u));
      out[dig[dgt] + off[dgt * ntiles + tile] + run[dgt] + pre + below] = e;
    }
    __syncthreads();
    uint32_t sum = 0;
    for (uint32_t q = 0; q < kRsThreads / 32; ++q) sum += wc[q][t];
    run[t] += sum;
    __syncthreads();
  }
}

// Merge-path splits of the window's merge: split[b] = A items among the first b * kMpTile
// outputs, one thread per tile boundary (all searches at once).
__device__ __forceinline__ void gaq_win_merge_inputs(const gpq_item* arr0, const gpq_item* arr1, const gpq_item* ch,
                                                     const gpq_item* ch_tmp, const GaqWin* w, const gpq_item** A,
                                                     uint32_t* na, const gpq_item** B, uint32_t* nb) {
  *A = (w->cur ? arr1 : arr0) + w->c;
  *na = w->n - w->c;
  *B = (w->passes & 1u) ? ch_tmp : ch;
  *nb = w->nc;
}

static __global__ void gaq_win_splits_kernel(const gpq_item* arr0, const gpq_item* arr1, const gpq_item* ch,
                                             const gpq_item* ch_tmp, const GaqWin* w, uint32_t* split) {
  if (!w->gate) return;
  const uint32_t total = w->total;
  const uint32_t tiles = (total + kMpTile - 1) / kMpTile;
  const gpq_item *A, *B;
  uint32_t na, nb;
  gaq_win_merge_inputs(arr0, arr1, ch, ch_tmp, w, &A, &na, &B, &nb);
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= tiles; b += gridDim.x * blockDim.x)
    split[b] = mp_search(A, na, B, nb, min(b * kMpTile, total));
}

// Merge the array's unsafe suffix with the sorted children into the other buffer.
static __global__ void gaq_win_merge_kernel(gpq_item* arr0, gpq_item* arr1, const gpq_item* ch, const gpq_item* ch_tmp,
                                            const GaqWin* w, const uint32_t* __restrict__ split, uint32_t* err) {
  if (!w->gate) return;
  const uint32_t total = w->total;
  const uint32_t d0 = blockIdx.x * kMpTile;
  if (d0 >= total) return;
  const gpq_item *A, *B;
  uint32_t na, nb;
  gaq_win_merge_inputs(arr0, arr1, ch, ch_tmp, w, &A, &na, &B, &nb);
  gpq_item* out = w->cur ? arr0 : arr1;
  extern __shared__ __align__(16) unsigned char mp_smem[];
  gpq_item* s = reinterpret_cast<gpq_item*>(mp_smem);  // [kMpTile] inputs
  __shared__ uint32_t kp[kMpTile + kMpTile / 32];
  __shared__ uint16_t src[kMpTile];
  const uint32_t d1 = min(d0 + kMpTile, total);
  const uint32_t a0 = split[blockIdx.x], a1 = split[blockIdx.x + 1];
  const uint32_t b0 = d0 - a0, b1 = d1 - a1;
  const uint32_t la = a1 - a0, lb = b1 - b0;
  __shared__ __align__(8) uint64_t bar;
  if (!mp_stage_inputs(s, A, a0, la, B, b0, lb, &bar, err)) return;
  mp_merge_tile(s, la, lb, kp, src, out + d0);
}

static __global__ void gaq_win_end_kernel(GaqWin* w) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || !w->gate) return;
  w->n = w->total;
  w->cur ^= 1u;
}
