// Many PHOLD instances in one persistent launch (batched and served PHOLD).
//
// The instances share one LP space: instance i owns LPs [lp0_i, lp0_i + L_i) of the
// local array queues (src/local_array_queue.cu as rebuilt in laq.cuh), and every LP
// knows its instance (lp_inst).  All instances advance together, one window per grid
// barrier, but each with its own window: LP lp of instance i drains the events below
// min_i + lookahead_i (and end_time_i), where min_i is instance i's minimum from the
// previous window (src/des.cu:154-214 per instance).  An instance whose minimum reached
// its end time is finished and its LPs are skipped until the host collects it.
//
// A lane group of G lanes handles one LP per turn: merge the children of the previous
// window into the ring (laq_merge), then drain the safe prefix G events at a time, each
// lane processing one event (hashes, child, insert) -- the one-pass form of the single
// instance engine, with the instance's parameters looked up per LP.
#pragma once

#include "laq.cuh"

struct PmInstDev {
  gpq_phold_params p;  // num_lps = L_i
  uint32_t lp0;
  uint32_t per_lp;     // initial events per LP
  uint32_t err;
  uint32_t windows;    // windows this instance took part in
  uint32_t w0;         // its first window; it runs windows [w0, w0 + windows)
  uint32_t aux;        // bucketed sessions: 1 / bucket width of the run (float bits)
};

struct PmCtl {
  uint32_t err;
  uint32_t phase;    // next window
  unsigned long long bar;
};

struct PmDev {
  PmInstDev* inst;
  uint32_t* mins;        // [max_inst][3] window minimum slots (float bits)
  uint32_t* errs;        // [max_inst][3] error seen in the window before (slots like mins)
  const uint8_t* on;     // slot in use
  uint32_t n_inst;       // slots [0, n_inst) may be in use
  uint32_t* lp_inst;     // [n_lps] owning slot, ~0u when free
  uint32_t n_lps;        // LPs [0, n_lps) may be in use
  gpq_item* ring;        // [max_lps << cap_log2]
  uint32_t* rd;
  uint32_t* wr;
  uint32_t cap_log2;
  gpq_item* ibuf;        // [2][max_lps][ibc]
  uint32_t* icnt;        // [2][max_lps]
  uint32_t ibc;
  uint32_t max_lps;
  uint32_t* count;
  unsigned long long* csum;
  unsigned long long* ohash;
  PmCtl* ctl;
  uint64_t spin_limit;
};

// Instance i runs window s: in use, minimum below its end time, no error in window s - 1.
// Every block decides from the same slots, written before the last grid barrier.
__device__ __forceinline__ bool pm_active(const PmDev& d, uint32_t i, uint32_t s) {
  return d.on[i] && gpq_u2f(ld_relaxed_u32(&d.mins[3 * i + s % 3u])) < d.inst[i].p.end_time &&
         ld_relaxed_u32(&d.errs[3 * i + s % 3u]) == 0u;
}

__device__ __forceinline__ void pm_error(const PmDev& d, uint32_t inst, uint32_t s, uint32_t code) {
  gpq_set_error(&d.inst[inst].err, code);
  atomicOr(&d.errs[3 * inst + (s + 1u) % 3u], 1u);
}

// One LP of one window (all lanes of the group).  Returns nothing; folds the LP's next
// minimum into the instance's slot for window s + 1 through the warp-level reduction.
template <int G>
__device__ __forceinline__ void pm_lp_window(const PmDev& d, uint32_t lp, uint32_t s, const LaqGroupSmem& sm,
                                             const LaneGroup<G>& g) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t inst = ~0u, vmin = kInfBits;
  if (lp < d.n_lps) inst = d.lp_inst[lp];
  bool run = inst != ~0u;
  float m = 0.f, T = 0.f;
  PmInstDev* Ip = nullptr;
  if (run) {
    Ip = d.inst + inst;
    m = gpq_u2f(ld_relaxed_u32(&d.mins[3 * inst + s % 3u]));
    T = Ip->p.end_time;
    run = d.on[inst] && m < T && ld_relaxed_u32(&d.errs[3 * inst + s % 3u]) == 0u;
  }
  if (run) {
    const gpq_phold_params p = Ip->p;
    const uint32_t lp0 = Ip->lp0;
    const float bound = GPQ_FADD(m, p.lookahead);
    const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
    const uint32_t cap = 1u << d.cap_log2, mask = cap - 1u;
    gpq_item* ring = d.ring + ((size_t)lp << d.cap_log2);
    const uint32_t rd = d.rd[lp];
    uint32_t n = d.wr[lp] - rd;
    uint32_t k = d.icnt[(size_t)prevb * d.max_lps + lp];
    bool head_in_smem = false;
    if (k > 0) {
      if (k > d.ibc) k = d.ibc;  // overflow was flagged by the inserter
      if (n + k > cap) {
        if (g.gl == 0) pm_error(d, inst, s, GPQ_ERR_QUEUE_FULL);
        k = cap - n;
      }
      head_in_smem = laq_merge<G>(ring, mask, rd, n, d.ibuf + ((size_t)prevb * d.max_lps + lp) * d.ibc, k, sm, g);
      n += k;
      if (g.gl == 0) {
        d.wr[lp] = rd + n;
        d.icnt[(size_t)prevb * d.max_lps + lp] = 0;
      }
    }
    const uint32_t c0 = d.count[lp];
    uint64_t cs = 0, oh = 0;
    uint32_t done = 0, head = kInfBits, cmin = kInfBits;
    while (done < n) {
      const uint32_t i = done + g.gl;
      gpq_item e;
      bool safe = false;
      if (i < n) {
        e = (head_in_smem && i < (uint32_t)G) ? sm.head[i] : ring[(rd + i) & mask];
        safe = (e.ts < bound) && (e.ts < T);
      }
      const uint32_t c = __popc(g.ballot(safe));  // the run is sorted: a prefix is safe
      if (safe) {
        const uint32_t tb = gpq_f2u(e.ts);
        const uint64_t h = gpq_ev_hash(e.id, tb);
        cs += h;
        oh += gpq_seq_hash(h, (uint64_t)c0 + i);
        gpq_item pe = e;
        pe.lp = lp - lp0;
        gpq_item ch = gpq_phold_child(p, pe);
        ch.lp += lp0;
        const uint32_t pos = atomicAdd(&d.icnt[(size_t)curb * d.max_lps + ch.lp], 1u);
        if (pos < d.ibc) d.ibuf[((size_t)curb * d.max_lps + ch.lp) * d.ibc + pos] = ch;
        else pm_error(d, inst, s, GPQ_ERR_INSERT_FULL);
        cmin = min(cmin, gpq_f2u(ch.ts));
      }
      if (c < (uint32_t)G) {
        head = g.shfl((i < n) ? gpq_f2u(e.ts) : kInfBits, c);
        done += c;
        break;
      }
      done += G;
    }
    cs = g.sum(cs);
    oh = g.sum(oh);
    if (g.gl == 0 && done > 0) {
      d.count[lp] = c0 + done;
      d.csum[lp] += cs;
      d.ohash[lp] += oh;
      d.rd[lp] = rd + done;
    }
    vmin = min(head, g.umin(cmin));
  } else {
    inst = ~0u;
  }
  // one atomic per instance per warp
  const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, inst);
  const uint32_t red = __reduce_min_sync(peers, vmin);
  if (inst != ~0u && lane == (uint32_t)(__ffs(peers) - 1) && red != kInfBits)
    atomicMin(&d.mins[3 * inst + (s + 1u) % 3u], red);
}

// Windows s0, s0 + 1, ... while some instance is running, at most step_windows of them
// (0 = no limit).  Dynamic shared memory: laq_group_smem_bytes(ibc, G) per lane group.
template <int G>
static __global__ void __launch_bounds__(256, 4) pm_persistent_kernel(PmDev d, uint32_t s0, uint32_t step_windows) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_any;
  const LaneGroup<G> g;
  const uint32_t gib = threadIdx.x / G, gpb = blockDim.x / G;
  const LaqGroupSmem sm = laq_group_smem(smem_raw + (size_t)gib * laq_group_smem_bytes(d.ibc, G), d.ibc, G);
  const uint32_t ngroups = gridDim.x * gpb;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  unsigned long long target = 0;
  uint32_t s = s0;
  for (;; ++s) {
    // every block takes the same decision from the same slots
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    int any = 0;
    for (uint32_t i = threadIdx.x; i < d.n_inst && !any; i += blockDim.x) any = pm_active(d, i, s);
    if (any) s_any = 1;
    __syncthreads();
    if (!s_any || ld_relaxed_u32(&d.ctl->err) != 0u || (step_windows && s - s0 >= step_windows)) break;
    for (uint32_t i = tid; i < d.n_inst; i += nthreads) {
      if (pm_active(d, i, s)) d.inst[i].windows += 1u;
      d.mins[3 * i + (s + 2u) % 3u] = kInfBits;  // slots of window s + 2, last read in window s - 1
      d.errs[3 * i + (s + 2u) % 3u] = 0u;
    }
    // LPs in lane-group turns; the loop bound is uniform per warp
    const uint32_t turns = (d.n_lps + ngroups - 1) / ngroups;
    for (uint32_t r = 0; r < turns; ++r) pm_lp_window<G>(d, r * ngroups + blockIdx.x * gpb + gib, s, sm, g);
    target += gridDim.x;
    if (!grid_barrier(&d.ctl->bar, target, d.spin_limit, &d.ctl->err)) {
      s += 1u;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctl->phase = s;
}

// Initial events of the instances in list[0, n): one warp per LP of each, sorted into
// the ring (ids lp * per_lp + k over local LPs), per-LP outputs zeroed, the instance's
// first minimum into its slot for window s.  blockIdx.y = position in the list.
// Dynamic shared memory: per_lp items and keys per warp.
static __global__ void pm_populate_kernel(PmDev d, const uint32_t* list, uint32_t s) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t inst = list[blockIdx.y];
  const PmInstDev I = d.inst[inst];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const uint32_t P = I.per_lp;
  gpq_item* s_it = reinterpret_cast<gpq_item*>(smem_raw) + (size_t)wib * P;
  uint64_t* s_key = reinterpret_cast<uint64_t*>(reinterpret_cast<gpq_item*>(smem_raw) + (size_t)wpb * P) + (size_t)wib * P;
  for (uint32_t l = blockIdx.x * wpb + wib; l < I.p.num_lps; l += gridDim.x * wpb) {
    const uint32_t lp = I.lp0 + l;
    gpq_item* ring = d.ring + ((size_t)lp << d.cap_log2);
    uint32_t mn = kInfBits;
    for (uint32_t j = lane; j < P; j += 32) {
      const gpq_item e = gpq_phold_initial(I.p, l, j, P);
      s_it[j] = e;
      s_key[j] = gpq_lp_key(e);
      mn = min(mn, gpq_f2u(e.ts));
    }
    __syncwarp();
    for (uint32_t j = lane; j < P; j += 32) {
      const uint64_t kj = s_key[j];
      uint32_t r = 0;  // rank among the LP's initial events
      for (uint32_t i = 0; i < P; ++i) r += s_key[i] < kj ? 1u : 0u;
      gpq_item e = s_it[j];
      e.lp = lp;
      ring[r] = e;
    }
    __syncwarp();
    mn = warp_min_u32(mn);
    if (lane == 0) {
      d.rd[lp] = 0;
      d.wr[lp] = P;
      d.icnt[lp] = 0;
      d.icnt[(size_t)d.max_lps + lp] = 0;
      d.count[lp] = 0;
      d.csum[lp] = 0;
      d.ohash[lp] = 0;
      d.lp_inst[lp] = inst;
      if (mn != kInfBits) atomicMin(&d.mins[3 * inst + s % 3u], mn);
    }
  }
}

// Results of the finished instances in list[0, n): committed count, pending events (ring
// contents and the unmerged children of the instance's last window), the digest over
// local LP numbers, the pending minimum.  blockIdx.y = position in the list.
struct PmAcc {
  unsigned long long committed, pending, pending_csum, digest;
  uint32_t pending_min;
  uint32_t pad;
};

static __global__ void pm_finalize_kernel(PmDev d, const uint32_t* list, PmAcc* acc) {
  const uint32_t j = blockIdx.y;
  const PmInstDev I = d.inst[list[j]];
  const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
  const uint32_t s = I.w0 + I.windows;  // the instance's first inactive window
  const uint32_t prevb = (s + 1u) & 1u;
  const uint32_t mask = (1u << d.cap_log2) - 1u;
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t pmin = kInfBits;
  for (uint32_t l = blockIdx.x * wpb + (threadIdx.x >> 5); l < I.p.num_lps; l += gridDim.x * wpb) {
    const uint32_t lp = I.lp0 + l;
    const gpq_item* ring = d.ring + ((size_t)lp << d.cap_log2);
    const uint32_t rd = d.rd[lp], n = d.wr[lp] - rd;
    for (uint32_t q = lane; q < n; q += 32) {
      const gpq_item e = ring[(rd + q) & mask];
      pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
      pend += 1;
      pmin = min(pmin, gpq_f2u(e.ts));
    }
    const uint32_t k = min(d.icnt[(size_t)prevb * d.max_lps + lp], d.ibc);
    const gpq_item* src = d.ibuf + ((size_t)prevb * d.max_lps + lp) * d.ibc;
    for (uint32_t q = lane; q < k; q += 32) {
      const gpq_item e = src[q];
      pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
      pend += 1;
      pmin = min(pmin, gpq_f2u(e.ts));
    }
    if (lane == 0) {
      const uint32_t c = d.count[lp];
      com += c;
      dig += gpq_mix64(gpq_mix64(gpq_mix64(((uint64_t)l << 32) | c) ^ d.csum[lp]) + d.ohash[lp]);
    }
  }
  pend = warp_sum_u64(pend);
  pcs = warp_sum_u64(pcs);
  dig = warp_sum_u64(dig);
  com = warp_sum_u64(com);
  pmin = warp_min_u32(pmin);
  if (lane == 0) {
    atomicAdd(&acc[j].pending, (unsigned long long)pend);
    atomicAdd(&acc[j].pending_csum, (unsigned long long)pcs);
    atomicAdd(&acc[j].digest, (unsigned long long)dig);
    atomicAdd(&acc[j].committed, (unsigned long long)com);
    atomicMin(&acc[j].pending_min, pmin);
  }
}

// Slots in use whose run ended (minimum at or past the end time, or an error) at window s.
static __global__ void pm_done_list_kernel(PmDev d, uint32_t s, uint32_t* out, uint32_t* out_n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n_inst; i += gridDim.x * blockDim.x)
    if (d.on[i] && !pm_active(d, i, s)) out[atomicAdd(out_n, 1u)] = i;
}

// Release the LPs of the instances in list[0, n).
static __global__ void pm_release_kernel(PmDev d, const uint32_t* list) {
  const PmInstDev I = d.inst[list[blockIdx.y]];
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < I.p.num_lps; l += gridDim.x * blockDim.x)
    d.lp_inst[I.lp0 + l] = ~0u;
}
