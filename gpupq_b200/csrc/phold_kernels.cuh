// PHOLD engine kernels over the per-LP queues (local array, local heap, local splay):
// population, one window per launch (plain loop, like the reference's des_run), all
// windows in one persistent launch, and the end-of-run reduction.  The window body is
// shared; the queue kind enters through a policy class (LaqPolicy, LhqPolicy,
// LsqPolicy) that merges/pushes one LP's new items and stages its safe events.
#pragma once

#include "laq.cuh"
#include "lhq.cuh"
#include "lsq.cuh"
#include "las.cuh"

// Union of the per-LP queue layouts (host-visible; kernels build the policy's view).
struct LpQueueDev {
  uint32_t kind;       // gpq_queue_kind
  uint32_t cap_log2;
  gpq_item* items;     // num_lps << cap_log2: LAQ ring / LHQ heap / LSQ node pool
  uint32_t* a;         // LAQ rd   | LHQ size | LSQ root
  uint32_t* b;         // LAQ wr   |          | LSQ size
  uint32_t* c;         //          |          | LSQ free-stack height
  uint32_t* links;     // LSQ link words
  uint16_t* freestk;   // LSQ free stacks
};

template <int G>
struct LaqP : LaqPolicy<G> {
  __device__ static LaqDev dev(const LpQueueDev& l) { return LaqDev{l.items, l.a, l.b, l.cap_log2}; }
};
template <int G>
struct LasP : LasPolicy<G> {
  __device__ static LaqDev dev(const LpQueueDev& l) { return LaqDev{l.items, l.a, l.b, l.cap_log2}; }
};
template <int G>
struct LhqP : LhqPolicy<G> {
  __device__ static LhqDev dev(const LpQueueDev& l) { return LhqDev{l.items, l.a, l.cap_log2}; }
};
struct LsqP : LsqPolicy {
  __device__ static LsqDev dev(const LpQueueDev& l) {
    return LsqDev{l.items, l.links, l.freestk, l.a, l.b, l.c, l.cap_log2};
  }
};

// Accumulators filled by the finalize kernel.
struct PholdAcc {
  unsigned long long committed;
  unsigned long long pending;
  unsigned long long pending_csum;
  unsigned long long digest;
  uint32_t pending_min;
  uint32_t pad[3];
};

// ---------------------------------------------------------------------------------
// Population (src/phold.cu:63-79,124-163): LP l receives events id = l*P + k.  One warp
// per LP ranks its P events in shared memory and writes them sorted to slots [0, P) of
// its item array (a sorted array is also a valid heap; for the splay queue the slots
// become a left-leaning chain whose root is the largest item).  `src` = NULL generates
// the events from the seed; otherwise src holds them grouped by LP (src[l*P + k]).
// Also computes the first window minimum into mins[0].
// ---------------------------------------------------------------------------------
static __global__ void phold_populate_kernel(PholdDev d, LpQueueDev q, uint32_t per_lp,
                                             const gpq_item* __restrict__ src) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t red[32];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t wpb = blockDim.x >> 5;
  gpq_item* s_it = reinterpret_cast<gpq_item*>(smem_raw) + (size_t)wib * per_lp;
  uint64_t* s_key = reinterpret_cast<uint64_t*>(reinterpret_cast<gpq_item*>(smem_raw) + (size_t)wpb * per_lp) +
                    (size_t)wib * per_lp;
  const uint32_t lp = d.lp_begin + blockIdx.x * wpb + wib;
  const uint32_t cap = 1u << q.cap_log2;
  uint32_t mn = kInfBits;
  if (lp < d.lp_end) {
    for (uint32_t j = lane; j < per_lp; j += 32) {
      gpq_item e;
      if (src) {
        e = src[(size_t)lp * per_lp + j];
        if (e.lp != lp) gpq_set_error(&d.ctrl->err, GPQ_ERR_INVALID);
        e.lp = lp;
      } else {
        e = gpq_phold_initial(d.p, lp, j, per_lp);
      }
      s_it[j] = e;
      s_key[j] = gpq_lp_key(e);
      mn = min(mn, gpq_f2u(e.ts));
    }
    __syncwarp();
    const size_t base = (size_t)lp << q.cap_log2;
    gpq_item* items = q.items + base;
    for (uint32_t j = lane; j < per_lp; j += 32) {
      const uint64_t kj = s_key[j];
      uint32_t r = 0;
      for (uint32_t i = 0; i < per_lp; ++i) r += (s_key[i] < kj) ? 1u : 0u;
      items[r] = s_it[j];
    }
    if (q.kind == GPQ_QUEUE_LSQ) {
      for (uint32_t j = lane; j < cap; j += 32) {
        if (j < per_lp) {
          q.links[base + j] = ((j == 0 ? kLsqNil : j - 1) << 16) | kLsqNil;
        } else {
          items[j].lp = 0xffffffffu;
          q.freestk[base + (j - per_lp)] = (uint16_t)j;
        }
      }
    }
    if (lane == 0) {
      if (q.kind == GPQ_QUEUE_LAQ) { q.a[lp] = 0; q.b[lp] = per_lp; }
      else if (q.kind == GPQ_QUEUE_LHQ) { q.a[lp] = per_lp; }
      else { q.a[lp] = per_lp - 1; q.b[lp] = per_lp; q.c[lp] = cap - per_lp; }
      d.count[lp] = 0;
      d.csum[lp] = 0;
      d.ohash[lp] = 0;
    }
  }
  mn = block_min_u32(mn, red);
  if (threadIdx.x == 0 && mn != kInfBits) atomicMin(&d.ctrl->mins[0], mn);
}

// Per-CTA staging of one super-round (shared memory): room for 8 safe events per LP on
// average; a lane group that finds the area full handles its events itself.
static constexpr uint32_t kStageRounds = 4;  // rounds (LPs per lane group) per super-round

__host__ __device__ inline uint32_t phold_stage_cap(uint32_t block, uint32_t group) {
  const uint32_t c = kStageRounds * (block / group) * 8u;
  return c < 512u ? 512u : (c > 2048u ? 2048u : c);
}

__host__ __device__ inline size_t phold_stage_smem_bytes(uint32_t block, uint32_t group) {
  const size_t slots = (size_t)kStageRounds * (block / group);
  return (size_t)phold_stage_cap(block, group) * 16 + slots * (8 + 8 + 4 + 4) + 16;
}

__host__ __device__ inline size_t phold_window_smem_bytes(uint32_t block, uint32_t group, size_t group_smem) {
  return (size_t)(block / group) * group_smem + phold_stage_smem_bytes(block, group);
}

// Shared body of one window for all LPs owned by this CTA.  The CTA's LPs are
// lp = blockIdx.x * gpb + gib + r * ngroups for rounds r = 0, 1, ...; they are handled
// in super-rounds of kStageRounds rounds, each in three passes:
//   A  every lane group merges and stages its LP of each round (lane-group parallel);
//   B  every thread of the CTA processes staged events (one event per thread);
//   C  per-LP checksums go back to global memory.
// Folds the CTA's minimum into mins[(s+1)%3].
template <class Q>
__device__ __forceinline__ void phold_window_body(const PholdDev& d, const typename Q::Dev& q, const InsDev& ib,
                                                  uint32_t s, float m, unsigned char* smem_raw, uint32_t* red) {
  constexpr int G = Q::G;
  const LaneGroup<G> g;
  const uint32_t gib = threadIdx.x / G;  // group in block
  const uint32_t gpb = blockDim.x / G;
  const size_t gbytes = Q::group_smem_bytes(ib.ibc);
  const typename Q::Smem sm = Q::smem(smem_raw + (size_t)gib * gbytes, ib.ibc);
  unsigned char* sbase = smem_raw + (size_t)gpb * gbytes;
  const uint32_t nslots = kStageRounds * gpb;
  const uint32_t stage_cap = phold_stage_cap(blockDim.x, G);
  PholdStage st;
  st.ev = reinterpret_cast<gpq_item*>(sbase);
  st.csum = reinterpret_cast<unsigned long long*>(sbase + (size_t)stage_cap * 16);
  st.ohash = st.csum + nslots;
  st.seq0 = reinterpret_cast<uint32_t*>(st.ohash + nslots);
  st.lp = st.seq0 + nslots;
  st.cnt = st.lp + nslots;
  st.cap = stage_cap;

  const float bound = GPQ_FADD(m, d.p.lookahead);
  uint32_t* err_slot = &d.ctrl->errs[(s + 1u) % 3u];
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const uint32_t ngroups = gridDim.x * gpb;
  const uint32_t first = d.lp_begin + blockIdx.x * gpb;
  uint32_t mn = kInfBits;
  for (uint32_t r0 = 0; first + r0 * ngroups < d.lp_end; r0 += kStageRounds) {
    if (threadIdx.x == 0) *st.cnt = 0;
    for (uint32_t t = threadIdx.x; t < nslots; t += blockDim.x) st.lp[t] = ~0u;
    __syncthreads();
    // A: merge + stage, one LP per lane group per round (metadata prefetched one round ahead)
    uint32_t lp = first + gib + r0 * ngroups;
    typename Q::Meta next;
    if (lp < d.lp_end) next = Q::load_meta(d, q, ib, lp, prevb);
    for (uint32_t r = 0; r < kStageRounds && lp < d.lp_end; ++r, lp += ngroups) {
      const typename Q::Meta cur = next;
      if (r + 1 < kStageRounds && lp + ngroups < d.lp_end) next = Q::load_meta(d, q, ib, lp + ngroups, prevb);
      mn = min(mn, Q::stage_lp(d, q, ib, lp, r * gpb + gib, s, bound, sm, st, g, err_slot, cur));
    }
    __syncthreads();
    // B: one staged event per thread
    const uint32_t ns = min(*st.cnt, st.cap);
    for (uint32_t t = threadIdx.x; t < ns; t += blockDim.x) {
      const gpq_item e = st.ev[t];
      if (e.aux != kStageHole) mn = min(mn, phold_process_event(d, ib, st, e, curb, err_slot));
    }
    __syncthreads();
    // C: checksums back to the LPs that committed events
    for (uint32_t t = threadIdx.x; t < nslots; t += blockDim.x) {
      const uint32_t l = st.lp[t];
      if (l != ~0u) {
        d.csum[l] = st.csum[t];
        d.ohash[l] = st.ohash[t];
      }
    }
    __syncthreads();
  }
  mn = block_min_u32(mn, red);
  if (threadIdx.x == 0 && mn != kInfBits) atomicMin(&d.ctrl->mins[(s + 1u) % 3u], mn);
}

// Plain form: one launch per window; the kernel boundary is the barrier.
template <class Q>
static __global__ void phold_window_kernel(PholdDev d, LpQueueDev lq, InsDev ib, uint32_t s) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t red[32];
  const uint32_t mb = d.ctrl->mins[s % 3u];
  const float m = gpq_u2f(mb);
  if (!(m < d.p.end_time)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.ctrl->mins[(s + 2u) % 3u] = kInfBits;  // slot for window s+2 (last read in window s-1)
    d.ctrl->errs[(s + 2u) % 3u] = 0u;
    d.ctrl->steps += 1ull;
    d.ctrl->phase = s + 1u;
  }
  phold_window_body<Q>(d, Q::dev(lq), ib, s, m, smem_raw, red);
}

// Persistent form: all windows in one cooperative launch; a bounded grid barrier
// separates windows.  Every block takes the same exit decision from the same
// (minimum, error) slot written before the barrier.
template <class Q>
static __global__ void phold_persistent_kernel(PholdDev d, LpQueueDev lq, InsDev ib, uint32_t s0, uint32_t max_steps) {
  const typename Q::Dev q = Q::dev(lq);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t red[32];
  unsigned long long target = 0;
  uint32_t s = s0;
  for (;; ++s) {
    const uint32_t mb = ld_relaxed_u32(&d.ctrl->mins[s % 3u]);
    const uint32_t eb = ld_relaxed_u32(&d.ctrl->errs[s % 3u]);
    const float m = gpq_u2f(mb);
    if (!(m < d.p.end_time) || eb != 0u || (max_steps != 0u && s - s0 >= max_steps)) break;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      d.ctrl->mins[(s + 2u) % 3u] = kInfBits;
      d.ctrl->errs[(s + 2u) % 3u] = 0u;
      d.ctrl->steps += 1ull;
    }
    phold_window_body<Q>(d, q, ib, s, m, smem_raw, red);
    target += gridDim.x;
    if (!grid_barrier(&d.ctrl->bar, target, d.spin_limit, &d.ctrl->err)) {
      s += 1u;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctrl->phase = s;
}

// Kernel pointers of one (queue kind, lane-group size) pair (host-side dispatch).
struct PholdKernelSet {
  const void* window;
  const void* persistent;
  uint32_t group;
  size_t group_smem;  // per lane group, for insert capacity ibc
};

inline bool phold_kernel_set(uint32_t kind, uint32_t group, uint32_t ibc, PholdKernelSet* out, uint32_t laq_mode = 0) {
#define GPQ_KS(P) *out = {(const void*)phold_window_kernel<P>, (const void*)phold_persistent_kernel<P>, \
                          (uint32_t)P::G, P::group_smem_bytes(ibc)}; return true
  if (kind == GPQ_QUEUE_LAQ && laq_mode == 1) {
    switch (group) {
      case 4: GPQ_KS(LasP<4>);
      case 8: GPQ_KS(LasP<8>);
      case 16: GPQ_KS(LasP<16>);
      case 32: GPQ_KS(LasP<32>);
    }
  } else if (kind == GPQ_QUEUE_LAQ) {
    switch (group) {
      case 4: GPQ_KS(LaqP<4>);
      case 8: GPQ_KS(LaqP<8>);
      case 16: GPQ_KS(LaqP<16>);
      case 32: GPQ_KS(LaqP<32>);
    }
  } else if (kind == GPQ_QUEUE_LHQ) {
    switch (group) {
      case 1: GPQ_KS(LhqP<1>);
      case 4: GPQ_KS(LhqP<4>);
      case 8: GPQ_KS(LhqP<8>);
      case 16: GPQ_KS(LhqP<16>);
      case 32: GPQ_KS(LhqP<32>);
    }
  } else if (kind == GPQ_QUEUE_LSQ) {
    GPQ_KS(LsqP);
  }
#undef GPQ_KS
  return false;
}

// End of run: committed total, pending events (queue contents + the unmerged children
// of the last window) and the order-sensitive digest over the per-LP outputs.  One warp
// per LP.
static __global__ void phold_finalize_kernel(PholdDev d, LpQueueDev q, InsDev ib, PholdAcc* acc) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const uint32_t nwarps = gridDim.x * wpb;
  const uint32_t s = d.ctrl->phase;
  const uint32_t prevb = (s + 1u) & 1u;
  const uint32_t cap = 1u << q.cap_log2, mask = cap - 1u;
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t pmin = kInfBits;
  for (uint32_t lp = d.lp_begin + blockIdx.x * wpb + (threadIdx.x >> 5); lp < d.lp_end; lp += nwarps) {
    const gpq_item* items = q.items + ((size_t)lp << q.cap_log2);
    uint32_t first = 0, n = 0;
    if (q.kind == GPQ_QUEUE_LAQ) { first = q.a[lp]; n = q.b[lp] - first; }
    else if (q.kind == GPQ_QUEUE_LHQ) { n = q.a[lp]; }
    else { n = cap; }
    for (uint32_t j = lane; j < n; j += 32) {
      const gpq_item e = items[(first + j) & mask];
      if (q.kind == GPQ_QUEUE_LSQ && e.lp == 0xffffffffu) continue;  // free pool slot
      pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
      pend += 1;
      pmin = min(pmin, gpq_f2u(e.ts));
    }
    const uint32_t k = min(ib.cnt[(size_t)prevb * d.L + lp], ib.ibc);
    const gpq_item* src = ib.buf + ((size_t)prevb * d.L + lp) * ib.ibc;
    for (uint32_t j = lane; j < k; j += 32) {
      const gpq_item e = src[j];
      pcs += gpq_ev_hash(e.id, gpq_f2u(e.ts));
      pend += 1;
      pmin = min(pmin, gpq_f2u(e.ts));
    }
    if (lane == 0) {
      const uint32_t c = d.count[lp];
      com += c;
      const uint64_t lph = gpq_mix64(gpq_mix64(((uint64_t)lp << 32) | c) ^ d.csum[lp]) + d.ohash[lp];
      dig += gpq_mix64(lph);
    }
  }
  pend = warp_sum_u64(pend);
  pcs = warp_sum_u64(pcs);
  dig = warp_sum_u64(dig);
  com = warp_sum_u64(com);
  pmin = warp_min_u32(pmin);
  if (lane == 0) {
    atomicAdd(&acc->pending, (unsigned long long)pend);
    atomicAdd(&acc->pending_csum, (unsigned long long)pcs);
    atomicAdd(&acc->digest, (unsigned long long)dig);
    atomicAdd(&acc->committed, (unsigned long long)com);
    atomicMin(&acc->pending_min, pmin);
  }
}

// Children of n events (the model's event function on the device).
static __global__ void phold_children_kernel(gpq_phold_params p, const gpq_item* __restrict__ ev, gpq_item* out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = gpq_phold_child(p, ev[i]);
}

// Sharded runs: items handed over from other shards after window s go into the insert
// buffers that window s filled (parity curb), so window s + 1 merges them with this
// shard's own children.  Items for LPs outside the shard are an argument error.
static __global__ void phold_inject_kernel(PholdDev d, InsDev ib, const gpq_item* __restrict__ items, uint64_t n,
                                           uint32_t curb) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const gpq_item it = items[i];
    if (it.lp < d.lp_begin || it.lp >= d.lp_end) {
      gpq_set_error(&d.ctrl->err, GPQ_ERR_INVALID);
      continue;
    }
    const uint32_t pos = atomicAdd(&ib.cnt[(size_t)curb * d.L + it.lp], 1u);
    if (pos < ib.ibc) ib.buf[((size_t)curb * d.L + it.lp) * ib.ibc + pos] = it;
    else gpq_set_error(&d.ctrl->err, GPQ_ERR_INSERT_FULL);
  }
}
