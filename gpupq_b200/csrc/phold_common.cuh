// Shared device code of the PHOLD engine: control block, lane groups, the staging
// area and the per-event pass (the PHOLD handler of the reference, src/phold.cu:81-117).
#pragma once

#include "common.cuh"
#include "gpq/model.h"

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
  // Sharded runs (per-LP queue kinds): this handle processes LPs [lp_begin, lp_end) of the
  // L-LP arrays; a child for another shard's LP goes to outbox[dest][out_cap] (dest =
  // lp / shard_lps, count out_n[dest]) for the host to hand over between windows.
  // Unsharded: [0, L) and outbox == nullptr.
  uint32_t lp_begin, lp_end;
  uint32_t shard_lps;
  uint32_t out_cap;
  gpq_item* outbox;
  uint32_t* out_n;
  // Sharded runs of the bucketed local array queue connected for direct hand-over: every
  // shard's bucket arrays ([world] LabPeer, lab.cuh); a child for another shard's LP is
  // filed straight into that shard's buckets.  nullptr: hand-over through the outbox.
  const void* peers;
};

// A group of G consecutive lanes of one warp working on one LP.
template <int G>
struct LaneGroup {
  static_assert(G == 1 || G == 2 || G == 4 || G == 8 || G == 16 || G == 32, "group size");
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
  // Group-wide minimum of a 64-bit key; returns the key and the lane that holds it.
  __device__ __forceinline__ uint64_t kmin(uint64_t v, uint32_t* who) const {
    uint32_t w = gl;
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const uint64_t ov = __shfl_xor_sync(mask, v, o, G);
      const uint32_t ow = __shfl_xor_sync(mask, w, o, G);
      if (ov < v || (ov == v && ow < w)) { v = ov; w = ow; }
    }
    *who = w;
    return v;
  }
  __device__ __forceinline__ uint32_t shfl(uint32_t v, uint32_t src) const { return __shfl_sync(mask, v, src, G); }
  __device__ __forceinline__ uint64_t sum(uint64_t v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
  }
  __device__ __forceinline__ uint32_t umin(uint32_t v) const { return __reduce_min_sync(mask, v); }
};

static constexpr uint32_t kStageHole = 0xffffffffu;  // aux of a reserved but unused staging slot

// Per-CTA shared staging of one super-round: the safe events found by the lane groups
// (aux = slot << 16 | index in the LP's safe prefix) and per-LP-slot accumulators.
struct PholdStage {
  gpq_item* ev;              // [cap] staged events
  uint32_t* cnt;             // number of staged events
  uint32_t* seq0;            // [slots] LP's committed count before this window
  unsigned long long* csum;  // [slots] LP checksum (value before the window + this window's events)
  unsigned long long* ohash; // [slots]
  uint32_t* lp;              // [slots] LP of the slot (~0u = unused)
  uint32_t cap;
};

// Process one safe event: per-LP hashes into the slot accumulators, the child into the
// window's insert buffers.  Returns the child's timestamp bits.
__device__ __forceinline__ uint32_t phold_process_event(const PholdDev& d, const InsDev& ib, const PholdStage& st,
                                                      const gpq_item e, uint32_t curb, uint32_t* err_slot) {
  const uint32_t slot = e.aux >> 16;
  const uint32_t idx = e.aux & 0xffffu;
  const uint32_t tb = gpq_f2u(e.ts);
  const uint64_t h = gpq_ev_hash(e.id, tb);
  atomicAdd(&st.csum[slot], (unsigned long long)h);
  atomicAdd(&st.ohash[slot], (unsigned long long)gpq_seq_hash(h, (uint64_t)st.seq0[slot] + idx));
  gpq_item pe = e;
  pe.aux = e.lp;
  const gpq_item ch = gpq_phold_child(d.p, pe);
  if (d.outbox && (ch.lp < d.lp_begin || ch.lp >= d.lp_end)) {  // another shard's LP
    const uint32_t dest = ch.lp / d.shard_lps;
    const uint32_t pos = atomicAdd(&d.out_n[dest], 1u);
    if (pos < d.out_cap) {
      d.outbox[(size_t)dest * d.out_cap + pos] = ch;
    } else {
      gpq_set_error(&d.ctrl->err, GPQ_ERR_INSERT_FULL);
      atomicOr(err_slot, 1u);
    }
    return gpq_f2u(ch.ts);
  }
  const uint32_t pos = atomicAdd(&ib.cnt[(size_t)curb * d.L + ch.lp], 1u);
  if (pos < ib.ibc) {
    ib.buf[((size_t)curb * d.L + ch.lp) * ib.ibc + pos] = ch;
  } else {
    gpq_set_error(&d.ctrl->err, GPQ_ERR_INSERT_FULL);
    atomicOr(err_slot, 1u);
  }
  return gpq_f2u(ch.ts);
}


// Slot accumulators start from the LP's values before this window (group leader).
__device__ __forceinline__ void phold_stage_slot_init(const PholdStage& st, uint32_t slot, uint32_t count,
                                                      unsigned long long csum, unsigned long long ohash) {
  st.seq0[slot] = count;
  st.csum[slot] = csum;
  st.ohash[slot] = ohash;
}

// Stage one batch of a group's safe events.  Lane gl holds event index idx (its position
// in the LP's safe sequence) when `safe`; the safe lanes are lanes 0..c-1.  If the staging
// area is full the events are processed here (their reserved slots inside the area are
// marked as holes).  Returns the min of the children processed here.  All lanes of the
// group, convergent.
template <int G>
__device__ __forceinline__ uint32_t phold_stage_batch(const PholdDev& d, const InsDev& ib, const PholdStage& st,
                                                      const LaneGroup<G>& g, gpq_item e, bool safe, uint32_t idx,
                                                      uint32_t c, uint32_t slot, uint32_t curb, uint32_t* err_slot) {
  uint32_t cmin = kInfBits;
  if (c == 0) return cmin;
  uint32_t base = 0;
  if (g.gl == 0) base = atomicAdd(st.cnt, c);
  base = g.shfl(base, 0);
  if (safe) {
    e.aux = (slot << 16) | idx;
    if (base + c <= st.cap) {
      st.ev[base + g.gl] = e;
    } else {
      if (base + g.gl < st.cap) {
        gpq_item hole = e;
        hole.aux = kStageHole;
        st.ev[base + g.gl] = hole;
      }
      cmin = phold_process_event(d, ib, st, e, curb, err_slot);
    }
  }
  return cmin;
}
