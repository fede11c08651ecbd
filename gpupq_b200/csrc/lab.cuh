// Local array queue, bucketed form (laq_mode 2).
//
// Reference: src/local_array_queue.cu keeps each LP's events in one sorted ring and, on
// every queue_post, insertion-sorts each new event into it (d_insertion_sort,
// :254-299, src/sort.cu:329-353) although a window only dequeues the events below its
// bound (queue_peek, :760-779).
//
// Here each LP's array is split into NB time buckets of C slots.  An event is stored as
// its 8-byte per-LP key (ts bits << 32 | id: the LP is implied by the array, and the key
// orders the LP's events exactly like (ts bits, lp, id)).  Bucket j holds the events with
// floor(ts * inv_w) == j in arrival order; absolute bucket j lives in slot j mod NB.  The
// bucket function is monotone, so bucket order is timestamp order.
//
// Window s (minimum m, bound = m + lookahead): every safe event lies in the buckets
// j0 = bi(m) .. j1 = bi(bound).  Children (ts >= bound) land in buckets >= j1, so the
// buckets below j1 belong to their LP's lane group alone during the window, while bucket
// j1 and the ones above take appends (atomicAdd on the bucket count) at any time.  Pass A
// (one lane group per LP) reads the range buckets and the LP's spill list of window s-1,
// ranks the safe keys in shared memory (their positions in the LP's sequence), stages
// them for the CTA-wide event pass, compacts the buckets below j1, re-files the spill
// list and finds the LP's next minimum.  Pass B appends each child to its bucket; a full
// bucket or one beyond the horizon sends it to the LP's spill list of this window's
// parity.  There is no merge and no ordering work beyond the ranks of each window's safe
// events.
//
// Consumed events are not erased from bucket j1 (it may be appended to meanwhile): a key
// with ts < m is dead.  Every read filters on m <= ts <= +inf, which also skips slots
// never written (all ones) and slots reserved by an append whose store is not visible
// yet (they still hold a dead key of an earlier use of the slot).  A bucket's count is
// reset when the window leaves it behind: the buckets below j1 by their compaction, and
// bucket j1(s-1) and any bucket skipped by a jump of m in pass A of window s.  Appends
// in window s reach at most bucket j1(s-1) + NB - 1, so no append meets a slot whose
// count is not reset yet.  The next minimum of an LP is the smallest live key that stays
// at or below j1 (spill list included); only when there is none does the LP scan the
// buckets above j1, whose live keys are pending events either way, so the minimum over
// the LPs and the children is exactly the minimum over the pending events.
#pragma once

#include "phold_kernels.cuh"

struct LabDev {
  unsigned long long* keys;   // [num_lps][NB][C]; slots [0, min(cnt, C)) of a bucket hold keys (live or dead)
  uint32_t* cnt;              // [num_lps][NB] appends per bucket (above C: the excess went to spill)
  unsigned long long* spill;  // [2][num_lps][F] per-LP spill lists, by window parity
  uint32_t* scnt;             // [2][num_lps]
  uint32_t* wj;               // [4] j1 of window s in wj[s & 3] (wj[3] = 0 before window 0)
  uint32_t nb_log2, c_log2, F;
  float inv_w;                // 1 / bucket width
  uint32_t chunk;             // LPs per warp chunk (lab_chunk_lps)
};

// One shard's bucket arrays, for another shard's direct hand-over.
struct LabPeer {
  unsigned long long* keys;
  uint32_t* cnt;
  unsigned long long* spill;
  uint32_t* scnt;
};

static constexpr uint32_t kLabSafeCap = 32;  // safe keys of one LP per window ranked in shared memory

__host__ __device__ inline size_t lab_group_smem_bytes() { return (size_t)kLabSafeCap * 8; }

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bucket of a timestamp (bits); monotone non-decreasing in ts, saturating at 2^32 - 1.
__device__ __forceinline__ uint32_t lab_bucket(uint32_t tsb, float inv_w) {
  return __float2uint_rz(__fmul_rn(gpq_u2f(tsb), inv_w));
}

__device__ __forceinline__ unsigned long long lab_key(uint32_t tsb, uint32_t id) {
  return ((unsigned long long)tsb << 32) | id;
}

// Window constants (the same in every thread).
struct LabWin {
  uint32_t mb;        // m as float bits: keys below are dead
  uint32_t safe_lim;  // a live key is safe iff its ts bits < safe_lim (= min(bound, end_time) bits)
  uint32_t j0, j1;    // bucket range that holds every safe event
  uint32_t j1p;       // j1 of the previous window: appends reach at most j1p + NB - 1
  uint32_t curb, prevb;
  float inv_w;        // 1 / bucket width of the run
};

__device__ __forceinline__ bool lab_live(uint32_t t, const LabWin& w) { return t >= w.mb && t <= kInfBits; }

// The run a window belongs to: its model, where its LPs sit in the LP space, and where its
// errors go.  One PHOLD run per launch uses lp_base 0 and L = its LP count; runs that share
// an LP space number their LPs from lp_base (events carry LP-space numbers; the model sees
// numbers local to the run).
struct LabCtx {
  gpq_phold_params p;  // the run's model (num_lps = its LP count)
  uint32_t L;          // LP-space size: stride of the spill lists
  uint32_t lp_base;    // the run's first LP in the LP space
  uint32_t* err;       // the run's sticky error word
  uint32_t* err_slot;  // error slot read by the next window's exit decision
  // A shard of a sharded run owns LPs [lp_begin, lp_end); a child for another shard's LP
  // goes to outbox[dest][out_cap] (dest = lp / shard_lps, count out_n[dest]) for the host
  // to hand over between windows.  outbox == nullptr: every LP is local.
  gpq_item* outbox = nullptr;
  uint32_t* out_n = nullptr;
  uint32_t out_cap = 0, shard_lps = 1, lp_begin = 0, lp_end = 0xffffffffu;
  const LabPeer* peers = nullptr;  // direct hand-over: every shard's bucket arrays
};

__device__ __forceinline__ void lab_fail(const LabCtx& x, uint32_t code) {
  gpq_set_error(x.err, code);
  atomicOr(x.err_slot, 1u);
}

// Child of staged event e (LP-space numbers in and out).
__device__ __forceinline__ gpq_item lab_child(const LabCtx& x, const gpq_item e) {
  gpq_item pe = e;
  pe.lp = e.lp - x.lp_base;
  pe.aux = pe.lp;
  gpq_item ch = gpq_phold_child(x.p, pe);
  ch.lp += x.lp_base;
  return ch;
}

// Window s of a run with minimum m, model p, bucket width 1 / inv_w, and top bucket of its
// previous window j1p.
__device__ __forceinline__ LabWin lab_window_of(const gpq_phold_params& p, float inv_w, uint32_t s, float m,
                                                uint32_t j1p) {
  LabWin w;
  const float bound = GPQ_FADD(m, p.lookahead);
  w.mb = gpq_f2u(m);
  const uint32_t bb = gpq_f2u(bound), tb = gpq_f2u(p.end_time);
  w.safe_lim = bb < tb ? bb : tb;  // timestamps, bound and end time are >= +0: bit order = value order
  w.j0 = lab_bucket(w.mb, inv_w);
  w.j1 = lab_bucket(bb, inv_w);
  w.j1p = j1p;
  w.curb = s & 1u;
  w.prevb = (s + 1u) & 1u;
  w.inv_w = inv_w;
  return w;
}

__device__ __forceinline__ LabWin lab_window(const PholdDev& d, const LabDev& q, uint32_t s, float m) {
  return lab_window_of(d.p, q.inv_w, s, m, ld_relaxed_u32(&q.wj[(s + 3u) & 3u]));
}

// Files one pending key of LP `lp` (bucket jb) during window w: into its bucket when jb is
// in [j1, j1p + NB) and the bucket has room, else into the spill list of this window's
// parity.
__device__ __forceinline__ void lab_push(const LabCtx& x, const LabDev& q, uint32_t lp, unsigned long long key,
                                         uint32_t jb, const LabWin& w) {
  const uint32_t nbm = (1u << q.nb_log2) - 1u;
  if (jb >= w.j1 && jb - w.j1p <= nbm) {
    const size_t b = ((size_t)lp << q.nb_log2) + (jb & nbm);
    const uint32_t pos = atomicAdd(&q.cnt[b], 1u);
    if (pos < (1u << q.c_log2)) {
      st_relaxed_u64(q.keys + (b << q.c_log2) + pos, key);
      return;
    }
  }
  const size_t sl = (size_t)w.curb * x.L + lp;
  const uint32_t pos = atomicAdd(&q.scnt[sl], 1u);
  if (pos < q.F) {
    q.spill[sl * q.F + pos] = key;
  } else {
    lab_fail(x, GPQ_ERR_QUEUE_FULL);
  }
}

// A child of another shard's LP: filed straight into that shard's buckets (connected
// shards: the same append rule as a local child -- every shard runs window w with the same
// bound and bucket geometry, and an append lands at or above j1, which the owner does not
// compact during the window), or into the outbox.  Returns false for a local child.
__device__ __forceinline__ bool lab_handover(const LabCtx& x, const LabDev& q, const LabWin& w, const gpq_item& ch) {
  if (x.outbox == nullptr || (ch.lp >= x.lp_begin && ch.lp < x.lp_end)) return false;
  const uint32_t dest = ch.lp / x.shard_lps;
  if (x.peers != nullptr) {
    const LabPeer P = x.peers[dest];
    LabDev qd = q;
    qd.keys = P.keys;
    qd.cnt = P.cnt;
    qd.spill = P.spill;
    qd.scnt = P.scnt;
    const uint32_t cb = gpq_f2u(ch.ts);
    lab_push(x, qd, ch.lp, lab_key(cb, ch.id), lab_bucket(cb, w.inv_w), w);
    return true;
  }
  const uint32_t slot = atomicAdd(&x.out_n[dest], 1u);
  if (slot < x.out_cap) {
    x.outbox[(size_t)dest * x.out_cap + slot] = ch;
  } else {
    gpq_set_error(x.err, GPQ_ERR_INSERT_FULL);
    atomicOr(x.err_slot, 1u);
  }
  return true;
}

// Process one staged event: per-LP hashes into the slot accumulators, the child into its
// bucket (kShard: a child of another shard's LP is handed over).  Returns the child's
// timestamp bits.
template <bool kShard>
__device__ __forceinline__ uint32_t lab_process_event(const LabCtx& x, const LabDev& q, const PholdStage& st,
                                                      const gpq_item e, const LabWin& w) {
  const uint32_t slot = e.aux >> 16;
  const uint32_t idx = e.aux & 0xffffu;
  const uint32_t tb = gpq_f2u(e.ts);
  const uint64_t h = gpq_ev_hash(e.id, tb);
  atomicAdd(&st.csum[slot], (unsigned long long)h);
  atomicAdd(&st.ohash[slot], (unsigned long long)gpq_seq_hash(h, (uint64_t)st.seq0[slot] + idx));
  const gpq_item ch = lab_child(x, e);
  const uint32_t cb = gpq_f2u(ch.ts);
  if (!(kShard && lab_handover(x, q, w, ch))) lab_push(x, q, ch.lp, lab_key(cb, ch.id), lab_bucket(cb, w.inv_w), w);
  return cb;
}

// Per-LP words read at the start of its turn on the general path: the spill count of
// window s-1 and (lane gl) the count of bucket j0 + gl.
struct LabMeta {
  uint32_t sc, bc;
};

__device__ __forceinline__ LabMeta lab_load_meta(const LabCtx& x, const LabDev& q, uint32_t lp, const LabWin& w,
                                                 uint32_t gl) {
  LabMeta mt;
  mt.sc = q.scnt[(size_t)w.prevb * x.L + lp];
  const uint32_t nbm = (1u << q.nb_log2) - 1u;
  mt.bc = ld_relaxed_u32(&q.cnt[((size_t)lp << q.nb_log2) + ((w.j0 + gl) & nbm)]);
  return mt;
}

// Number of appends to bucket j0 + r of the LP (lane r of the prefetch, or a load).
template <int G>
__device__ __forceinline__ uint32_t lab_range_count(const LabDev& q, const uint32_t* cnt, const LabWin& w, uint32_t r,
                                                    const LabMeta& mt, const LaneGroup<G>& g) {
  if (r < (uint32_t)G) return g.shfl(mt.bc, r);
  return ld_relaxed_u32(&cnt[(w.j0 + r) & ((1u << q.nb_log2) - 1u)]);
}

// Key i of candidate source r of the LP: range bucket j0 + r (r < nr; bucket j1 may be
// appended to meanwhile, so it is read with relaxed loads) or the spill list (r == nr).
__device__ __forceinline__ unsigned long long lab_cand(const unsigned long long* src, uint32_t i, bool shared) {
  return shared ? ld_relaxed_u64(src + i) : src[i];
}

// One LP, one window, by a lane group (the general path: any bucket range, any number of
// candidates): rank and stage the safe events (slot = the LP's index in its chunk, whose
// accumulators st.seq0/csum/ohash hold the LP's outputs), compact the buckets below j1,
// re-file the spill list, store the number of safe events in nsafe_out[slot], and return
// the LP's next minimum (ts bits) min'ed with any child processed here.  All lanes of the
// group, convergent.
template <int G, bool kShard>
__device__ uint32_t lab_lp_stage(const LabCtx& x, const LabDev& q, uint32_t lp, uint32_t slot, const LabWin& w,
                                 unsigned long long* skeys, const PholdStage& st, const LaneGroup<G>& g, const LabMeta& mt, uint32_t* nsafe_out) {
  const uint32_t L = x.L;
  const uint32_t NB = 1u << q.nb_log2, nbm = NB - 1u, C = 1u << q.c_log2;
  const size_t lpb = (size_t)lp << q.nb_log2;
  unsigned long long* keys = q.keys + (lpb << q.c_log2);
  uint32_t* cnt = q.cnt + lpb;
  const unsigned long long* sp = q.spill + ((size_t)w.prevb * L + lp) * q.F;
  const uint32_t nr = w.j1 - w.j0 + 1u;
  const uint32_t sc = mt.sc < q.F ? mt.sc : q.F;
  const uint32_t lt = (1u << g.gl) - 1u;

  // 1. read-only scan of the range buckets and the spill list: count the safe events and
  //    keep up to kLabSafeCap of their keys
  uint32_t nsafe = 0;
  for (uint32_t r = 0; r <= nr; ++r) {
    uint32_t c;
    const unsigned long long* src;
    if (r < nr) {
      c = min(lab_range_count<G>(q, cnt, w, r, mt, g), C);
      src = keys + ((size_t)((w.j0 + r) & nbm) << q.c_log2);
    } else {
      c = sc;
      src = sp;
    }
    const bool shared = r == nr - 1u;
    for (uint32_t i0 = 0; i0 < c; i0 += G) {
      const uint32_t i = i0 + g.gl;
      const unsigned long long k = (i < c) ? lab_cand(src, i, shared) : ~0ull;
      const uint32_t t = (uint32_t)(k >> 32);
      const bool sf = t >= w.mb && t < w.safe_lim;
      const uint32_t b = g.ballot(sf);
      if (sf) {
        const uint32_t p = nsafe + __popc(b & lt);
        if (p < kLabSafeCap) skeys[p] = k;
      }
      nsafe += __popc(b);
    }
  }
  if (nsafe > 0xffffu) {  // ranks are 16-bit in the staged events
    if (g.gl == 0) lab_fail(x, GPQ_ERR_INVALID);
    nsafe = 0;
  }
  g.sync();

  // 2. ranks (positions in the LP's sequence) and staging
  uint32_t cmin = kInfBits;
  if (nsafe > 0) {
    uint32_t base = 0;
    if (g.gl == 0) base = atomicAdd(st.cnt, nsafe);
    base = g.shfl(base, 0);
    const bool fits = base + nsafe <= st.cap;
    auto stage = [&](unsigned long long k, uint32_t rank) {
      gpq_item e;
      e.ts = gpq_u2f((uint32_t)(k >> 32));
      e.lp = lp;
      e.id = (uint32_t)k;
      e.aux = (slot << 16) | rank;
      if (fits) {
        st.ev[base + rank] = e;
      } else {
        if (base + rank < st.cap) {
          gpq_item hole = e;
          hole.aux = kStageHole;
          st.ev[base + rank] = hole;
        }
        cmin = min(cmin, lab_process_event<kShard>(x, q, st, e, w));
      }
    };
    if (nsafe <= kLabSafeCap) {
      for (uint32_t u = g.gl; u < nsafe; u += G) {
        const unsigned long long k = skeys[u];
        uint32_t rank = 0;
        for (uint32_t v = 0; v < nsafe; ++v) rank += (skeys[v] < k) ? 1u : 0u;
        stage(k, rank);
      }
    } else {
      // more safe events than the shared list holds: rank each against every candidate
      // (safe keys are neither moved nor erased before step 3)
      for (uint32_t r = 0; r <= nr; ++r) {
        uint32_t c;
        const unsigned long long* src;
        if (r < nr) {
          c = min(ld_relaxed_u32(&cnt[(w.j0 + r) & nbm]), C);
          src = keys + ((size_t)((w.j0 + r) & nbm) << q.c_log2);
        } else {
          c = sc;
          src = sp;
        }
        for (uint32_t i = g.gl; i < c; i += G) {
          const unsigned long long k = lab_cand(src, i, r == nr - 1u);
          const uint32_t t = (uint32_t)(k >> 32);
          if (!(t >= w.mb && t < w.safe_lim)) continue;
          uint32_t rank = 0;
          for (uint32_t r2 = 0; r2 <= nr; ++r2) {
            uint32_t c2;
            const unsigned long long* s2;
            if (r2 < nr) {
              c2 = min(ld_relaxed_u32(&cnt[(w.j0 + r2) & nbm]), C);
              s2 = keys + ((size_t)((w.j0 + r2) & nbm) << q.c_log2);
            } else {
              c2 = sc;
              s2 = sp;
            }
            for (uint32_t v = 0; v < c2; ++v) {
              const unsigned long long k2 = lab_cand(s2, v, r2 == nr - 1u);
              const uint32_t t2 = (uint32_t)(k2 >> 32);
              rank += (t2 >= w.mb && t2 < w.safe_lim && k2 < k) ? 1u : 0u;
            }
          }
          stage(k, rank);
        }
      }
    }
  }
  g.sync();

  // 3. compact the buckets below j1 (keep the live keys that are not safe: ts >= end
  //    time, or a float-rounding edge), note the live keys left in j1, re-file the spill list
  uint32_t rmin = kInfBits;
  bool low_lane = false;  // something live stays at or below bucket j1
  for (uint32_t r = 0; r < nr; ++r) {
    const uint32_t raw = lab_range_count<G>(q, cnt, w, r, mt, g);
    const uint32_t c = min(raw, C);
    unsigned long long* bk = keys + ((size_t)((w.j0 + r) & nbm) << q.c_log2);
    if (r == nr - 1u) {
      for (uint32_t i = g.gl; i < c; i += G) {
        const uint32_t t = (uint32_t)(ld_relaxed_u64(bk + i) >> 32);
        if (lab_live(t, w) && t >= w.safe_lim) {
          rmin = min(rmin, t);
          low_lane = true;
        }
      }
      continue;
    }
    uint32_t kept = 0;
    for (uint32_t i0 = 0; i0 < c; i0 += G) {
      const uint32_t i = i0 + g.gl;
      const unsigned long long k = (i < c) ? bk[i] : ~0ull;
      const uint32_t t = (uint32_t)(k >> 32);
      const bool keep = lab_live(t, w) && t >= w.safe_lim;
      const uint32_t kb = g.ballot(keep);
      g.sync();  // every load of the chunk precedes every store (stores go to positions <= i)
      if (keep) {
        const uint32_t p = kept + __popc(kb & lt);
        if (p != i) bk[p] = k;
        rmin = min(rmin, t);
        low_lane = true;
      }
      kept += __popc(kb);
    }
    if (g.gl == 0 && kept != raw) cnt[(w.j0 + r) & nbm] = kept;
  }
  for (uint32_t i = g.gl; i < sc; i += G) {
    const unsigned long long k = sp[i];
    const uint32_t t = (uint32_t)(k >> 32);
    if (t < w.safe_lim) continue;
    const uint32_t jb = lab_bucket(t, w.inv_w);
    rmin = min(rmin, t);
    low_lane = low_lane || jb <= w.j1;
    lab_push(x, q, lp, k, jb, w);
  }
  const bool low = g.ballot(low_lane) != 0u;
  if (g.gl == 0 && mt.sc != 0) q.scnt[(size_t)w.prevb * L + lp] = 0;
  uint32_t lpmin = g.umin(rmin);

  // 4. nothing live stays at or below j1: the LP's next minimum is in the first bucket above
  //    j1 that holds a live key (read while pass B may append to it)
  if (!low) {
    uint32_t found = kInfBits;
    for (uint32_t jb0 = w.j1 + 1u; jb0 - w.j0 < NB && found == kInfBits; jb0 += G) {
      const uint32_t j = jb0 + g.gl;
      uint32_t c = 0;
      if (j - w.j0 < NB) c = min(ld_relaxed_u32(&cnt[j & nbm]), C);
      uint32_t nz = g.ballot(c > 0);
      while (nz != 0u && found == kInfBits) {
        const uint32_t l = (uint32_t)__ffs(nz) - 1u;
        nz &= nz - 1u;
        const uint32_t cj = g.shfl(c, l);
        const unsigned long long* bk = keys + ((size_t)((jb0 + l) & nbm) << q.c_log2);
        uint32_t v = kInfBits;
        for (uint32_t i = g.gl; i < cj; i += G) {
          const uint32_t t = (uint32_t)(ld_relaxed_u64(bk + i) >> 32);
          if (lab_live(t, w) && t < v) v = t;
        }
        found = g.umin(v);
      }
    }
    lpmin = min(lpmin, found);
  }

  if (g.gl == 0) nsafe_out[slot] = nsafe;
  return min(lpmin, g.umin(cmin));
}


// ---------------------------------------------------------------------------------
// Warp-owned window.  A CTA owns a contiguous LP range, split evenly among its warps; a
// warp works through its share in chunks of up to kLabWarpLps LPs, and every phase of a
// chunk runs inside the warp (no CTA-wide synchronisation until the window's minimum), so
// the warps of an SM overlap one another's memory waits.  The PHOLD outputs of a chunk live
// in the warp's shared memory (for the whole persistent launch when the warp owns at most
// one chunk).  On the common path every phase covers all LPs of the chunk at once:
//   P1  counts of the range buckets and spill lists, and of the two buckets above j1;
//   P2  a prefix sum gives each (LP, source) its place in the warp's candidate list;
//   P3  every lane loads up to 8 candidate keys (independent loads);
//   P4  per candidate: dead / safe (rank among the LP's safe keys) / staying (LP minimum,
//       compaction below j1, spill re-filing);
//   P5  bucket and spill counts written back; prefix sum of the LPs' safe counts;
//   P6  safe events staged in (LP, rank) order; loads of the next-minimum scan issued;
//   P7  the event pass (children appended), then each LP's next minimum.
// Bucket ranges wider than kLabSegMax - 1 buckets or more candidates than kLabCandCap take
// the general path: the warp as one lane group per LP (lab_lp_stage<32>).
// ---------------------------------------------------------------------------------
static constexpr uint32_t kLabWarpLps = 16;    // LPs per warp chunk
static constexpr uint32_t kLabSegMax = 5;      // candidate sources per LP on the common path
static constexpr uint32_t kLabCandCap = 256;   // candidate keys per warp chunk on the common path
static constexpr uint32_t kLabStageCap = 128;  // staged events per warp chunk (4-byte entries)
static constexpr uint32_t kLabSafePerLp = 32;  // safe keys of one LP ranked on the common path
static constexpr uint32_t kLabItemStageCap = kLabStageCap * 4 / 16;  // staged items on the general path
static_assert(kLabCandCap <= 256 && kLabSafePerLp <= 256 && kLabWarpLps <= 65536, "staging entry fields");

struct LabWarpSmem {
  unsigned long long* ls_csum;   // [kLabWarpLps] LP checksum
  unsigned long long* ls_ohash;  // [kLabWarpLps] LP order-sensitive hash
  unsigned long long* cand;      // [kLabCandCap] candidate keys (general path: the safe-key list)
  uint32_t* cstage;              // [kLabStageCap] staged events: candidate index | rank << 8 | LP index << 16
  gpq_item* stage;               // [kLabItemStageCap] staged items on the general path (same bytes as cstage)
  uint32_t* ls_cnt;              // [kLabWarpLps] LP committed count (before the window: the sequence base)
  uint32_t* seg_raw;             // [kLabWarpLps * kLabSegMax] bucket count / spill count as read
  uint32_t* seg_off;             // [kLabWarpLps * kLabSegMax + 1] candidate offsets
  uint32_t* seg_kept;            // [kLabWarpLps * kLabSegMax] keys kept by a bucket below j1
  uint32_t* lp_nsafe;            // [kLabWarpLps]
  uint32_t* lp_soff;             // [kLabWarpLps + 1] staging offsets
  uint32_t* lp_rmin;             // [kLabWarpLps] smallest staying key (ts bits)
  uint32_t* lp_low;              // [kLabWarpLps] something stays at or below j1
  uint32_t* lp_nmin;             // [kLabWarpLps] smallest live key of the first bucket above j1 holding one
  uint32_t* nx_cnt;              // [kLabWarpLps * 2] counts of the two buckets above j1
  uint32_t* misc;                // [4] staging count
  uint16_t* cseg;                // [kLabCandCap] source of each candidate: lpi << 3 | r
  uint16_t* sidx;                // [kLabWarpLps * kLabSafePerLp] safe candidates of each LP
};

__host__ __device__ constexpr size_t lab_warp_smem_bytes() {
  return ((size_t)kLabWarpLps * 16 + (size_t)kLabCandCap * 8 + (size_t)kLabStageCap * 4 +
          (size_t)(kLabWarpLps + 3 * kLabWarpLps * kLabSegMax + 1 + 7 * kLabWarpLps + 1 + 4) * 4 +
          (size_t)kLabCandCap * 2 + (size_t)kLabWarpLps * kLabSafePerLp * 2 + 15) & ~(size_t)15;
}

// LPs per warp chunk for a run with lookahead la, bucket width 1 / inv_w and E events per
// LP: the chunk's candidate keys (its LPs' range buckets, each holding about
// occ = E / (inv_w * (la + 1)) live keys, plus dead ones) within kLabCandCap and its safe
// events (about E * la / (la + 1) per LP per window) within kLabStageCap, with a margin,
// so that windows stay on the common path.
__host__ __device__ inline uint32_t lab_chunk_lps(float la, float inv_w, uint32_t E) {
  const float occ = (float)E / (inv_w * (la + 1.0f));
  const float cand = occ * (la * inv_w + 1.5f) + 1.0f;
  const float ev = (float)E * la / (la + 1.0f) + 0.5f;
  float n = 0.9f * (float)kLabCandCap / cand;
  const float n2 = 0.9f * (float)kLabStageCap / ev;
  if (n2 < n) n = n2;
  if (n > (float)kLabWarpLps) n = (float)kLabWarpLps;
  return n < 1.0f ? 1u : (uint32_t)n;
}

__host__ __device__ inline size_t lab_cta_smem_bytes(uint32_t block) { return (size_t)(block / 32) * lab_warp_smem_bytes(); }

__device__ __forceinline__ LabWarpSmem lab_warp_smem(unsigned char* base) {
  LabWarpSmem s;
  s.ls_csum = reinterpret_cast<unsigned long long*>(base);
  s.ls_ohash = s.ls_csum + kLabWarpLps;
  s.cand = s.ls_ohash + kLabWarpLps;
  s.cstage = reinterpret_cast<uint32_t*>(s.cand + kLabCandCap);
  s.stage = reinterpret_cast<gpq_item*>(s.cstage);
  s.ls_cnt = s.cstage + kLabStageCap;
  s.seg_raw = s.ls_cnt + kLabWarpLps;
  s.seg_off = s.seg_raw + kLabWarpLps * kLabSegMax;
  s.seg_kept = s.seg_off + kLabWarpLps * kLabSegMax + 1;
  s.lp_nsafe = s.seg_kept + kLabWarpLps * kLabSegMax;
  s.lp_soff = s.lp_nsafe + kLabWarpLps;
  s.lp_rmin = s.lp_soff + kLabWarpLps + 1;
  s.lp_low = s.lp_rmin + kLabWarpLps;
  s.lp_nmin = s.lp_low + kLabWarpLps;
  s.nx_cnt = s.lp_nmin + kLabWarpLps;
  s.misc = s.nx_cnt + 2 * kLabWarpLps;
  s.cseg = reinterpret_cast<uint16_t*>(s.misc + 4);
  s.sidx = s.cseg + kLabCandCap;
  return s;
}

// In-place exclusive prefix sum of a[0, n) by one warp (a[n] = the total, returned to every lane).
__device__ __forceinline__ uint32_t lab_warp_scan(uint32_t* a, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t per = (n + 31u) >> 5;
  const uint32_t b = min(n, lane * per), e = min(n, b + per);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; ++i) sum += a[i];
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(GPQ_FULL_MASK, incl, o);
    if (lane >= (uint32_t)o) incl += v;
  }
  const uint32_t total = __shfl_sync(GPQ_FULL_MASK, incl, 31);
  uint32_t run = incl - sum;
  for (uint32_t i = b; i < e; ++i) {
    const uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
  if (lane == 0) a[n] = total;
  __syncwarp();
  return total;
}

__device__ __forceinline__ void lab_state_load(const uint32_t* count, const unsigned long long* csum,
                                               const unsigned long long* ohash, const LabWarpSmem& sm, uint32_t lp0,
                                               uint32_t n) {
  for (uint32_t x = threadIdx.x & 31u; x < n; x += 32u) {
    sm.ls_cnt[x] = count[lp0 + x];
    sm.ls_csum[x] = csum[lp0 + x];
    sm.ls_ohash[x] = ohash[lp0 + x];
  }
  __syncwarp();
}

__device__ __forceinline__ void lab_state_load(const PholdDev& d, const LabWarpSmem& sm, uint32_t lp0, uint32_t n) {
  lab_state_load(d.count, d.csum, d.ohash, sm, lp0, n);
}

__device__ __forceinline__ void lab_state_store(uint32_t* count, unsigned long long* csum, unsigned long long* ohash,
                                                const LabWarpSmem& sm, uint32_t lp0, uint32_t n) {
  __syncwarp();
  for (uint32_t x = threadIdx.x & 31u; x < n; x += 32u) {
    count[lp0 + x] = sm.ls_cnt[x];
    csum[lp0 + x] = sm.ls_csum[x];
    ohash[lp0 + x] = sm.ls_ohash[x];
  }
}

__device__ __forceinline__ void lab_state_store(const PholdDev& d, const LabWarpSmem& sm, uint32_t lp0, uint32_t n) {
  lab_state_store(d.count, d.csum, d.ohash, sm, lp0, n);
}

// Next minimum of an LP with nothing live at or below j1: the smallest live key of the
// first bucket above j1 that holds one (kInfBits if none).  All lanes of one warp.
__device__ __forceinline__ uint32_t lab_scan_above(const LabDev& q, uint32_t lp, const LabWin& w) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t NB = 1u << q.nb_log2, nbm = NB - 1u, C = 1u << q.c_log2;
  const size_t lpb = (size_t)lp << q.nb_log2;
  uint32_t found = kInfBits;
  for (uint32_t jb0 = w.j1 + 1u; jb0 - w.j0 < NB && found == kInfBits; jb0 += 32u) {
    const uint32_t j = jb0 + lane;
    uint32_t c = 0;
    if (j - w.j0 < NB) c = min(ld_relaxed_u32(&q.cnt[lpb + (j & nbm)]), C);
    uint32_t nz = __ballot_sync(GPQ_FULL_MASK, c > 0);
    while (nz != 0u && found == kInfBits) {
      const uint32_t l = (uint32_t)__ffs(nz) - 1u;
      nz &= nz - 1u;
      const uint32_t cj = __shfl_sync(GPQ_FULL_MASK, c, l);
      const unsigned long long* bk = q.keys + ((lpb + ((jb0 + l) & nbm)) << q.c_log2);
      uint32_t v = kInfBits;
      for (uint32_t i = lane; i < cj; i += 32u) {
        const uint32_t t = (uint32_t)(ld_relaxed_u64(bk + i) >> 32);
        if (lab_live(t, w) && t < v) v = t;
      }
      found = warp_min_u32(v);
    }
  }
  return found;
}

// Events x0, x0 + stride, ... (up to four per thread) of a staging area (`get(x)` returns
// staged event x, or one whose aux is kStageHole): hashes into the LP accumulators and the
// children first, then all bucket reservations (independent atomics in flight together),
// then the stores.  Returns the children's minimum.
template <bool kShard, class Get>
__device__ __forceinline__ uint32_t lab_event_batch(const LabCtx& x, const LabDev& q, const PholdStage& st,
                                                    uint32_t ns, uint32_t x0, uint32_t stride, const LabWin& w, Get get) {
  constexpr int U = 4;
  const uint32_t nbm = (1u << q.nb_log2) - 1u, C = 1u << q.c_log2;
  unsigned long long key[U];
  uint32_t lp[U], jb[U], pos[U];
  uint32_t mn = kInfBits;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const uint32_t xi = x0 + (uint32_t)u * stride;
    lp[u] = ~0u;
    if (xi < ns) {
      const gpq_item e = get(xi);
      if (e.aux != kStageHole) {
        const uint32_t slot = e.aux >> 16, idx = e.aux & 0xffffu, tb = gpq_f2u(e.ts);
        const uint64_t h = gpq_ev_hash(e.id, tb);
        atomicAdd(&st.csum[slot], (unsigned long long)h);
        atomicAdd(&st.ohash[slot], (unsigned long long)gpq_seq_hash(h, (uint64_t)st.seq0[slot] + idx));
        const gpq_item ch = lab_child(x, e);
        const uint32_t cb = gpq_f2u(ch.ts);
        mn = min(mn, cb);
        if (!(kShard && lab_handover(x, q, w, ch))) {
          key[u] = lab_key(cb, ch.id);
          lp[u] = ch.lp;
          jb[u] = lab_bucket(cb, w.inv_w);
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    pos[u] = ~0u;
    if (lp[u] != ~0u && jb[u] >= w.j1 && jb[u] - w.j1p <= nbm)
      pos[u] = atomicAdd(&q.cnt[((size_t)lp[u] << q.nb_log2) + (jb[u] & nbm)], 1u);
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (lp[u] == ~0u) continue;
    if (pos[u] < C) {
      st_relaxed_u64(q.keys + ((((size_t)lp[u] << q.nb_log2) + (jb[u] & nbm)) << q.c_log2) + pos[u], key[u]);
    } else {
      const size_t sl = (size_t)w.curb * x.L + lp[u];
      const uint32_t sp = atomicAdd(&q.scnt[sl], 1u);
      if (sp < q.F) {
        q.spill[sl * q.F + sp] = key[u];
      } else {
        lab_fail(x, GPQ_ERR_QUEUE_FULL);
      }
    }
  }
  return mn;
}

// Key of candidate source r, slot i, of LP lp (bucket j1 read with relaxed loads: it may be
// appended to meanwhile).
__device__ __forceinline__ unsigned long long lab_load_cand(const LabCtx& x, const LabDev& q, const LabWin& w,
                                                            uint32_t nr, uint32_t lp, uint32_t r, uint32_t i) {
  const uint32_t nbm = (1u << q.nb_log2) - 1u;
  if (r < nr) {
    const unsigned long long* p = q.keys + ((((size_t)lp << q.nb_log2) + ((w.j0 + r) & nbm)) << q.c_log2) + i;
    return (r + 1u == nr) ? ld_relaxed_u64(p) : *p;
  }
  return q.spill[((size_t)w.prevb * x.L + lp) * q.F + i];
}

// y / d for the small operands of a warp chunk (y < 2^16 / d): inv = ceil(2^16 / d), and
// the error of the scaled reciprocal, below y / 2^16 < 1 / d, never reaches the next integer.
__device__ __forceinline__ uint32_t lab_recip16(uint32_t d) { return (65536u + d - 1u) / d; }
__device__ __forceinline__ uint32_t lab_div16(uint32_t y, uint32_t inv) { return (y * inv) >> 16; }

// One window for the chunk [lp0, lp0 + n) of one warp (outputs in sm.ls_*).  Returns this
// lane's part of the chunk minimum (LP next minima and children).  All lanes of the warp.
template <bool kShard = false>
static __device__ uint32_t lab_warp_window(const LabCtx& x, const LabDev& q, const LabWin& w, uint32_t lp0, uint32_t n,
                                    const LabWarpSmem& sm) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t L = x.L, NB = 1u << q.nb_log2, nbm = NB - 1u, C = 1u << q.c_log2;
  const uint32_t nr = w.j1 - w.j0 + 1u, S = nr + 1u;
  uint32_t mn = kInfBits;
  PholdStage st;
  st.ev = sm.stage;
  st.cnt = &sm.misc[0];
  st.seq0 = sm.ls_cnt;
  st.csum = sm.ls_csum;
  st.ohash = sm.ls_ohash;
  st.lp = nullptr;
  st.cap = kLabStageCap;

  // buckets the window left behind without a compaction: j1 of the previous window and any
  // bucket skipped by a jump of m (no append reaches their next use before this window)
  if (w.j0 > w.j1p) {
    const uint32_t nres = min(w.j0, w.j1p + NB) - w.j1p;
    for (uint32_t y = lane; y < n * nres; y += 32u) {
      const uint32_t lpi = y / nres, j = w.j1p + (y - lpi * nres);
      q.cnt[((size_t)(lp0 + lpi) << q.nb_log2) + (j & nbm)] = 0u;
    }
  }
  if (lane < n) {
    sm.lp_nsafe[lane] = 0u;
    sm.lp_rmin[lane] = kInfBits;
    sm.lp_low[lane] = 0u;
    sm.lp_nmin[lane] = kInfBits;
  }
  if (lane == 0) sm.misc[0] = 0u;

  uint32_t K = 0xffffffffu;
  if (S <= kLabSegMax) {
    // P1: range-bucket and spill counts, and the counts of the two buckets above j1 (every
    // load of a lane issued before any of its stores, so that they are in flight together)
    const uint32_t inv2 = lab_recip16(S + 2u), ny = n * (S + 2u);
    constexpr uint32_t kP1 = (kLabWarpLps * (kLabSegMax + 2u) + 31u) / 32u;
    uint32_t raw[kP1];
#pragma unroll
    for (uint32_t u = 0; u < kP1; ++u) {
      const uint32_t y = lane + 32u * u;
      raw[u] = 0u;
      if (y < ny) {
        const uint32_t lpi = lab_div16(y, inv2), r = y - lpi * (S + 2u), lp = lp0 + lpi;
        if (r < nr) {
          raw[u] = ld_relaxed_u32(&q.cnt[((size_t)lp << q.nb_log2) + ((w.j0 + r) & nbm)]);
        } else if (r == nr) {
          raw[u] = q.scnt[(size_t)w.prevb * L + lp];
        } else {
          const uint32_t j = w.j1 + 1u + (r - S);
          if (j - w.j0 < NB) raw[u] = ld_relaxed_u32(&q.cnt[((size_t)lp << q.nb_log2) + (j & nbm)]);
        }
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < kP1; ++u) {
      const uint32_t y = lane + 32u * u;
      if (y < ny) {
        const uint32_t lpi = lab_div16(y, inv2), r = y - lpi * (S + 2u);
        if (r < S) {
          const uint32_t ys = lpi * S + r;
          sm.seg_raw[ys] = raw[u];
          sm.seg_off[ys] = min(raw[u], r < nr ? C : q.F);
          sm.seg_kept[ys] = 0u;
        } else {
          sm.nx_cnt[lpi * 2u + (r - S)] = min(raw[u], C);
        }
      }
    }
    __syncwarp();
    // P2
    K = lab_warp_scan(sm.seg_off, n * S);
  }

  uint32_t scan_min = kInfBits, scan_lpi = ~0u;
  if (K <= kLabCandCap) {
    if (q.c_log2 <= 4u) {
      // buckets of at most 16 slots: each (LP, source) segment writes its code (LP index << 3 |
      // source) over its candidate slots, and the candidate loads read it
      const uint32_t invs = lab_recip16(S);
      for (uint32_t y = lane; y < n * S; y += 32u) {
        const uint32_t a = sm.seg_off[y], b = sm.seg_off[y + 1u], lpi = lab_div16(y, invs);
        const uint16_t code = (uint16_t)((lpi << 3) | (y - lpi * S));
        for (uint32_t k = a; k < b; ++k) sm.cseg[k] = code;
      }
      __syncwarp();
      // P3: candidate keys, up to 8 per lane, all loads in flight together
      constexpr uint32_t U = kLabCandCap / 32u;
      unsigned long long v[U];
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t k = lane + 32u * u;
        v[u] = 0;
        if (k < K) {
          const uint32_t sg = sm.cseg[k], lo = sg >> 3, r = sg & 7u;
          v[u] = lab_load_cand(x, q, w, nr, lp0 + lo, r, k - sm.seg_off[lo * S + r]);
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t k = lane + 32u * u;
        if (k < K) sm.cand[k] = v[u];
      }
    } else {
      // larger buckets (long segments, few LPs a chunk): each candidate finds its segment
      // by a search next to its load
      constexpr uint32_t U = kLabCandCap / 32u;
      unsigned long long v[U];
      uint32_t sg[U];
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t k = lane + 32u * u;
        sg[u] = ~0u;
        v[u] = 0;
        if (k < K) {
          uint32_t lo = 0, hi = n;  // LP: seg_off[lo * S] <= k < seg_off[hi * S]
          while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.seg_off[mid * S] <= k) lo = mid; else hi = mid;
          }
          uint32_t r = 0;
          while (r + 1u < S && sm.seg_off[lo * S + r + 1u] <= k) ++r;
          sg[u] = (lo << 3) | r;
          v[u] = lab_load_cand(x, q, w, nr, lp0 + lo, r, k - sm.seg_off[lo * S + r]);
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        if (sg[u] != ~0u) {
          const uint32_t k = lane + 32u * u;
          sm.cand[k] = v[u];
          sm.cseg[k] = (uint16_t)sg[u];
        }
      }
    }
    __syncwarp();
    // P4a (read-only): safe candidates into their LP's list; the minimum and the "stays at
    // or below j1" flag of each LP
#pragma unroll 4
    for (uint32_t k = lane; k < K; k += 32u) {
      const uint32_t sg = sm.cseg[k], lpi = sg >> 3, r = sg & 7u;
      const uint32_t t = (uint32_t)(sm.cand[k] >> 32);
      if (!lab_live(t, w)) continue;  // dead, or a slot not written yet
      if (t < w.safe_lim) {
        const uint32_t p = atomicAdd(&sm.lp_nsafe[lpi], 1u);
        if (p < kLabSafePerLp) sm.sidx[lpi * kLabSafePerLp + p] = (uint16_t)k;
        continue;
      }
      atomicMin(&sm.lp_rmin[lpi], t);
      if (r < nr || lab_bucket(t, w.inv_w) <= w.j1) sm.lp_low[lpi] = 1u;
    }
    __syncwarp();
  }
  const bool common = K <= kLabCandCap && !__any_sync(GPQ_FULL_MASK, lane < n && sm.lp_nsafe[lane] > kLabSafePerLp);
  if (common) {
    // P4b: compaction of the buckets below j1 and re-filing of the spill list
    for (uint32_t k = lane; k < K; k += 32u) {
      const uint32_t sg = sm.cseg[k], lpi = sg >> 3, r = sg & 7u;
      const unsigned long long key = sm.cand[k];
      const uint32_t t = (uint32_t)(key >> 32);
      if (!lab_live(t, w) || t < w.safe_lim) continue;
      const uint32_t lp = lp0 + lpi;
      if (r < nr) {
        if (r + 1u < nr) {  // a bucket below j1: compact (the staying keys keep their order)
          const uint32_t sgi = lpi * S + r, a = sm.seg_off[sgi];
          uint32_t p = 0;
          for (uint32_t y = a; y < k; ++y) {
            const uint32_t t2 = (uint32_t)(sm.cand[y] >> 32);
            p += (lab_live(t2, w) && t2 >= w.safe_lim) ? 1u : 0u;
          }
          atomicAdd(&sm.seg_kept[sgi], 1u);
          if (p != k - a) q.keys[((((size_t)lp << q.nb_log2) + ((w.j0 + r) & nbm)) << q.c_log2) + p] = key;
        }
      } else {
        lab_push(x, q, lp, key, lab_bucket(t, w.inv_w), w);
      }
    }
    __syncwarp();
    // P5
    if (lane < n) {
      const uint32_t lp = lp0 + lane;
      for (uint32_t r = 0; r + 1u < nr; ++r) {
        const uint32_t y = lane * S + r;
        if (sm.seg_kept[y] != sm.seg_raw[y]) q.cnt[((size_t)lp << q.nb_log2) + ((w.j0 + r) & nbm)] = sm.seg_kept[y];
      }
      if (sm.seg_raw[lane * S + nr] != 0u) q.scnt[(size_t)w.prevb * L + lp] = 0u;
      sm.lp_soff[lane] = sm.lp_nsafe[lane];
    }
    __syncwarp();
    const uint32_t nsafe = lab_warp_scan(sm.lp_soff, n);
    if (lane == 0) sm.misc[0] = nsafe;
    // LP of every staging position below kLabStageCap (a byte map in seg_kept, free after P5)
    uint8_t* spl = reinterpret_cast<uint8_t*>(sm.seg_kept);
    static_assert(kLabWarpLps * kLabSegMax * 4 >= kLabStageCap && kLabWarpLps <= 256, "staging map");
    if (lane < n) {
      const uint32_t e = min(sm.lp_soff[lane + 1u], kLabStageCap);
      for (uint32_t u = sm.lp_soff[lane]; u < e; ++u) spl[u] = (uint8_t)lane;
    }
    __syncwarp();
    // P6: rank each safe key among its LP's safe keys and stage it at (LP offset + rank)
    for (uint32_t u = lane; u < nsafe; u += 32u) {
      uint32_t lo = 0, hi = n;  // LP: lp_soff[lo] <= u < lp_soff[lo + 1]
      if (u < kLabStageCap) {
        lo = spl[u];
      } else {
        while (hi - lo > 1u) {
          const uint32_t mid = (lo + hi) >> 1;
          if (sm.lp_soff[mid] <= u) lo = mid; else hi = mid;
        }
      }
      const uint16_t* li = sm.sidx + lo * kLabSafePerLp;
      const uint32_t ns_lp = sm.lp_nsafe[lo];
      const uint32_t k = li[u - sm.lp_soff[lo]];
      const unsigned long long key = sm.cand[k];
      uint32_t rank = 0;
#pragma unroll 4  // the keys' loads overlap
      for (uint32_t y = 0; y < ns_lp; ++y) rank += (sm.cand[li[y]] < key) ? 1u : 0u;
      const uint32_t pos = sm.lp_soff[lo] + rank;
      if (pos < kLabStageCap) {
        sm.cstage[pos] = k | (rank << 8) | (lo << 16);
      } else {
        gpq_item e;
        e.ts = gpq_u2f((uint32_t)(key >> 32));
        e.lp = lp0 + lo;
        e.id = (uint32_t)key;
        e.aux = (lo << 16) | rank;
        mn = min(mn, lab_process_event<kShard>(x, q, st, e, w));
      }
    }
    // next-minimum scan of the LPs with nothing live at or below j1, when one of the two
    // buckets above j1 holds keys: two lanes per LP issue their loads here and use them
    // after the event pass
    if (lane < 2u * n) {
      const uint32_t lpi = lane >> 1;
      if (sm.lp_low[lpi] == 0u) {
        const uint32_t c0 = sm.nx_cnt[2u * lpi], c1 = sm.nx_cnt[2u * lpi + 1u];
        const uint32_t r = c0 ? 0u : 1u, c = c0 ? c0 : c1;
        if (c > 0u && c <= 16u) {
          const unsigned long long* bk =
              q.keys + ((((size_t)(lp0 + lpi) << q.nb_log2) + ((w.j1 + 1u + r) & nbm)) << q.c_log2);
          uint32_t tv[8];
#pragma unroll
          for (uint32_t u = 0; u < 8u; ++u) {
            const uint32_t i = (lane & 1u) + 2u * u;
            tv[u] = (i < c) ? (uint32_t)(ld_relaxed_u64(bk + i) >> 32) : 0xffffffffu;
          }
          scan_lpi = lpi;
#pragma unroll
          for (uint32_t u = 0; u < 8u; ++u)
            if (lab_live(tv[u], w) && tv[u] < scan_min) scan_min = tv[u];
        }
      }
    }
    __syncwarp();
  } else {
    // general path: the warp as one lane group per LP
    const LaneGroup<32> g;
    st.cap = kLabItemStageCap;
    if (lane < n) sm.lp_nsafe[lane] = 0u;
    __syncwarp();
    for (uint32_t lpi = 0; lpi < n; ++lpi) {
      const uint32_t lp = lp0 + lpi;
      const LabMeta mt = lab_load_meta(x, q, lp, w, g.gl);
      mn = min(mn, lab_lp_stage<32, kShard>(x, q, lp, lpi, w, sm.cand, st, g, mt, sm.lp_nsafe));
    }
    __syncwarp();
  }

  // P7: events (four in flight per lane), then the next minimum of each LP
  if (common) {
    const uint32_t ns = min(sm.misc[0], kLabStageCap);
    auto get = [&](uint32_t y) {
      const uint32_t c = sm.cstage[y], lpi = c >> 16;
      const unsigned long long key = sm.cand[c & 0xffu];
      gpq_item e;
      e.ts = gpq_u2f((uint32_t)(key >> 32));
      e.lp = lp0 + lpi;
      e.id = (uint32_t)key;
      e.aux = (lpi << 16) | ((c >> 8) & 0xffu);
      return e;
    };
    for (uint32_t x0 = lane; x0 < ns; x0 += 128u) mn = min(mn, lab_event_batch<kShard>(x, q, st, ns, x0, 32u, w, get));
  } else {
    const uint32_t ns = min(sm.misc[0], kLabItemStageCap);
    auto get = [&](uint32_t y) { return sm.stage[y]; };
    for (uint32_t x0 = lane; x0 < ns; x0 += 128u) mn = min(mn, lab_event_batch<kShard>(x, q, st, ns, x0, 32u, w, get));
  }
  if (common) {
    if (scan_lpi != ~0u && scan_min != kInfBits) atomicMin(&sm.lp_nmin[scan_lpi], scan_min);
    __syncwarp();
    bool deep = false;
    if (lane < n) {
      uint32_t lm = sm.lp_rmin[lane];
      if (sm.lp_low[lane] == 0u) {
        const uint32_t nm = sm.lp_nmin[lane];
        if (nm != kInfBits) lm = min(lm, nm);
        else deep = true;
      }
      mn = min(mn, lm);
    }
    uint32_t dz = __ballot_sync(GPQ_FULL_MASK, deep);
    while (dz != 0u) {  // rare: scan bucket by bucket above j1
      const uint32_t l = (uint32_t)__ffs(dz) - 1u;
      dz &= dz - 1u;
      mn = min(mn, lab_scan_above(q, lp0 + l, w));
    }
  }
  __syncwarp();
  if (lane < n) sm.ls_cnt[lane] += sm.lp_nsafe[lane];
  __syncwarp();
  return mn;
}

// One window for the LPs [lp_lo, lp_hi) of this CTA, split evenly among its warps.  Each
// warp min's its part of the next window's minimum into red[0] (shared); the caller
// publishes the CTA's minimum to mins[(s+1)%3].  `resident`: every warp owns at most one
// chunk, whose outputs stay in shared memory between windows.
template <bool kShard>
__device__ __forceinline__ void lab_window_body(const PholdDev& d, const LabDev& q, uint32_t s, float m, uint32_t j1p,
                                                unsigned char* smem_raw, uint32_t* red, uint32_t lp_lo,
                                                uint32_t lp_hi, bool resident) {
  const LabWin w = lab_window_of(d.p, q.inv_w, s, m, j1p);
  LabCtx x{d.p, d.L, 0u, &d.ctrl->err, &d.ctrl->errs[(s + 1u) % 3u]};
  if (kShard && d.outbox != nullptr) {
    x.outbox = d.outbox;
    x.out_n = d.out_n;
    x.out_cap = d.out_cap;
    x.shard_lps = d.shard_lps;
    x.lp_begin = d.lp_begin;
    x.lp_end = d.lp_end;
    x.peers = static_cast<const LabPeer*>(d.peers);
  }
  const uint32_t warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const LabWarpSmem sm = lab_warp_smem(smem_raw + (size_t)warp * lab_warp_smem_bytes());
  const uint32_t pw = (lp_hi - lp_lo + nw - 1u) / nw;
  const uint32_t wlo = min(lp_hi, lp_lo + warp * pw), whi = min(lp_hi, wlo + pw);
  uint32_t mn = kInfBits;
  for (uint32_t c0 = wlo; c0 < whi; c0 += q.chunk) {
    const uint32_t n = min(q.chunk, whi - c0);
    if (!resident) lab_state_load(d, sm, c0, n);
    mn = min(mn, lab_warp_window<kShard>(x, q, w, c0, n, sm));
    if (!resident) lab_state_store(d, sm, c0, n);
  }
  mn = warp_min_u32(mn);
  if ((threadIdx.x & 31u) == 0 && mn != kInfBits) atomicMin(&red[0], mn);  // the CTA's minimum (kInfBits: none)
}

// LPs a CTA of `block` threads covers in one launch of the plain form.
__host__ __device__ inline uint32_t lab_plain_lps_per_cta(uint32_t block, uint32_t chunk) { return (block / 32u) * chunk; }

// Plain form: one launch per window (kShard: the window of one shard of a sharded run,
// children of other shards' LPs handed over).
template <bool kShard>
static __global__ void __launch_bounds__(1024, 1) lab_window_kernel(PholdDev d, LabDev q, uint32_t s) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t red[32];
  const uint32_t mb = d.ctrl->mins[s % 3u];
  const float m = gpq_u2f(mb);
  if (!(m < d.p.end_time)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.ctrl->mins[(s + 2u) % 3u] = kInfBits;
    d.ctrl->errs[(s + 2u) % 3u] = 0u;
    d.ctrl->steps += 1ull;
    d.ctrl->phase = s + 1u;
    q.wj[s & 3u] = lab_bucket(gpq_f2u(GPQ_FADD(m, d.p.lookahead)), q.inv_w);
  }
  const uint32_t per = (blockDim.x / 32u) * q.chunk;  // a shard works its own LPs [lp_begin, lp_end)
  const uint32_t lp_lo = min(d.lp_end, d.lp_begin + blockIdx.x * per), lp_hi = min(d.lp_end, lp_lo + per);
  if (threadIdx.x == 0) red[0] = kInfBits;
  __syncthreads();
  lab_window_body<kShard>(d, q, s, m, ld_relaxed_u32(&q.wj[(s + 3u) & 3u]), smem_raw, red, lp_lo, lp_hi, false);
  __syncthreads();
  if (threadIdx.x == 0 && red[0] != kInfBits) atomicMin(&d.ctrl->mins[(s + 1u) % 3u], red[0]);
}

// Persistent form: all windows in one cooperative launch, a bounded grid barrier per window.
static __global__ void __launch_bounds__(1024, 1) lab_persistent_kernel(PholdDev d, LabDev q, uint32_t s0,
                                                                       uint32_t max_steps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t red[32];
  const uint32_t per = (d.L + gridDim.x - 1u) / gridDim.x;
  const uint32_t lp_lo = min(d.L, blockIdx.x * per), lp_hi = min(d.L, lp_lo + per);
  const uint32_t warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t pw = (lp_hi - lp_lo + nw - 1u) / nw;
  const uint32_t wlo = min(lp_hi, lp_lo + warp * pw), whi = min(lp_hi, wlo + pw);
  const bool resident = (per + nw - 1u) / nw <= q.chunk;
  const LabWarpSmem sm = lab_warp_smem(smem_raw + (size_t)warp * lab_warp_smem_bytes());
  if (resident) lab_state_load(d, sm, wlo, whi - wlo);
  if (threadIdx.x == 0) red[0] = kInfBits;  // the CTA's part of the next window's minimum
  __syncthreads();
  unsigned long long target = 0;
  uint32_t s = s0;
  // j1 of the previous window: read once, then carried in registers (every CTA computes
  // what block 0 records in q.wj for the plain form and the next launch)
  uint32_t j1p = ld_relaxed_u32(&q.wj[(s0 + 3u) & 3u]);
  for (;; ++s) {
    const uint32_t mb = ld_relaxed_u32(&d.ctrl->mins[s % 3u]);
    const uint32_t eb = ld_relaxed_u32(&d.ctrl->errs[s % 3u]);
    const float m = gpq_u2f(mb);
    if (!(m < d.p.end_time) || eb != 0u || (max_steps != 0u && s - s0 >= max_steps)) break;
    const uint32_t j1 = lab_bucket(gpq_f2u(GPQ_FADD(m, d.p.lookahead)), q.inv_w);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      d.ctrl->mins[(s + 2u) % 3u] = kInfBits;
      d.ctrl->errs[(s + 2u) % 3u] = 0u;
      d.ctrl->steps += 1ull;
      q.wj[s & 3u] = j1;
    }
    lab_window_body<false>(d, q, s, m, j1p, smem_raw, red, lp_lo, lp_hi, resident);
    j1p = j1;
    target += gridDim.x;
    if (!grid_barrier_min(&d.ctrl->bar, target, d.spin_limit, &d.ctrl->err, &red[0], &d.ctrl->mins[(s + 1u) % 3u])) {
      s += 1u;
      break;
    }
  }
  if (resident) lab_state_store(d, sm, wlo, whi - wlo);
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctrl->phase = s;
}

// Population (src/phold.cu:63-79,124-163), one thread per initial event: event k of LP l
// (id l*per_lp + k) goes to its bucket of the absolute range [0, NB), or to the spill list
// read by window 0.  Keys, counts and spill counts were reset by the host.  Also computes
// the first window minimum into mins[0] and zeroes the PHOLD outputs.
static __global__ void lab_populate_kernel(PholdDev d, LabDev q, uint32_t per_lp, const gpq_item* __restrict__ src) {
  __shared__ uint32_t red[32];
  const uint64_t n = (uint64_t)d.L * per_lp;
  const uint32_t NB = 1u << q.nb_log2, C = 1u << q.c_log2;
  uint32_t mn = kInfBits;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t lp = (uint32_t)(i / per_lp), k = (uint32_t)(i % per_lp);
    if (lp < d.lp_begin || lp >= d.lp_end) {  // another shard's LP: outputs only
      if (k == 0) {
        d.count[lp] = 0;
        d.csum[lp] = 0;
        d.ohash[lp] = 0;
      }
      continue;
    }
    gpq_item e;
    if (src) {
      e = src[i];
      if (e.lp != lp) gpq_set_error(&d.ctrl->err, GPQ_ERR_INVALID);
    } else {
      e = gpq_phold_initial(d.p, lp, k, per_lp);
    }
    const uint32_t tb = gpq_f2u(e.ts);
    const unsigned long long key = lab_key(tb, e.id);
    const uint32_t jb = lab_bucket(tb, q.inv_w);
    bool placed = false;
    if (jb < NB) {
      const size_t b = ((size_t)lp << q.nb_log2) + jb;
      const uint32_t pos = atomicAdd(&q.cnt[b], 1u);
      if (pos < C) {
        q.keys[(b << q.c_log2) + pos] = key;
        placed = true;
      }
    }
    if (!placed) {
      const size_t sl = (size_t)d.L + lp;  // parity 1: the list window 0 reads
      const uint32_t pos = atomicAdd(&q.scnt[sl], 1u);
      if (pos < q.F) q.spill[sl * q.F + pos] = key;
      else gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL);
    }
    mn = min(mn, tb);
    if (k == 0) {
      d.count[lp] = 0;
      d.csum[lp] = 0;
      d.ohash[lp] = 0;
    }
  }
  mn = block_min_u32(mn, red);
  if (threadIdx.x == 0 && mn != kInfBits) atomicMin(&d.ctrl->mins[0], mn);
}

// A shard's handed-over children of window s (made by other shards, all for this shard's
// LPs), filed as if this shard had pushed them during window s: bucket or spill list of the
// window's parity.
static __global__ void lab_inject_kernel(PholdDev d, LabDev q, const gpq_item* __restrict__ items, uint64_t n,
                                         uint32_t s) {
  const float m = gpq_u2f(d.ctrl->mins[s % 3u]);
  const LabWin w = lab_window(d, q, s, m);
  const LabCtx x{d.p, d.L, 0u, &d.ctrl->err, &d.ctrl->errs[(s + 1u) % 3u]};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const gpq_item it = items[i];
    if (it.lp < d.lp_begin || it.lp >= d.lp_end) {
      gpq_set_error(&d.ctrl->err, GPQ_ERR_INVALID);
      continue;
    }
    const uint32_t tb = gpq_f2u(it.ts);
    lab_push(x, q, it.lp, lab_key(tb, it.id), lab_bucket(tb, w.inv_w), w);
  }
}

// End of run: committed total, pending events (the live keys of the buckets + the spill
// list of the last window) and the order-sensitive digest.  One warp per LP.
static __global__ void lab_finalize_kernel(PholdDev d, LabDev q, PholdAcc* acc) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t wpb = blockDim.x >> 5;
  const uint32_t nwarps = gridDim.x * wpb;
  const uint32_t phase = d.ctrl->phase;
  const uint32_t prevb = (phase + 1u) & 1u;
  const uint32_t mb = d.ctrl->mins[phase % 3u];  // every pending event is >= the next window's minimum
  const uint32_t NB = 1u << q.nb_log2, C = 1u << q.c_log2;
  uint64_t pend = 0, pcs = 0, dig = 0, com = 0;
  uint32_t pmin = kInfBits;
  for (uint32_t lp = d.lp_begin + blockIdx.x * wpb + (threadIdx.x >> 5); lp < d.lp_end; lp += nwarps) {  // a shard: its LPs
    const size_t lpb = (size_t)lp << q.nb_log2;
    for (uint32_t b0 = 0; b0 < NB; b0 += 32) {
      const uint32_t c = (b0 + lane < NB) ? min(q.cnt[lpb + b0 + lane], C) : 0u;
      uint32_t nz = __ballot_sync(GPQ_FULL_MASK, c > 0);
      while (nz) {
        const uint32_t l = (uint32_t)__ffs(nz) - 1u;
        nz &= nz - 1u;
        const uint32_t cl = __shfl_sync(GPQ_FULL_MASK, c, l);
        const unsigned long long* bk = q.keys + ((lpb + b0 + l) << q.c_log2);
        for (uint32_t i = lane; i < cl; i += 32) {
          const unsigned long long k = bk[i];
          const uint32_t t = (uint32_t)(k >> 32);
          if (t < mb || t > kInfBits) continue;  // dead: consumed in an earlier window
          pcs += gpq_ev_hash((uint32_t)k, t);
          pend += 1;
          pmin = min(pmin, t);
        }
      }
    }
    const size_t sl = (size_t)prevb * d.L + lp;
    const uint32_t sc = min(q.scnt[sl], q.F);
    for (uint32_t i = lane; i < sc; i += 32) {
      const unsigned long long k = q.spill[sl * q.F + i];
      const uint32_t t = (uint32_t)(k >> 32);
      pcs += gpq_ev_hash((uint32_t)k, t);
      pend += 1;
      pmin = min(pmin, t);
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

// Kernel pointers (host-side dispatch).  The window is warp-owned for every lanes_per_lp;
// a shard of a sharded run (which runs window by window) takes the window that hands
// children over, every other run the one without that code.
struct LabKernelSet {
  const void* window;
  const void* persistent;
};

inline bool lab_kernel_set(uint32_t group, LabKernelSet* out, bool sharded = false) {
  if (group != 4 && group != 8 && group != 16 && group != 32) return false;
  *out = {sharded ? (const void*)lab_window_kernel<true> : (const void*)lab_window_kernel<false>,
          (const void*)lab_persistent_kernel};
  return true;
}
