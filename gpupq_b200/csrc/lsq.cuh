// Local splay queue (LSQ), B200 form.
//
// Reference: src/local_splay_queue.cu.  Each LP owns a top-down splay tree (Sleator's
// public-domain code, credited in the reference's header comment) over a per-LP node
// pool of 32-byte nodes with two child pointers (:108-156 splay, :158-202 insert,
// :233-273 delete_min); free nodes are found by scanning the pool (:72-93);
// queue_post inserts the buffered items one by one (:435-454).
//
// Here nodes are pool indices, not pointers: an LP's pool is items[lp << cap_log2 ...]
// (16-byte items) plus a 32-bit link word per node (left << 16 | right, 0xffff = none),
// so a node costs 20 bytes and the structure is relocatable.  Free nodes come from a
// per-LP stack (O(1) instead of a pool scan).  Free pool slots carry lp = 0xffffffff.
// A splay tree is a pointer-chasing sequential structure, so each LP is handled by one
// lane; the window's safe events are popped with splay-to-minimum (top-down splay with
// a key below every item) and staged for the CTA-wide event pass.
#pragma once

#include "phold_common.cuh"

static constexpr uint32_t kLsqNil = 0xffffu;
static constexpr uint32_t kLsqHdr = 0x10000u;  // the splay's header node (not in the pool)

struct LsqDev {
  gpq_item* items;   // num_lps << cap_log2 node items
  uint32_t* links;   // num_lps << cap_log2 link words
  uint16_t* freestk; // num_lps << cap_log2 free-node stacks
  uint32_t* root;    // per-LP root index (kLsqNil = empty)
  uint32_t* size;    // per-LP node count
  uint32_t* freetop; // per-LP free-stack height
  uint32_t cap_log2;
};

struct LsqView {
  gpq_item* it;
  uint32_t* ln;
  __device__ __forceinline__ uint32_t left(uint32_t x) const { return ln[x] >> 16; }
  __device__ __forceinline__ uint32_t right(uint32_t x) const { return ln[x] & 0xffffu; }
  __device__ __forceinline__ void set_left(uint32_t x, uint32_t v) const { ln[x] = (ln[x] & 0xffffu) | (v << 16); }
  __device__ __forceinline__ void set_right(uint32_t x, uint32_t v) const { ln[x] = (ln[x] & 0xffff0000u) | v; }
  __device__ __forceinline__ uint64_t key(uint32_t x) const { return gpq_lp_key(it[x]); }
};

// Top-down splay of `key` in the tree rooted at t (Sleator-Tarjan 1985, top-down
// variant): returns the new root, the last node on the search path for `key`.
__device__ __forceinline__ uint32_t lsq_splay(const LsqView& v, uint32_t t, uint64_t key) {
  if (t == kLsqNil) return t;
  uint32_t n_left = kLsqNil, n_right = kLsqNil;  // the header's left and right trees
  uint32_t l = kLsqHdr, r = kLsqHdr;
  for (;;) {
    if (key <= v.key(t)) {
      uint32_t tl = v.left(t);
      if (tl == kLsqNil) break;
      if (key < v.key(tl)) {  // rotate right
        v.set_left(t, v.right(tl));
        v.set_right(tl, t);
        t = tl;
        tl = v.left(t);
        if (tl == kLsqNil) break;
      }
      if (r == kLsqHdr) n_left = t; else v.set_left(r, t);  // link right
      r = t;
      t = tl;
    } else {
      uint32_t tr = v.right(t);
      if (tr == kLsqNil) break;
      if (key > v.key(tr)) {  // rotate left
        v.set_right(t, v.left(tr));
        v.set_left(tr, t);
        t = tr;
        tr = v.right(t);
        if (tr == kLsqNil) break;
      }
      if (l == kLsqHdr) n_right = t; else v.set_right(l, t);  // link left
      l = t;
      t = tr;
    }
  }
  const uint32_t tl = v.left(t), tr = v.right(t);  // assemble
  if (l == kLsqHdr) n_right = tl; else v.set_right(l, tl);
  if (r == kLsqHdr) n_left = tr; else v.set_left(r, tr);
  v.ln[t] = (n_right << 16) | n_left;
  return t;
}

// Insert node x (item already stored) into the tree rooted at t; returns the new root.
__device__ __forceinline__ uint32_t lsq_insert(const LsqView& v, uint32_t t, uint32_t x) {
  if (t == kLsqNil) {
    v.ln[x] = (kLsqNil << 16) | kLsqNil;
    return x;
  }
  const uint64_t kx = v.key(x);
  t = lsq_splay(v, t, kx);
  if (kx <= v.key(t)) {
    v.ln[x] = (v.left(t) << 16) | t;
    v.set_left(t, kLsqNil);
  } else {
    v.ln[x] = (t << 16) | v.right(t);
    v.set_right(t, kLsqNil);
  }
  return x;
}

struct LsqMeta {
  uint32_t k, root, size, freetop, count;
  unsigned long long csum, ohash;
};

__device__ __forceinline__ LsqMeta lsq_load_meta(const PholdDev& d, const LsqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t prevb) {
  LsqMeta m;
  m.k = ib.cnt[(size_t)prevb * d.L + lp];
  m.root = q.root[lp];
  m.size = q.size[lp];
  m.freetop = q.freetop[lp];
  m.count = d.count[lp];
  m.csum = d.csum[lp];
  m.ohash = d.ohash[lp];
  return m;
}

// One LP (one lane), one window s: insert the children of window s-1, then remove the
// minimum while it is safe and stage it.  Returns the new minimum's timestamp bits,
// min'ed with any child processed here.
__device__ __forceinline__ uint32_t lsq_lp_stage(const PholdDev& d, const LsqDev& q, const InsDev& ib, uint32_t lp,
                                                 uint32_t slot, uint32_t s, float bound, const PholdStage& st,
                                                 const LaneGroup<1>& g, uint32_t* err_slot, const LsqMeta& mt) {
  const uint32_t L = d.L;
  const uint32_t prevb = (s + 1u) & 1u, curb = s & 1u;
  const size_t base = (size_t)lp << q.cap_log2;
  const LsqView v{q.items + base, q.links + base};
  uint16_t* fs = q.freestk + base;
  const float T = d.p.end_time;
  uint32_t root = mt.root, size = mt.size, ftop = mt.freetop;
  uint32_t k = mt.k;
  if (k > 0) {
    if (k > ib.ibc) k = ib.ibc;
    const gpq_item* src = ib.buf + ((size_t)prevb * L + lp) * ib.ibc;
    for (uint32_t j = 0; j < k; ++j) {
      if (ftop == 0) {
        gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL);
        atomicOr(err_slot, 1u);
        break;
      }
      const uint32_t x = fs[--ftop];
      v.it[x] = src[j];
      root = lsq_insert(v, root, x);
      ++size;
    }
    ib.cnt[(size_t)prevb * L + lp] = 0;
  }
  phold_stage_slot_init(st, slot, mt.count, mt.csum, mt.ohash);
  uint32_t done = 0, cmin = kInfBits, head = kInfBits;
  while (root != kLsqNil) {
    root = lsq_splay(v, root, 0ull);  // the minimum becomes the root, with no left child
    gpq_item e = v.it[root];
    if (!((e.ts < bound) && (e.ts < T))) { head = gpq_f2u(e.ts); break; }
    cmin = min(cmin, phold_stage_batch<1>(d, ib, st, g, e, true, done, 1, slot, curb, err_slot));
    const uint32_t x = root;
    root = v.right(x);
    v.it[x].lp = 0xffffffffu;  // free pool slot
    fs[ftop++] = (uint16_t)x;
    --size;
    ++done;
  }
  q.root[lp] = root;
  q.size[lp] = size;
  q.freetop[lp] = ftop;
  st.lp[slot] = done > 0 ? lp : ~0u;
  if (done > 0) d.count[lp] = mt.count + done;
  return min(head, cmin);
}

struct LsqPolicy {
  static constexpr int G = 1;
  using Dev = LsqDev;
  using Meta = LsqMeta;
  struct Smem {};
  __host__ __device__ static size_t group_smem_bytes(uint32_t) { return 0; }
  __device__ static Smem smem(unsigned char*, uint32_t) { return Smem{}; }
  __device__ static Meta load_meta(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t prevb) {
    return lsq_load_meta(d, q, ib, lp, prevb);
  }
  __device__ static uint32_t stage_lp(const PholdDev& d, const Dev& q, const InsDev& ib, uint32_t lp, uint32_t slot,
                                      uint32_t s, float bound, const Smem&, const PholdStage& st,
                                      const LaneGroup<1>& g, uint32_t* err_slot, const Meta& mt) {
    return lsq_lp_stage(d, q, ib, lp, slot, s, bound, st, g, err_slot, mt);
  }
};
