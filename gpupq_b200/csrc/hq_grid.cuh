// Parallel heap queue with large nodes, worked by the whole GPU (PHOLD engine, node sizes
// above the one-CTA limit kHqMaxR).
//
// Reference: src/heap_queue.cu merges a root of HQ_NODE_SIZE items (256 K by default,
// src/config.h:88) with moderngpu over the whole GPU, node by node, driven from host
// threads (:1541-1553, :1609-1774).  Here the heap keeps the layout and the operations of
// hq.cuh -- sorted r-item nodes with max(parent) <= min(child), insert-update pieces along
// root-to-target paths, the root's safe prefix in batches, copy-last and delete-update --
// inside one persistent cooperative launch over every SM:
//   * merges are tiled: a CTA takes kHqgTile outputs, finds where they start and end in
//     both inputs with a block-wide search (each round probes 256 positions at once, so a
//     split costs three or four global round trips, not twenty), stages both input slices
//     in shared memory and merges kHqgIpt outputs per thread there;
//   * sorts are a block merge sort per chunk (a sorting network in registers, then
//     merge rounds in shared memory) followed by tiled merge rounds over the chunks;
//   * the heap's control state (root buffer and offset, root count, last node and its
//     count: every node between the root and the last one is full) lives in registers of
//     every thread, and every block takes each decision itself from data that no block
//     writes in the same phase, so phases are separated by data barriers only;
//   * the root has two buffers and an offset: a batch's removal advances the offset, and
//     every merge into the root writes the other buffer;
//   * the refill takes the largest items of the last node(s) -- suffixes of sorted nodes,
//     so one merge of at most two runs replaces a sort;
//   * when the root holds every item (the global array queue's layout; the reference's
//     256 K root on small populations), a window is three phases over bucket lists that
//     each phase fills for the next, instead of grid-wide sorts (see the list section).
// A batch's per-LP ranks (the order-sensitive hash needs each event's position in its
// LP's sequence) come from a sort of (lp, position) keys: an event's rank is its LP's
// count so far plus its distance from the first key of its LP.
#pragma once

#include "hq.cuh"

static constexpr uint32_t kHqgThreads = 512;
static constexpr uint32_t kHqgIpt = 8;                          // items per thread (sorts, merges)
static constexpr uint32_t kHqgTile = kHqgThreads * kHqgIpt;     // 4,096 items per CTA tile
static constexpr uint32_t kHqgKpt = 16;                         // keys per thread
static constexpr uint32_t kHqgKeyTile = kHqgThreads * kHqgKpt;  // 8,192 keys per CTA tile
static constexpr uint32_t kHqgMaxR = 1u << 22;                  // node size limit of the grid form

// Shared memory: two tiles, padded by one element per kPer (a thread's run), so that a
// thread's kPer consecutive elements and its neighbours' fall in different banks; then an
// auxiliary area of kHqgAux words (bin counts, and one packed word per element of a tile)
// for the counting sorts and the bucket lists.
static constexpr uint32_t kHqgAux = 16384;
static constexpr uint32_t kHqgBins = kHqgAux / 2;  // bins of a counting sort
__host__ __device__ inline size_t hqg_tiles_bytes() {
  return 2 * (size_t)(kHqgTile + kHqgTile / kHqgIpt) * sizeof(gpq_item);
}
__host__ __device__ inline size_t hqg_smem_bytes() { return hqg_tiles_bytes() + (size_t)kHqgAux * sizeof(uint32_t); }
__device__ __forceinline__ uint32_t* hqg_aux(unsigned char* smem) {
  return reinterpret_cast<uint32_t*>(smem + hqg_tiles_bytes());
}

struct HqgItemOps {
  using T = gpq_item;
  static constexpr uint32_t kPer = kHqgIpt;
  static __device__ __forceinline__ bool less(const T& a, const T& b) { return hq_less(a, b); }
  static __device__ __forceinline__ T maxv() { return hq_max_item(); }
};

struct HqgKeyOps {
  using T = unsigned long long;
  static constexpr uint32_t kPer = kHqgKpt;
  static __device__ __forceinline__ bool less(T a, T b) { return a < b; }
  static __device__ __forceinline__ T maxv() { return ~0ull; }
};

template <class Ops>
__device__ __forceinline__ uint32_t hqg_pad(uint32_t j) { return j + j / Ops::kPer; }
template <class Ops>
__host__ __device__ constexpr uint32_t hqg_tile_cap() { return kHqgThreads * (Ops::kPer + 1); }

struct HqgDev {
  HqDev h;
  gpq_item* root2;          // [r] the root's second buffer
  gpq_item* t0;             // [2r] merge output of a non-root node / delete-update
  gpq_item* t1;             // [3r] delete-update
  gpq_item* pa;             // [r] insert pieces (alternating)
  gpq_item* pb;             // [r]
  gpq_item* e2;             // [population] sort scratch of the children
  gpq_item* bref;           // [r] refill: the two suffixes merged
  unsigned long long* k0;   // [r] (lp, position) keys of a batch
  unsigned long long* k1;   // [r]
  uint32_t* rank;           // [r] an event's position in its LP's sequence
  uint32_t* addc;           // [r] run length at the last event of an LP's run, else 0
  uint32_t* ovf;            // bucket overflows of the one-phase paths (zeroed per launch)
  // Bucket lists that each phase fills for the next (heaps whose root holds every item;
  // null otherwise).  Counts are double-buffered by window parity and zeroed per launch.
  gpq_item* ilist;            // [max buckets][kHqgListCapI] children by root-quantile bucket
  uint32_t* icnt;             // [2][max buckets]
  unsigned long long* plist;  // [max buckets][kHqgListCapP] next batch's (lp, position) keys by LP range
  uint32_t* pcnt;             // [2][max buckets]
};

struct HqgSync {
  const PholdDev* d;
  unsigned long long target;
  bool ok;
};

__device__ __forceinline__ bool hqg_bar(HqgSync& s) {
  s.target += gridDim.x;
  if (s.ok && !grid_barrier(&s.d->ctrl->bar, s.target, s.d->spin_limit, &s.d->ctrl->err)) s.ok = false;
  return s.ok;
}

__device__ __forceinline__ uint32_t hqg_tid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// Asynchronous 16-byte copies from this GPU's global memory into the CTA's shared memory
// (cp.async, no cluster multicast), completed per thread by commit groups.
__device__ __forceinline__ void hqg_cp16(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void hqg_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void hqg_cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ uint32_t hqg_nthreads() { return gridDim.x * blockDim.x; }

// ---------------------------------------------------------------------------------------
// Block-wide searches.

// First i in [lo, hi) with pred(i) true (pred monotone: false ... false true ... true), or
// hi; every thread of the block gets the answer.  Each round probes blockDim.x positions.
template <class Pred>
__device__ uint32_t hqg_cta_search(uint32_t lo, uint32_t hi, Pred pred) {
  __shared__ uint32_t s_lo, s_hi, s_first;
  if (threadIdx.x == 0) { s_lo = lo; s_hi = hi; }
  __syncthreads();
  const uint32_t m = blockDim.x, k = threadIdx.x;
  for (;;) {
    const uint32_t l = s_lo, h = s_hi;
    if (l >= h) break;
    if (k == 0) s_first = m;
    __syncthreads();
    const uint32_t i = l + (uint32_t)(((uint64_t)(h - l) * (k + 1)) / (m + 1));
    if (pred(i)) atomicMin(&s_first, k);
    __syncthreads();
    if (k == 0) {
      const uint32_t f = s_first;
      s_lo = f > 0 ? l + (uint32_t)(((uint64_t)(h - l) * f) / (m + 1)) + 1 : l;
      s_hi = f < m ? l + (uint32_t)(((uint64_t)(h - l) * (f + 1)) / (m + 1)) : h;
    }
    __syncthreads();
  }
  const uint32_t r = s_lo;
  __syncthreads();
  return r;
}

// Merge-path splits of diagonals d0 and d1 of merge(A, B) (A first on ties): the number
// of A items among the first d outputs.  Two halves of the block search one each.
template <class Ops>
__device__ void hqg_cta_split2(const typename Ops::T* A, uint32_t na, const typename Ops::T* B, uint32_t nb,
                               uint32_t d0, uint32_t d1, uint32_t* x0, uint32_t* x1) {
  __shared__ uint32_t s_lo[2], s_hi[2], s_first[2];
  const uint32_t half = blockDim.x >> 1;
  const uint32_t which = threadIdx.x >= half ? 1u : 0u, k = threadIdx.x - which * half;
  const uint32_t d = which ? d1 : d0;
  if (k == 0) {
    s_lo[which] = d > nb ? d - nb : 0u;
    s_hi[which] = min(d, na);
  }
  __syncthreads();
  for (;;) {
    const uint32_t l = s_lo[which], h = s_hi[which];
    if (s_lo[0] >= s_hi[0] && s_lo[1] >= s_hi[1]) break;
    if (k == 0) s_first[which] = half;
    __syncthreads();
    if (l < h) {
      const uint32_t i = l + (uint32_t)(((uint64_t)(h - l) * (k + 1)) / (half + 1));
      if (Ops::less(B[d - 1 - i], A[i])) atomicMin(&s_first[which], k);
    }
    __syncthreads();
    if (k == 0 && l < h) {
      const uint32_t f = s_first[which];
      s_lo[which] = f > 0 ? l + (uint32_t)(((uint64_t)(h - l) * f) / (half + 1)) + 1 : l;
      s_hi[which] = f < half ? l + (uint32_t)(((uint64_t)(h - l) * (f + 1)) / (half + 1)) : h;
    }
    __syncthreads();
  }
  *x0 = s_lo[0];
  *x1 = s_lo[1];
  __syncthreads();
}

// Merge-path split of diagonal `diag` of merge(A, B) with A = XA[aoff, aoff + na) and
// B = XB[boff, boff + nb), both in padded shared-memory tiles.
template <class Ops>
__device__ __forceinline__ uint32_t hqg_split(const typename Ops::T* XA, uint32_t aoff, uint32_t na,
                                              const typename Ops::T* XB, uint32_t boff, uint32_t nb, uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0u, hi = min(diag, na);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (!Ops::less(XB[hqg_pad<Ops>(boff + diag - 1 - mid)], XA[hqg_pad<Ops>(aoff + mid)])) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Outputs [dg, dg + per) of merge(A, B) (A, B as above; fewer at the end; per defaults to
// kPer) to out(k, v), k = 0, 1, ...  The two heads are kept in registers: one shared-memory
// load per output.
template <class Ops, class Out>
__device__ __forceinline__ void hqg_merge_run(const typename Ops::T* XA, uint32_t aoff, uint32_t na,
                                              const typename Ops::T* XB, uint32_t boff, uint32_t nb, uint32_t dg,
                                              Out out, uint32_t per = Ops::kPer) {
  using T = typename Ops::T;
  uint32_t ia = hqg_split<Ops>(XA, aoff, na, XB, boff, nb, dg), ib = dg - ia;
  T a = ia < na ? XA[hqg_pad<Ops>(aoff + ia)] : Ops::maxv();
  T b = ib < nb ? XB[hqg_pad<Ops>(boff + ib)] : Ops::maxv();
  const uint32_t n = min(per, na + nb - dg);
  for (uint32_t k = 0; k < n; ++k) {
    const bool take_a = ib >= nb || (ia < na && !Ops::less(b, a));
    if (take_a) {
      out(k, a);
      if (++ia < na) a = XA[hqg_pad<Ops>(aoff + ia)];
    } else {
      out(k, b);
      if (++ib < nb) b = XB[hqg_pad<Ops>(boff + ib)];
    }
  }
}

// ---------------------------------------------------------------------------------------
// Tiled merge: one CTA produces outputs [d0, d1) of merge(A, B) through out(o, v); sa and
// sb are two padded tiles.

template <class Ops, class Out>
__device__ void hqg_merge_tile(const typename Ops::T* A, uint32_t na, const typename Ops::T* B, uint32_t nb,
                               uint32_t d0, uint32_t d1, typename Ops::T* sa, typename Ops::T* sb, Out out) {
  uint32_t a0, a1;
  hqg_cta_split2<Ops>(A, na, B, nb, d0, d1, &a0, &a1);
  const uint32_t la = a1 - a0, lb = (d1 - a1) - (d0 - a0), b0 = d0 - a0, n = la + lb;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sa[hqg_pad<Ops>(i)] = i < la ? A[a0 + i] : B[b0 + i - la];
  __syncthreads();
  const uint32_t ld = threadIdx.x * Ops::kPer;
  if (ld < n)
    hqg_merge_run<Ops>(sa, 0, la, sa, la, lb, ld, [&](uint32_t k, const typename Ops::T& v) { sb[hqg_pad<Ops>(ld + k)] = v; });
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) out(d0 + i, sb[hqg_pad<Ops>(i)]);
}

// out(o, v) for every output of merge(A, B); all CTAs; ends with a barrier.
template <class Ops, class Out>
__device__ void hqg_merge(const typename Ops::T* A, uint32_t na, const typename Ops::T* B, uint32_t nb,
                          unsigned char* smem, HqgSync& s, Out out) {
  constexpr uint32_t tile = kHqgThreads * Ops::kPer;
  typename Ops::T* sa = reinterpret_cast<typename Ops::T*>(smem);
  typename Ops::T* sb = sa + hqg_tile_cap<Ops>();
  const uint32_t total = na + nb;
  for (uint32_t t = blockIdx.x; t * tile < total; t += gridDim.x)
    hqg_merge_tile<Ops>(A, na, B, nb, t * tile, min(t * tile + tile, total), sa, sb, out);
  hqg_bar(s);
}

struct HqgStore {
  gpq_item* p;
  __device__ __forceinline__ void operator()(uint32_t o, const gpq_item& v) const { p[o] = v; }
};

// The first `n` outputs to p, the rest to q.
struct HqgStore2 {
  gpq_item* p;
  gpq_item* q;
  uint32_t n;
  __device__ __forceinline__ void operator()(uint32_t o, const gpq_item& v) const {
    if (o < n) p[o] = v; else q[o - n] = v;
  }
};

// ---------------------------------------------------------------------------------------
// Sorts.

// Odd-even transposition network over kPer values in registers.
template <class Ops>
__device__ __forceinline__ void hqg_reg_sort(typename Ops::T (&v)[Ops::kPer]) {
#pragma unroll
  for (uint32_t r = 0; r < Ops::kPer; ++r) {
#pragma unroll
    for (uint32_t i = r & 1u; i + 1 < Ops::kPer; i += 2) {
      if (Ops::less(v[i + 1], v[i])) {
        const typename Ops::T x = v[i];
        v[i] = v[i + 1];
        v[i + 1] = x;
      }
    }
  }
}

static constexpr uint32_t kHqgRankSortMax = 512;

// Block merge sort of the padded tile sa holding n values (n <= kThreads * kPer; sb is a
// second padded tile).  Returns the tile that holds the sorted values in [0, n).  Up to
// kHqgRankSortMax values (all distinct, as items and (lp, position) keys are) are placed
// by rank instead: each thread counts the values below its own, reading the tile in step
// with the other threads (broadcast reads), one pass without dependent rounds.
template <class Ops>
__device__ typename Ops::T* hqg_cta_sort(typename Ops::T* sa, typename Ops::T* sb, uint32_t n) {
  using T = typename Ops::T;
  constexpr uint32_t P = Ops::kPer;
  if (n <= kHqgRankSortMax) {
    // G lanes (a power of two dividing 32) share one value's count when the block has
    // G threads per value
    uint32_t G = 1;
    while (G < 32 && (G * 2) * n <= blockDim.x) G *= 2;
    const uint32_t e = threadIdx.x / G, sub = threadIdx.x % G;
    const bool valid = e < n;
    T x{};
    uint32_t rk = 0;
    if (valid) {
      x = sa[hqg_pad<Ops>(e)];
      for (uint32_t j = sub; j < n; j += G) rk += Ops::less(sa[hqg_pad<Ops>(j)], x) ? 1u : 0u;
    }
    for (uint32_t o = G / 2; o > 0; o >>= 1) rk += __shfl_xor_sync(GPQ_FULL_MASK, rk, o, G);
    if (valid && sub == 0) sb[hqg_pad<Ops>(rk)] = x;
    __syncthreads();
    return sb;
  }
  const uint32_t nn = (n + P - 1) / P * P;
  const uint32_t b = threadIdx.x * P;
  if (b < nn) {
    T v[P];
#pragma unroll
    for (uint32_t k = 0; k < P; ++k) v[k] = (b + k < n) ? sa[hqg_pad<Ops>(b + k)] : Ops::maxv();
    hqg_reg_sort<Ops>(v);
#pragma unroll
    for (uint32_t k = 0; k < P; ++k) sa[hqg_pad<Ops>(b + k)] = v[k];
  }
  __syncthreads();
  for (uint32_t w = P; w < nn; w <<= 1) {
    if (b < nn) {
      const uint32_t p0 = b / (2 * w) * (2 * w);
      const uint32_t na = min(w, nn - p0), nb = min(w, nn - p0 - na);
      hqg_merge_run<Ops>(sa, p0, na, sa, p0 + na, nb, b - p0, [&](uint32_t k, const T& v) { sb[hqg_pad<Ops>(b + k)] = v; });
    }
    __syncthreads();
    T* x = sa;
    sa = sb;
    sb = x;
  }
  return sa;
}

// Sorts n values, value j given by load(j), into buf (tmp: scratch of n); all CTAs.
// Returns the buffer holding the result; ends with a barrier.
template <class Ops, class Load>
__device__ typename Ops::T* hqg_sort(typename Ops::T* buf, typename Ops::T* tmp, uint32_t n, unsigned char* smem,
                                     HqgSync& s, Load load) {
  using T = typename Ops::T;
  constexpr uint32_t tile = kHqgThreads * Ops::kPer;
  T* sa = reinterpret_cast<T*>(smem);
  T* sb = sa + hqg_tile_cap<Ops>();
  for (uint32_t c = blockIdx.x; c * tile < n; c += gridDim.x) {
    const uint32_t c0 = c * tile, cn = min(tile, n - c0);
    for (uint32_t i = threadIdx.x; i < cn; i += blockDim.x) sa[hqg_pad<Ops>(i)] = load(c0 + i);
    __syncthreads();
    const T* sorted = hqg_cta_sort<Ops>(sa, sb, cn);
    for (uint32_t i = threadIdx.x; i < cn; i += blockDim.x) buf[c0 + i] = sorted[hqg_pad<Ops>(i)];
    __syncthreads();
  }
  hqg_bar(s);
  for (uint32_t w = tile; w < n; w <<= 1) {  // runs of w into runs of 2w, tile by tile
    for (uint32_t t = blockIdx.x; t * tile < n; t += gridDim.x) {
      const uint32_t o0 = t * tile, p0 = o0 / (2 * w) * (2 * w);
      const uint32_t na = min(w, n - p0), nb = min(w, n - p0 - na);
      const uint32_t d0 = o0 - p0, d1 = min(d0 + tile, na + nb);
      hqg_merge_tile<Ops>(buf + p0, na, buf + p0 + na, nb, d0, d1, sa, sb,
                          [&](uint32_t o, const T& v) { tmp[p0 + o] = v; });
      __syncthreads();
    }
    hqg_bar(s);
    T* x = buf;
    buf = tmp;
    tmp = x;
  }
  return buf;
}

// ---------------------------------------------------------------------------------------
// The heap's control state, the same in every thread of the grid.

struct HqgState {
  gpq_item* root;   // buffer holding the root
  gpq_item* spare;  // the root's other buffer
  uint32_t off;     // first live item of the root
  uint32_t cnt0;    // live items of the root
  uint32_t last;    // last non-empty node
  uint32_t cntl;    // items of node `last` (last > 0)
  __device__ __forceinline__ uint32_t cnt(uint32_t p, uint32_t r) const {
    return p == 0 ? cnt0 : (p == last ? cntl : r);
  }
  __device__ __forceinline__ void swap_root() {
    gpq_item* x = root;
    root = spare;
    spare = x;
    off = 0;
  }
};

__device__ __forceinline__ gpq_item* hqg_node(const HqgDev& g, const HqgState& q, uint32_t p) {
  return p == 0 ? q.root + q.off : g.h.nodes + (size_t)p * g.h.r;
}

__device__ __forceinline__ void hqg_copy(gpq_item* dst, const gpq_item* src, uint32_t n, HqgSync& s) {
  for (uint32_t i = hqg_tid(); i < n; i += hqg_nthreads()) dst[i] = src[i];
  hqg_bar(s);
}

// Inserts the sorted items src[0, k) (insert-update pieces: each piece fills the last
// node or a new one and walks the root-to-target path, every full ancestor keeping the
// smallest r).  Returns false if the heap ran out of nodes (error recorded) or a barrier
// failed.
__device__ bool hqg_insert(const PholdDev& d, const HqgDev& g, HqgState& q, const gpq_item* src, uint32_t k,
                           unsigned char* smem, HqgSync& s) {
  const uint32_t r = g.h.r;
  uint32_t done = 0;
  while (done < k) {
    uint32_t tgt = q.last;
    if (q.cnt(q.last, r) == r) {
      tgt = q.last + 1;
      if (tgt >= g.h.maxnodes) {
        if (hqg_tid() == 0) gpq_set_error(&d.ctrl->err, GPQ_ERR_QUEUE_FULL);
        return false;
      }
      q.last = tgt;
      q.cntl = 0;
    }
    const uint32_t nt = q.cnt(tgt, r), px = min(k - done, r - nt);
    uint32_t depth = 0;
    while (((tgt + 1) >> (depth + 1)) != 0) ++depth;
    const gpq_item* piece = src + done;
    bool use_a = true;
    for (uint32_t l = 0; l < depth; ++l) {  // full ancestors on the path
      const uint32_t p = ((tgt + 1) >> (depth - l)) - 1;
      gpq_item* pout = use_a ? g.pa : g.pb;
      use_a = !use_a;
      if (p == 0) {
        hqg_merge<HqgItemOps>(q.root + q.off, r, piece, px, smem, s, HqgStore2{q.spare, pout, r});
        q.swap_root();
      } else {
        gpq_item* node = g.h.nodes + (size_t)p * r;
        hqg_merge<HqgItemOps>(node, r, piece, px, smem, s, HqgStore2{g.t0, pout, r});
        hqg_copy(node, g.t0, r, s);
      }
      piece = pout;
    }
    if (tgt == 0) {
      hqg_merge<HqgItemOps>(q.root + q.off, nt, piece, px, smem, s, HqgStore{q.spare});
      q.swap_root();
      q.cnt0 = nt + px;
    } else {
      gpq_item* node = g.h.nodes + (size_t)tgt * r;
      hqg_merge<HqgItemOps>(node, nt, piece, px, smem, s, HqgStore{g.t0});
      hqg_copy(node, g.t0, nt + px, s);
      q.cntl = nt + px;
    }
    done += px;
    if (!s.ok) return false;
  }
  return true;
}

// After a batch: refill the root from the largest items of the last nodes (copy-last) and
// restore the order along one path (delete-update).  Returns false if a barrier failed.
__device__ bool hqg_refill(const HqgDev& g, HqgState& q, unsigned char* smem, HqgSync& s) {
  const uint32_t r = g.h.r;
  if (q.last == 0) return true;  // the root holds every item
  const uint32_t keep = q.cnt0, want = r - keep;
  // The taken items are suffixes of one or two sorted nodes: node `last` (cntl items) and,
  // if it runs out, the full node before it (never the root).
  const uint32_t l1 = q.last, n1 = q.cntl, t1 = min(want, n1);
  const gpq_item* s1 = g.h.nodes + (size_t)l1 * r + (n1 - t1);
  q.cntl = n1 - t1;
  if (q.cntl == 0) {
    q.last = l1 - 1;
    q.cntl = r;
  }
  uint32_t t2 = 0;
  const gpq_item* s2 = nullptr;
  if (t1 < want && q.last > 0) {
    t2 = want - t1;  // <= r: node last - 1 is full
    s2 = g.h.nodes + (size_t)q.last * r + (r - t2);
    q.cntl = r - t2;
    if (q.cntl == 0) {
      q.last -= 1;
      q.cntl = r;
    }
  }
  const gpq_item* run = s1;
  if (t2 > 0) {
    hqg_merge<HqgItemOps>(s1, t1, s2, t2, smem, s, HqgStore{g.bref});
    run = g.bref;
  }
  hqg_merge<HqgItemOps>(q.root + q.off, keep, run, t1 + t2, smem, s, HqgStore{q.spare});
  q.swap_root();
  q.cnt0 = keep + t1 + t2;
  if (q.last == 0) q.cntl = 0;
  // delete-update
  uint32_t p = 0;
  while (s.ok) {
    const uint32_t c1 = 2 * p + 1, c2 = 2 * p + 2;
    const uint32_t np = q.cnt(p, r);
    const uint32_t m1 = (c1 <= q.last) ? q.cnt(c1, r) : 0u;
    const uint32_t m2 = (c2 <= q.last) ? q.cnt(c2, r) : 0u;
    if (np == 0 || (m1 == 0 && m2 == 0)) break;
    const gpq_item* P = hqg_node(g, q, p);
    const gpq_item* C1 = g.h.nodes + (size_t)c1 * r;
    const gpq_item* C2 = g.h.nodes + (size_t)c2 * r;
    const gpq_item pmax = P[np - 1];
    const bool ok1 = m1 == 0 || hq_less(pmax, C1[0]);
    const bool ok2 = m2 == 0 || hq_less(pmax, C2[0]);
    if (ok1 && ok2) break;
    // The child with the larger old maximum (or a partial c2, the last node) takes the
    // middle items, the other one the largest, and the walk continues there
    // (delete_update_post, src/heap_queue.cu:728-784).
    uint32_t mid, lrg;
    if (m2 == 0) {
      mid = lrg = c1;
    } else if (m1 == 0) {
      mid = lrg = c2;
    } else {
      const bool mid2 = m2 < r || hq_less(C1[m1 - 1], C2[m2 - 1]);
      mid = mid2 ? c2 : c1;
      lrg = mid2 ? c1 : c2;
    }
    hqg_merge<HqgItemOps>(P, np, C1, m1, smem, s, HqgStore{g.t0});
    hqg_merge<HqgItemOps>(g.t0, np + m1, C2, m2, smem, s, HqgStore{g.t1});
    const uint32_t nmid = (mid == c1) ? m1 : m2;
    gpq_item* Pw = hqg_node(g, q, p);
    gpq_item* Mw = g.h.nodes + (size_t)mid * r;
    gpq_item* Lw = g.h.nodes + (size_t)lrg * r;
    for (uint32_t i = hqg_tid(); i < np + m1 + m2; i += hqg_nthreads()) {
      const gpq_item v = g.t1[i];
      if (i < np) Pw[i] = v;
      else if (i < np + nmid) Mw[i - np] = v;
      else Lw[i - np - nmid] = v;
    }
    hqg_bar(s);
    p = lrg;
  }
  return s.ok;
}

// ---------------------------------------------------------------------------------------
// Per-LP ranks of a batch.

// Positions [t0, t0 + tn) of the sorted keys K[0, n) (staged in sk): rank[i] = count[lp]
// + p - (first position of lp's run) and addc[i] = run length at the run's last key.
// gseg = first position of the run holding position t0.
// sk is a padded shared-memory tile.
__device__ void hqg_rank_tile(const PholdDev& d, const HqgDev& g, const unsigned long long* sk, uint32_t t0,
                              uint32_t tn, uint32_t n, uint32_t gseg, const unsigned long long* K) {
  auto at = [sk](uint32_t j) { return sk[hqg_pad<HqgKeyOps>(j)]; };
  const uint32_t lp0 = (uint32_t)(at(0) >> 32);
  for (uint32_t j = threadIdx.x; j < tn; j += blockDim.x) {
    const unsigned long long key = at(j);
    const uint32_t lp = (uint32_t)(key >> 32), i = (uint32_t)key;
    uint32_t seg;
    if (lp == lp0) {
      seg = gseg;
    } else {
      const unsigned long long lo_key = (unsigned long long)lp << 32;
      uint32_t lo = 0, hi = j;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (at(mid) < lo_key) lo = mid + 1; else hi = mid;
      }
      seg = t0 + lo;
    }
    const uint32_t p = t0 + j;
    g.rank[i] = d.count[lp] + (p - seg);
    const uint64_t nxt = (j + 1 < tn) ? at(j + 1) : (p + 1 < n ? K[p + 1] : ~0ull);
    g.addc[i] = ((uint32_t)(nxt >> 32) != lp || p + 1 == n) ? p - seg + 1 : 0u;
  }
}

// Ranks of the c events root[0, c); ends with a barrier.
__device__ void hqg_ranks(const PholdDev& d, const HqgDev& g, const gpq_item* root, uint32_t c, unsigned char* smem,
                          HqgSync& s) {
  auto load = [root](uint32_t j) { return ((unsigned long long)root[j].lp << 32) | j; };
  unsigned long long* sa = reinterpret_cast<unsigned long long*>(smem);
  if (c <= kHqgKeyTile) {  // one CTA sorts and ranks the whole batch
    if (blockIdx.x == gridDim.x - 1) {
      for (uint32_t j = threadIdx.x; j < c; j += blockDim.x) sa[hqg_pad<HqgKeyOps>(j)] = load(j);
      __syncthreads();
      const unsigned long long* sk = hqg_cta_sort<HqgKeyOps>(sa, sa + hqg_tile_cap<HqgKeyOps>(), c);
      hqg_rank_tile(d, g, sk, 0, c, c, 0, nullptr);
      __syncthreads();
    }
    hqg_bar(s);
    return;
  }
  const unsigned long long* K = hqg_sort<HqgKeyOps>(g.k0, g.k1, c, smem, s, load);
  for (uint32_t t = blockIdx.x; t * kHqgKeyTile < c; t += gridDim.x) {
    const uint32_t t0 = t * kHqgKeyTile, tn = min(kHqgKeyTile, c - t0);
    for (uint32_t j = threadIdx.x; j < tn; j += blockDim.x) sa[hqg_pad<HqgKeyOps>(j)] = K[t0 + j];
    __syncthreads();
    const unsigned long long lo_key = sa[0] & 0xffffffff00000000ull;
    const uint32_t gseg = hqg_cta_search(0, t0, [K, lo_key](uint32_t i) { return K[i] >= lo_key; });
    hqg_rank_tile(d, g, sa, t0, tn, c, gseg, K);
    __syncthreads();
  }
  hqg_bar(s);
}

// ---------------------------------------------------------------------------------------
// One-phase paths for small windows.  Buckets whose contents one CTA holds in shared
// memory replace the sorts: each CTA scans the whole input and keeps its bucket's share.

static constexpr uint32_t kHqgScanMax = 32768;  // children a one-phase insert scans
static constexpr uint32_t kHqgScanPer = 128;    // items per bucket aimed at

// visit(i, v, i < n) for i in [0, n) rounded up, v = load(i) (a zero value past n), every
// thread of the CTA with all lanes of each warp together (visit may use warp
// collectives); U loads in flight per thread.
template <uint32_t U, class Load, class Visit>
__device__ __forceinline__ void hqg_cta_scan(uint32_t n, Load load, Visit visit) {
  using V = decltype(load(0u));
  for (uint32_t base = 0; base < n; base += blockDim.x * U) {
    V x[U];
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      x[u] = (i < n) ? load(i) : V{};
    }
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      visit(i, x[u], i < n);
    }
  }
}

// A slot of a shared-memory counter for every lane with `take` set, one atomic per warp.
__device__ __forceinline__ uint32_t hqg_warp_slot(uint32_t* ctr, bool take) {
  const uint32_t m = __ballot_sync(GPQ_FULL_MASK, take);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t leader = m != 0u ? (uint32_t)(__ffs(m) - 1) : 0u;
  uint32_t b = 0;
  if (m != 0u && lane == leader) b = atomicAdd(ctr, (uint32_t)__popc(m));
  b = __shfl_sync(GPQ_FULL_MASK, b, (int)leader);
  return b + __popc(m & ((1u << lane) - 1u));
}

// Buckets of the one-phase insert into a root of nr items with nch children (0 = the
// general path).
__device__ __forceinline__ uint32_t hqg_insert_buckets(const HqgState& q, uint32_t r, uint32_t nch) {
  const uint32_t nr = q.cnt0, total = nr + nch;
  if (q.last != 0 || total > r || nch > kHqgScanMax) return 0;
  uint32_t B = min(gridDim.x, max(1u, total / kHqgScanPer));
  if (nr < B) B = max(1u, nr);
  return (nr / B + 1 <= kHqgTile) ? B : 0u;
}

// The children C[0, nch) into a heap whose root holds every item and has room for them:
// the new root is R u C (R = the root's items) in one phase.  The splitters are R's
// quantiles (R is sorted): bucket b holds R's b-th slice and the children from that
// slice's first item up to the next slice's first item.  CTA b collects its children by
// scanning all of them, sorts them in shared memory, merges them with its slice and
// writes the result at (slice start + children below the slice) of the root's other
// buffer.  Returns false when a bucket overflowed shared memory (the heap is unchanged;
// the caller takes the general path) or a barrier failed.
__device__ bool hqg_insert_scan(const HqgDev& g, HqgState& q, const gpq_item* C, uint32_t nch, uint32_t B,
                                unsigned char* smem, HqgSync& s, uint32_t& ovf_seen) {
  const gpq_item* R = q.root + q.off;
  const uint32_t nr = q.cnt0;
  gpq_item* sa = reinterpret_cast<gpq_item*>(smem);
  gpq_item* sb = sa + hqg_tile_cap<HqgItemOps>();
  __shared__ uint32_t s_nc, s_below;
  for (uint32_t b = blockIdx.x; b < B; b += gridDim.x) {
    const uint32_t r0 = (uint32_t)((uint64_t)b * nr / B), r1 = (uint32_t)((uint64_t)(b + 1) * nr / B);
    const bool has_lo = b > 0, has_hi = b + 1 < B;
    const gpq_item lo = has_lo ? R[r0] : hq_max_item(), hi = has_hi ? R[r1] : hq_max_item();
    if (threadIdx.x == 0) {
      s_nc = 0;
      s_below = 0;
    }
    __syncthreads();
    uint32_t below = 0;
    hqg_cta_scan<4>(nch, [C](uint32_t i) { return C[i]; }, [&](uint32_t, const gpq_item& x, bool valid) {
      const bool lo_ok = valid && !(has_lo && hq_less(x, lo));
      below += (valid && !lo_ok) ? 1u : 0u;
      const bool take = lo_ok && (!has_hi || hq_less(x, hi));
      const uint32_t slot = hqg_warp_slot(&s_nc, take);
      if (take && slot < kHqgTile) sa[hqg_pad<HqgItemOps>(slot)] = x;
    });
    below = warp_sum_u32(below);
    if ((threadIdx.x & 31u) == 0 && below) atomicAdd(&s_below, below);
    __syncthreads();
    const uint32_t nc = s_nc, nbw = s_below, nrb = r1 - r0;
    if (nc > kHqgTile) {
      if (threadIdx.x == 0) atomicAdd(g.ovf, 1u);
      __syncthreads();
      continue;
    }
    gpq_item* X = hqg_cta_sort<HqgItemOps>(sa, sb, nc);
    gpq_item* Y = (X == sa) ? sb : sa;
    for (uint32_t j = threadIdx.x; j < nrb; j += blockDim.x) Y[hqg_pad<HqgItemOps>(j)] = R[r0 + j];
    __syncthreads();
    gpq_item* dst = q.spare + r0 + nbw;
    const uint32_t ld = threadIdx.x * kHqgIpt;
    if (ld < nc + nrb)
      hqg_merge_run<HqgItemOps>(Y, 0, nrb, X, 0, nc, ld, [&](uint32_t k, const gpq_item& v) { dst[ld + k] = v; });
    __syncthreads();
  }
  if (!hqg_bar(s)) return false;
  const uint32_t o = ld_relaxed_u32(g.ovf);
  if (o != ovf_seen) {
    ovf_seen = o;
    return false;
  }
  q.swap_root();
  q.cnt0 = nr + nch;
  return true;
}

// ---------------------------------------------------------------------------------------
// Bucket lists passed between phases (heaps whose root holds every item, the global
// array queue's layout).  A window is three phases whose CTAs read only their own
// buckets: the batch's (lp, position) keys filed into LP-range lists by equal slices of
// the batch; each LP range sorted and processed by one CTA, which files every child into
// a bucket of the root's remainder R (splitters: R's quantiles, as in the one-phase
// insert); each insert bucket's children sorted in shared memory and merged with its R
// slice into the root's other buffer.  A list that overflows sends its phase down the
// paths above (the children are also kept in h.ch).

static constexpr uint32_t kHqgListCapI = kHqgTile;     // children per insert bucket
static constexpr uint32_t kHqgListCapP = kHqgKeyTile;  // keys per LP-range bucket
static constexpr uint32_t kHqgMaxBuckets = 160;        // >= the grid (one CTA per SM)

struct HqgLists {
  bool ins;     // this window's children are filed in the insert lists
  uint32_t BI;  // insert buckets
};

// LP-range buckets: LP lp belongs to bucket floor(lp * B / L), whose first LP is
// ceil(b * L / B).
__device__ __forceinline__ uint32_t hqg_lp_bucket(uint32_t lp, uint32_t B, uint32_t L) {
  return (uint32_t)((uint64_t)lp * B / L);
}
__device__ __forceinline__ uint32_t hqg_lp_first(uint32_t b, uint32_t B, uint32_t L) {
  return (uint32_t)(((uint64_t)b * L + B - 1) / B);
}

// Insert buckets for a batch of c events leaving nr items in the root.
__device__ __forceinline__ uint32_t hqg_list_ibuckets(uint32_t nr, uint32_t c) {
  if (nr == 0) return 1u;
  return min(gridDim.x, max(1u, min(nr, (nr + c) / 256u)));
}

// Where a batch phase files its children (ins.on == false: nowhere).
struct HqgIns {
  bool on;
  uint32_t BI;
  const gpq_item* spl;  // [BI - 1] splitters (shared memory)
  uint32_t* icnt;       // [BI] this window's counts
  gpq_item* ilist;
};

// Bucket of x among the splitters: the number of splitters below it.
__device__ __forceinline__ uint32_t hqg_bucket_of(const gpq_item* spl, uint32_t ns, const gpq_item& x) {
  uint32_t lo = 0, hi = ns;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (hq_less(spl[mid], x)) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Appends v to list `bucket` (cap entries each) for every lane with `take`; lanes of a warp
// that share a bucket take one atomic.  All lanes of the warp.  Returns false if the
// bucket was full (the entry is counted, not stored: the reader sees the overflow).
template <class T>
__device__ __forceinline__ void hqg_list_append(uint32_t* cnt, T* list, uint32_t cap, bool take, uint32_t bucket,
                                                const T& v) {
  const uint32_t key = take ? bucket : (0x80000000u | (threadIdx.x & 31u));
  const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, key);
  const uint32_t lane = threadIdx.x & 31u, leader = (uint32_t)(__ffs(peers) - 1);
  uint32_t b = 0;
  if (take && lane == leader) b = atomicAdd(&cnt[bucket], (uint32_t)__popc(peers));
  b = __shfl_sync(GPQ_FULL_MASK, b, (int)leader);
  const uint32_t slot = b + __popc(peers & ((1u << lane) - 1u));
  if (take && slot < cap) list[(size_t)bucket * cap + slot] = v;
}

// Loads the BI - 1 splitters of the root remainder R[0, nr) into shared memory.
__device__ __forceinline__ void hqg_load_splitters(gpq_item* spl, const gpq_item* R, uint32_t nr, uint32_t BI) {
  for (uint32_t k = threadIdx.x; k + 1 < BI; k += blockDim.x) spl[k] = R[(uint32_t)((uint64_t)(k + 1) * nr / BI)];
  __syncthreads();
}

// Exclusive scan of a[0, n) in shared memory by the CTA (n <= kHqgBins); returns the total
// and sets *mx to the largest entry.  All threads.
__device__ uint32_t hqg_block_scan(uint32_t* a, uint32_t n, uint32_t* mx) {
  __shared__ uint32_t s_w[32], s_m[32];
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t b0 = min(n, threadIdx.x * per), b1 = min(n, b0 + per);
  uint32_t sum = 0, m = 0;
  for (uint32_t i = b0; i < b1; ++i) {
    sum += a[i];
    m = max(m, a[i]);
  }
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(GPQ_FULL_MASK, incl, o);
    if (lane >= (uint32_t)o) incl += v;
  }
  m = __reduce_max_sync(GPQ_FULL_MASK, m);
  if (lane == 31) s_w[warp] = incl;
  if (lane == 0) s_m[warp] = m;
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = blockDim.x >> 5;
    const uint32_t v = lane < nw ? s_w[lane] : 0u;
    uint32_t wi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(GPQ_FULL_MASK, wi, o);
      if (lane >= (uint32_t)o) wi += u;
    }
    const uint32_t mm = __reduce_max_sync(GPQ_FULL_MASK, lane < nw ? s_m[lane] : 0u);
    s_w[lane] = wi - v;
    if (lane == 31) s_m[0] = wi;  // total
    if (lane == 30) s_m[1] = mm;
  }
  __syncthreads();
  uint32_t run = s_w[warp] + incl - sum;
  for (uint32_t i = b0; i < b1; ++i) {
    const uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
  const uint32_t total = s_m[0];
  *mx = s_m[1];
  __syncthreads();
  return total;
}

static constexpr uint32_t kHqgRunMax = 64;  // longest bin a thread sorts by insertion

// Sorts the n items of the padded tile in (n <= kHqgTile; LPs below L) into out: a
// counting sort over bins of v = (ts bits - min) * 2^16 + lp * 2^16 / L (monotone in the
// item order; the LP part spreads equal timestamps, frequent where float32 spacing is
// coarse), bin = v * NB / (v range), then each bin sorted by the full item order
// (insertion sort, one thread per bin).  Returns false, with out unusable, when some bin
// has more than kHqgRunMax items.  bins: kHqgBins words.  All threads.
__device__ bool hqg_bin_sort_items(const gpq_item* in, gpq_item* out, uint32_t n, uint32_t L, uint32_t* bins) {
  __shared__ uint32_t s_tmin, s_tmax;
  if (threadIdx.x == 0) {
    s_tmin = 0xffffffffu;
    s_tmax = 0u;
  }
  __syncthreads();
  uint32_t tmin = 0xffffffffu, tmax = 0u;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t t = gpq_f2u(in[hqg_pad<HqgItemOps>(j)].ts);
    tmin = min(tmin, t);
    tmax = max(tmax, t);
  }
  tmin = warp_min_u32(tmin);
  tmax = __reduce_max_sync(GPQ_FULL_MASK, tmax);
  if ((threadIdx.x & 31u) == 0) {
    atomicMin(&s_tmin, tmin);
    atomicMax(&s_tmax, tmax);
  }
  const uint32_t NB = max(1u, min(kHqgBins, n));
  for (uint32_t b = threadIdx.x; b < NB; b += blockDim.x) bins[b] = 0u;
  __syncthreads();
  const uint32_t t0 = s_tmin;
  const uint64_t span = ((uint64_t)(s_tmax - t0) + 1u) << 16;  // <= 2^48
  auto bin_of = [t0, span, NB, L](const gpq_item& x) {
    const uint64_t v = ((uint64_t)(gpq_f2u(x.ts) - t0) << 16) + (((uint64_t)x.lp << 16) / L);
    return (uint32_t)(v * NB / span);  // v * NB < 2^61
  };
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) atomicAdd(&bins[bin_of(in[hqg_pad<HqgItemOps>(j)])], 1u);
  __syncthreads();
  uint32_t mx = 0;
  hqg_block_scan(bins, NB, &mx);
  if (mx > kHqgRunMax) return false;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const gpq_item x = in[hqg_pad<HqgItemOps>(j)];
    const uint32_t pos = atomicAdd(&bins[bin_of(x)], 1u);
    if (pos < n) out[hqg_pad<HqgItemOps>(pos)] = x;
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < NB; b += blockDim.x) {
    const uint32_t e = bins[b], st = b ? bins[b - 1] : 0u;
    for (uint32_t x = st + 1; x < e; ++x) {
      const gpq_item v = out[hqg_pad<HqgItemOps>(x)];
      uint32_t y = x;
      while (y > st && hq_less(v, out[hqg_pad<HqgItemOps>(y - 1)])) {
        out[hqg_pad<HqgItemOps>(y)] = out[hqg_pad<HqgItemOps>(y - 1)];
        --y;
      }
      out[hqg_pad<HqgItemOps>(y)] = v;
    }
  }
  __syncthreads();
  return true;
}

// Groups the n (lp, position) keys of in (padded tile) by LP into out (padded tile): a
// counting sort over the LP range [lp0, lp0 + W), then each LP's run sorted by position
// (insertion sort, one thread per LP).  On return bins[b] is the end of LP lp0 + b's run
// (its start: bins[b - 1], or 0).  Returns false, with out unusable, when W exceeds
// kHqgBins or some LP has more than kHqgRunMax keys.  All threads.
__device__ bool hqg_group_by_lp(const unsigned long long* in, unsigned long long* out, uint32_t n, uint32_t lp0,
                                uint32_t W, uint32_t* bins) {
  __shared__ int s_outside;
  if (W > kHqgBins || W == 0) return false;
  for (uint32_t b = threadIdx.x; b < W; b += blockDim.x) bins[b] = 0u;
  if (threadIdx.x == 0) s_outside = 0;
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t bi = (uint32_t)(in[hqg_pad<HqgKeyOps>(j)] >> 32) - lp0;
    if (bi < W) atomicAdd(&bins[bi], 1u);
    else s_outside = 1;  // a key outside the range: not binned (the merge sort takes any keys)
  }
  __syncthreads();
  if (s_outside) return false;
  uint32_t mx = 0;
  hqg_block_scan(bins, W, &mx);
  if (mx > kHqgRunMax) return false;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const unsigned long long k = in[hqg_pad<HqgKeyOps>(j)];
    const uint32_t pos = atomicAdd(&bins[(uint32_t)(k >> 32) - lp0], 1u);
    if (pos < n) out[hqg_pad<HqgKeyOps>(pos)] = k;
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < W; b += blockDim.x) {
    const uint32_t e = bins[b], st = b ? bins[b - 1] : 0u;
    for (uint32_t x = st + 1; x < e; ++x) {  // insertion sort of the run by position
      const unsigned long long v = out[hqg_pad<HqgKeyOps>(x)];
      uint32_t y = x;
      while (y > st && out[hqg_pad<HqgKeyOps>(y - 1)] > v) {
        out[hqg_pad<HqgKeyOps>(y)] = out[hqg_pad<HqgKeyOps>(y - 1)];
        --y;
      }
      out[hqg_pad<HqgKeyOps>(y)] = v;
    }
  }
  __syncthreads();
  return true;
}

// The n (lp, position) keys K of one LP range (padded tile, grouped by LP with positions
// ascending -- every LP's events of the batch), seg(j, lp) = the first position of lp's run:
// each event folded into its LP's outputs in order (the per-LP sums of a warp's run added
// by one lane), its child written to ch[base + position] and filed by `ins` (counted per
// bucket in shared memory, one reservation per bucket, then written), the LP's count
// advanced.  aux: kHqgBins words for the children's bucket slots.  All threads.
template <class Seg>
__device__ void hqg_process_keys(const PholdDev& d, const HqgDev& g, const gpq_item* root,
                                 const unsigned long long* K, uint32_t n, uint32_t base, const HqgIns& ins,
                                 uint32_t* slots, Seg seg) {
  __shared__ uint32_t s_bc[kHqgMaxBuckets], s_gb[kHqgMaxBuckets];
  if (ins.on) {
    for (uint32_t k = threadIdx.x; k < ins.BI; k += blockDim.x) s_bc[k] = 0u;
    __syncthreads();
  }
  const uint32_t lane = threadIdx.x & 31u;
  const bool direct = n <= blockDim.x;
  for (uint32_t j0 = 0; j0 < n; j0 += blockDim.x) {
    const uint32_t j = j0 + threadIdx.x;
    const bool valid = j < n;
    uint32_t lp = 0;
    unsigned long long cs = 0, oh = 0;
    gpq_item chd{};
    if (valid) {
      const unsigned long long key = K[hqg_pad<HqgKeyOps>(j)];
      lp = (uint32_t)(key >> 32);
      const uint32_t i = (uint32_t)key;
      const gpq_item e = root[i];
      const uint64_t hh = gpq_ev_hash(e.id, gpq_f2u(e.ts));
      cs = hh;
      oh = gpq_seq_hash(hh, (uint64_t)d.count[lp] + (j - seg(j, lp)));
      const gpq_item ch = gpq_phold_child(d.p, e);
      g.h.ch[base + i] = ch;
      if (ins.on && !direct && j < kHqgBins) {
        const uint32_t bk = hqg_bucket_of(ins.spl, ins.BI - 1, ch);
        slots[j] = (bk << 16) | atomicAdd(&s_bc[bk], 1u);
      }
      if (ins.on && direct) chd = ch;
    }
    if (ins.on && direct) {  // one round: each warp files its children directly
      const uint32_t bk = valid ? hqg_bucket_of(ins.spl, ins.BI - 1, chd) : 0u;
      hqg_list_append<gpq_item>(ins.icnt, ins.ilist, kHqgListCapI, valid, bk, chd);
    }
    // the LP's runs are contiguous in the warp: sum each run into its first lane
    const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, valid ? lp : (0x80000000u | lane));
    const uint32_t last = 31u - __clz(peers);
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const unsigned long long c2 = __shfl_down_sync(GPQ_FULL_MASK, cs, o);
      const unsigned long long o2 = __shfl_down_sync(GPQ_FULL_MASK, oh, o);
      if (lane + o <= last) {
        cs += c2;
        oh += o2;
      }
    }
    if (valid && lane == (uint32_t)(__ffs(peers) - 1)) {
      atomicAdd(&d.csum[lp], cs);
      atomicAdd(&d.ohash[lp], oh);
    }
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t lp = (uint32_t)(K[hqg_pad<HqgKeyOps>(j)] >> 32);
    if (j + 1 == n || (uint32_t)(K[hqg_pad<HqgKeyOps>(j + 1)] >> 32) != lp) d.count[lp] += j - seg(j, lp) + 1;
  }
  if (ins.on && !direct) {  // one reservation per bucket, then the children into their lists
    for (uint32_t k = threadIdx.x; k < ins.BI; k += blockDim.x)
      s_gb[k] = s_bc[k] ? atomicAdd(&ins.icnt[k], s_bc[k]) : 0u;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
      const uint32_t i = (uint32_t)K[hqg_pad<HqgKeyOps>(j)];
      const gpq_item ch = g.h.ch[base + i];
      if (j < kHqgBins) {
        const uint32_t sv = slots[j], bk = sv >> 16, slot = s_gb[bk] + (sv & 0xffffu);
        if (slot < kHqgListCapI) ins.ilist[(size_t)bk * kHqgListCapI + slot] = ch;
      } else {  // beyond the slot area (more than kHqgBins keys): one atomic each
        const uint32_t bk = hqg_bucket_of(ins.spl, ins.BI - 1, ch);
        const uint32_t slot = atomicAdd(&ins.icnt[bk], 1u);
        if (slot < kHqgListCapI) ins.ilist[(size_t)bk * kHqgListCapI + slot] = ch;
      }
    }
  }
  __syncthreads();
}

// Sorts the n keys of sa (an LP range of W LPs from lp0) for hqg_process_keys and runs it:
// grouped by LP when it can, else the block merge sort.
__device__ void hqg_sort_and_process(const PholdDev& d, const HqgDev& g, const gpq_item* root,
                                     unsigned long long* sa, unsigned long long* sb, uint32_t n, uint32_t lp0,
                                     uint32_t W, uint32_t base, const HqgIns& ins, uint32_t* aux) {
  uint32_t* bins = aux;
  uint32_t* slots = aux + kHqgBins;
  if (hqg_group_by_lp(sa, sb, n, lp0, W, bins)) {
    hqg_process_keys(d, g, root, sb, n, base, ins, slots,
                     [bins, lp0](uint32_t, uint32_t lp) { return lp > lp0 ? bins[lp - lp0 - 1] : 0u; });
  } else {
    const unsigned long long* K = hqg_cta_sort<HqgKeyOps>(sa, sb, n);
    hqg_process_keys(d, g, root, K, n, base, ins, slots, [K](uint32_t j, uint32_t lp) {
      const unsigned long long lo_key = (unsigned long long)lp << 32;
      uint32_t l = 0, h = j;
      while (l < h) {
        const uint32_t mid = (l + h) >> 1;
        if (K[hqg_pad<HqgKeyOps>(mid)] < lo_key) l = mid + 1; else h = mid;
      }
      return l;
    });
  }
}

static constexpr uint32_t kHqgScanBatchMax = 2 * kHqgKeyTile;  // batches the one-phase form scans

// A batch of c <= kHqgScanBatchMax events root[0, c) in one phase: LP-range buckets (one
// per CTA), so that every LP's events of the batch are in one CTA, which collects their
// (lp, position) keys by scanning the batch, sorts them in shared memory and processes
// them in order (hqg_sort_and_process).  Every CTA also counts every bucket while it
// scans, so all of them see the same largest bucket: when one holds more keys than a tile,
// nothing is processed and false is returned (in every CTA, without a barrier).  Else ends
// with a barrier.
__device__ bool hqg_process_scan(const PholdDev& d, const HqgDev& g, const gpq_item* root, uint32_t c, uint32_t base,
                                 const HqgIns& ins, unsigned char* smem, HqgSync& s) {
  const uint32_t L = d.L;
  const uint32_t B = min(gridDim.x, max(1u, c / 64u));
  unsigned long long* sa = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* sb = sa + hqg_tile_cap<HqgKeyOps>();
  __shared__ uint32_t s_n, s_hist[kHqgMaxBuckets], s_first[kHqgMaxBuckets + 1];
  __shared__ int s_big;
  const uint32_t b = blockIdx.x;  // this CTA's bucket (B <= gridDim.x)
  // a batch that fits a tile cannot overflow a bucket; a larger one is counted per bucket
  // (bucket of an LP: a float estimate corrected against the buckets' first LPs)
  const bool count = c > kHqgKeyTile;
  for (uint32_t k = threadIdx.x; k <= B; k += blockDim.x) {
    if (k < B) s_hist[k] = 0u;
    s_first[k] = hqg_lp_first(k, B, L);
  }
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lo_b = s_first[min(b, B)], hi_b = s_first[min(b + 1, B)];
  const float scale = (float)B / (float)L;
  hqg_cta_scan<8>(c, [root](uint32_t i) { return root[i].lp; }, [&](uint32_t i, uint32_t lp, bool valid) {
    if (count) {
      uint32_t bk = 0x80000000u | lane;
      if (valid) {
        bk = min(B - 1, __float2uint_rd((float)lp * scale));
        while (bk > 0 && lp < s_first[bk]) --bk;
        while (lp >= s_first[bk + 1]) ++bk;
      }
      const uint32_t peers = __match_any_sync(GPQ_FULL_MASK, bk);
      if (valid && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&s_hist[bk], (uint32_t)__popc(peers));
    }
    const bool take = valid && lp >= lo_b && lp < hi_b;
    const uint32_t slot = hqg_warp_slot(&s_n, take);
    if (take && slot < kHqgKeyTile) sa[hqg_pad<HqgKeyOps>(slot)] = ((unsigned long long)lp << 32) | i;
  });
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t mx = 0;
    if (count)
      for (uint32_t k = 0; k < B; ++k) mx = max(mx, s_hist[k]);
    s_big = mx > kHqgKeyTile;
  }
  __syncthreads();
  if (s_big) return false;
  if (b < B) hqg_sort_and_process(d, g, root, sa, sb, s_n, lo_b, hi_b - lo_b, base, ins, hqg_aux(smem));
  hqg_bar(s);
  return true;
}

// A batch whose keys the insert phase filed into BP LP-range lists (counts pc, none above
// kHqgListCapP): each CTA sorts its list and processes it.  Ends with a barrier.
__device__ void hqg_process_lists(const PholdDev& d, const HqgDev& g, const gpq_item* root, const uint32_t* pc,
                                  uint32_t BP, uint32_t base, const HqgIns& ins, unsigned char* smem, HqgSync& s) {
  unsigned long long* sa = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* sb = sa + hqg_tile_cap<HqgKeyOps>();
  const uint32_t L = d.L;
  for (uint32_t b = blockIdx.x; b < BP; b += gridDim.x) {
    const uint32_t n = min(pc[b], kHqgListCapP);
    const uint32_t lo = hqg_lp_first(b, BP, L), hi = hqg_lp_first(b + 1, BP, L);
    const unsigned long long* src = g.plist + (size_t)b * kHqgListCapP;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) sa[hqg_pad<HqgKeyOps>(j)] = src[j];
    __syncthreads();
    hqg_sort_and_process(d, g, root, sa, sb, n, lo, hi - lo, base, ins, hqg_aux(smem));
  }
  hqg_bar(s);
}

// The items root[lo, hi) filed into BP LP-range lists (counts pc, zero before the window)
// for hqg_process_lists: the CTA counts its keys per range in shared memory, reserves each
// range's share with one atomic and writes them.
__device__ void hqg_file_range(const HqgDev& g, const gpq_item* root, uint32_t lo, uint32_t hi, uint32_t BP,
                               uint32_t* pc, uint32_t L, uint32_t* aux) {
  __shared__ uint32_t s_pb[kHqgMaxBuckets];
  for (uint32_t p0 = lo; p0 < hi; p0 += kHqgAux) {
    const uint32_t pn = min(kHqgAux, hi - p0);
    for (uint32_t k = threadIdx.x; k < BP; k += blockDim.x) s_pb[k] = 0u;
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < pn; p += blockDim.x) {
      const uint32_t bk = hqg_lp_bucket(root[p0 + p].lp, BP, L);
      aux[p] = (bk << 16) | atomicAdd(&s_pb[bk], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < BP; k += blockDim.x) s_pb[k] = s_pb[k] ? atomicAdd(&pc[k], s_pb[k]) : 0u;
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < pn; p += blockDim.x) {
      const uint32_t sv = aux[p], bk = sv >> 16, slot = s_pb[bk] + (sv & 0xffffu);
      if (slot < kHqgListCapP) g.plist[(size_t)bk * kHqgListCapP + slot] = ((unsigned long long)root[p0 + p].lp << 32) | (p0 + p);
    }
    __syncthreads();
  }
}

// The children of the last batch, filed in BI insert lists (this window's counts ic), into
// the root (all of whose items stay: R = root[off, off + cnt0)): CTA b sorts its list in
// shared memory and streams R's slice b past it -- an R item lands at (slice start +
// children below the slice + its index + children below it), the children between two R
// items right after the first -- into the root's other buffer.  Returns false, with
// nothing written, when a list overflowed.
//
// pre.on: the next window's batch is also filed into its LP-range lists (pre.BP ranges,
// counts pre.pc) here, so that the window needs no filing phase: the new root's head is the
// smaller of R's head and the smallest child (in the first non-empty list), which fixes the
// window's bound; each CTA's outputs below it are a prefix of its output range, filed by
// that CTA after its merge.
struct HqgPre {
  bool on;
  float la, T;   // lookahead and end time: the bound is min(head + la, T)
  uint32_t BP;   // LP ranges
  uint32_t* pc;  // their counts (zeroed before the window)
};

__device__ bool hqg_insert_lists(const HqgDev& g, HqgState& q, uint32_t nch, uint32_t BI, const uint32_t* ic,
                                 uint32_t L, const HqgPre& pre, unsigned char* smem, HqgSync& s) {
  __shared__ uint32_t s_pre[kHqgMaxBuckets + 1];
  __shared__ int s_ovf;
  __shared__ uint32_t s_b0, s_red[32];
  uint32_t* aux = hqg_aux(smem);
  const gpq_item* R = q.root + q.off;
  const uint32_t nr = q.cnt0;
  for (uint32_t k = threadIdx.x; k < BI; k += blockDim.x) s_pre[k] = ic[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    int ovf = 0;
    for (uint32_t k = 0; k < BI; ++k) {
      const uint32_t v = s_pre[k];
      ovf |= v > kHqgListCapI ? 1 : 0;
      s_pre[k] = run;
      run += v;
    }
    s_pre[BI] = run;
    s_ovf = ovf || run != nch;
  }
  __syncthreads();
  if (s_ovf) return false;  // the same decision in every block: nothing written
  uint32_t lim = 0;  // pre.on: the next window's bound (ts bits), the same in every block
  if (pre.on) {
    if (threadIdx.x == 0) {
      uint32_t b0 = BI;
      for (uint32_t k = 0; k < BI && b0 == BI; ++k)
        if (s_pre[k + 1] > s_pre[k]) b0 = k;
      s_b0 = b0;
    }
    __syncthreads();
    uint32_t mn = (threadIdx.x == 0 && nr > 0) ? gpq_f2u(R[0].ts) : kInfBits;
    if (s_b0 < BI) {
      const gpq_item* l0 = g.ilist + (size_t)s_b0 * kHqgListCapI;
      for (uint32_t j = threadIdx.x; j < s_pre[s_b0 + 1] - s_pre[s_b0]; j += blockDim.x) mn = min(mn, gpq_f2u(l0[j].ts));
    }
    mn = block_min_u32(mn, s_red);
    lim = min(gpq_f2u(GPQ_FADD(gpq_u2f(mn), pre.la)), gpq_f2u(pre.T));
  }
  gpq_item* sa = reinterpret_cast<gpq_item*>(smem);
  gpq_item* sb = sa + hqg_tile_cap<HqgItemOps>();
  gpq_item* out = q.spare;
  for (uint32_t b = blockIdx.x; b < BI; b += gridDim.x) {
    const uint32_t nc = s_pre[b + 1] - s_pre[b];
    const gpq_item* src = g.ilist + (size_t)b * kHqgListCapI;
    for (uint32_t j = threadIdx.x; j < nc; j += blockDim.x) sa[hqg_pad<HqgItemOps>(j)] = src[j];
    __syncthreads();
    const gpq_item* X = hqg_bin_sort_items(sa, sb, nc, L, aux) ? sb : hqg_cta_sort<HqgItemOps>(sa, sb, nc);
    gpq_item* Y = (X == sa) ? sb : sa;  // two of the three staging buffers for R's tiles
    const uint32_t r0 = (uint32_t)((uint64_t)b * nr / BI), r1 = (uint32_t)((uint64_t)(b + 1) * nr / BI);
    const uint32_t nrb = r1 - r0, base = r0 + s_pre[b];
    // R's slice in tiles of kStreamTile, copied into shared memory asynchronously two tiles
    // ahead (three staging buffers: the two halves of the free tile and the auxiliary
    // area); each tile merged with the children between its first item and the next tile's
    // (merge path, an equal run of outputs a thread).  chis[t]: the children below tile t + 1's
    // first item, for all tiles at once.
    constexpr uint32_t kStreamTile = 2048;
    constexpr uint32_t kHalf = kStreamTile + kStreamTile / kHqgIpt;  // a padded tile
    constexpr uint32_t kChis = 2048;                                 // words at the end of aux
    static_assert(kHalf * sizeof(gpq_item) <= (kHqgAux - kChis) * sizeof(uint32_t), "third staging buffer");
    const uint32_t ntiles = (nrb + kStreamTile - 1) / kStreamTile;
    uint32_t* chis = aux + (kHqgAux - kChis);
    gpq_item* const stg[3] = {Y, Y + kHalf, reinterpret_cast<gpq_item*>(aux)};
    auto issue = [&](uint32_t tt, gpq_item* Yh) {  // tile tt's copies, one group per thread
      const uint32_t t0 = tt * kStreamTile;
      for (uint32_t i = threadIdx.x; i < kStreamTile; i += blockDim.x)
        if (t0 + i < nrb) hqg_cp16(&Yh[hqg_pad<HqgItemOps>(i)], &R[r0 + t0 + i]);
      hqg_cp_commit();
    };
    uint32_t cpos = 0;  // children below the current tile's first item
    for (uint32_t tb = 0; tb < ntiles; tb += kChis) {  // boundaries, kChis at a time
      const uint32_t tcnt = min(kChis, ntiles - tb);
      for (uint32_t t = threadIdx.x; t < tcnt; t += blockDim.x) {
        const uint32_t tt = tb + t, nxt = (tt + 1) * kStreamTile;
        uint32_t chi = nc;
        if (nxt < nrb) {
          const gpq_item nx = R[r0 + nxt];
          uint32_t lo = 0, hi = nc;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (hq_less(X[hqg_pad<HqgItemOps>(mid)], nx)) lo = mid + 1; else hi = mid;
          }
          chi = lo;
        }
        chis[t] = chi;
      }
      issue(tb, stg[0]);
      if (tcnt > 1) issue(tb + 1, stg[1]); else hqg_cp_commit();
      for (uint32_t t = 0; t < tcnt; ++t) {
        hqg_cp_wait<1>();  // this tile's copies have landed (the next one's may be in flight)
        __syncthreads();
        const uint32_t tt = tb + t, t0 = tt * kStreamTile;
        const gpq_item* Yh = stg[t % 3];
        if (t + 2 < tcnt) issue(tt + 2, stg[(t + 2) % 3]); else hqg_cp_commit();  // read in the last round
        const uint32_t tn = min(kStreamTile, nrb - t0), chi = chis[t], cn = chi - cpos, total = tn + cn;
        gpq_item* dst = out + base + t0 + cpos;
        // every thread one run of about total / blockDim outputs (at most kHqgIpt, the
        // padding's stride, so the lanes' heads stay in different bank groups)
        const uint32_t per = min(kHqgIpt, (total + blockDim.x - 1u) / blockDim.x);
        for (uint32_t o0 = threadIdx.x * per; o0 < total; o0 += blockDim.x * per)
          hqg_merge_run<HqgItemOps>(Yh, 0, tn, X, cpos, cn, o0, [&](uint32_t k, const gpq_item& v) { dst[o0 + k] = v; },
                                    per);
        cpos = chi;
      }
      hqg_cp_wait<0>();
      __syncthreads();
    }
    for (uint32_t j = cpos + threadIdx.x; j < nc; j += blockDim.x) out[base + nrb + j] = X[hqg_pad<HqgItemOps>(j)];
    __syncthreads();
    if (pre.on) {  // this CTA's outputs below the bound: R's and the children's below it
      const uint32_t nR = hqg_cta_search(0, nrb, [R, r0, lim](uint32_t i) { return gpq_f2u(R[r0 + i].ts) >= lim; });
      const uint32_t nX =
          hqg_cta_search(0, nc, [X, lim](uint32_t i) { return gpq_f2u(X[hqg_pad<HqgItemOps>(i)].ts) >= lim; });
      hqg_file_range(g, out, base, base + nR + nX, pre.BP, pre.pc, L, aux);
    }
  }
  if (!hqg_bar(s)) return false;
  q.swap_root();
  q.cnt0 = nr + nch;
  return true;
}

// hqg_file_range over equal slices of the batch root[0, c), one per CTA; ends with a barrier.
__device__ void hqg_file_batch(const PholdDev& d, const HqgDev& g, const gpq_item* root, uint32_t c, uint32_t BP,
                               uint32_t* pc, unsigned char* smem, HqgSync& s) {
  const uint32_t per = (c + gridDim.x - 1) / gridDim.x;
  const uint32_t lo = min(c, blockIdx.x * per), hi = min(c, lo + per);
  hqg_file_range(g, root, lo, hi, BP, pc, d.L, hqg_aux(smem));
  hqg_bar(s);
}

// ---------------------------------------------------------------------------------------
// All windows of one heap (des_run over the parallel heap), the whole grid.  Per window:
// the previous window's children sorted and inserted, the bound fixed from the root's
// head, then batches -- the root's prefix below the bound, folded into the per-LP outputs
// with ranks from the key sort, its children appended to h.ch, the root refilled -- until
// the root's head reaches the bound.  The root always holds the r smallest items, so the
// batches come in global key order; a child is never safe in its parent's window.
static __global__ void __launch_bounds__(kHqgThreads, 1) hqg_phold_kernel(PholdDev d, HqgDev g, uint32_t max_steps) {
  extern __shared__ __align__(16) unsigned char smem[];
  const HqDev& h = g.h;
  const uint32_t r = h.r;
  HqgSync s{&d, 0ull, true};
  HqgState q;
  q.root = h.nodes;
  q.spare = g.root2;
  q.off = 0;
  q.last = h.meta[0];
  q.cnt0 = h.cnt[0];
  q.cntl = q.last > 0 ? h.cnt[q.last] : 0u;
  uint32_t steps = 0, nch = 0, ovf_seen = 0;
  uint32_t c_last = 0;    // size of the last batch
  bool prefiled = false;  // this window's batch was filed by the insert phase (pre_bp ranges)
  uint32_t pre_bp = 0;
  HqgLists lists{false, 0u};
  __shared__ gpq_item s_spl[kHqgMaxBuckets];
  __shared__ uint32_t s_pc[kHqgMaxBuckets];
  __shared__ int s_pc_ovf;
  __shared__ uint32_t s_pc_sum;
  while (s.ok) {
    if (nch > 0) {  // the previous window's children
      bool done = false;
      if (g.icnt != nullptr && blockIdx.x == 0)  // the next window's insert counts start at zero
        for (uint32_t k = threadIdx.x; k < kHqgMaxBuckets; k += blockDim.x)
          g.icnt[((steps + 1u) & 1u) * kHqgMaxBuckets + k] = 0u;
      if (lists.ins) {
        // a batch of a large share of the root (C1-like windows) is filed while the children
        // are merged; a small one (a long array) is filed by equal slices in a phase of its own
        HqgPre pre{};
        pre.on = g.plist != nullptr && q.last == 0 && 4ull * c_last >= (uint64_t)q.cnt0 + nch;
        pre.la = d.p.lookahead;
        pre.T = d.p.end_time;
        pre.BP = min(gridDim.x, max(1u, c_last / 64u));
        pre.pc = g.pcnt + ((steps + 1u) & 1u) * kHqgMaxBuckets;
        done = hqg_insert_lists(g, q, nch, lists.BI, g.icnt + (steps & 1u) * kHqgMaxBuckets, d.L, pre, smem, s);
        if (!s.ok) break;
        prefiled = done && pre.on;
        pre_bp = pre.BP;
      }
      lists.ins = false;
      if (!done) {
        const uint32_t B = hqg_insert_buckets(q, r, nch);
        const bool done1 = B != 0 && hqg_insert_scan(g, q, h.ch, nch, B, smem, s, ovf_seen);
        if (!s.ok) break;
        if (!done1) {
          const gpq_item* ch = h.ch;
          const gpq_item* sorted = hqg_sort<HqgItemOps>(h.ch, g.e2, nch, smem, s, [ch](uint32_t j) { return ch[j]; });
          if (!hqg_insert(d, g, q, sorted, nch, smem, s)) break;
        }
      }
      nch = 0;
    }
    if (q.cnt0 == 0 || (max_steps != 0 && steps >= max_steps)) break;
    const float m = q.root[q.off].ts;
    if (!(m < d.p.end_time)) break;
    const uint32_t lim = min(gpq_f2u(GPQ_FADD(m, d.p.lookahead)), gpq_f2u(d.p.end_time));
    ++steps;
    while (s.ok) {  // batches of the window
      const gpq_item* root = q.root + q.off;
      const uint32_t c = hqg_cta_search(0, q.cnt0, [root, lim](uint32_t i) { return gpq_f2u(root[i].ts) >= lim; });
      const bool use_pre = prefiled;  // only the window's first batch
      prefiled = false;
      if (c == 0) break;
      // LP-range lists for the batch (a heap whose root holds every item; other heaps scan
      // the batch in each CTA or take the general path)
      bool from_lists = false;
      uint32_t BP = 0;
      if (g.pcnt != nullptr && blockIdx.x == 0)  // the next window's range counts start at zero
        for (uint32_t k = threadIdx.x; k < kHqgMaxBuckets; k += blockDim.x)
          g.pcnt[((steps + 1u) & 1u) * kHqgMaxBuckets + k] = 0u;
      if (g.plist != nullptr && q.last == 0) {  // the root holds every item: file the batch
        uint32_t* pc = g.pcnt + (steps & 1u) * kHqgMaxBuckets;
        if (use_pre) {  // filed by the insert phase
          BP = pre_bp;
        } else {
          BP = min(gridDim.x, max(1u, c / 64u));
          hqg_file_batch(d, g, root, c, BP, pc, smem, s);
          if (!s.ok) break;
        }
        for (uint32_t k = threadIdx.x; k < BP; k += blockDim.x) s_pc[k] = ld_relaxed_u32(&pc[k]);
        __syncthreads();
        if (threadIdx.x == 0) {
          uint32_t sum = 0;
          int ovf = 0;
          for (uint32_t k = 0; k < BP; ++k) {
            sum += s_pc[k];
            ovf |= s_pc[k] > kHqgListCapP ? 1 : 0;
          }
          s_pc_sum = sum;
          s_pc_ovf = ovf;
        }
        __syncthreads();
        from_lists = !s_pc_ovf && s_pc_sum == c;
      }
      HqgIns ins{};
      ins.on = g.ilist != nullptr && q.last == 0 && nch == 0;
      if (ins.on) {
        const uint32_t nr = q.cnt0 - c;
        ins.BI = hqg_list_ibuckets(nr, c);
        hqg_load_splitters(s_spl, root + c, nr, ins.BI);
        ins.spl = s_spl;
        ins.icnt = g.icnt + (steps & 1u) * kHqgMaxBuckets;
        ins.ilist = g.ilist;
      }
      bool done = false;
      if (from_lists) {
        hqg_process_lists(d, g, root, s_pc, BP, nch, ins, smem, s);
        done = true;
      } else if (c <= kHqgScanBatchMax) {
        done = hqg_process_scan(d, g, root, c, nch, ins, smem, s);
      }
      if (!done) {
        hqg_ranks(d, g, root, c, smem, s);
        for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < c; i0 += hqg_nthreads()) {
          const uint32_t i = i0 + threadIdx.x;
          const bool valid = i < c;
          gpq_item ch{};
          if (valid) {
            const gpq_item e = root[i];
            const uint64_t hh = gpq_ev_hash(e.id, gpq_f2u(e.ts));
            const uint32_t add = g.addc[i];
            if (add) d.count[e.lp] += add;  // the LP's one writer in this batch
            atomicAdd(&d.csum[e.lp], (unsigned long long)hh);
            atomicAdd(&d.ohash[e.lp], (unsigned long long)gpq_seq_hash(hh, (uint64_t)g.rank[i]));
            ch = gpq_phold_child(d.p, e);
            h.ch[nch + i] = ch;
          }
          if (ins.on) {
            const uint32_t bk = valid ? hqg_bucket_of(ins.spl, ins.BI - 1, ch) : 0u;
            hqg_list_append<gpq_item>(ins.icnt, ins.ilist, kHqgListCapI, valid, bk, ch);
          }
        }
        hqg_bar(s);
      }
      lists.ins = ins.on;
      lists.BI = ins.BI;
      c_last = c;
      nch += c;
      q.off += c;
      q.cnt0 -= c;
      if (!hqg_refill(g, q, smem, s)) break;
    }
  }
  // Leave the root in node 0's storage at offset 0 and the counts in h.cnt / h.meta.
  if (s.ok && q.root != h.nodes) {
    hqg_copy(h.nodes, q.root + q.off, q.cnt0, s);
  } else if (s.ok && q.off != 0) {
    hqg_copy(g.root2, q.root + q.off, q.cnt0, s);
    hqg_copy(h.nodes, g.root2, q.cnt0, s);
  }
  if (blockIdx.x == 0) {
    for (uint32_t i = threadIdx.x; i <= q.last; i += blockDim.x) h.cnt[i] = q.cnt(i, r);
    if (threadIdx.x == 0) {
      h.meta[0] = q.last;
      h.meta[1] = steps;
      d.ctrl->steps = steps;
    }
  }
}
