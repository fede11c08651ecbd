// A* grid search on the GPU: many instances, each grid cut into square tiles (the
// shards of the open list), one persistent cooperative launch over rounds.
//
// Reference: src/a_star.cu:269-593 runs one best-first search per agent in one CTA,
// popping up to eight open-list minima per round from the agent's queue
// (queue_peek/queue_set_done/queue_insert_or_update, src/queue.cuh:46-70).  Here the
// open list of an instance is sharded by tile, and a round drains every tile's items
// inside the instance's current window f <= bound:
//
//   * phase P: each active tile is taken by one CTA.  Its inbox (items sent by other
//     tiles in the previous round) and, when the window moved, its open array are
//     scanned; stale items (g above the cell's current g) are dropped, items above the
//     instance's best goal cost UB are pruned, items with f <= bound join the CTA's
//     frontier in shared memory and the rest stay in the open array.  The CTA then
//     expands the frontier level by level: a child whose g improves (atomicMin on the
//     cell's g) goes to the next frontier when it lies in the tile and in the window,
//     to the tile's open array when above the window, or to the owning tile's inbox for
//     the next round.
//   * phase W: an instance whose tiles sent nothing for the next round has drained its
//     window; the window moves to [min f of its open arrays, + delta], or the instance
//     is done when that minimum exceeds UB.
//
// Work items are 8 bytes (cell, g); f = g + h(cell) is recomputed.  With a consistent
// heuristic every cell with g + h <= C* ends with its exact g, whatever the order of
// expansions, so the outputs (C*, the expanded set, the canonical path) do not depend
// on the schedule; re-expansions only cost time.
#pragma once

#include "common.cuh"
#include "gpq/astar.h"

static constexpr uint32_t kAstarInf = GPQ_ASTAR_INF;

struct AstarInstDev {
  gpq_astar_grid g;
  uint64_t cell0;      // first cell in the shared g array and bitmap (a multiple of 32)
  uint32_t tile0;      // first tile
  uint32_t tiles_x, tiles_y;
  uint32_t ub;         // best goal cost found so far
  uint32_t bound;      // window: items with f <= bound are expanded
  uint32_t active_next;
  uint32_t done;
  uint32_t err;
  uint32_t windows;
  uint32_t delta;      // window width on f
  unsigned long long pops;  // expansions performed (re-expansions included)
};

struct AstarTileDev {
  uint32_t inst;
  uint32_t tx, ty;
  uint32_t in_cnt[2];  // inbox fill per round parity
  uint32_t open_cnt;   // open array fill
  uint32_t open_min;   // min f in the open array (kAstarInf when empty)
  uint32_t queued[2];  // on the active list of the round with this parity
  uint32_t pad[3];
};

// Control words of one launch.
struct AstarCtl {
  uint32_t al_cnt[2];
  uint32_t work[2];
  uint32_t err;
  uint32_t rounds;
  unsigned long long bar;
};

struct AstarDev {
  AstarInstDev* inst;
  AstarTileDev* tiles;
  uint32_t* gcost;  // [cells]
  const uint32_t* blk;  // blocked bitmap, one bit per cell
  uint2* inbox;     // [2][n_tiles][in_cap] (cell, g)
  uint2* open;      // [n_tiles][open_cap]
  uint32_t* al;     // [2][n_tiles] active tiles per round parity
  AstarCtl* ctl;
  uint32_t n_inst, n_tiles;
  uint32_t in_cap, open_cap;
  uint32_t ts;      // tile side
  uint32_t max_rounds;
  uint32_t frontier_cap;  // per shared frontier buffer
  uint64_t spin_limit;
};

__device__ __forceinline__ uint32_t ldcg_u32(const uint32_t* p) { return __ldcg(p); }

__device__ __forceinline__ bool astar_blocked(const AstarDev& d, const AstarInstDev& I, uint32_t cell) {
  const uint64_t b = I.cell0 + cell;
  return (__ldg(&d.blk[b >> 5]) >> (b & 31u)) & 1u;
}

__device__ __forceinline__ uint32_t astar_tile_of(const AstarDev& d, const AstarInstDev& I, uint32_t cell) {
  const uint32_t x = cell % I.g.width, y = cell / I.g.width;
  return I.tile0 + (y / d.ts) * I.tiles_x + x / d.ts;
}

// Put tile t on the active list of round parity `par` (once per round).
__device__ __forceinline__ void astar_activate(const AstarDev& d, uint32_t t, uint32_t par, bool count) {
  if (atomicExch(&d.tiles[t].queued[par], 1u) == 0u) {
    const uint32_t pos = atomicAdd(&d.ctl->al_cnt[par], 1u);
    d.al[(size_t)par * d.n_tiles + pos] = t;
    if (count) atomicAdd(&d.inst[d.tiles[t].inst].active_next, 1u);
  }
}

__device__ __forceinline__ void astar_inbox_push(const AstarDev& d, AstarInstDev* Ip, uint32_t t, uint32_t par,
                                                 uint2 it) {
  const uint32_t pos = atomicAdd(&d.tiles[t].in_cnt[par], 1u);
  if (pos < d.in_cap) {
    d.inbox[((size_t)par * d.n_tiles + t) * d.in_cap + pos] = it;
  } else {
    gpq_set_error(&Ip->err, GPQ_ERR_INSERT_FULL);
  }
  astar_activate(d, t, par, true);
}

// Shared state of the CTA working on one tile.
struct AstarTileSmem {
  uint2* fa;  // frontier buffers
  uint2* fb;
  uint32_t n[2];
  uint32_t open_min;
  uint32_t open_cnt;
  uint32_t t;
  uint32_t inst;
  unsigned long long pops;
  uint32_t scan[33];
};

// Frontier push: into the shared buffer, or (when it is full) into the tile's own inbox
// for the next round.
__device__ __forceinline__ void astar_frontier_push(const AstarDev& d, AstarInstDev* Ip, AstarTileSmem& sm,
                                                    uint2* buf, uint32_t which, uint32_t t, uint32_t npar, uint2 it) {
  const uint32_t pos = atomicAdd(&sm.n[which], 1u);
  if (pos < d.frontier_cap) {
    buf[pos] = it;
  } else {
    astar_inbox_push(d, Ip, t, npar, it);
  }
}

__device__ __forceinline__ void astar_open_push(const AstarDev& d, AstarInstDev* Ip, AstarTileSmem& sm, uint32_t t,
                                                uint2 it, uint32_t f) {
  const uint32_t pos = atomicAdd(&sm.open_cnt, 1u);
  if (pos < d.open_cap) {
    d.open[(size_t)t * d.open_cap + pos] = it;
    atomicMin(&sm.open_min, f);
  } else {
    gpq_set_error(&Ip->err, GPQ_ERR_QUEUE_FULL);
  }
}

// Expand one frontier item of tile t (one thread).
__device__ __forceinline__ void astar_expand(const AstarDev& d, AstarInstDev* Ip, const AstarInstDev& I,
                                             AstarTileSmem& sm, uint2* next, uint32_t which, uint32_t t, uint32_t npar,
                                             uint2 it, uint32_t bound, uint32_t* pops) {
  const uint32_t cell = it.x, g = it.y;
  uint32_t* G = d.gcost + I.cell0;
  if (ldcg_u32(&G[cell]) != g) return;  // a better path reached the cell meanwhile
  ++*pops;
  const uint32_t w = I.g.width, h = I.g.height, conn = I.g.conn;
  const int x = (int)(cell % w), y = (int)(cell / w);
  const int nk = conn == 4 ? 4 : 8;
  for (int k = 0; k < nk; ++k) {
    const int nx = x + gpq_astar_dx(k), ny = y + gpq_astar_dy(k);
    if (nx < 0 || ny < 0 || nx >= (int)w || ny >= (int)h) continue;
    const uint32_t nb = (uint32_t)ny * w + (uint32_t)nx;
    if (astar_blocked(d, I, nb)) continue;
    if (k >= 4 && (astar_blocked(d, I, (uint32_t)y * w + (uint32_t)nx) || astar_blocked(d, I, (uint32_t)ny * w + (uint32_t)x)))
      continue;
    const uint32_t ng = g + gpq_astar_cost(conn, k);
    const uint32_t old = atomicMin(&G[nb], ng);
    if (ng >= old) continue;
    const uint32_t nf = ng + gpq_astar_h(conn, nb, I.g.goal, w);
    if (nb == I.g.goal) atomicMin(&Ip->ub, ng);
    if (nf > ldcg_u32(&Ip->ub)) continue;
    const uint2 child = make_uint2(nb, ng);
    const uint32_t nt = astar_tile_of(d, I, nb);
    if (nt == t) {
      if (nf <= bound) astar_frontier_push(d, Ip, sm, next, which, t, npar, child);
      else astar_open_push(d, Ip, sm, t, child, nf);
    } else {
      astar_inbox_push(d, Ip, nt, npar, child);
    }
  }
}

// Block-wide exclusive prefix sum of 0/1 flags; returns this thread's offset and writes
// the total to *total.  All threads call.
__device__ __forceinline__ uint32_t astar_block_scan(uint32_t flag, uint32_t* scratch, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(GPQ_FULL_MASK, flag);
  const uint32_t below = __popc(bal & ((1u << lane) - 1u));
  if (lane == 0) scratch[warp] = __popc(bal);
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = blockDim.x >> 5;
    uint32_t v = lane < nw ? scratch[lane] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(GPQ_FULL_MASK, incl, o);
      if (lane >= (uint32_t)o) incl += u;
    }
    if (lane < nw) scratch[lane] = incl - v;
    if (lane == 31) scratch[32] = incl;
  }
  __syncthreads();
  const uint32_t off = scratch[warp] + below;
  *total = scratch[32];
  __syncthreads();
  return off;
}

// Process tile t in round s (the whole CTA).
__device__ void astar_process_tile(const AstarDev& d, uint32_t t, uint32_t s, AstarTileSmem& sm) {
  const uint32_t par = s & 1u, npar = par ^ 1u;
  AstarTileDev* T = d.tiles + t;
  AstarInstDev* Ip = d.inst + T->inst;
  const AstarInstDev I = *Ip;  // static fields; ub/bound are read through Ip
  uint32_t* G = d.gcost + I.cell0;
  if (threadIdx.x == 0) {
    sm.n[0] = 0;
    sm.n[1] = 0;
    sm.pops = 0;
    sm.open_cnt = T->open_cnt;
    sm.open_min = kAstarInf;
  }
  __syncthreads();
  const uint32_t k_in = min(ldcg_u32(&T->in_cnt[par]), d.in_cap);
  const uint32_t bound = ldcg_u32(&Ip->bound);
  if (ldcg_u32(&Ip->done)) {
    if (threadIdx.x == 0) {
      T->in_cnt[par] = 0;
      T->queued[par] = 0;
      T->open_cnt = 0;
      T->open_min = kAstarInf;
    }
    __syncthreads();
    return;
  }
  uint32_t ub = ldcg_u32(&Ip->ub);
  // 1. the open array, when the window reached it: expand-now items leave, the rest is
  //    compacted in place (a chunk is read completely before any of it is written)
  const uint32_t n_open = sm.open_cnt;
  if (n_open > 0 && ldcg_u32(&T->open_min) <= bound) {
    uint2* O = d.open + (size_t)t * d.open_cap;
    uint32_t kept = 0;
    for (uint32_t c0 = 0; c0 < n_open; c0 += blockDim.x) {
      const uint32_t i = c0 + threadIdx.x;
      uint2 it = make_uint2(0, kAstarInf);
      uint32_t keep = 0, f = kAstarInf;
      if (i < n_open) {
        it = O[i];
        if (ldcg_u32(&G[it.x]) == it.y) {
          f = it.y + gpq_astar_h(I.g.conn, it.x, I.g.goal, I.g.width);
          if (f <= ub) {
            if (f <= bound) astar_frontier_push(d, Ip, sm, sm.fa, 0, t, npar, it);
            else keep = 1;
          }
        }
      }
      uint32_t total;
      const uint32_t off = astar_block_scan(keep, sm.scan, &total);
      if (keep) {
        O[kept + off] = it;
        atomicMin(&sm.open_min, f);
      }
      kept += total;
    }
    if (threadIdx.x == 0) sm.open_cnt = kept;
    __syncthreads();
  } else if (threadIdx.x == 0) {
    sm.open_min = ldcg_u32(&T->open_min);
  }
  __syncthreads();
  // 2. the inbox
  {
    const uint2* B = d.inbox + ((size_t)par * d.n_tiles + t) * d.in_cap;
    for (uint32_t i = threadIdx.x; i < k_in; i += blockDim.x) {
      const uint2 it = B[i];
      if (ldcg_u32(&G[it.x]) != it.y) continue;
      const uint32_t f = it.y + gpq_astar_h(I.g.conn, it.x, I.g.goal, I.g.width);
      if (f > ub) continue;
      if (f <= bound) astar_frontier_push(d, Ip, sm, sm.fa, 0, t, npar, it);
      else astar_open_push(d, Ip, sm, t, it, f);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T->in_cnt[par] = 0;
    T->queued[par] = 0;
  }
  // 3. level-by-level expansion of the frontier inside the tile
  uint32_t pops = 0;
  uint32_t cur = 0;
  for (;;) {
    const uint32_t n = min(sm.n[cur], d.frontier_cap);
    if (n == 0) break;
    uint2* src = cur ? sm.fb : sm.fa;
    uint2* dst = cur ? sm.fa : sm.fb;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
      astar_expand(d, Ip, I, sm, dst, cur ^ 1u, t, npar, src[i], bound, &pops);
    __syncthreads();
    if (threadIdx.x == 0) sm.n[cur] = 0;
    cur ^= 1u;
    __syncthreads();
  }
  pops = warp_sum_u32(pops);
  if ((threadIdx.x & 31u) == 0 && pops) atomicAdd(&sm.pops, (unsigned long long)pops);
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t oc = min(sm.open_cnt, d.open_cap);
    T->open_cnt = oc;
    T->open_min = oc ? sm.open_min : kAstarInf;
    if (sm.pops) atomicAdd(&Ip->pops, sm.pops);
  }
  __syncthreads();
}

// Phase W for one instance (one warp): a drained window moves on, or the instance ends.
__device__ void astar_window_step(const AstarDev& d, uint32_t i, uint32_t npar) {
  AstarInstDev* Ip = d.inst + i;
  const uint32_t lane = threadIdx.x & 31u;
  if (ldcg_u32(&Ip->done)) return;
  const uint32_t a = ldcg_u32(&Ip->active_next);
  __syncwarp();
  if (lane == 0) Ip->active_next = 0;
  if (a > 0) return;
  const uint32_t nt = Ip->tiles_x * Ip->tiles_y, t0 = Ip->tile0;
  uint32_t m = kAstarInf;
  for (uint32_t j = lane; j < nt; j += 32) {
    const AstarTileDev* T = d.tiles + t0 + j;
    if (ldcg_u32(&T->open_cnt)) m = min(m, ldcg_u32(&T->open_min));
  }
  m = warp_min_u32(m);
  const uint32_t ub = ldcg_u32(&Ip->ub);
  if (m == kAstarInf || m > ub) {
    if (lane == 0) Ip->done = 1;
    return;
  }
  uint32_t bound = m + Ip->delta;
  if (bound < m || bound > ub) bound = ub;
  if (lane == 0) {
    Ip->bound = bound;
    Ip->windows += 1;
  }
  for (uint32_t j = lane; j < nt; j += 32) {
    AstarTileDev* T = d.tiles + t0 + j;
    if (ldcg_u32(&T->open_cnt) && ldcg_u32(&T->open_min) <= bound) astar_activate(d, t0 + j, npar, false);
  }
}

// The persistent search loop over all instances.  Dynamic shared memory: two frontier
// buffers of frontier_cap items.
static __global__ void __launch_bounds__(256) astar_persistent_kernel(AstarDev d) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ AstarTileSmem sm;
  __shared__ uint32_t s_t;
  if (threadIdx.x == 0) {
    sm.fa = reinterpret_cast<uint2*>(smem_raw);
    sm.fb = sm.fa + d.frontier_cap;
  }
  __syncthreads();
  const unsigned long long nb = gridDim.x;
  unsigned long long bar_target = 0;
  const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
  const uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (uint32_t s = 0;; ++s) {
    const uint32_t par = s & 1u, npar = par ^ 1u;
    const uint32_t n = ldcg_u32(&d.ctl->al_cnt[par]);
    for (;;) {
      if (threadIdx.x == 0) s_t = atomicAdd(&d.ctl->work[par], 1u);
      __syncthreads();
      const uint32_t j = s_t;
      __syncthreads();
      if (j >= n) break;
      astar_process_tile(d, d.al[(size_t)par * d.n_tiles + j], s, sm);
    }
    bar_target += nb;
    if (!grid_barrier(&d.ctl->bar, bar_target, d.spin_limit, &d.ctl->err)) return;
    for (uint32_t i = gwarp; i < d.n_inst; i += warps_total) astar_window_step(d, i, npar);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      d.ctl->al_cnt[par] = 0;
      d.ctl->work[par] = 0;
      d.ctl->rounds = s + 1;
    }
    bar_target += nb;
    if (!grid_barrier(&d.ctl->bar, bar_target, d.spin_limit, &d.ctl->err)) return;
    if (ldcg_u32(&d.ctl->al_cnt[npar]) == 0 || ldcg_u32(&d.ctl->err) != 0) break;
    if (d.max_rounds && s + 1 >= d.max_rounds) {
      if (blockIdx.x == 0 && threadIdx.x == 0) gpq_set_error(&d.ctl->err, GPQ_ERR_TIMEOUT);
      break;
    }
  }
}

// ---- set-up and results ----

// Blocked bitmap of all instances: one thread per 32-cell word.
static __global__ void astar_bitmap_kernel(const AstarInstDev* inst, uint32_t n_inst, const uint64_t* word0,
                                           uint64_t total_words, uint32_t* blk) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t wi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; wi < total_words; wi += stride) {
    uint32_t lo = 0, hi = n_inst - 1;  // last instance with word0 <= wi
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (word0[mid] <= wi) lo = mid; else hi = mid - 1;
    }
    const AstarInstDev& I = inst[lo];
    const uint64_t cells = (uint64_t)I.g.width * I.g.height;
    const uint64_t c0 = (wi - word0[lo]) * 32u;
    uint32_t w = 0;
    for (uint32_t b = 0; b < 32; ++b) {
      const uint64_t c = c0 + b;
      if (c < cells && gpq_astar_blocked(&I.g, (uint32_t)c)) w |= 1u << b;
    }
    blk[wi] = w;
  }
}

// Initial state: g = inf everywhere (done by a memset), g[start] = 0, the start item in
// the start tile's inbox, the start tiles on the round-0 active list.
static __global__ void astar_init_kernel(AstarDev d) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_inst) return;
  AstarInstDev& I = d.inst[i];
  d.gcost[I.cell0 + I.g.start] = 0;
  const uint32_t t = astar_tile_of(d, I, I.g.start);
  d.tiles[t].in_cnt[0] = 1;
  d.inbox[(size_t)t * d.in_cap] = make_uint2(I.g.start, 0);
  d.tiles[t].queued[0] = 1;
  d.al[i] = t;
  if (i == 0) d.ctl->al_cnt[0] = d.n_inst;
}

static __global__ void astar_tiles_init_kernel(AstarDev d) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  for (uint32_t inst = i; inst < d.n_inst; inst += nthreads) {
    const AstarInstDev& I = d.inst[inst];
    for (uint32_t ty = 0; ty < I.tiles_y; ++ty)
      for (uint32_t tx = 0; tx < I.tiles_x; ++tx) {
        AstarTileDev T{};
        T.inst = inst;
        T.tx = tx;
        T.ty = ty;
        T.open_min = kAstarInf;
        d.tiles[I.tile0 + ty * I.tiles_x + tx] = T;
      }
  }
}

// Per-instance expanded set (g + h <= C*, or every reached cell when the goal is not
// reachable): count and hash.  Block per (instance, chunk): blockIdx.y = instance.
static __global__ void astar_finalize_kernel(AstarDev d, unsigned long long* out /* [n_inst][2] */) {
  const uint32_t i = blockIdx.y;
  const AstarInstDev& I = d.inst[i];
  const uint32_t cs = I.ub;
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  const uint32_t* G = d.gcost + I.cell0;
  unsigned long long cnt = 0, hs = 0;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < cells;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = G[c];
    if (g == kAstarInf) continue;
    if (cs != kAstarInf && (uint64_t)g + gpq_astar_h(I.g.conn, (uint32_t)c, I.g.goal, I.g.width) > cs) continue;
    ++cnt;
    hs += gpq_astar_cell_hash((uint32_t)c, g);
  }
  cnt = warp_sum_u64(cnt);
  hs = warp_sum_u64(hs);
  if ((threadIdx.x & 31u) == 0 && cnt) {
    atomicAdd(&out[2 * i], cnt);
    atomicAdd(&out[2 * i + 1], hs);
  }
}

// Canonical path of each instance, one warp per instance: from the goal, step to the
// smallest-id neighbour p with g[p] + c(p, cell) == g[cell] and g[p] + h(p) <= C*.
// out[3 * i] = length, out[3 * i + 1] = hash, out[3 * i + 2] = 1 when the walk failed.
// When path != nullptr the cells of instance `want` are written (goal first, <= cap).
static __global__ void astar_path_kernel(AstarDev d, unsigned long long* out, uint32_t want, uint32_t* path,
                                         uint32_t cap) {
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (i >= d.n_inst) return;
  const AstarInstDev& I = d.inst[i];
  const uint32_t cs = I.ub;
  if (cs == kAstarInf) {
    if (lane == 0) { out[3 * i] = 0; out[3 * i + 1] = 0; out[3 * i + 2] = 0; }
    return;
  }
  const uint32_t* G = d.gcost + I.cell0;
  const uint32_t w = I.g.width, h = I.g.height, conn = I.g.conn;
  const uint64_t cells = (uint64_t)w * h;
  uint32_t cur = I.g.goal;
  unsigned long long hs = 0;
  uint32_t len = 0, fail = 0;
  for (uint64_t step = 0; step <= cells; ++step) {
    if (lane == 0) {
      hs += gpq_astar_path_hash(len, cur);
      if (path && i == want && len < cap) path[len] = cur;
    }
    ++len;
    if (cur == I.g.start) break;
    const uint32_t gc = G[cur];
    uint32_t cand = kAstarInf;
    const int k = (int)lane;
    if (k < (conn == 4 ? 4 : 8)) {
      const int x = (int)(cur % w), y = (int)(cur / w);
      const int nx = x + gpq_astar_dx(k), ny = y + gpq_astar_dy(k);
      if (nx >= 0 && ny >= 0 && nx < (int)w && ny < (int)h) {
        const uint32_t p = (uint32_t)ny * w + (uint32_t)nx;
        bool ok = !astar_blocked(d, I, p);
        if (ok && k >= 4)
          ok = !astar_blocked(d, I, (uint32_t)y * w + (uint32_t)nx) && !astar_blocked(d, I, (uint32_t)ny * w + (uint32_t)x);
        if (ok) {
          const uint32_t gp = G[p];
          if (gp != kAstarInf && (uint64_t)gp + gpq_astar_cost(conn, k) == gc &&
              (uint64_t)gp + gpq_astar_h(conn, p, I.g.goal, w) <= cs)
            cand = p;
        }
      }
    }
    cand = warp_min_u32(cand);
    if (cand == kAstarInf) { fail = 1; break; }
    cur = cand;
  }
  if (lane == 0) {
    out[3 * i] = len;
    out[3 * i + 1] = hs;
    out[3 * i + 2] = fail;
  }
}
