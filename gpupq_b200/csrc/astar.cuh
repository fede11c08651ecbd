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
// Work items are 8 bytes (y << 16 | x, g); f = g + h(x, y) is recomputed, so the hot loop
// needs no division.  With a consistent
// heuristic every cell with g + h <= C* ends with its exact g, whatever the order of
// expansions, so the outputs (C*, the expanded set, the canonical path) do not depend
// on the schedule; re-expansions only cost time.
#pragma once

#include "common.cuh"
#include "gpq/astar.h"

static constexpr uint32_t kAstarInf = GPQ_ASTAR_INF;

namespace gpq {
// Defaults and limits of the engine knobs (host side, astar.cu).
gpq_status astar_normalize(gpq_astar_config& c);
}  // namespace gpq

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
  uint32_t gx, gy;     // goal coordinates
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
  unsigned long long visits;  // tiles processed
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
  uint32_t lts;     // log2(ts)
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

__device__ __forceinline__ uint32_t astar_hxy(uint32_t conn, int x, int y, int gx, int gy) {
  const uint32_t dx = (uint32_t)abs(x - gx), dy = (uint32_t)abs(y - gy);
  return conn == 4 ? dx + dy : 10u * max(dx, dy) + 4u * min(dx, dy);
}

__device__ __forceinline__ uint32_t astar_pack(int x, int y) { return ((uint32_t)y << 16) | (uint32_t)x; }

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

// Shared state of the CTA working on one tile.  While a CTA holds a tile, the tile's g
// values live in shared memory (gt) and only this CTA changes them; other tiles lower the
// global copy with atomicMin (a filter for their sends) and the holder merges its copy
// back with atomicMin when it lets go of the tile.
struct AstarTileSmem {
  uint2* fa;      // frontier buffers [frontier_cap]
  uint2* fb;
  uint32_t* gt;   // [ts * ts] g of the tile's cells, local index ly * ts + lx
  uint32_t* blk;  // [ts * ts / 32] blocked bits of the tile
  uint32_t* chg;  // [ts * ts / 32] cells whose g dropped during this visit
  uint2* ob;      // [8 * ts] moves into other tiles, sent when the visit ends
  uint32_t ob_n;
  uint32_t n[3];  // frontier fill, rotating by level
  uint32_t ub;    // the instance's best goal cost as of this visit (stale values only prune less)
  uint32_t open_min;
  uint32_t open_cnt;
  unsigned long long pops;
  uint32_t scan[33];
};

__host__ __device__ inline uint32_t astar_outbox_cap(uint32_t ts) { return 8u * ts; }

__host__ __device__ inline size_t astar_smem_bytes(uint32_t ts, uint32_t frontier_cap) {
  return 2ull * frontier_cap * sizeof(uint2) + (size_t)astar_outbox_cap(ts) * sizeof(uint2) +
         (size_t)ts * ts * sizeof(uint32_t) + 2ull * (ts * ts / 32) * sizeof(uint32_t);
}

// Geometry of the tile being processed.
struct AstarTileGeo {
  uint32_t x0, y0, tw, th, ts;
  __device__ __forceinline__ bool inside(int x, int y) const {
    return x >= (int)x0 && y >= (int)y0 && x < (int)(x0 + tw) && y < (int)(y0 + th);
  }
  uint32_t lts;
  __device__ __forceinline__ uint32_t local(int x, int y) const {
    return (((uint32_t)y - y0) << lts) + ((uint32_t)x - x0);
  }
};

// The threads that process one tile visit: the whole CTA, or one warp (WARP), in which
// case every warp of the CTA works on its own tile with its own slice of shared memory.
template <bool WARP>
struct AstarWorker {
  uint32_t tid;  // thread within the worker
  uint32_t n;    // threads in the worker
  uint32_t id;   // worker within the CTA
  __device__ __forceinline__ AstarWorker() {
    if (WARP) {
      tid = threadIdx.x & 31u;
      n = 32u;
      id = threadIdx.x >> 5;
    } else {
      tid = threadIdx.x;
      n = blockDim.x;
      id = 0;
    }
  }
  __device__ __forceinline__ void sync() const {
    if (WARP) __syncwarp();
    else __syncthreads();
  }
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

__device__ __forceinline__ bool astar_cell_blocked(const AstarDev& d, const AstarInstDev& I, const AstarTileSmem& sm,
                                                   const AstarTileGeo& tg, int x, int y) {
  if (tg.inside(x, y)) {
    const uint32_t l = tg.local(x, y);
    return (sm.blk[l >> 5] >> (l & 31u)) & 1u;
  }
  return astar_blocked(d, I, (uint32_t)y * I.g.width + (uint32_t)x);
}

// A move into another tile: lower the cell's global g (the filter), and when that
// improves it, send the item to the owning tile's inbox for the next round.
__device__ __forceinline__ void astar_send(const AstarDev& d, AstarInstDev* Ip, const AstarInstDev& I, uint2 it,
                                           uint32_t npar) {
  const int x = (int)(it.x & 0xffffu), y = (int)(it.x >> 16);
  const uint32_t ng = it.y;
  if (ng >= atomicMin(&d.gcost[I.cell0 + (uint32_t)y * I.g.width + (uint32_t)x], ng)) return;
  const uint32_t nf = ng + astar_hxy(I.g.conn, x, y, (int)I.gx, (int)I.gy);
  if (x == (int)I.gx && y == (int)I.gy) atomicMin(&Ip->ub, ng);
  if (nf > ldcg_u32(&Ip->ub)) return;
  const uint32_t nt = I.tile0 + ((uint32_t)y >> d.lts) * I.tiles_x + ((uint32_t)x >> d.lts);
  astar_inbox_push(d, Ip, nt, npar, it);
}

// Expand frontier items src[ib .. ib + 32 / M) with one warp, one lane per (item, move):
// lane = item * M + move, M = 4 or 8 moves (all lanes call; ib is warp-uniform).  A level
// of few items thus costs the latency of one move, not of M moves in a row.  Children
// are appended with one shared atomic per warp and target: the frontier and the open
// array are the two hot counters of a level.
__device__ __forceinline__ void astar_expand_warp(const AstarDev& d, AstarInstDev* Ip, const AstarInstDev& I,
                                                  AstarTileSmem& sm, const AstarTileGeo& tg, const uint2* src,
                                                  uint32_t ib, uint32_t n, uint2* next, uint32_t which, uint32_t t,
                                                  uint32_t npar, uint32_t bound, uint32_t* pops) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t conn = I.g.conn;
  const uint32_t M = conn == 4 ? 4u : 8u;
  const uint32_t k = lane & (M - 1u);
  const uint32_t i = ib + lane / M;
  uint32_t kind = 0;  // 1 frontier, 2 open array, 4 outbox (another tile)
  uint2 child = make_uint2(0, 0);
  uint32_t nf = kAstarInf;
  if (i < n) {
    const uint2 it = src[i];
    const int x = (int)(it.x & 0xffffu), y = (int)(it.x >> 16);
    const uint32_t g = it.y;
    if (sm.gt[tg.local(x, y)] == g) {  // else a better path reached the cell meanwhile
      if (k == 0) ++*pops;
      const uint32_t w = I.g.width, h = I.g.height;
      const int nx = x + gpq_astar_dx((int)k), ny = y + gpq_astar_dy((int)k);
      if (nx >= 0 && ny >= 0 && nx < (int)w && ny < (int)h) {
        const bool in = tg.inside(nx, ny);
        const uint32_t l = in ? tg.local(nx, ny) : 0u;
        bool ok = !(in ? ((sm.blk[l >> 5] >> (l & 31u)) & 1u) : astar_blocked(d, I, (uint32_t)ny * w + (uint32_t)nx));
        if (ok && k >= 4) ok = !astar_cell_blocked(d, I, sm, tg, nx, y) && !astar_cell_blocked(d, I, sm, tg, x, ny);
        if (ok) {
          const uint32_t ng = g + gpq_astar_cost(conn, (int)k);
          if (in) {
            ok = ng < atomicMin(&sm.gt[l], ng);
            if (ok) atomicOr(&sm.chg[l >> 5], 1u << (l & 31u));
          } else {
            kind = 4u;  // to the outbox: filtered and sent when the visit ends
            child = make_uint2(astar_pack(nx, ny), ng);
            ok = false;
          }
          if (ok) {
            const int gx = (int)I.gx, gy = (int)I.gy;
            nf = ng + astar_hxy(conn, nx, ny, gx, gy);
            if (nx == gx && ny == gy) {
              atomicMin(&Ip->ub, ng);
              atomicMin(&sm.ub, ng);
            }
            if (nf <= sm.ub) {
              child = make_uint2(astar_pack(nx, ny), ng);
              kind = nf <= bound ? 1u : 2u;
            }
          }
        }
      }
    }
  }
  const uint32_t mf = __ballot_sync(GPQ_FULL_MASK, kind == 1u);
  if (mf) {
    const uint32_t leader = (uint32_t)(__ffs(mf) - 1);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&sm.n[which], (uint32_t)__popc(mf));
    base = __shfl_sync(GPQ_FULL_MASK, base, leader);
    if (kind == 1u) {
      const uint32_t pos = base + __popc(mf & lt);
      if (pos < d.frontier_cap) next[pos] = child;
      else astar_inbox_push(d, Ip, t, npar, child);  // full: the tile's own next round
    }
  }
  const uint32_t mx = __ballot_sync(GPQ_FULL_MASK, kind == 4u);
  if (mx) {
    const uint32_t leader = (uint32_t)(__ffs(mx) - 1);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&sm.ob_n, (uint32_t)__popc(mx));
    base = __shfl_sync(GPQ_FULL_MASK, base, leader);
    if (kind == 4u) {
      const uint32_t pos = base + __popc(mx & lt);
      if (pos < astar_outbox_cap(tg.ts)) sm.ob[pos] = child;
      else astar_send(d, Ip, I, child, npar);  // full: send now
    }
  }
  const uint32_t mo = __ballot_sync(GPQ_FULL_MASK, kind == 2u);
  if (mo) {
    const uint32_t leader = (uint32_t)(__ffs(mo) - 1);
    const uint32_t fmin = __reduce_min_sync(GPQ_FULL_MASK, kind == 2u ? nf : kAstarInf);
    uint32_t base = 0;
    if (lane == leader) {
      base = atomicAdd(&sm.open_cnt, (uint32_t)__popc(mo));
      atomicMin(&sm.open_min, fmin);
    }
    base = __shfl_sync(GPQ_FULL_MASK, base, leader);
    if (kind == 2u) {
      const uint32_t pos = base + __popc(mo & lt);
      if (pos < d.open_cap) d.open[(size_t)t * d.open_cap + pos] = child;
      else gpq_set_error(&Ip->err, GPQ_ERR_QUEUE_FULL);
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

template <bool WARP>
__device__ __forceinline__ uint32_t astar_worker_scan(uint32_t flag, uint32_t* scratch, uint32_t* total) {
  if (WARP) {
    const uint32_t bal = __ballot_sync(GPQ_FULL_MASK, flag);
    *total = (uint32_t)__popc(bal);
    return (uint32_t)__popc(bal & ((1u << (threadIdx.x & 31u)) - 1u));
  }
  return astar_block_scan(flag, scratch, total);
}

// Process tile t in round s (one worker).
template <bool WARP>
__device__ void astar_process_tile(const AstarDev& d, uint32_t t, uint32_t s, AstarTileSmem& sm,
                                   const AstarWorker<WARP>& wk) {
  const uint32_t par = s & 1u, npar = par ^ 1u;
  AstarTileDev* T = d.tiles + t;
  AstarInstDev* Ip = d.inst + T->inst;
  const AstarInstDev I = *Ip;  // static fields; ub/bound are read through Ip
  uint32_t* G = d.gcost + I.cell0;
  const uint32_t ts = d.ts, words = ts * ts / 32;
  AstarTileGeo tg;
  tg.ts = ts;
  tg.lts = d.lts;
  tg.x0 = T->tx * ts;
  tg.y0 = T->ty * ts;
  tg.tw = min(ts, I.g.width - tg.x0);
  tg.th = min(ts, I.g.height - tg.y0);
  if (wk.tid == 0) {
    sm.n[0] = 0;
    sm.n[1] = 0;
    sm.n[2] = 0;
    sm.ob_n = 0;
    sm.pops = 0;
    sm.open_cnt = T->open_cnt;
    sm.open_min = kAstarInf;
  }
  wk.sync();
  const uint32_t k_in = min(ldcg_u32(&T->in_cnt[par]), d.in_cap);
  const uint32_t bound = ldcg_u32(&Ip->bound);
  if (ldcg_u32(&Ip->done)) {
    if (wk.tid == 0) {
      T->in_cnt[par] = 0;
      T->queued[par] = 0;
      T->open_cnt = 0;
      T->open_min = kAstarInf;
    }
    wk.sync();
    return;
  }
  const uint32_t ub = ldcg_u32(&Ip->ub);
  if (wk.tid == 0) {
    sm.ub = ub;
    atomicAdd(&d.ctl->visits, 1ull);
  }
  // 0. the tile's g values and blocked bits into shared memory
  for (uint32_t j = wk.tid; j < words; j += wk.n) {
    sm.blk[j] = 0;
    sm.chg[j] = 0;
  }
  for (uint32_t l = wk.tid; l < ts * ts; l += wk.n) {
    const uint32_t lx = l % ts, ly = l / ts;
    sm.gt[l] = (lx < tg.tw && ly < tg.th) ? ldcg_u32(&G[(tg.y0 + ly) * I.g.width + tg.x0 + lx]) : kAstarInf;
  }
  wk.sync();
  {
    const uint32_t segw = ts < 32 ? ts : 32u, segs = ts / segw;
    for (uint32_t j = wk.tid; j < tg.th * segs; j += wk.n) {
      const uint32_t ly = j / segs, lx0 = (j % segs) * segw;
      if (lx0 >= tg.tw) continue;
      const uint64_t b0 = I.cell0 + (uint64_t)(tg.y0 + ly) * I.g.width + tg.x0 + lx0;
      uint32_t bits = __funnelshift_r(__ldg(&d.blk[b0 >> 5]), __ldg(&d.blk[(b0 >> 5) + 1]), (uint32_t)(b0 & 31u));
      const uint32_t nb = min(segw, tg.tw - lx0);
      if (nb < 32) bits &= (1u << nb) - 1u;
      const uint32_t l0 = ly * ts + lx0;
      atomicOr(&sm.blk[l0 >> 5], bits << (l0 & 31u));
    }
  }
  wk.sync();
  // 1. the open array, when the window reached it: expand-now items leave, the rest is
  //    compacted in place (a chunk is read completely before any of it is written)
  const uint32_t n_open = sm.open_cnt;
  if (n_open > 0 && ldcg_u32(&T->open_min) <= bound) {
    uint2* O = d.open + (size_t)t * d.open_cap;
    uint32_t kept = 0;
    for (uint32_t c0 = 0; c0 < n_open; c0 += wk.n) {
      const uint32_t i = c0 + wk.tid;
      uint2 it = make_uint2(0, kAstarInf);
      uint32_t keep = 0, f = kAstarInf;
      if (i < n_open) {
        it = O[i];
        const int x = (int)(it.x & 0xffffu), y = (int)(it.x >> 16);
        if (sm.gt[tg.local(x, y)] == it.y) {
          f = it.y + astar_hxy(I.g.conn, x, y, (int)I.gx, (int)I.gy);
          if (f <= ub) {
            if (f <= bound) astar_frontier_push(d, Ip, sm, sm.fa, 0, t, npar, it);
            else keep = 1;
          }
        }
      }
      uint32_t total;
      const uint32_t off = astar_worker_scan<WARP>(keep, sm.scan, &total);
      if (keep) {
        O[kept + off] = it;
        atomicMin(&sm.open_min, f);
      }
      kept += total;
    }
    if (wk.tid == 0) sm.open_cnt = kept;
    wk.sync();
  } else if (wk.tid == 0) {
    sm.open_min = ldcg_u32(&T->open_min);
  }
  wk.sync();
  // 2. the inbox (senders lowered the global g of these cells before sending)
  {
    const uint2* B = d.inbox + ((size_t)par * d.n_tiles + t) * d.in_cap;
    for (uint32_t i = wk.tid; i < k_in; i += wk.n) {
      const uint2 it = B[i];
      const int x = (int)(it.x & 0xffffu), y = (int)(it.x >> 16);
      if (sm.gt[tg.local(x, y)] != it.y) continue;
      const uint32_t f = it.y + astar_hxy(I.g.conn, x, y, (int)I.gx, (int)I.gy);
      if (f > ub) continue;
      if (f <= bound) astar_frontier_push(d, Ip, sm, sm.fa, 0, t, npar, it);
      else astar_open_push(d, Ip, sm, t, it, f);
    }
  }
  wk.sync();
  if (wk.tid == 0) {
    T->in_cnt[par] = 0;
    T->queued[par] = 0;
  }
  // 3. level-by-level expansion of the frontier inside the tile; level i reads buffer
  //    i % 2 with fill n[i % 3], fills the other buffer and n[(i + 1) % 3], and clears
  //    n[(i + 2) % 3] (read at level i - 1, filled at level i + 1): one barrier a level
  uint32_t pops = 0;
  for (uint32_t lv = 0;; ++lv) {
    const uint32_t c3 = lv % 3u;
    const uint32_t n = min(sm.n[c3], d.frontier_cap);
    if (n == 0) break;
    uint2* src = (lv & 1u) ? sm.fb : sm.fa;
    uint2* dst = (lv & 1u) ? sm.fa : sm.fb;
    if (wk.tid == 0) sm.n[(c3 + 2u) % 3u] = 0;
    const uint32_t ipw = I.g.conn == 4 ? 8u : 4u;  // items per warp pass
    for (uint32_t ib = (wk.tid >> 5) * ipw; ib < n; ib += (wk.n >> 5) * ipw)
      astar_expand_warp(d, Ip, I, sm, tg, src, ib, n, dst, (c3 + 1u) % 3u, t, npar, bound, &pops);
    wk.sync();
  }
  // 4. send the moves into other tiles
  {
    const uint32_t nob = min(sm.ob_n, astar_outbox_cap(ts));
    for (uint32_t i = wk.tid; i < nob; i += wk.n) astar_send(d, Ip, I, sm.ob[i], npar);
  }
  // 5. merge the tile's g values back
  for (uint32_t l = wk.tid; l < ts * ts; l += wk.n) {
    if ((sm.chg[l >> 5] >> (l & 31u)) & 1u) {
      const uint32_t lx = l % ts, ly = l / ts;
      atomicMin(&G[(tg.y0 + ly) * I.g.width + tg.x0 + lx], sm.gt[l]);
    }
  }
  pops = warp_sum_u32(pops);
  if ((threadIdx.x & 31u) == 0 && pops) atomicAdd(&sm.pops, (unsigned long long)pops);
  wk.sync();
  if (wk.tid == 0) {
    const uint32_t oc = min(sm.open_cnt, d.open_cap);
    T->open_cnt = oc;
    T->open_min = oc ? sm.open_min : kAstarInf;
    if (sm.pops) atomicAdd(&Ip->pops, sm.pops);
  }
  wk.sync();
}

// Phase W for one instance (one warp): a drained window moves on, or the instance ends.
static __device__ void astar_window_step(const AstarDev& d, uint32_t i, uint32_t npar) {
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

// The persistent search loop over all instances.  Dynamic shared memory: one slice of
// astar_worker_smem_bytes(ts, frontier_cap) per worker (per warp when WARP).
static constexpr uint32_t kAstarMaxWorkers = 8;  // 256 threads / 32

__host__ __device__ inline size_t astar_worker_smem_bytes(uint32_t ts, uint32_t frontier_cap) {
  return (astar_smem_bytes(ts, frontier_cap) + 15u) & ~(size_t)15u;
}

// Rounds s0, s0 + 1, ... until every instance is done, or until `step_rounds` rounds ran
// (0 = no limit): a resident session resumes at the next round in its next launch.
template <bool WARP>
static __global__ void __launch_bounds__(256) astar_persistent_kernel(AstarDev d, uint32_t s0, uint32_t step_rounds) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ AstarTileSmem sms[kAstarMaxWorkers];
  __shared__ uint32_t s_t;
  const AstarWorker<WARP> wk;
  AstarTileSmem& sm = sms[wk.id];
  if (wk.tid == 0) {
    unsigned char* base = smem_raw + (size_t)wk.id * astar_worker_smem_bytes(d.ts, d.frontier_cap);
    sm.fa = reinterpret_cast<uint2*>(base);
    sm.fb = sm.fa + d.frontier_cap;
    sm.ob = sm.fb + d.frontier_cap;
    sm.gt = reinterpret_cast<uint32_t*>(sm.ob + astar_outbox_cap(d.ts));
    sm.blk = sm.gt + d.ts * d.ts;
    sm.chg = sm.blk + d.ts * d.ts / 32;
  }
  __syncthreads();
  const unsigned long long nb = gridDim.x;
  unsigned long long bar_target = 0;
  const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
  const uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (uint32_t s = s0;; ++s) {
    const uint32_t par = s & 1u, npar = par ^ 1u;
    const uint32_t n = ldcg_u32(&d.ctl->al_cnt[par]);
    for (;;) {
      uint32_t j;
      if (WARP) {
        j = 0;
        if (wk.tid == 0) j = atomicAdd(&d.ctl->work[par], 1u);
        j = __shfl_sync(GPQ_FULL_MASK, j, 0);
      } else {
        if (threadIdx.x == 0) s_t = atomicAdd(&d.ctl->work[par], 1u);
        __syncthreads();
        j = s_t;
        __syncthreads();
      }
      if (j >= n) break;
      astar_process_tile<WARP>(d, d.al[(size_t)par * d.n_tiles + j], s, sm, wk);
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
    if (step_rounds && s + 1 - s0 >= step_rounds) break;
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

// Initial state of instances list[0, n) (all instances when list == nullptr): g = inf
// (done by a memset), g[start] = 0, the start item in the start tile's inbox of round
// parity par, the start tile on that round's active list.
static __global__ void astar_init_kernel(AstarDev d, const uint32_t* list, uint32_t n, uint32_t par) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = list ? list[j] : j;
  AstarInstDev& I = d.inst[i];
  d.gcost[I.cell0 + I.g.start] = 0;
  const uint32_t t = astar_tile_of(d, I, I.g.start);
  d.tiles[t].in_cnt[par] = 1;
  d.inbox[((size_t)par * d.n_tiles + t) * d.in_cap] =
      make_uint2(astar_pack((int)(I.g.start % I.g.width), (int)(I.g.start / I.g.width)), 0);
  astar_activate(d, t, par, false);
}

// Tile records of instances list[0, n) (all when list == nullptr): one block per instance.
static __global__ void astar_tiles_init_kernel(AstarDev d, const uint32_t* list, uint32_t n) {
  for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
    const uint32_t inst = list ? list[j] : j;
    const AstarInstDev& I = d.inst[inst];
    const uint32_t nt = I.tiles_x * I.tiles_y;
    for (uint32_t k = threadIdx.x; k < nt; k += blockDim.x) {
      AstarTileDev T{};
      T.inst = inst;
      T.tx = k % I.tiles_x;
      T.ty = k / I.tiles_x;
      T.open_min = kAstarInf;
      d.tiles[I.tile0 + k] = T;
    }
  }
}

// Blocked bits of instances list[0, n): blockIdx.y = position in the list.  Instance
// cell ranges start on 32-cell boundaries.
static __global__ void astar_bitmap_list_kernel(const AstarInstDev* inst, const uint32_t* list, uint32_t* blk) {
  const AstarInstDev& I = inst[list[blockIdx.y]];
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  const uint64_t words = (cells + 31) / 32, w0 = I.cell0 / 32;
  for (uint64_t wi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; wi < words; wi += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t w = 0;
    for (uint32_t b = 0; b < 32; ++b) {
      const uint64_t c = wi * 32 + b;
      if (c < cells && gpq_astar_blocked(&I.g, (uint32_t)c)) w |= 1u << b;
    }
    blk[w0 + wi] = w;
  }
}

// Slots that are in use (on[slot] != 0) and whose search has ended, appended to out.
static __global__ void astar_done_list_kernel(const AstarInstDev* inst, const uint8_t* on, uint32_t n_slots,
                                              uint32_t* out, uint32_t* out_n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_slots; i += gridDim.x * blockDim.x)
    if (on[i] && inst[i].done) out[atomicAdd(out_n, 1u)] = i;
}

// Per-instance expanded set (g + h <= C*, or every reached cell when the goal is not
// reachable): count and hash.  Block per (instance, chunk): blockIdx.y = instance.
static __global__ void astar_finalize_kernel(AstarDev d, const uint32_t* list, unsigned long long* out /* [n][2] */) {
  const uint32_t j = blockIdx.y;
  const uint32_t i = list ? list[j] : j;
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
    atomicAdd(&out[2 * j], cnt);
    atomicAdd(&out[2 * j + 1], hs);
  }
}

// Canonical path of each instance, one warp per instance: from the goal, step to the
// smallest-id neighbour p with g[p] + c(p, cell) == g[cell] and g[p] + h(p) <= C*.
// out[3 * i] = length, out[3 * i + 1] = hash, out[3 * i + 2] = 1 when the walk failed.
// When path != nullptr the cells of instance `want` are written (goal first, <= cap).
static __global__ void astar_path_kernel(AstarDev d, const uint32_t* list, uint32_t n, unsigned long long* out,
                                         uint32_t want, uint32_t* path, uint32_t cap) {
  const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (j >= n) return;
  const uint32_t i = list ? list[j] : j;
  const AstarInstDev& I = d.inst[i];
  const uint32_t cs = I.ub;
  if (cs == kAstarInf) {
    if (lane == 0) { out[3 * j] = 0; out[3 * j + 1] = 0; out[3 * j + 2] = 0; }
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
    out[3 * j] = len;
    out[3 * j + 1] = hs;
    out[3 * j + 2] = fail;
  }
}
