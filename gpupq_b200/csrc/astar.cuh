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
  uint8_t* pred;    // [cells + kAstarPredSlack] move to the canonical predecessor (astar_pred_kernel)
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

// Bytes after the last cell of the predecessor array: path windows read whole words.
static constexpr uint64_t kAstarPredSlack = 256;

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

// Move tested l-th (l = 0..7) when looking for a predecessor, numbered as in
// gpq_astar_dx/dy: the neighbours NW, N, NE, W, E, SW, S, SE, which is increasing cell id on
// every grid where two of them exist together.
__device__ __forceinline__ int astar_pred_order(int l) {
  return l == 0 ? 7 : l == 1 ? 3 : l == 2 ? 6 : l == 3 ? 1 : l == 4 ? 0 : l == 5 ? 5 : l == 6 ? 2 : 4;
}

static constexpr uint8_t kAstarNoPred = 0xFF;

// Instances of at least this many cells get predecessor moves from astar_pred_kernel and
// walk their path over them (long walks, few such instances at a time).
static constexpr uint64_t kAstarPredBytesCells = 1ull << 20;

__device__ __forceinline__ bool astar_pred_bytes(const AstarInstDev& I) {
  return (uint64_t)I.g.width * I.g.height >= kAstarPredBytesCells;
}

// The canonical predecessor of cell c (g = g[c], on an optimal path when g + h(c) <= C*):
// the neighbour p with the smallest id that is free (both orthogonal cells free for a
// diagonal), g[p] + c(p, c) == g and g[p] + h(p) <= C*.  Encoded as (dy + 1) << 2 | (dx + 1)
// for the move from c to p; kAstarNoPred when there is none.  Lanes without a cell that
// needs it pass cand = false; the blocked bits and g values of all eight neighbours are
// loaded in one batch and the choice is made in registers, without divergent branches.
__device__ __forceinline__ uint8_t astar_pred_move(const AstarDev& d, const AstarInstDev& I, const uint32_t* G,
                                                   bool cand, uint32_t c, uint32_t g, uint32_t cs) {
  const uint32_t w = I.g.width, h = I.g.height, conn = I.g.conn;
  const int x = (int)(c % w), y = (int)(c / w);
  bool fr[8];
  uint32_t gp[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    const int k = astar_pred_order(l);
    const int nx = x + gpq_astar_dx(k), ny = y + gpq_astar_dy(k);
    const bool in = cand && (conn == 8u || k < 4) && nx >= 0 && ny >= 0 && nx < (int)w && ny < (int)h;
    const uint32_t p = (uint32_t)ny * w + (uint32_t)nx;
    fr[l] = in && !astar_blocked(d, I, p);
    gp[l] = in ? __ldg(&G[p]) : kAstarInf;
  }
  // diagonals (lanes 0 NW, 2 NE, 5 SW, 7 SE) also need their two orthogonal cells free
  const bool diag = conn == 8u;
  const bool ok[8] = {diag && fr[0] && fr[3] && fr[1], fr[1], diag && fr[2] && fr[1] && fr[4], fr[3],
                      fr[4], diag && fr[5] && fr[3] && fr[6], fr[6], diag && fr[7] && fr[4] && fr[6]};
  uint8_t best = kAstarNoPred;
#pragma unroll
  for (int l = 7; l >= 0; --l) {  // the smallest valid l is assigned last
    const int k = astar_pred_order(l);
    const int dx = gpq_astar_dx(k), dy = gpq_astar_dy(k);
    if (ok[l] && gp[l] != kAstarInf && (uint64_t)gp[l] + gpq_astar_cost(conn, k) == g &&
        (uint64_t)gp[l] + astar_hxy(conn, x + dx, y + dy, (int)I.gx, (int)I.gy) <= cs)
      best = (uint8_t)((dy + 1) << 2 | (dx + 1));
  }
  return best;
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

// Predecessor move of every expanded cell (g + h <= C*) of the instances in list[0, n)
// that reached their goal and have at least kAstarPredBytesCells cells; the others
// return at once.  Block per (instance, chunk): blockIdx.y = instance.  Whole warps step
// together (blockDim is a multiple of 32), so a warp without expanded cells skips the
// neighbour loads.
static __global__ void astar_pred_kernel(AstarDev d, const uint32_t* list) {
  const uint32_t i = list ? list[blockIdx.y] : blockIdx.y;
  const AstarInstDev& I = d.inst[i];
  const uint32_t cs = I.ub;
  if (cs == kAstarInf || !astar_pred_bytes(I)) return;
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  const uint32_t* G = d.gcost + I.cell0;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x - lane); base < cells;
       base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = base + lane;
    const uint32_t g = c < cells ? G[c] : kAstarInf;
    const bool exp = g != kAstarInf && (uint64_t)g + gpq_astar_h(I.g.conn, (uint32_t)c, I.g.goal, I.g.width) <= cs;
    if (__any_sync(GPQ_FULL_MASK, exp)) {
      const uint8_t mv = astar_pred_move(d, I, G, exp, (uint32_t)c, g, cs);
      if (exp) d.pred[I.cell0 + c] = mv;
    }
  }
}

// ---- canonical path ----
// From the goal, step to the neighbour p with g[p] + c(p, cell) == g[cell] and
// g[p] + h(p) <= C* that has the smallest id, until the start.  The walk is serial, so
// one CTA per instance keeps everything else off its critical path: all warps stage a
// window of the grid in shared memory, one thread (or warp) walks inside it, and all
// warps hash and store the cells it recorded.  Windows are placed around the current cell
// with most of their room on the side of the start, where the path is heading.  Two forms:
//  - instances of at least kAstarPredBytesCells cells (long walks, few of them at a time)
//    use the predecessor moves that astar_pred_kernel wrote for every expanded cell:
//    128 x 128 windows of move bytes, one shared-memory byte per step;
//  - smaller instances (many at a time, where a pass over every expanded cell would
//    cost more than it saves) stage 64 x 64 windows of g values and blocked
//    bits, and warp 0 finds each step: lane l tests the l-th neighbour in increasing
//    cell id, and the first lane whose test passes (one ballot) is the step.
static constexpr uint32_t kPathThreads = 512;
static constexpr uint32_t kPathWalkCap = 2048;
static constexpr int kPathWinB = 128;                  // move-byte window side
static constexpr int kPathRowWords = kPathWinB / 4 + 1;  // aligned words that cover 128 bytes
static constexpr int kPathWinC = 64;                   // g-value window side
static constexpr int kPathHalo = kPathWinC + 2;         // plus the cells its moves reach
static constexpr int kPathStageBytes = kPathHalo * kPathHalo * 5 > kPathWinB * kPathRowWords * 4
                                           ? kPathHalo * kPathHalo * 5
                                           : kPathWinB * kPathRowWords * 4;

// First column (row) of a window of side win around coordinate c on an axis of n cells,
// with the start at coordinate s: 7/8 of the room towards the start.
__device__ __forceinline__ int astar_path_origin(int c, int s, int n, int win) {
  if (n <= win) return 0;
  const int o = s < c ? c - (win - win / 8) : s > c ? c - (win / 8 - 1) : c - win / 2;
  return min(max(o, 0), n - win);
}

struct AstarPathSmem {
  uint32_t* walk;  // [kPathWalkCap] cells recorded in the current window
  uint32_t* cur;   // next cell to record
  uint32_t* nwalk;
  uint32_t* done;  // 0 walking, 1 reached the start, 2 no predecessor
};

// One window of the move-byte form: stage, then thread 0 walks.  Ends with a barrier.
__device__ __forceinline__ void astar_path_window_bytes(const AstarDev& d, const AstarInstDev& I, uint32_t* s_pw,
                                                        const AstarPathSmem& sm) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const int w = (int)I.g.width, h = (int)I.g.height;
  const uint32_t start = I.g.start, cur = *sm.cur;
  const int cx = (int)(cur % (uint32_t)w), cy = (int)(cur / (uint32_t)w);
  const int tx0 = astar_path_origin(cx, (int)(start % (uint32_t)w), w, kPathWinB);
  const int ty0 = astar_path_origin(cy, (int)(start / (uint32_t)w), h, kPathWinB);
  const uint32_t* PW = reinterpret_cast<const uint32_t*>(d.pred);
  const int rows = min(kPathWinB, h - ty0);
  for (int r = (int)warp; r < rows; r += (int)(kPathThreads / 32)) {  // row r: its bytes from (tx0, ty0 + r) on
    const uint64_t w0 = (I.cell0 + (uint64_t)(ty0 + r) * (uint64_t)w + (uint64_t)tx0) >> 2;
    const uint32_t a = __ldg(&PW[w0 + lane]);
    const uint32_t b = lane == 0 ? __ldg(&PW[w0 + 32]) : 0u;
    s_pw[r * kPathRowWords + (int)lane] = a;
    if (lane == 0) s_pw[r * kPathRowWords + 32] = b;
  }
  __syncthreads();
  if (tid == 0) {
    const uint8_t* s_pb = reinterpret_cast<const uint8_t*>(s_pw);
    uint32_t c = cur, q = 0, done = 0;
    uint32_t pc = (uint32_t)(I.cell0 + cur);  // its low two bits give each row's offset in its words
    int lx = cx - tx0, ly = cy - ty0;
    while (lx >= 0 && ly >= 0 && lx < kPathWinB && ly < kPathWinB && q < kPathWalkCap) {
      sm.walk[q++] = c;
      if (c == start) { done = 1; break; }
      const uint32_t mv = s_pb[ly * (kPathRowWords * 4) + lx + (int)((pc - (uint32_t)lx) & 3u)];
      if (mv == kAstarNoPred) { done = 2; break; }
      const int dx = (int)(mv & 3u) - 1, dy = (int)(mv >> 2) - 1;
      lx += dx;
      ly += dy;
      const uint32_t step = (uint32_t)(dy * w + dx);  // modulo 2^32: a step back is a wrapped add
      c += step;
      pc += step;
    }
    *sm.cur = c;
    *sm.nwalk = q;
    *sm.done = done;
  }
  __syncthreads();
}

// One window of the g-value form: stage g values and blocked bits (one grid row per warp
// and pass), then warp 0 walks.  Ends with a barrier.
__device__ __forceinline__ void astar_path_window_cells(const AstarDev& d, const AstarInstDev& I, uint32_t* s_g,
                                                        uint8_t* s_b, const AstarPathSmem& sm) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t* G = d.gcost + I.cell0;
  const int w = (int)I.g.width, h = (int)I.g.height;
  const uint32_t conn = I.g.conn, start = I.g.start, cs = I.ub, cur = *sm.cur;
  const int cx = (int)(cur % (uint32_t)w), cy = (int)(cur / (uint32_t)w);
  const int tx0 = astar_path_origin(cx, (int)(start % (uint32_t)w), w, kPathWinC);
  const int ty0 = astar_path_origin(cy, (int)(start / (uint32_t)w), h, kPathWinC);
  // the window and its halo, clipped to the grid (moves never leave the grid)
  const int sx0 = max(tx0 - 1, 0), sx1 = min(tx0 + kPathWinC, w - 1);
  const int sy0 = max(ty0 - 1, 0), sy1 = min(ty0 + kPathWinC, h - 1);
  for (int y = sy0 + (int)warp; y <= sy1; y += (int)(kPathThreads / 32)) {
    const uint32_t row = (uint32_t)y * (uint32_t)w;
    const int hrow = (y - ty0 + 1) * kPathHalo - tx0 + 1;  // + x = halo index of (x, y)
    uint32_t gv[3];
    bool bv[3];
#pragma unroll
    for (int u = 0; u < 3; ++u) {  // 3 x 32 >= kPathHalo columns
      const int x = sx0 + (int)lane + 32 * u;
      if (x <= sx1) {
        gv[u] = __ldg(&G[row + (uint32_t)x]);
        bv[u] = astar_blocked(d, I, row + (uint32_t)x);
      }
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int x = sx0 + (int)lane + 32 * u;
      if (x <= sx1) {
        s_g[hrow + x] = gv[u];
        s_b[hrow + x] = bv[u] ? 1 : 0;
      }
    }
  }
  __syncthreads();
  if (warp == 0) {
    // this lane's move, offset and cost (lanes 8..31 and the diagonals of 4-conn grids idle)
    const int lk = astar_pred_order((int)(lane & 7u));
    const bool lane_on = lane < 8u && (conn == 8u || lk < 4);
    const int ldx = gpq_astar_dx(lk), ldy = gpq_astar_dy(lk);
    const int loff = ldy * kPathHalo + ldx;
    const uint32_t lcost = gpq_astar_cost(conn, lk);
    uint32_t c = cur, q = 0, done = 0;
    int x = cx, y = cy, lx = cx - tx0, ly = cy - ty0;
    while (lx >= 0 && ly >= 0 && lx < kPathWinC && ly < kPathWinC && q < kPathWalkCap) {
      if (lane == 0) sm.walk[q] = c;
      ++q;
      if (c == start) { done = 1; break; }
      const int hi = (ly + 1) * kPathHalo + (lx + 1);
      bool ok = false;
      if (lane_on) {
        const int nx = x + ldx, ny = y + ldy;
        if (nx >= 0 && ny >= 0 && nx < w && ny < h && !s_b[hi + loff] &&
            (ldx == 0 || ldy == 0 || (!s_b[hi + ldx] && !s_b[hi + ldy * kPathHalo]))) {
          const uint32_t gp = s_g[hi + loff], gc = s_g[hi];
          ok = gp != kAstarInf && (uint64_t)gp + lcost == gc &&
               (uint64_t)gp + astar_hxy(conn, nx, ny, (int)I.gx, (int)I.gy) <= cs;
        }
      }
      const uint32_t m = __ballot_sync(GPQ_FULL_MASK, ok);
      if (m == 0u) { done = 2; break; }
      const int k = astar_pred_order(__ffs(m) - 1);
      const int dx = gpq_astar_dx(k), dy = gpq_astar_dy(k);
      x += dx;
      y += dy;
      lx += dx;
      ly += dy;
      c += (uint32_t)(dy * w + dx);  // modulo 2^32: a step back is a wrapped add
    }
    if (lane == 0) {
      *sm.cur = c;
      *sm.nwalk = q;
      *sm.done = done;
    }
  }
  __syncthreads();
}

// Canonical path of the instances in list[0, n) (list == NULL: instances 0..n-1), one CTA
// per instance.  out[3j..3j+2] = path length, path hash, failure flag; the path of
// instance `want` is written to path[0, cap).
static __global__ void __launch_bounds__(kPathThreads) astar_path_kernel(AstarDev d, const uint32_t* list, uint32_t n,
                                                                         unsigned long long* out, uint32_t want,
                                                                         uint32_t* path, uint32_t cap) {
  __shared__ __align__(16) uint8_t s_stage[kPathStageBytes];
  __shared__ uint32_t s_walk[kPathWalkCap];
  __shared__ uint32_t s_cur, s_len, s_done, s_nwalk;
  __shared__ unsigned long long s_hs;
  const uint32_t j = blockIdx.x;
  if (j >= n) return;
  const uint32_t i = list ? list[j] : j;
  const AstarInstDev& I = d.inst[i];
  const uint32_t tid = threadIdx.x;
  if (I.ub == kAstarInf) {
    if (tid == 0) { out[3 * j] = 0; out[3 * j + 1] = 0; out[3 * j + 2] = 0; }
    return;
  }
  const bool bytes = astar_pred_bytes(I);
  const AstarPathSmem sm{s_walk, &s_cur, &s_nwalk, &s_done};
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  if (tid == 0) {
    s_cur = I.g.goal;
    s_len = 0;
    s_done = 0;
    s_hs = 0;
  }
  __syncthreads();
  // every window records at least one cell: at most cells + 1 windows
  for (uint64_t it = 0; it <= cells && s_done == 0u; ++it) {
    if (bytes)
      astar_path_window_bytes(d, I, reinterpret_cast<uint32_t*>(s_stage), sm);
    else
      astar_path_window_cells(d, I, reinterpret_cast<uint32_t*>(s_stage), s_stage + kPathHalo * kPathHalo * 4, sm);
    const uint32_t nw = s_nwalk, len0 = s_len;
    unsigned long long part = 0;
    for (uint32_t q = tid; q < nw; q += kPathThreads) {
      const uint32_t c = s_walk[q];
      part += gpq_astar_path_hash(len0 + q, c);
      if (path && i == want && len0 + q < cap) path[len0 + q] = c;
    }
    part = warp_sum_u64(part);
    if ((tid & 31u) == 0 && part) atomicAdd(&s_hs, part);
    __syncthreads();
    if (tid == 0) s_len = len0 + nw;  // read again only after the next window's barriers
  }
  __syncthreads();
  if (tid == 0) {
    out[3 * j] = s_len;
    out[3 * j + 1] = s_hs;
    out[3 * j + 2] = s_done == 1u ? 0u : 1u;
  }
}
