/*
 * gpq/astar.h -- A* grid-search semantics shared by the host and device code of gpupq_b200.
 *
 * The reference's A* (src/a_star.cu:269-593) runs one best-first search per agent
 * with a half-precision f, eight parallel pops per round and a stop at the first sight
 * of the goal, so its expansion count and its path depend on the schedule.  Here the
 * search is pinned so that cost, path and expansion count are functions of the grid:
 *
 *   grid      W x H cells, cell id = y * W + x; a cell is blocked iff the top 24 bits of
 *             its draw are below `block_thr` (= density * 2^24); start and goal are free;
 *   moves     4-connected with cost 1, or 8-connected with costs 10 (straight) and 14
 *             (diagonal), a diagonal move needing both orthogonal cells free;
 *   h         Manhattan (4-connected) or octile 10*max + 4*min (8-connected); both are
 *             consistent, so every cell whose final f = g + h is at most the optimal cost
 *             C* carries its exact distance g*;
 *   expanded  the cells with g + h <= C* (all reachable cells when the goal is not);
 *   path      from the goal back to the start, each step to the neighbour p with
 *             g[p] + c(p, cell) == g[cell] and g[p] + h(p) <= C* that has the smallest id.
 *
 * Open-list items are gpq_items: ts = (float)f (exact, f < 2^24), lp = shard, id = cell,
 * aux = g, so the queues order them by (f, shard, cell).
 */
#ifndef GPQ_ASTAR_H
#define GPQ_ASTAR_H

#include "gpq/model.h"

#define GPQ_ASTAR_INF 0xFFFFFFFFu
#define GPQ_ASTAR_CELL_DOMAIN 0x41535452u  /* ts-bits key of the obstacle draws */
#define GPQ_ASTAR_QUERY_DOMAIN 0x51525931u /* id key of the query-parameter draws */

typedef struct gpq_astar_grid {
  uint64_t seed;      /* obstacle seed */
  uint32_t width, height;
  uint32_t block_thr; /* blocked iff (draw >> 40) < block_thr */
  uint32_t conn;      /* 4 or 8 */
  uint32_t start, goal;
} gpq_astar_grid;

GPQ_HD int gpq_astar_raw_blocked(uint64_t seed, uint32_t thr, uint32_t cell) {
  return (uint32_t)(gpq_draw(seed, cell, GPQ_ASTAR_CELL_DOMAIN, 0) >> 40) < thr;
}

GPQ_HD int gpq_astar_blocked(const gpq_astar_grid* g, uint32_t cell) {
  return cell != g->start && cell != g->goal && gpq_astar_raw_blocked(g->seed, g->block_thr, cell);
}

GPQ_HD uint32_t gpq_astar_h(uint32_t conn, uint32_t cell, uint32_t goal, uint32_t w) {
  uint32_t x = cell % w, y = cell / w, gx = goal % w, gy = goal / w;
  uint32_t dx = x > gx ? x - gx : gx - x, dy = y > gy ? y - gy : gy - y;
  if (conn == 4) return dx + dy;
  uint32_t mx = dx > dy ? dx : dy, mn = dx > dy ? dy : dx;
  return 10u * mx + 4u * mn;
}

/* Move k (0..3 straight E, W, S, N; 4..7 diagonal SE, SW, NE, NW) as (dx, dy). */
GPQ_HD int gpq_astar_dx(int k) { return (k == 0 || k == 4 || k == 6) ? 1 : (k == 1 || k == 5 || k == 7) ? -1 : 0; }
GPQ_HD int gpq_astar_dy(int k) { return (k == 2 || k == 4 || k == 5) ? 1 : (k == 3 || k == 6 || k == 7) ? -1 : 0; }
GPQ_HD uint32_t gpq_astar_cost(uint32_t conn, int k) { return conn == 4 ? 1u : (k < 4 ? 10u : 14u); }

/* Neighbour of `cell` by move k, or GPQ_ASTAR_INF when it is off the grid, blocked, or a
 * diagonal whose orthogonal cells are not both free.  `blocked(c)` is evaluated by the
 * caller's predicate object through the macro argument. */
#define GPQ_ASTAR_NEIGHBOUR(OUT, GRID, CELL, K, BLOCKED)                                    \
  do {                                                                                      \
    const uint32_t _w = (GRID).width, _h = (GRID).height;                                  \
    const int _x = (int)((CELL) % _w), _y = (int)((CELL) / _w);                             \
    const int _dx = gpq_astar_dx(K), _dy = gpq_astar_dy(K);                                 \
    const int _nx = _x + _dx, _ny = _y + _dy;                                               \
    (OUT) = GPQ_ASTAR_INF;                                                                  \
    if (_nx >= 0 && _ny >= 0 && _nx < (int)_w && _ny < (int)_h) {                           \
      const uint32_t _n = (uint32_t)_ny * _w + (uint32_t)_nx;                               \
      int _ok = !BLOCKED(_n);                                                               \
      if (_ok && (K) >= 4)                                                                  \
        _ok = !BLOCKED((uint32_t)_y * _w + (uint32_t)_nx) && !BLOCKED((uint32_t)_ny * _w + (uint32_t)_x); \
      if (_ok) (OUT) = _n;                                                                  \
    }                                                                                       \
  } while (0)

/* Order-insensitive hash of one expanded cell and its distance. */
GPQ_HD uint64_t gpq_astar_cell_hash(uint32_t cell, uint32_t g) {
  return gpq_mix64(((uint64_t)cell << 32) | (uint64_t)g);
}

/* Hash of the path cell at position i counted from the goal (i = 0). */
GPQ_HD uint64_t gpq_astar_path_hash(uint32_t i, uint32_t cell) {
  return gpq_mix64((((uint64_t)i << 32) | (uint64_t)cell) + GPQ_GOLDEN64);
}

#endif /* GPQ_ASTAR_H */
