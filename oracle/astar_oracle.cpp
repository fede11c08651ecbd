// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the A* grid-search hot path.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this file's
// library; the product (gpupq_b200) never includes, links or calls it.
//
// A sequential best-first search with one std::priority_queue, restating what the
// reference's a_star kernel computes per agent (src/a_star.cu:269-593: pop the open
// list's minimum, close it, relax the neighbours, push the improved ones; heuristic
// src/a_star.cu:124-135), under the pinned semantics that make the result a function of
// the grid alone: integer g, 4-connected unit or 8-connected 10/14 moves (diagonals need
// both orthogonal cells free), Manhattan or octile heuristic, every cell with
// f <= C* expanded, canonical path (smallest-id predecessor on an optimal path).
// The grid, heuristic and hashes are restated independently of the product's
// include/gpq/astar.h so that the two cross-check each other.
//
// The reference has no A* test and no golden vector (parity unpinned by the reference);
// the oracle checks itself: the number of closed cells must equal the number of cells
// with g + h <= C*, the defining property of the pinned expansion set.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <queue>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t kInf = 0xFFFFFFFFu;
constexpr uint32_t kCellDomain = 0x41535452u;
constexpr uint32_t kQueryDomain = 0x51525931u;
constexpr uint64_t kPhi = 0x9E3779B97F4A7C15ULL;

inline uint64_t mix(uint64_t z) {  // SplitMix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
inline uint64_t rnd(uint64_t seed, uint32_t id, uint32_t tsb, uint32_t k) {
  return mix(mix(seed ^ ((uint64_t)id * kPhi)) ^ (((uint64_t)tsb << 8) | (k & 0xffu)));
}
inline uint32_t below(uint64_t r, uint32_t n) { return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32); }

struct Grid {
  uint64_t seed;
  uint32_t width, height, block_thr, conn, start, goal;
};

struct Result {
  uint32_t cost, path_len;
  uint64_t expanded, gsum, path_hash, pops;
  double seconds;
};

inline bool raw_blocked(uint64_t seed, uint32_t thr, uint32_t c) {
  return (uint32_t)(rnd(seed, c, kCellDomain, 0) >> 40) < thr;
}

struct Search {
  const Grid& G;
  std::vector<uint8_t> blk;
  std::vector<uint32_t> g;
  explicit Search(const Grid& grid) : G(grid) {
    const uint64_t n = (uint64_t)G.width * G.height;
    blk.resize(n);
    for (uint64_t c = 0; c < n; ++c)
      blk[c] = (c != G.start && c != G.goal && raw_blocked(G.seed, G.block_thr, (uint32_t)c)) ? 1 : 0;
    g.assign(n, kInf);
  }
  uint32_t h(uint32_t c) const {
    const int64_t x = c % G.width, y = c / G.width, gx = G.goal % G.width, gy = G.goal / G.width;
    const uint32_t dx = (uint32_t)std::llabs(x - gx), dy = (uint32_t)std::llabs(y - gy);
    if (G.conn == 4) return dx + dy;
    return 10 * std::max(dx, dy) + 4 * std::min(dx, dy);
  }
  // Calls f(neighbour, cost) for every legal move out of c.
  template <class F>
  void moves(uint32_t c, F&& f) const {
    static const int DX[8] = {1, -1, 0, 0, 1, -1, 1, -1};
    static const int DY[8] = {0, 0, 1, -1, 1, 1, -1, -1};
    const int x = (int)(c % G.width), y = (int)(c / G.width);
    const int nk = G.conn == 4 ? 4 : 8;
    for (int k = 0; k < nk; ++k) {
      const int nx = x + DX[k], ny = y + DY[k];
      if (nx < 0 || ny < 0 || nx >= (int)G.width || ny >= (int)G.height) continue;
      const uint32_t n = (uint32_t)ny * G.width + (uint32_t)nx;
      if (blk[n]) continue;
      if (k >= 4 && (blk[(uint32_t)y * G.width + (uint32_t)nx] || blk[(uint32_t)ny * G.width + (uint32_t)x])) continue;
      f(n, G.conn == 4 ? 1u : (k < 4 ? 10u : 14u));
    }
  }

  // Returns 0, or -1 when the self-check fails.
  int run(Result* r, uint32_t* path_out, uint32_t path_cap) {
    const uint64_t n = g.size();
    std::vector<uint8_t> closed(n, 0);
    using Key = uint64_t;  // f << 32 | cell
    std::priority_queue<Key, std::vector<Key>, std::greater<Key>> open;
    uint32_t ub = kInf;
    g[G.start] = 0;
    open.push(((uint64_t)h(G.start) << 32) | G.start);
    if (G.start == G.goal) ub = 0;
    uint64_t pops = 0;
    while (!open.empty()) {
      const Key k = open.top();
      const uint32_t f = (uint32_t)(k >> 32), c = (uint32_t)k;
      if (ub != kInf && f > ub) break;
      open.pop();
      if (closed[c]) continue;
      closed[c] = 1;
      ++pops;
      const uint32_t gc = g[c];
      moves(c, [&](uint32_t nb, uint32_t cost) {
        if (closed[nb]) return;
        const uint32_t ng = gc + cost;
        if (ng < g[nb]) {
          g[nb] = ng;
          open.push(((uint64_t)(ng + h(nb)) << 32) | nb);
          if (nb == G.goal) ub = std::min(ub, ng);
        }
      });
    }
    const uint32_t cs = g[G.goal];
    uint64_t expanded = 0, gsum = 0;
    for (uint64_t c = 0; c < n; ++c) {
      if (g[c] == kInf) continue;
      if (cs != kInf && (uint64_t)g[c] + h((uint32_t)c) > cs) continue;
      ++expanded;
      gsum += mix(((uint64_t)c << 32) | g[c]);
    }
    r->cost = cs;
    r->expanded = expanded;
    r->gsum = gsum;
    r->pops = pops;
    r->path_len = 0;
    r->path_hash = 0;
    if (cs != kInf) {
      uint32_t cur = G.goal, i = 0;
      for (;;) {
        if (path_out && i < path_cap) path_out[i] = cur;
        r->path_hash += mix((((uint64_t)i << 32) | cur) + kPhi);
        ++i;
        if (cur == G.start) break;
        uint32_t best = kInf;
        const uint32_t gcur = g[cur];
        // predecessor p: a move p -> cur of cost c with g[p] + c == g[cur], p expanded;
        // moves are symmetric, so enumerate the moves out of cur
        moves(cur, [&](uint32_t p, uint32_t cost) {
          if (g[p] == kInf || (uint64_t)g[p] + cost != gcur) return;
          if ((uint64_t)g[p] + h(p) > cs) return;
          best = std::min(best, p);
        });
        if (best == kInf) return -1;
        cur = best;
      }
      r->path_len = i;
    }
    // self-check: the closed cells are exactly the cells with g + h <= C*
    return pops == expanded ? 0 : -1;
  }
};

}  // namespace

extern "C" {

struct OracleAstarGrid {
  uint64_t seed;
  uint32_t width, height, block_thr, conn, start, goal;
};

struct OracleAstarResult {
  uint32_t cost, path_len;
  uint64_t expanded, gsum, path_hash, pops;
  double seconds;
};

// Parameters of query `index` of a batch: grid side log-uniform in [side_lo, side_hi],
// obstacle density uniform in [dens_lo, dens_hi], start and goal uniform over the free
// cells (distinct), all drawn from seed = base_seed + index.
void oracle_astar_query(uint64_t base_seed, uint32_t index, uint32_t conn, uint32_t side_lo, uint32_t side_hi,
                        double dens_lo, double dens_hi, OracleAstarGrid* out) {
  const uint64_t seed = base_seed + index;
  const double u0 = (double)(rnd(seed, kQueryDomain, 0, 0) >> 11) * 0x1.0p-53;
  const double u1 = (double)(rnd(seed, kQueryDomain, 0, 1) >> 11) * 0x1.0p-53;
  uint32_t side = (uint32_t)std::floor((double)side_lo * std::exp2(u0 * std::log2((double)side_hi / side_lo)));
  side = std::min(std::max(side, side_lo), side_hi);
  const uint32_t thr = (uint32_t)((dens_lo + (dens_hi - dens_lo) * u1) * 16777216.0);
  const uint32_t cells = side * side;
  uint32_t s = 0, gl = 0;
  for (uint32_t k = 0;; ++k) {
    s = below(rnd(seed, kQueryDomain, k, 2), cells);
    if (!raw_blocked(seed, thr, s)) break;
  }
  for (uint32_t k = 0;; ++k) {
    gl = below(rnd(seed, kQueryDomain, k, 3), cells);
    if (gl != s && !raw_blocked(seed, thr, gl)) break;
  }
  *out = OracleAstarGrid{seed, side, side, thr, conn, s, gl};
}

int oracle_astar_solve(const OracleAstarGrid* grid, OracleAstarResult* res, uint32_t* g_out, uint32_t* path_out,
                       uint32_t path_cap) {
  const Grid G{grid->seed, grid->width, grid->height, grid->block_thr, grid->conn, grid->start, grid->goal};
  const auto t0 = std::chrono::steady_clock::now();
  Search s(G);
  Result r{};
  const int rc = s.run(&r, path_out, path_cap);
  r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (g_out) std::memcpy(g_out, s.g.data(), s.g.size() * sizeof(uint32_t));
  *res = OracleAstarResult{r.cost, r.path_len, r.expanded, r.gsum, r.path_hash, r.pops, r.seconds};
  return rc;
}

// Many independent queries, one per std::thread at a time (the batched CPU baseline).
// Returns wall seconds; per-query results in res[0, n).
double oracle_astar_batch(const OracleAstarGrid* grids, uint32_t n, int threads, OracleAstarResult* res) {
  std::atomic<uint32_t> next{0};
  std::atomic<int> bad{0};
  const auto t0 = std::chrono::steady_clock::now();
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(1);
      if (i >= n) break;
      if (oracle_astar_solve(&grids[i], &res[i], nullptr, nullptr, 0) != 0) bad.fetch_add(1);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return bad.load() ? -sec : sec;
}

}  // extern "C"
