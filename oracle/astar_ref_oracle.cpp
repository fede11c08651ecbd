// TEST INFRASTRUCTURE ONLY -- CPU oracle of the reference-semantics A* mode.
//
// Only tests/ and bench.py's CPU-baseline leg load this; the product never does.  It
// restates the reference's agent (src/a_star.cu:269-593) sequentially, one agent at a
// time, written independently of include/gpq/astar_ref.h:
//   * a round pops min(open length, 8) vertices in key order (f, then h, then cell: the
//     reference's operator< of src/queue_item.h:56-73 with its schedule-dependent ties
//     fixed by cell) and closes them (src/a_star.cu:331-374);
//   * if one of them is the goal, the agent ends with that vertex's f
//     (src/a_star.cu:401-442);
//   * else each popped vertex explores its 3 x 3 square with clamped coordinates
//     (src/a_star.cu:384-399); a cell neither closed nor a wall gets
//     g = f(cur) - h(cur, goal) + h(cur, nb) and f = half(g + h(nb, goal))
//     (src/a_star.cu:474-496);
//   * duplicates of the round keep the first position and the smallest f
//     (src/a_star.cu:508-530); a survivor is inserted only if its f beats the best f the
//     cell was ever inserted with (src/a_star.cu:537-560);
//   * an empty open list after a round ends the agent without a path (src/a_star.cu:564-580).
// h is sqrt(2) * min + max - min evaluated in double and rounded to float
// (src/a_star.cu:124-135); the half conversion rounds to nearest even, here through
// frexp/ldexp arithmetic rather than bit manipulation.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

namespace {

float href(int x0, int y0, int x1, int y1) {
  const int dx = std::abs(x0 - x1), dy = std::abs(y0 - y1);
  const int mn = std::min(dx, dy), mx = std::max(dx, dy);
  volatile double a = 1.4142135623730951 * (double)mn;  // no contraction into an fma
  volatile double b = a + (double)mx;
  volatile double c = b - (double)mn;
  return (float)c;
}

// float -> binary16 value (round to nearest even), returned as the exact float value.
float to_half(float v) {
  if (v == 0.0f) return 0.0f;
  int e;
  const double m = std::frexp((double)v, &e);  // v = m * 2^e, m in [0.5, 1)
  // a half has 11 significant bits for exponents >= -13 (normal), fewer below
  const int keep = (e - 1 >= -14) ? 11 : 11 - (-14 - (e - 1));
  if (keep <= 0) {
    const double q = std::ldexp((double)v, 24);  // units of 2^-24
    return (float)std::ldexp(std::nearbyint(q), -24);
  }
  const double scaled = std::ldexp(m, keep);      // keep bits before the point
  const double r = std::nearbyint(scaled);        // ties to even (default rounding mode)
  const double out = std::ldexp(r, e - keep);
  if (out > 65504.0) return INFINITY;
  return (float)out;
}

uint32_t half_bits(float hv) {  // bits of a value that is exactly a non-negative half
  if (hv == 0.0f) return 0;
  if (std::isinf(hv)) return 0x7c00u;
  int e;
  const double m = std::frexp((double)hv, &e);  // hv = m * 2^e
  const int ue = e - 1;                          // hv = 1.f * 2^ue
  if (ue >= -14) {
    const uint32_t frac = (uint32_t)std::ldexp(m * 2.0 - 1.0, 10);
    return ((uint32_t)(ue + 15) << 10) | frac;
  }
  return (uint32_t)std::ldexp((double)hv, 24);  // subnormal: units of 2^-24
}

struct V {
  uint32_t f;  // half bits
  float h;
  uint32_t cell;
  float fv;    // f as a float
};
struct Greater {
  bool operator()(const V& a, const V& b) const {
    if (a.f != b.f) return a.f > b.f;
    if (a.h != b.h) return a.h > b.h;
    return a.cell > b.cell;
  }
};

}  // namespace

extern "C" {

typedef struct oracle_astar_ref_result {
  uint32_t found;
  float cost;
  uint32_t pops;
  uint32_t rounds;
} oracle_astar_ref_result;

void oracle_astar_ref_agent(uint32_t W, uint32_t H, const uint8_t* map, uint32_t start, uint32_t goal,
                            oracle_astar_ref_result* out) {
  const uint32_t cells = W * H;
  std::vector<uint8_t> closed(cells, 0);
  std::vector<float> f_ol(cells, 0.0f);
  std::priority_queue<V, std::vector<V>, Greater> open;
  const int gx = (int)(goal % W), gy = (int)(goal / W);
  const float h0 = href((int)(start % W), (int)(start / W), gx, gy);
  const float f0 = to_half(h0);
  open.push({half_bits(f0), h0, start, f0});
  uint32_t rounds = 0, pops = 0, found = 0;
  float cost = 0.0f;
  struct Cand { uint32_t cell; float f; bool live; };
  while (!open.empty()) {
    ++rounds;
    const uint32_t npop = std::min<size_t>(open.size(), 8);
    V popped[8];
    for (uint32_t p = 0; p < npop; ++p) {
      popped[p] = open.top();
      open.pop();
      closed[popped[p].cell] = 1;
    }
    pops += npop;
    bool hit = false;
    for (uint32_t p = 0; p < npop && !hit; ++p)
      if (popped[p].cell == goal) { hit = true; cost = popped[p].fv; }
    if (hit) { found = 1; break; }
    Cand cand[64];
    for (uint32_t c = 0; c < 64; ++c) {
      cand[c].live = false;
      const uint32_t p = c / 8, k = c % 8;
      if (p >= npop) continue;
      const int x = (int)(popped[p].cell % W), y = (int)(popped[p].cell / W);
      const int l = (int)(k >= 4 ? k + 1 : k);
      const int nx = std::max(0, std::min((int)W - 1, x - 1 + l % 3));
      const int ny = std::max(0, std::min((int)H - 1, y - 1 + l / 3));
      const uint32_t nc = (uint32_t)ny * W + (uint32_t)nx;
      if (closed[nc] || map[nc]) continue;
      const float g = (popped[p].fv - href(x, y, gx, gy)) + href(x, y, nx, ny);
      cand[c] = {nc, to_half(g + href(nx, ny, gx, gy)), true};
    }
    for (uint32_t i = 0; i < 64; ++i) {  // de-duplicate in order
      if (!cand[i].live) continue;
      for (uint32_t j = i + 1; j < 64; ++j) {
        if (!cand[j].live || cand[j].cell != cand[i].cell) continue;
        if (cand[i].f > cand[j].f) cand[i].f = cand[j].f;
        cand[j].live = false;
      }
    }
    std::vector<uint32_t> better;
    for (uint32_t i = 0; i < 64; ++i)
      if (cand[i].live && (f_ol[cand[i].cell] == 0.0f || f_ol[cand[i].cell] > cand[i].f)) better.push_back(i);
    for (uint32_t i : better) {
      const Cand& c = cand[i];
      open.push({half_bits(c.f), href((int)(c.cell % W), (int)(c.cell / W), gx, gy), c.cell, c.f});
      f_ol[c.cell] = c.f;
    }
  }
  out->found = found;
  out->cost = cost;
  out->pops = pops;
  out->rounds = rounds;
}

// All agents, spread over `threads` host threads; returns the wall seconds.
double oracle_astar_ref_run(uint32_t W, uint32_t H, const uint8_t* map, const uint32_t* start_goal, uint32_t n,
                            int threads, oracle_astar_ref_result* out) {
  if (threads < 1) threads = 1;
  std::atomic<uint32_t> next{0};
  auto t0 = std::chrono::steady_clock::now();
  auto work = [&]() {
    for (uint32_t i; (i = next.fetch_add(1)) < n;)
      oracle_astar_ref_agent(W, H, map, start_goal[2 * i], start_goal[2 * i + 1], out + i);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < threads; ++t) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The half conversion of the oracle, for its own tests.
float oracle_to_half(float v) { return to_half(v); }
uint32_t oracle_half_bits(float v) { return half_bits(to_half(v)); }
float oracle_astar_ref_h(int x0, int y0, int x1, int y1) { return href(x0, y0, x1, y1); }

}  // extern "C"
