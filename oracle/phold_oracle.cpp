// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the PHOLD hot path.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
// file's library; the product (gpupq_b200) never includes, links or calls it.
//
// It restates, in plain sequential C++, what the reference computes on its hot path:
//   * the PHOLD event handler, src/phold.cu:81-117 (peek the LP's earliest safe event,
//     count it, draw destination and Exp increment, set_done, insert the child);
//   * the conservative safe-window loop, src/des.cu:154-214 (global minimum ->
//     window [min, min + LOOKAHEAD) -> handle -> queue_post), with the minimum as in
//     src/local_array_queue.cu:116-146,460-478;
//   * the per-LP queue ordering of src/queue_item.h:20-26 (by timestamp), with ties
//     broken by (ts bits, LP, id).
// The event semantics (counter-based draws, own logarithm, float32 timestamps) are
// restated independently of the product's include/gpq/model.h so that the two
// cross-check each other.  Parity for the ring helpers is pinned by the reference's
// own known-answer tests (src/test_laq.cu:39-236), see oracle_ring_* below.
//
// Three drivers produce identical per-LP outputs:
//   oracle_phold_seq     one global std::priority_queue, events popped in key order;
//   oracle_phold_window  one std::priority_queue per LP, LPs split over host threads,
//                        window-synchronous steps (the reference's loop run on CPU cores;
//                        used as the timed CPU baseline);
//   oracle_phold_one_per_lp  the reference's own schedule: every window handles at most
//                        ONE event per LP (src/phold.cu:84-94 peeks one item per LP per
//                        call; src/local_array_queue.cu:760-779), so it takes more windows;
//                        its window count is what the reference's loop reports.
// The first two count windows in which every LP drains all of its safe events.
// Build: g++ -O2 -std=c++20 -ffp-contract=off -fPIC -shared (see oracle/build.py).

#include <algorithm>
#include <atomic>
#include <barrier>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

namespace {

struct Ev {
  float ts;
  uint32_t lp, id, aux;
};

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float ffrom(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// (ts bits, lp, id) order; timestamps are finite and >= +0.
inline bool key_less(const Ev& a, const Ev& b) {
  uint32_t ta = fbits(a.ts), tb = fbits(b.ts);
  if (ta != tb) return ta < tb;
  if (a.lp != b.lp) return a.lp < b.lp;
  return a.id < b.id;
}
struct KeyGreater {
  bool operator()(const Ev& a, const Ev& b) const { return key_less(b, a); }
};
using MinHeap = std::priority_queue<Ev, std::vector<Ev>, KeyGreater>;

// SplitMix64 finaliser (Steele, Lea, Flood 2014).
inline uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

inline uint64_t rng(uint64_t seed, uint32_t id, uint32_t tsb, uint32_t k) {
  uint64_t key = mix(seed ^ ((uint64_t)id * kGolden));
  return mix(key ^ (((uint64_t)tsb << 8) | (uint64_t)(k & 0xffu)));
}

// ln(x) by range reduction to [sqrt(1/2), sqrt(2)) and the atanh series
// 2*(s + s^3/3 + ... + s^9/9), s = (m-1)/(m+1); one float rounding per operation.
inline float ln_own(float x) {
  uint32_t b = fbits(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = ffrom((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 0.222222224f;
  p = p * z + 0.285714298f;
  p = p * z + 0.400000006f;
  p = p * z + 0.666666687f;
  p = p * z + 2.0f;
  float lm = s * p;
  return (float)e * 0.693147182f + lm;
}

inline float exp_draw(uint64_t r) {
  float u = (float)((uint32_t)(r >> 40) + 1u) * 5.9604644775390625e-8f;  // (0, 1]
  return 0.0f - ln_own(u);
}

inline uint32_t below(uint64_t r, uint32_t n) { return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32); }

}  // namespace

extern "C" {

typedef struct oracle_phold_cfg {
  uint64_t seed;
  uint32_t num_lps;
  uint32_t events_per_lp;
  uint32_t dest_mode;       // 0 uniform, 1 ring
  uint32_t ring_width;
  uint32_t ring_threshold;  // ring with probability threshold / 2^32
  float lookahead;
  float end_time;
} oracle_phold_cfg;

typedef struct oracle_phold_summary {
  uint64_t committed;
  uint64_t steps;
  uint64_t pending;
  uint64_t pending_csum;
  double seconds;  // wall time of the event loop (population excluded)
} oracle_phold_summary;

}  // extern "C"

namespace {

struct Model {
  oracle_phold_cfg c;
  uint32_t dest(uint32_t lp, uint64_t r) const {
    if (c.dest_mode == 1 && (uint32_t)r < c.ring_threshold) {
      uint32_t w = c.ring_width;
      uint32_t k = below(r, 2 * w);
      int64_t off = (k < w) ? (int64_t)k - w : (int64_t)k - w + 1;
      int64_t d = ((int64_t)lp + off) % (int64_t)c.num_lps;
      if (d < 0) d += c.num_lps;
      return (uint32_t)d;
    }
    return below(r, c.num_lps);
  }
  // src/phold.cu:95-114: new event at ts + LOOKAHEAD + Exp on a drawn node.
  Ev child(const Ev& e) const {
    uint32_t tb = fbits(e.ts);
    uint64_t r0 = rng(c.seed, e.id, tb, 0);
    uint64_t r1 = rng(c.seed, e.id, tb, 1);
    float delta = c.lookahead + exp_draw(r1);
    Ev n;
    n.ts = e.ts + delta;
    n.lp = dest(e.lp, r0);
    n.id = e.id;
    n.aux = e.lp;
    return n;
  }
  // src/phold.cu:63-79 populates randomly; here LP l holds events id = l*P + k.
  Ev initial(uint32_t lp, uint32_t k) const {
    Ev e;
    e.id = lp * c.events_per_lp + k;
    e.lp = lp;
    e.aux = lp;
    e.ts = exp_draw(rng(c.seed, e.id, 0xFFFFFFFFu, 0));
    return e;
  }
};

inline uint64_t ev_hash(const Ev& e) { return mix(((uint64_t)e.id << 32) | fbits(e.ts)); }

struct LpOut {
  uint32_t* count;
  uint64_t* csum;
  uint64_t* ohash;
  // src/phold.cu:91-92: save_lp_ts + num_events[lp]++ ; plus the two checksums.
  void commit(const Ev& e) {
    uint64_t h = ev_hash(e);
    uint64_t seq = count[e.lp];
    count[e.lp] = (uint32_t)(seq + 1);
    csum[e.lp] += h;
    ohash[e.lp] += mix(h + seq * kGolden);
  }
};

}  // namespace

extern "C" {

// Sequential driver: one global priority queue popped in key order.  A new window
// starts whenever the popped event is not below the current window bound.
int oracle_phold_seq(const oracle_phold_cfg* cfg, uint32_t* count, uint64_t* csum, uint64_t* ohash,
                     oracle_phold_summary* out) {
  if (!cfg || !count || !csum || !ohash || !out || cfg->num_lps == 0) return 1;
  Model m{*cfg};
  const uint32_t L = cfg->num_lps;
  std::memset(count, 0, sizeof(uint32_t) * L);
  std::memset(csum, 0, sizeof(uint64_t) * L);
  std::memset(ohash, 0, sizeof(uint64_t) * L);
  LpOut o{count, csum, ohash};

  std::vector<Ev> init;
  init.reserve((size_t)L * cfg->events_per_lp);
  for (uint32_t lp = 0; lp < L; ++lp)
    for (uint32_t k = 0; k < cfg->events_per_lp; ++k) init.push_back(m.initial(lp, k));
  MinHeap pq(KeyGreater{}, std::move(init));

  auto t0 = std::chrono::steady_clock::now();
  uint64_t committed = 0, steps = 0;
  bool have_bound = false;
  float bound = 0.0f;
  const float T = cfg->end_time;
  while (!pq.empty()) {
    Ev e = pq.top();
    if (!(e.ts < T)) break;
    if (!have_bound || !(e.ts < bound)) {  // window [m, m + LOOKAHEAD), m = e.ts
      ++steps;
      bound = e.ts + cfg->lookahead;
      have_bound = true;
    }
    pq.pop();
    o.commit(e);
    ++committed;
    pq.push(m.child(e));
  }
  auto t1 = std::chrono::steady_clock::now();
  uint64_t pend = 0, pcs = 0;
  while (!pq.empty()) { pcs += ev_hash(pq.top()); ++pend; pq.pop(); }
  out->committed = committed;
  out->steps = steps;
  out->pending = pend;
  out->pending_csum = pcs;
  out->seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}

// Window-synchronous driver over per-LP queues on `nthreads` host threads
// (the loop of src/des.cu:154-214 with one std::priority_queue per LP).
int oracle_phold_window(const oracle_phold_cfg* cfg, int nthreads, uint32_t* count, uint64_t* csum,
                        uint64_t* ohash, oracle_phold_summary* out) {
  if (!cfg || !count || !csum || !ohash || !out || cfg->num_lps == 0) return 1;
  if (nthreads < 1) nthreads = 1;
  const uint32_t L = cfg->num_lps;
  if ((uint32_t)nthreads > L) nthreads = (int)L;
  Model m{*cfg};
  std::memset(count, 0, sizeof(uint32_t) * L);
  std::memset(csum, 0, sizeof(uint64_t) * L);
  std::memset(ohash, 0, sizeof(uint64_t) * L);
  LpOut o{count, csum, ohash};

  std::vector<MinHeap> q(L);
  for (uint32_t lp = 0; lp < L; ++lp)
    for (uint32_t k = 0; k < cfg->events_per_lp; ++k) q[lp].push(m.initial(lp, k));

  const int P = nthreads;
  auto lp_begin = [&](int t) { return (uint32_t)(((uint64_t)L * t) / P); };
  auto owner = [&](uint32_t lp) {
    // inverse of lp_begin: largest t with lp_begin(t) <= lp
    int t = (int)(((uint64_t)lp * P) / L);
    while (t + 1 < P && lp_begin(t + 1) <= lp) ++t;
    while (t > 0 && lp_begin(t) > lp) --t;
    return t;
  };
  // outbox[src * P + dst]
  std::vector<std::vector<Ev>> outbox((size_t)P * P);
  std::vector<float> tmin(P, ffrom(0x7f800000u));
  std::vector<uint64_t> tcommit(P, 0);
  const float inf = ffrom(0x7f800000u);
  const float T = cfg->end_time;
  float gmin = inf;
  uint64_t steps = 0;
  bool done = false;

  // Barriers alternate: even-numbered ones reduce the per-thread minima into the
  // next window (and decide termination), odd-numbered ones separate drain and insert.
  uint64_t barrier_no = 0;
  auto reduce = [&]() noexcept {
    if ((barrier_no++ & 1u) != 0) return;
    float mn = inf;
    for (int t = 0; t < P; ++t) mn = std::min(mn, tmin[t]);
    gmin = mn;
    if (!(gmin < T)) done = true; else ++steps;
  };
  std::barrier sync(P, reduce);

  auto local_min = [&](int t) {
    float mn = inf;
    for (uint32_t lp = lp_begin(t); lp < lp_begin(t + 1); ++lp)
      if (!q[lp].empty()) mn = std::min(mn, q[lp].top().ts);
    tmin[t] = mn;
  };

  auto t0 = std::chrono::steady_clock::now();
  auto worker = [&](int t) {
    local_min(t);
    sync.arrive_and_wait();  // reduce -> gmin, steps
    while (!done) {
      const float bound = gmin + cfg->lookahead;
      // drain: src/phold.cu:81-117 for every safe event of the LP, in key order
      for (uint32_t lp = lp_begin(t); lp < lp_begin(t + 1); ++lp) {
        MinHeap& h = q[lp];
        while (!h.empty()) {
          const Ev e = h.top();
          if (!(e.ts < bound) || !(e.ts < T)) break;
          h.pop();
          o.commit(e);
          ++tcommit[t];
          Ev c = m.child(e);
          outbox[(size_t)t * P + owner(c.lp)].push_back(c);
        }
      }
      sync.arrive_and_wait();
      // queue_post: insert the children
      for (int s = 0; s < P; ++s) {
        auto& box = outbox[(size_t)s * P + t];
        for (const Ev& c : box) q[c.lp].push(c);
        box.clear();
      }
      local_min(t);
      sync.arrive_and_wait();  // reduce
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < P; ++t) th.emplace_back(worker, t);
  worker(0);
  for (auto& x : th) x.join();
  auto t1 = std::chrono::steady_clock::now();

  uint64_t committed = 0, pend = 0, pcs = 0;
  for (int t = 0; t < P; ++t) committed += tcommit[t];
  for (uint32_t lp = 0; lp < L; ++lp) {
    while (!q[lp].empty()) { pcs += ev_hash(q[lp].top()); ++pend; q[lp].pop(); }
  }
  out->committed = committed;
  out->steps = steps;
  out->pending = pend;
  out->pending_csum = pcs;
  out->seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}

// The reference's schedule (src/des.cu:154-214 with src/phold.cu:81-117): each window
// m = minimum pending timestamp; the loop stops when m >= T; every LP whose earliest event
// e has e.ts < m + lookahead and e.ts < T handles that ONE event; the children enter the
// queues after the window (queue_post).  Sequential; meant for small and medium sizes.
int oracle_phold_one_per_lp(const oracle_phold_cfg* cfg, uint32_t* count, uint64_t* csum, uint64_t* ohash,
                            oracle_phold_summary* out) {
  if (!cfg || !count || !csum || !ohash || !out || cfg->num_lps == 0) return 1;
  Model m{*cfg};
  const uint32_t L = cfg->num_lps;
  std::memset(count, 0, sizeof(uint32_t) * L);
  std::memset(csum, 0, sizeof(uint64_t) * L);
  std::memset(ohash, 0, sizeof(uint64_t) * L);
  LpOut o{count, csum, ohash};
  std::vector<MinHeap> q(L);
  for (uint32_t lp = 0; lp < L; ++lp)
    for (uint32_t k = 0; k < cfg->events_per_lp; ++k) q[lp].push(m.initial(lp, k));
  const float inf = ffrom(0x7f800000u), T = cfg->end_time;
  std::vector<Ev> children;
  auto t0 = std::chrono::steady_clock::now();
  uint64_t committed = 0, steps = 0;
  for (;;) {
    float mn = inf;
    for (uint32_t lp = 0; lp < L; ++lp)
      if (!q[lp].empty()) mn = std::min(mn, q[lp].top().ts);
    if (!(mn < T)) break;
    ++steps;
    const float bound = mn + cfg->lookahead;
    children.clear();
    for (uint32_t lp = 0; lp < L; ++lp) {
      if (q[lp].empty()) continue;
      const Ev e = q[lp].top();
      if (!(e.ts < bound) || !(e.ts < T)) continue;
      q[lp].pop();
      o.commit(e);
      ++committed;
      children.push_back(m.child(e));
    }
    for (const Ev& c : children) q[c.lp].push(c);
  }
  auto t1 = std::chrono::steady_clock::now();
  uint64_t pend = 0, pcs = 0;
  for (uint32_t lp = 0; lp < L; ++lp)
    while (!q[lp].empty()) { pcs += ev_hash(q[lp].top()); ++pend; q[lp].pop(); }
  out->committed = committed;
  out->steps = steps;
  out->pending = pend;
  out->pending_csum = pcs;
  out->seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}

// Order-sensitive digest over the per-LP outputs, as the GPU engine reports it:
// sum over LPs of mix(mix(mix(lp << 32 | count) ^ csum) + ohash).
uint64_t oracle_phold_digest(uint32_t num_lps, const uint32_t* count, const uint64_t* csum, const uint64_t* ohash) {
  uint64_t d = 0;
  for (uint32_t lp = 0; lp < num_lps; ++lp)
    d += mix(mix(mix(((uint64_t)lp << 32) | count[lp]) ^ csum[lp]) + ohash[lp]);
  return d;
}

// The PHOLD child and the initial events as seen by the oracle (for spot checks of the
// event function against the product, item by item).
void oracle_phold_child(const oracle_phold_cfg* cfg, const float* ts, const uint32_t* lp,
                        const uint32_t* id, uint64_t n, float* out_ts, uint32_t* out_lp) {
  Model m{*cfg};
  for (uint64_t i = 0; i < n; ++i) {
    Ev e{ts[i], lp[i], id[i], lp[i]};
    Ev c = m.child(e);
    out_ts[i] = c.ts;
    out_lp[i] = c.lp;
  }
}

void oracle_phold_initial(const oracle_phold_cfg* cfg, float* out_ts, uint32_t* out_lp, uint32_t* out_id) {
  Model m{*cfg};
  uint64_t i = 0;
  for (uint32_t lp = 0; lp < cfg->num_lps; ++lp)
    for (uint32_t k = 0; k < cfg->events_per_lp; ++k, ++i) {
      Ev e = m.initial(lp, k);
      out_ts[i] = e.ts;
      out_lp[i] = e.lp;
      out_id[i] = e.id;
    }
}

float oracle_logf(float x) { return ln_own(x); }

// ---------------------------------------------------------------------------------
// Ring helpers of the reference's local array queue, restated for its known-answer
// tests.  The ring holds integer timestamps in slots [0, cap); [read, write) is the
// sorted occupied range and may wrap.
// ---------------------------------------------------------------------------------

static inline int ring_wrap(int i, int cap) {  // src/sort.cu:17-26
  int r = i % cap;
  return r >= 0 ? r : cap + r;
}

// src/sort.cu:48-66: position after which `item` belongs, scanning from read-1.
int oracle_ring_search(const int64_t* ring, int cap, int read, int write, int64_t item) {
  int start = ring_wrap(read - 1, cap);
  int end = ring_wrap(write + 1, cap);
  int i;
  for (i = start; i != end; i = (i + 1) % cap) {
    int next = (i + 1) % cap;
    if (i + 1 == write) return i + 1;
    if (ring[next] > item) return i;
  }
  return i;
}

// src/sort.cu:329-353 (LOCAL_ARRAY_QUEUE_BACKWARD): insert `item` into the sorted
// range [read, write), shifting larger items one slot towards write.
void oracle_ring_insert_sorted(int64_t* ring, int cap, int read, int write, int64_t item) {
  int start = ring_wrap(write - 1, cap);
  int end = ring_wrap(read - 1, cap);
  if (read == write || ring[start] <= item) { ring[write] = item; return; }
  for (int i = start; i != end; i = ring_wrap(i - 1, cap)) {
    if (ring[i] > item) ring[ring_wrap(i + 1, cap)] = ring[i];
    int prev = ring_wrap(i - 1, cap);
    if (i == read || ring[prev] <= item) { ring[i] = item; return; }
  }
}

// src/sort.cu:74-131: in-place quicksort of the ring range [left, right] (inclusive;
// right < left means the range wraps), middle-element pivot, explicit stack.
void oracle_ring_quicksort(int64_t* ring, int cap, int left, int right) {
  if (left == right) return;
  if (left > right) right = cap + right;
  auto at = [&](int i) -> int64_t& { return ring[ring_wrap(i, cap)]; };
  std::vector<std::pair<int, int>> stack;
  stack.push_back({left, right});
  while (!stack.empty()) {
    auto [l, r] = stack.back();
    stack.pop_back();
    if (l >= r) continue;
    int mid = l + (r - l) / 2;
    int64_t pivot = at(mid);
    std::swap(at(mid), at(l));
    int i = l + 1, j = r;
    while (i <= j) {
      while (i <= j && at(i) <= pivot) ++i;
      while (i <= j && at(j) > pivot) --j;
      if (i < j) std::swap(at(i), at(j));
    }
    std::swap(at(i - 1), at(l));
    int part = i - 1;
    stack.push_back({l, part - 1});
    stack.push_back({part + 1, r});
  }
}

}  // extern "C"
