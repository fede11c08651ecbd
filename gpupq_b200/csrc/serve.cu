// Serving (gpq_serve_*): a stream of A* queries and PHOLD runs, admitted as they arrive
// against a device-memory budget and run with continuous batching -- every admitted
// request stays resident in its engine's session and advances a bounded number of
// rounds or windows per step, next to whatever else is running, until it finishes --
// or, for comparison, one request per launch in arrival order (the plain path).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <thread>
#include <vector>

#include "host_common.h"

using gpq::set_last_error;

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

void wait_until(Clock::time_point t0, double t) {
  const double now = seconds_since(t0);
  if (t > now) std::this_thread::sleep_for(std::chrono::duration<double>(t - now));
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const size_t i = (size_t)std::min<double>((double)v.size() - 1, std::ceil(q * v.size()) - 1);
  return v[i];
}

struct Sessions {
  gpq_astar_session* astar = nullptr;
  gpq_phold_session* phold = nullptr;
  ~Sessions() {
    gpq_astar_session_destroy(astar);
    gpq_phold_session_destroy(phold);
  }
};

gpq_status serve_batched(const gpq_serve_config& c, const gpq_serve_request* reqs, uint32_t n,
                         gpq_serve_response* out, gpq_serve_stats* stats) {
  // split the budget: A* cells (5.125 B each: g, predecessor move, blocked bit) and tiles, PHOLD LPs
  const uint64_t budget = c.hbm_budget;
  const double share = c.astar_share > 0.0 ? c.astar_share : 0.75;
  gpq_astar_config ac = c.astar;
  const uint32_t tile = ac.tile ? ac.tile : 64;
  const uint64_t in_cap = ac.inbox_capacity ? ac.inbox_capacity : 8ull * tile;
  const uint64_t open_cap = ac.open_capacity ? ac.open_capacity : (uint64_t)tile * tile;
  const uint64_t tile_bytes = 64 + 8 * (2 * in_cap + open_cap) + 8;
  const uint64_t a_bytes = (uint64_t)(budget * share);
  // a tile for every tile*tile cells, plus room for ragged edges
  const double per_cell = 5.125 + (double)tile_bytes / ((double)tile * tile) * 1.25;
  const uint64_t max_cells = std::max<uint64_t>((uint64_t)(a_bytes / per_cell), 1u << 20);
  const uint32_t max_tiles = (uint32_t)std::min<uint64_t>(max_cells / ((uint64_t)tile * tile) * 5 / 4 + 1024, 1u << 30);
  const uint32_t max_inst = 65536;
  const uint32_t cap = c.phold_capacity ? c.phold_capacity : 256;
  const uint32_t ibc = c.phold_insert_capacity ? c.phold_insert_capacity : 64;
  const uint64_t p_bytes = budget - std::min(budget, a_bytes);
  const bool buckets = c.phold_form == 1;
  const uint64_t per_lp = buckets ? gpq_phold_session_bytes_bucketed(1, 0, 0, 0) : 16ull * cap + 32ull * ibc + 40;
  const uint32_t max_lps = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(p_bytes / per_lp, 1024), 1u << 30);
  Sessions ss;
  gpq_status st = gpq_astar_session_create(&ac, max_cells, max_tiles, max_inst, &ss.astar);
  if (st != GPQ_OK) return st;
  st = buckets ? gpq_phold_session_create_bucketed(max_lps, 0, 0, max_inst, &ss.phold)
               : gpq_phold_session_create(max_lps, cap, ibc, max_inst, c.phold_lanes_per_lp, &ss.phold);
  if (st != GPQ_OK) return st;
  const uint32_t R = c.astar_rounds ? c.astar_rounds : 32;
  const uint32_t W = c.phold_windows ? c.phold_windows : 32;
  std::vector<uint32_t> owner_a(max_inst, ~0u), owner_p(max_inst, ~0u);
  std::vector<uint32_t> slots(max_inst);
  std::vector<gpq_astar_result> ares(max_inst);
  std::vector<gpq_phold_result> pres(max_inst);
  uint32_t next = 0, done = 0, resident_a = 0, resident_p = 0, max_res = 0;
  uint64_t steps = 0;
  const Clock::time_point t0 = Clock::now();
  while (done < n) {
    const double now = seconds_since(t0);
    // admission in arrival order; the first request that does not fit waits
    while (next < n && (!c.realtime || reqs[next].arrival <= now)) {
      const gpq_serve_request& q = reqs[next];
      uint32_t slot = 0;
      gpq_status a;
      if (q.kind == GPQ_REQ_ASTAR) a = gpq_astar_session_admit(ss.astar, &q.astar, &slot);
      else if (q.kind == GPQ_REQ_PHOLD) a = gpq_phold_session_admit(ss.phold, &q.phold, &slot);
      else a = GPQ_ERR_INVALID;
      if (a == GPQ_ERR_NOMEM && (resident_a + resident_p) > 0) break;  // room frees up later
      out[next].admitted = seconds_since(t0);
      if (a != GPQ_OK) {  // never fits, or invalid
        out[next].status = a;
        out[next].finished = out[next].admitted;
        ++done;
        ++next;
        continue;
      }
      if (q.kind == GPQ_REQ_ASTAR) {
        owner_a[slot] = next;
        ++resident_a;
      } else {
        owner_p[slot] = next;
        ++resident_p;
      }
      ++next;
    }
    max_res = std::max(max_res, resident_a + resident_p);
    if (resident_a + resident_p == 0) {
      if (next < n && c.realtime) wait_until(t0, reqs[next].arrival);
      continue;
    }
    uint32_t running = 0, got = 0;
    if (resident_a) {
      if ((st = gpq_astar_session_step(ss.astar, R, &running, nullptr)) != GPQ_OK) return st;
      if ((st = gpq_astar_session_collect(ss.astar, slots.data(), ares.data(), max_inst, &got, nullptr)) != GPQ_OK)
        return st;
      const double t = seconds_since(t0);
      for (uint32_t j = 0; j < got; ++j) {
        const uint32_t r = owner_a[slots[j]];
        out[r].astar = ares[j];
        out[r].status = ares[j].status;
        out[r].finished = t;
        owner_a[slots[j]] = ~0u;
      }
      resident_a -= got;
      done += got;
    }
    if (resident_p) {
      if ((st = gpq_phold_session_step(ss.phold, W, &running, nullptr)) != GPQ_OK) return st;
      if ((st = gpq_phold_session_collect(ss.phold, slots.data(), pres.data(), max_inst, &got, nullptr)) != GPQ_OK)
        return st;
      const double t = seconds_since(t0);
      for (uint32_t j = 0; j < got; ++j) {
        const uint32_t r = owner_p[slots[j]];
        out[r].phold = pres[j];
        out[r].status = pres[j].status;
        out[r].finished = t;
        owner_p[slots[j]] = ~0u;
      }
      resident_p -= got;
      done += got;
    }
    ++steps;
  }
  stats->steps = steps;
  stats->max_resident = max_res;
  return GPQ_OK;
}

gpq_status serve_plain(const gpq_serve_config& c, const gpq_serve_request* reqs, uint32_t n, gpq_serve_response* out,
                       gpq_serve_stats* stats) {
  gpq_astar* a = nullptr;
  gpq_status st = gpq_astar_create(&c.astar, &a);
  if (st != GPQ_OK) return st;
  const Clock::time_point t0 = Clock::now();
  for (uint32_t i = 0; i < n; ++i) {
    const gpq_serve_request& q = reqs[i];
    if (c.realtime) wait_until(t0, q.arrival);
    out[i].admitted = seconds_since(t0);
    if (q.kind == GPQ_REQ_ASTAR) {
      st = gpq_astar_solve(a, &q.astar, 1, &out[i].astar, nullptr);
      out[i].status = st != GPQ_OK ? st : out[i].astar.status;
    } else if (q.kind == GPQ_REQ_PHOLD) {
      gpq_phold_config pc = q.phold;
      pc.queue_kind = GPQ_QUEUE_LAQ;
      pc.loop_mode = GPQ_LOOP_PERSISTENT;
      pc.capacity = c.phold_capacity ? c.phold_capacity : 256;
      pc.insert_capacity = c.phold_insert_capacity ? c.phold_insert_capacity : 64;
      gpq_phold* h = nullptr;
      st = gpq_phold_create(&pc, &h);
      if (st == GPQ_OK) st = gpq_phold_populate(h, nullptr, 0, nullptr);
      if (st == GPQ_OK) st = gpq_phold_run(h, nullptr);
      if (st == GPQ_OK) st = gpq_phold_result_get(h, &out[i].phold, nullptr);
      gpq_phold_destroy(h);
      out[i].status = st != GPQ_OK ? st : out[i].phold.status;
    } else {
      out[i].status = GPQ_ERR_INVALID;
    }
    out[i].finished = seconds_since(t0);
  }
  gpq_astar_destroy(a);
  stats->steps = n;
  stats->max_resident = 1;
  return GPQ_OK;
}

}  // namespace

extern "C" {

gpq_status gpq_serve_run(const gpq_serve_config* cfg, const gpq_serve_request* reqs, uint32_t n,
                         gpq_serve_response* out, gpq_serve_stats* stats) {
  GPQ_CHECK_ARG(cfg && (reqs || n == 0) && (out || n == 0) && stats, "NULL argument");
  gpq_serve_config c = *cfg;
  if (c.hbm_budget == 0) c.hbm_budget = 120ull << 30;
  for (uint32_t i = 0; i < n; ++i) out[i] = gpq_serve_response{};
  *stats = gpq_serve_stats{};
  gpq_status st = c.mode == GPQ_SERVE_PLAIN ? serve_plain(c, reqs, n, out, stats)
                                            : serve_batched(c, reqs, n, out, stats);
  if (st != GPQ_OK) return st;
  std::vector<double> lat(n);
  double last = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    const double arrival = c.realtime ? reqs[i].arrival : 0.0;
    lat[i] = out[i].finished - arrival;
    last = std::max(last, out[i].finished);
  }
  stats->makespan = last;
  stats->throughput = last > 0.0 ? n / last : 0.0;
  stats->p50 = percentile(lat, 0.50);
  stats->p99 = percentile(lat, 0.99);
  stats->p999 = percentile(lat, 0.999);
  return GPQ_OK;
}

gpq_status gpq_serve_stream(uint64_t seed, double rate, double duration, double astar_fraction,
                            gpq_serve_request* out, uint32_t capacity, uint32_t* n) {
  GPQ_CHECK_ARG(n && rate > 0.0 && duration >= 0.0 && astar_fraction >= 0.0 && astar_fraction <= 1.0,
                "need rate > 0, duration >= 0, 0 <= astar_fraction <= 1");
  double t = 0.0;
  uint32_t k = 0;
  for (;; ++k) {
    const uint64_t r = gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN + 1u, k, 0);
    const double u = ((double)(r >> 11) + 1.0) * 0x1.0p-53;  // (0, 1]
    t += -std::log(u) / rate;  // exponential gaps: Poisson arrivals
    if (t > duration) break;
    if (k >= capacity) {
      if (out) break;
      continue;
    }
    if (!out) continue;
    gpq_serve_request& q = out[k];
    q = gpq_serve_request{};
    q.arrival = t;
    const double kind_u = (double)(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN + 1u, k, 1) >> 11) * 0x1.0p-53;
    if (kind_u < astar_fraction) {
      q.kind = GPQ_REQ_ASTAR;
      const gpq_status st = gpq_astar_query(seed, k, 4, 128, 4096, 0.2, 0.2, &q.astar);
      if (st != GPQ_OK) return st;
    } else {
      q.kind = GPQ_REQ_PHOLD;
      const double lu = (double)(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN + 1u, k, 2) >> 11) * 0x1.0p-53;
      uint32_t lps = (uint32_t)std::floor(256.0 * std::exp2(lu * 8.0));  // log-uniform in [256, 65536]
      lps = std::min<uint32_t>(std::max<uint32_t>(lps, 256), 65536);
      gpq_phold_config& p = q.phold;
      p.seed = seed + k;
      p.num_lps = lps;
      p.events_per_lp = 32;
      p.lookahead = 0.5f;
      p.end_time = 200.0f;
      p.dest_mode = GPQ_DEST_UNIFORM;
      p.queue_kind = GPQ_QUEUE_LAQ;
      p.loop_mode = GPQ_LOOP_PERSISTENT;
    }
  }
  *n = out ? std::min(k, capacity) : k;
  return GPQ_OK;
}

}  // extern "C"
