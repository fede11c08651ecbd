// Reference-semantics A* (gpq_astar_ref_*): the reference's agent model
// (src/a_star.cu:269-593, semantics in include/gpq/astar_ref.h) on the B200.
//
// The reference runs one CUDA block per concurrent agent and one kernel launch per round
// for all agents (model_handle_next, src/a_star.cu:854-872); thread 0 pops up to eight
// vertices from the agent's local array queue, 64 threads explore the 3 x 3 squares,
// thread 0 de-duplicates serially, and a new agent clears its 65,536-cell f_ol array
// with one thread.  Agents never interact, so here one warp owns a slot and runs its
// agents to completion without any grid-wide step: a persistent launch whose warps take
// agents from the pool with one atomicAdd (get_new_agent, src/a_star.cu:150-164).  A
// slot's open list is a 4-ary heap in global memory worked by the whole warp: a pop
// loads the four children of a level in one round trip, an insert loads every ancestor
// of the new leaf in one round trip and shifts the larger ones down in one store round;
// the 64 candidates of a round are de-duplicated with one lane per candidate; f_ol and
// the closed set are cleared with 16-byte stores of all lanes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "common.cuh"
#include "gpq/astar_ref.h"
#include "host_common.h"

namespace {

struct RefItem {  // open-list vertex: key (f half bits, h bits), cell
  uint32_t f, h, cell, pad;
};

__device__ __forceinline__ bool ref_less(const RefItem& a, const RefItem& b) {
  if (a.f != b.f) return a.f < b.f;
  if (a.h != b.h) return a.h < b.h;
  return a.cell < b.cell;
}

__device__ __forceinline__ RefItem ref_load(const RefItem* p) {
  const uint4 v = *reinterpret_cast<const uint4*>(p);
  return RefItem{v.x, v.y, v.z, v.w};
}

__device__ __forceinline__ void ref_store(RefItem* p, const RefItem& x) {
  *reinterpret_cast<uint4*>(p) = make_uint4(x.f, x.h, x.cell, x.pad);
}

__device__ __forceinline__ RefItem ref_shfl(const RefItem& x, int src) {
  return RefItem{__shfl_sync(GPQ_FULL_MASK, x.f, src), __shfl_sync(GPQ_FULL_MASK, x.h, src),
                 __shfl_sync(GPQ_FULL_MASK, x.cell, src), 0u};
}

struct RefDev {
  uint32_t width, height, cells, words;  // words: 32-bit words of one cell bitset
  const uint32_t* wall;                  // [words] map bitmap
  const gpq_astar_ref_agent* agents;
  gpq_astar_ref_result* results;
  uint32_t n_agents;
  uint32_t* next_agent;
  RefItem* heap;                         // [slots][cap]
  uint32_t cap;
  uint16_t* f_ol;                        // [slots][fol_stride] best f ever inserted (half bits; 0 = never)
  uint32_t fol_stride;                   // cells rounded up to 8 (16-byte rows)
  uint32_t* closed;                      // [slots][words]
  uint32_t slots;
};

__device__ __forceinline__ bool bit(const uint32_t* b, uint32_t i) { return (b[i >> 5] >> (i & 31u)) & 1u; }

// Removes the smallest item of a heap of n >= 1 items; all lanes, returns it in every lane.
__device__ RefItem ref_pop(RefItem* hp, uint32_t n, uint32_t lane) {
  const RefItem top = ref_load(hp);
  const RefItem last = ref_load(hp + n - 1);
  const uint32_t m = n - 1;
  uint32_t pos = 0;
  if (m > 0) {
    for (;;) {
      const uint32_t fc = 4u * pos + 1u;
      if (fc >= m) break;
      RefItem c{0xffffffffu, 0xffffffffu, 0xffffffffu, 0u};
      uint32_t ci = 0xffffffffu;
      if (lane < 4u && fc + lane < m) {
        c = ref_load(hp + fc + lane);
        ci = fc + lane;
      }
#pragma unroll
      for (int o = 1; o < 4; o <<= 1) {  // minimum over lanes 0..3
        const RefItem oc = ref_shfl(c, (int)(lane ^ (uint32_t)o));
        const uint32_t oi = __shfl_xor_sync(GPQ_FULL_MASK, ci, o);
        if (ref_less(oc, c)) { c = oc; ci = oi; }
      }
      c = ref_shfl(c, 0);
      ci = __shfl_sync(GPQ_FULL_MASK, ci, 0);
      if (!ref_less(c, last)) break;
      if (lane == 0) ref_store(hp + pos, c);
      pos = ci;
    }
    if (lane == 0) ref_store(hp + pos, last);
  }
  __syncwarp();
  return top;
}

// Inserts x into a heap of n items (n < capacity); all lanes.
__device__ void ref_push(RefItem* hp, uint32_t n, const RefItem& x, uint32_t lane) {
  // ancestor lane+1 of leaf n: a_0 = n, a_{k+1} = (a_k - 1) / 4
  uint32_t a = n, depth_ok = 1u;
  for (uint32_t k = 0; k <= lane; ++k) {
    if (a == 0) { depth_ok = 0u; break; }
    a = (a - 1u) >> 2;
  }
  RefItem anc{0u, 0u, 0u, 0u};
  bool greater = false;
  if (depth_ok) {
    anc = ref_load(hp + a);
    greater = ref_less(x, anc);
  }
  // the ancestors above x form a prefix (heap order): lanes 0..j-1
  const uint32_t j = (uint32_t)__popc(__ballot_sync(GPQ_FULL_MASK, greater));
  // ancestor k+1 moves into the place of ancestor k (ancestor 0 = the new leaf)
  const uint32_t below = __shfl_up_sync(GPQ_FULL_MASK, a, 1);
  if (greater) ref_store(hp + (lane == 0 ? n : below), anc);
  const uint32_t at = __shfl_sync(GPQ_FULL_MASK, a, (int)(j == 0 ? 0 : j - 1));
  if (lane == 0) ref_store(hp + (j == 0 ? n : at), x);
  __syncwarp();
}

__device__ __forceinline__ RefItem ref_vertex(uint32_t cell, uint32_t f_half, uint32_t w, uint32_t goal) {
  const float h = gpq_astar_ref_h((int)(cell % w), (int)(cell / w), (int)(goal % w), (int)(goal / w));
  return RefItem{f_half, gpq_f2u(h), cell, 0u};
}

__global__ void __launch_bounds__(256) astar_ref_kernel(RefDev d) {
  __shared__ uint32_t s_cell[8][64];
  __shared__ uint32_t s_f[8][64];
  __shared__ RefItem s_pop[8][GPQ_ASTAR_REF_POPS];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wib;
  if (slot >= d.slots) return;
  RefItem* hp = d.heap + (size_t)slot * d.cap;
  uint16_t* fol = d.f_ol + (size_t)slot * d.fol_stride;
  uint32_t* cl = d.closed + (size_t)slot * d.words;
  uint32_t* cand_cell = s_cell[wib];
  uint32_t* cand_f = s_f[wib];
  RefItem* popped = s_pop[wib];
  const uint32_t W = d.width, H = d.height;

  for (;;) {
    uint32_t agent = 0;
    if (lane == 0) agent = atomicAdd(d.next_agent, 1u);  // get_new_agent
    agent = __shfl_sync(GPQ_FULL_MASK, agent, 0);
    if (agent >= d.n_agents) break;
    const gpq_astar_ref_agent ag = d.agents[agent];
    // init_agent (src/a_star.cu:170-242): f_ol and the closed set cleared, start inserted
    {
      uint4* p = reinterpret_cast<uint4*>(fol);
      const uint32_t n16 = (d.cells * 2u) / 16u;
      for (uint32_t i = lane; i < n16; i += 32u) p[i] = make_uint4(0u, 0u, 0u, 0u);
      for (uint32_t i = n16 * 8u + lane; i < d.cells; i += 32u) fol[i] = 0;
      for (uint32_t i = lane; i < d.words; i += 32u) cl[i] = 0u;
    }
    __syncwarp();
    const uint32_t gx = ag.goal % W, gy = ag.goal / W;
    const float h0 = gpq_astar_ref_h((int)(ag.start % W), (int)(ag.start / W), (int)gx, (int)gy);
    if (lane == 0) ref_store(hp, RefItem{gpq_f32_to_f16_bits(h0), gpq_f2u(h0), ag.start, 0u});
    __syncwarp();
    uint32_t n = 1, rounds = 0, pops = 0, found = 0, status = 0;
    float cost = 0.f;
    while (n > 0) {
      ++rounds;
      const uint32_t npop = min(n, GPQ_ASTAR_REF_POPS);
      for (uint32_t p = 0; p < npop; ++p) {
        const RefItem v = ref_pop(hp, n, lane);
        --n;
        if (lane == 0) popped[p] = v;
      }
      pops += npop;
      __syncwarp();
      // close the popped vertices; is one of them the goal?
      uint32_t goal_lane = 32u;
      if (lane < npop) {
        const RefItem v = popped[lane];
        atomicOr(&cl[v.cell >> 5], 1u << (v.cell & 31u));
      }
      const uint32_t gm = __ballot_sync(GPQ_FULL_MASK, lane < npop && popped[lane].cell == ag.goal);
      __syncwarp();
      if (gm) {  // found_goal: the agent ends, its open list is dropped
        goal_lane = (uint32_t)__ffs(gm) - 1u;
        found = 1;
        cost = gpq_f16_bits_to_f32(popped[goal_lane].f);
        n = 0;
        break;
      }
      // explore: candidate c = popped vertex c / 8, square cell c % 8 (the centre skipped)
#pragma unroll
      for (uint32_t r = 0; r < 2; ++r) {
        const uint32_t c = lane + 32u * r, p = c >> 3, k = c & 7u;
        uint32_t cell = 0xffffffffu, fh = 0;
        if (p < npop) {
          const RefItem v = popped[p];
          const int x = (int)(v.cell % W), y = (int)(v.cell / W);
          const uint32_t l = k >= 4u ? k + 1u : k;
          int nx = x - 1 + (int)(l % 3u), ny = y - 1 + (int)(l / 3u);
          nx = max(0, min((int)W - 1, nx));
          ny = max(0, min((int)H - 1, ny));
          const uint32_t nc = (uint32_t)ny * W + (uint32_t)nx;
          if (!bit(cl, nc) && !bit(d.wall, nc)) {
            const float g = GPQ_FADD(GPQ_FSUB(gpq_f16_bits_to_f32(v.f), gpq_astar_ref_h(x, y, (int)gx, (int)gy)),
                                     gpq_astar_ref_h(x, y, nx, ny));
            fh = gpq_f32_to_f16_bits(GPQ_FADD(g, gpq_astar_ref_h(nx, ny, (int)gx, (int)gy)));
            cell = nc;
          }
        }
        cand_cell[c] = cell;
        cand_f[c] = fh;
      }
      __syncwarp();
      // de-duplicate (src/a_star.cu:508-530): the first entry of a cell keeps the smallest
      // f of its duplicates; then the f_ol test (src/a_star.cu:537-560)
      uint32_t ins_cell[2], ins_f[2];
#pragma unroll
      for (uint32_t r = 0; r < 2; ++r) {
        const uint32_t c = lane + 32u * r;
        const uint32_t cell = cand_cell[c];
        uint32_t fh = cand_f[c];
        ins_cell[r] = 0xffffffffu;
        ins_f[r] = 0;
        if (cell == 0xffffffffu) continue;
        bool first = true;
        for (uint32_t o = 0; o < 64u; ++o) {
          if (cand_cell[o] != cell || o == c) continue;
          if (o < c) { first = false; break; }
          fh = min(fh, cand_f[o]);  // halves >= 0: bit order = value order
        }
        if (!first) continue;
        const uint32_t old = fol[cell];
        if (old == 0u || old > fh) {
          ins_cell[r] = cell;
          ins_f[r] = fh;
        }
      }
      __syncwarp();
#pragma unroll
      for (uint32_t r = 0; r < 2; ++r)
        if (ins_cell[r] != 0xffffffffu) fol[ins_cell[r]] = (uint16_t)ins_f[r];
      // queue_insert_or_update of the survivors, in candidate order
#pragma unroll
      for (uint32_t r = 0; r < 2; ++r) {
        uint32_t m = __ballot_sync(GPQ_FULL_MASK, ins_cell[r] != 0xffffffffu);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1u;
          const uint32_t cell = __shfl_sync(GPQ_FULL_MASK, ins_cell[r], src);
          const uint32_t fh = __shfl_sync(GPQ_FULL_MASK, ins_f[r], src);
          if (n >= d.cap) {
            status = GPQ_ERR_QUEUE_FULL;
            continue;
          }
          ref_push(hp, n, ref_vertex(cell, fh, W, ag.goal), lane);
          ++n;
        }
      }
      if (status) break;
    }
    if (lane == 0) {
      gpq_astar_ref_result res;
      res.found = found;
      res.cost = cost;
      res.pops = pops;
      res.rounds = rounds;
      res.status = status;
      res.reserved = 0;
      d.results[agent] = res;
    }
    __syncwarp();
  }
}

__global__ void astar_ref_map_kernel(const uint8_t* map, uint32_t cells, uint32_t* wall) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < (cells + 31u) / 32u; w += gridDim.x * blockDim.x) {
    uint32_t v = 0;
    for (uint32_t b = 0; b < 32u; ++b) {
      const uint32_t c = w * 32u + b;
      if (c < cells && map[c]) v |= 1u << b;
    }
    wall[w] = v;
  }
}

}  // namespace

struct gpq_astar_ref {
  gpq_astar_ref_config cfg{};
  cudaStream_t own = nullptr;
  uint32_t cells = 0, words = 0;
  RefItem* heap = nullptr;
  uint16_t* f_ol = nullptr;
  uint32_t* closed = nullptr;
  uint32_t* wall = nullptr;
  uint8_t* map = nullptr;
  gpq_astar_ref_agent* agents = nullptr;
  gpq_astar_ref_result* results = nullptr;
  uint32_t agent_cap = 0;
  uint32_t* next = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  float last_ms = 0.f;
  ~gpq_astar_ref() {
    if (own) cudaStreamSynchronize(own);
    for (void* p : {(void*)heap, (void*)f_ol, (void*)closed, (void*)wall, (void*)map, (void*)agents, (void*)results,
                    (void*)next})
      if (p) cudaFree(p);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (own) cudaStreamDestroy(own);
  }
};

extern "C" {

gpq_status gpq_astar_ref_create(const gpq_astar_ref_config* cfg_in, gpq_astar_ref** out) {
  GPQ_CHECK_ARG(cfg_in && out, "NULL argument");
  *out = nullptr;
  gpq_astar_ref_config c = *cfg_in;
  GPQ_CHECK_ARG(c.width >= 1 && c.height >= 1 && (uint64_t)c.width * c.height <= (1u << 24),
                "width * height must be in [1, 2^24]");
  if (c.slots == 0) c.slots = 2048;
  GPQ_CHECK_ARG(c.slots <= 65536, "slots must be <= 65536");
  const uint32_t cells = c.width * c.height;
  if (c.open_capacity == 0) c.open_capacity = std::max(64u, 4u * cells);
  std::unique_ptr<gpq_astar_ref> h(new (std::nothrow) gpq_astar_ref());
  if (!h) return GPQ_ERR_NOMEM;
  h->cfg = c;
  h->cells = cells;
  h->words = (cells + 31u) / 32u;
  GPQ_CUDA_TRY(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  GPQ_CUDA_TRY(cudaEventCreate(&h->ev[0]));
  GPQ_CUDA_TRY(cudaEventCreate(&h->ev[1]));
  GPQ_CUDA_TRY(cudaMalloc(&h->heap, (size_t)c.slots * c.open_capacity * sizeof(RefItem)));
  // f_ol rows padded to 16 bytes so the clears use 16-byte stores
  const size_t fol_row = (size_t)((cells + 7u) & ~7u) * 2u;
  GPQ_CUDA_TRY(cudaMalloc(&h->f_ol, (size_t)c.slots * fol_row));
  GPQ_CUDA_TRY(cudaMalloc(&h->closed, (size_t)c.slots * h->words * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&h->wall, (size_t)h->words * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&h->map, cells));
  GPQ_CUDA_TRY(cudaMalloc(&h->next, sizeof(uint32_t)));
  *out = h.release();
  return GPQ_OK;
}

gpq_status gpq_astar_ref_destroy(gpq_astar_ref* h) {
  if (!h) return GPQ_ERR_INVALID;
  delete h;
  return GPQ_OK;
}

gpq_status gpq_astar_ref_solve(gpq_astar_ref* h, const uint8_t* map, const gpq_astar_ref_agent* agents, uint32_t n,
                               gpq_astar_ref_result* results, void* stream) {
  GPQ_CHECK_ARG(h && map && (agents || n == 0) && (results || n == 0), "NULL argument");
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  const gpq_astar_ref_config& c = h->cfg;
  for (uint32_t i = 0; i < n; ++i)
    GPQ_CHECK_ARG(agents[i].start < h->cells && agents[i].goal < h->cells, "agent start/goal outside the map");
  if (n > h->agent_cap) {
    if (h->agents) cudaFree(h->agents);
    if (h->results) cudaFree(h->results);
    h->agents = nullptr;
    h->results = nullptr;
    h->agent_cap = 0;
    GPQ_CUDA_TRY(cudaMalloc(&h->agents, (size_t)n * sizeof(gpq_astar_ref_agent)));
    GPQ_CUDA_TRY(cudaMalloc(&h->results, (size_t)n * sizeof(gpq_astar_ref_result)));
    h->agent_cap = n;
  }
  if (n == 0) return GPQ_OK;
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->map, map, h->cells, cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->agents, agents, (size_t)n * sizeof(gpq_astar_ref_agent), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemsetAsync(h->next, 0, sizeof(uint32_t), st));
  astar_ref_map_kernel<<<std::max(1u, std::min((h->words + 255u) / 256u, 1024u)), 256, 0, st>>>(h->map, h->cells,
                                                                                              h->wall);
  GPQ_CUDA_TRY(cudaGetLastError());
  RefDev d;
  d.width = c.width;
  d.height = c.height;
  d.cells = h->cells;
  d.words = h->words;
  d.wall = h->wall;
  d.agents = h->agents;
  d.results = h->results;
  d.n_agents = n;
  d.next_agent = h->next;
  d.heap = h->heap;
  d.cap = c.open_capacity;
  d.f_ol = h->f_ol;
  d.fol_stride = (h->cells + 7u) & ~7u;
  d.closed = h->closed;
  d.slots = std::min(c.slots, std::max(1u, n));
  const uint32_t warps_per_cta = 8;
  GPQ_CUDA_TRY(cudaEventRecord(h->ev[0], st));
  astar_ref_kernel<<<(d.slots + warps_per_cta - 1) / warps_per_cta, warps_per_cta * 32, 0, st>>>(d);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaEventRecord(h->ev[1], st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(results, h->results, (size_t)n * sizeof(gpq_astar_ref_result), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  GPQ_CUDA_TRY(cudaEventElapsedTime(&h->last_ms, h->ev[0], h->ev[1]));
  return GPQ_OK;
}

gpq_status gpq_astar_ref_last_ms(gpq_astar_ref* h, float* ms) {
  GPQ_CHECK_ARG(h && ms, "NULL argument");
  *ms = h->last_ms;
  return GPQ_OK;
}

// The reference's random map (src/a_star.cu:747-765): `squares` obstacle squares at
// uniform positions, side max(1, (int)(-size_mean * ln u)), clipped at the map edge;
// draws from this project's counter-based generator keyed by seed.
gpq_status gpq_astar_ref_map(uint32_t width, uint32_t height, float obstacle_frac, float size_mean, uint64_t seed,
                             uint8_t* map) {
  GPQ_CHECK_ARG(map && width >= 1 && height >= 1 && (uint64_t)width * height <= (1u << 24), "map size");
  GPQ_CHECK_ARG(obstacle_frac >= 0.f && obstacle_frac <= 16.f && size_mean >= 0.f, "obstacle parameters");
  std::memset(map, 0, (size_t)width * height);
  const uint32_t squares = (uint32_t)((double)obstacle_frac * width * height);
  for (uint32_t i = 0; i < squares; ++i) {
    const uint32_t x = gpq_uniform_below(gpq_draw(seed, i, 0x4f425331u, 0), width);
    const uint32_t y = gpq_uniform_below(gpq_draw(seed, i, 0x4f425331u, 1), height);
    const float u = gpq_unit_open0(gpq_draw(seed, i, 0x4f425331u, 2));
    const float len = size_mean * (0.0f - gpq_logf(u));
    const int s = std::max(1, (int)len);
    for (int dy = 0; dy < s && y + dy < height; ++dy)
      for (int dx = 0; dx < s && x + dx < width; ++dx) map[(size_t)(y + dy) * width + (x + dx)] = 1;
  }
  return GPQ_OK;
}

// Agents with uniformly random free start and goal cells (src/a_star.cu:768-789), drawn
// from this project's generator: agent i redraws its start (goal) until the cell is free.
gpq_status gpq_astar_ref_agents(const uint8_t* map, uint32_t width, uint32_t height, uint32_t n, uint64_t seed,
                                gpq_astar_ref_agent* out) {
  GPQ_CHECK_ARG(map && (out || n == 0), "NULL argument");
  const uint64_t cells = (uint64_t)width * height;
  GPQ_CHECK_ARG(cells >= 1 && cells <= (1u << 24), "map size");
  bool any = false;
  for (uint64_t c = 0; c < cells && !any; ++c) any = map[c] == 0;
  GPQ_CHECK_ARG(any, "the map has no free cell");
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t k = 0;
    auto pick = [&](uint32_t which) {
      for (;;) {
        const uint32_t c = gpq_uniform_below(gpq_draw(seed, i, 0x41474e54u + which, k++), (uint32_t)cells);
        if (!map[c]) return c;
      }
    };
    out[i].start = pick(0);
    out[i].goal = pick(1);
  }
  return GPQ_OK;
}

}  // extern "C"
