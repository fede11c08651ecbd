// Host side of the A* engine (gpq_astar_*): instance layout, buffers, the persistent
// launch and the per-instance results.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "astar.cuh"
#include "host_common.h"

using gpq::set_last_error;

struct gpq_astar {
  gpq_astar_config cfg{};
  cudaStream_t own = nullptr;
  cudaEvent_t ev[4] = {};
  // device buffers and their capacities
  uint32_t* gcost = nullptr;
  uint8_t* pred = nullptr;  // [cap_cells + kAstarPredSlack]
  uint64_t cap_cells = 0;
  uint32_t* blk = nullptr;
  uint64_t* word0 = nullptr;
  AstarInstDev* inst = nullptr;
  unsigned long long* fin = nullptr;   // [n][2]
  unsigned long long* pout = nullptr;  // [n][3]
  uint32_t cap_inst = 0;
  AstarTileDev* tiles = nullptr;
  uint2* inbox = nullptr;
  uint2* open = nullptr;
  uint32_t* al = nullptr;
  uint32_t cap_tiles = 0;
  AstarCtl* ctl = nullptr;
  uint32_t* path_buf = nullptr;
  uint32_t path_cap = 0;
  // last solve
  std::vector<AstarInstDev> h_inst;
  std::vector<uint64_t> h_word0;
  uint32_t n_inst = 0, n_tiles = 0;
  uint64_t n_cells = 0;
  float total_ms = 0.f, search_ms = 0.f;
  uint32_t rounds = 0, grid = 0, block = 0;
  uint64_t visits = 0;
  bool solved = false;
};

namespace {

template <class T>
gpq_status grow(T** p, uint64_t have, uint64_t need) {
  if (need <= have && *p) return GPQ_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  GPQ_CUDA_TRY(cudaMalloc(p, std::max<uint64_t>(need, 1) * sizeof(T)));
  return GPQ_OK;
}

#define GPQ_TRY(expr)                  \
  do {                                 \
    gpq_status s_ = (expr);            \
    if (s_ != GPQ_OK) return s_;       \
  } while (0)

bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }

}  // namespace

namespace gpq {

gpq_status astar_normalize(gpq_astar_config& c) {
  if (c.tile == 0) c.tile = 64;
  GPQ_CHECK_ARG(is_pow2(c.tile) && c.tile >= 8 && c.tile <= 128, "tile must be a power of two in [8, 128]");
  if (c.inbox_capacity == 0) c.inbox_capacity = 8 * c.tile;
  if (c.open_capacity == 0) c.open_capacity = c.tile * c.tile;
  GPQ_CHECK_ARG(c.tile_worker <= 1, "tile_worker must be 0 (CTA) or 1 (warp)");
  if (c.frontier_capacity == 0) c.frontier_capacity = c.tile_worker ? 256 : 2048;
  GPQ_CHECK_ARG(c.frontier_capacity >= 64 && c.frontier_capacity <= 8192, "frontier_capacity in [64, 8192]");
  if (c.block_threads == 0) c.block_threads = 256;
  GPQ_CHECK_ARG(c.block_threads == 64 || c.block_threads == 128 || c.block_threads == 256,
                "block_threads must be 64, 128 or 256");
  if (c.max_rounds == 0) c.max_rounds = 1u << 20;
  return GPQ_OK;
}

}  // namespace gpq

extern "C" {

gpq_status gpq_astar_create(const gpq_astar_config* cfg, gpq_astar** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  gpq_astar_config c{};
  if (cfg) c = *cfg;
  GPQ_TRY(gpq::astar_normalize(c));
  gpq_astar* a = new (std::nothrow) gpq_astar();
  if (!a) return GPQ_ERR_NOMEM;
  a->cfg = c;
  cudaError_t e = cudaStreamCreateWithFlags(&a->own, cudaStreamNonBlocking);
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&a->ev[i]);
  if (e == cudaSuccess) e = cudaMalloc(&a->ctl, sizeof(AstarCtl));
  if (e != cudaSuccess) {
    set_last_error("gpq_astar_create: %s", cudaGetErrorString(e));
    gpq_astar_destroy(a);
    return GPQ_ERR_CUDA;
  }
  *out = a;
  return GPQ_OK;
}

gpq_status gpq_astar_destroy(gpq_astar* a) {
  if (!a) return GPQ_OK;
  void* bufs[] = {a->gcost, a->pred, a->blk, a->word0, a->inst, a->fin, a->pout, a->tiles, a->inbox, a->open, a->al,
                  a->ctl, a->path_buf};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (auto& e : a->ev)
    if (e) cudaEventDestroy(e);
  if (a->own) cudaStreamDestroy(a->own);
  delete a;
  return GPQ_OK;
}

gpq_status gpq_astar_query(uint64_t base_seed, uint32_t index, uint32_t conn, uint32_t side_lo, uint32_t side_hi,
                           double dens_lo, double dens_hi, gpq_astar_grid* out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  GPQ_CHECK_ARG(conn == 4 || conn == 8, "conn must be 4 or 8");
  GPQ_CHECK_ARG(side_lo >= 2 && side_lo <= side_hi && side_hi <= 65535, "need 2 <= side_lo <= side_hi <= 65535");
  GPQ_CHECK_ARG(dens_lo >= 0.0 && dens_lo <= dens_hi && dens_hi < 1.0, "need 0 <= dens_lo <= dens_hi < 1");
  const uint64_t seed = base_seed + index;
  const double u0 = (double)(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN, 0, 0) >> 11) * 0x1.0p-53;
  const double u1 = (double)(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN, 0, 1) >> 11) * 0x1.0p-53;
  uint32_t side = (uint32_t)std::floor((double)side_lo * std::exp2(u0 * std::log2((double)side_hi / side_lo)));
  side = std::min(std::max(side, side_lo), side_hi);
  const uint32_t thr = (uint32_t)((dens_lo + (dens_hi - dens_lo) * u1) * 16777216.0);
  const uint32_t cells = side * side;
  uint32_t s = 0, g = 0;
  for (uint32_t k = 0;; ++k) {
    s = gpq_uniform_below(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN, k, 2), cells);
    if (!gpq_astar_raw_blocked(seed, thr, s)) break;
  }
  for (uint32_t k = 0;; ++k) {
    g = gpq_uniform_below(gpq_draw(seed, GPQ_ASTAR_QUERY_DOMAIN, k, 3), cells);
    if (g != s && !gpq_astar_raw_blocked(seed, thr, g)) break;
  }
  *out = gpq_astar_grid{seed, side, side, thr, conn, s, g};
  return GPQ_OK;
}

}  // extern "C"

// One launch over the batch with the current tile capacities.
static gpq_status astar_solve_pass(gpq_astar* a, const gpq_astar_grid* grids, uint32_t n, gpq_astar_result* results,
                                   cudaStream_t st) {
  const gpq_astar_config& c = a->cfg;
  const uint32_t ts = c.tile;
  // layout
  a->h_inst.assign(n, AstarInstDev{});
  a->h_word0.assign(n, 0);
  uint64_t cell0 = 0;
  uint32_t tile0 = 0;
  uint64_t max_cells = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const gpq_astar_grid& g = grids[i];
    GPQ_CHECK_ARG(g.width >= 1 && g.height >= 1 && (uint64_t)g.width * g.height <= 0xFFFFFFFFull,
                  "grid must have 1 .. 2^32-1 cells");
    GPQ_CHECK_ARG(g.width <= 65535 && g.height <= 65535, "grid sides must be <= 65535");
    GPQ_CHECK_ARG(g.conn == 4 || g.conn == 8, "conn must be 4 or 8");
    const uint64_t cells = (uint64_t)g.width * g.height;
    GPQ_CHECK_ARG(g.start < cells && g.goal < cells, "start and goal must be cells of the grid");
    AstarInstDev& I = a->h_inst[i];
    I.g = g;
    I.cell0 = cell0;
    I.tile0 = tile0;
    I.tiles_x = (g.width + ts - 1) / ts;
    I.tiles_y = (g.height + ts - 1) / ts;
    I.ub = (g.start == g.goal) ? 0u : kAstarInf;
    I.delta = c.window ? c.window : (g.conn == 4 ? 4u : 40u);
    I.gx = g.goal % g.width;
    I.gy = g.goal / g.width;
    const uint32_t h0 = gpq_astar_h(g.conn, g.start, g.goal, g.width);
    I.bound = (uint32_t)std::min<uint64_t>((uint64_t)h0 + I.delta, 0xFFFFFFFEull);
    I.done = 0;
    a->h_word0[i] = cell0 / 32;
    cell0 += (cells + 31) / 32 * 32;
    const uint64_t nt = (uint64_t)I.tiles_x * I.tiles_y;
    GPQ_CHECK_ARG((uint64_t)tile0 + nt < 0x7FFFFFFFull, "too many tiles");
    tile0 += (uint32_t)nt;
    max_cells = std::max(max_cells, cells);
  }
  a->n_inst = n;
  a->n_tiles = tile0;
  a->n_cells = cell0;
  // buffers
  GPQ_TRY(grow(&a->gcost, a->cap_cells, cell0));
  GPQ_TRY(grow(&a->blk, a->cap_cells / 32 + 1, cell0 / 32 + 1));  // +1: tile loads read one word ahead
  GPQ_TRY(grow(&a->pred, a->cap_cells + kAstarPredSlack, cell0 + kAstarPredSlack));
  a->cap_cells = std::max(a->cap_cells, cell0);
  if (n > a->cap_inst) {
    GPQ_TRY(grow(&a->word0, 0, n));
    GPQ_TRY(grow(&a->inst, 0, n));
    GPQ_TRY(grow(&a->fin, 0, 2ull * n));
    GPQ_TRY(grow(&a->pout, 0, 3ull * n));
    a->cap_inst = n;
  }
  if (tile0 > a->cap_tiles) {
    GPQ_TRY(grow(&a->tiles, 0, tile0));
    GPQ_TRY(grow(&a->inbox, 0, 2ull * tile0 * c.inbox_capacity));
    GPQ_TRY(grow(&a->open, 0, (uint64_t)tile0 * c.open_capacity));
    GPQ_TRY(grow(&a->al, 0, 2ull * tile0));
    a->cap_tiles = tile0;
  }
  AstarDev d{};
  d.inst = a->inst;
  d.tiles = a->tiles;
  d.gcost = a->gcost;
  d.blk = a->blk;
  d.pred = a->pred;
  d.inbox = a->inbox;
  d.open = a->open;
  d.al = a->al;
  d.ctl = a->ctl;
  d.n_inst = n;
  d.n_tiles = tile0;
  d.in_cap = c.inbox_capacity;
  d.open_cap = c.open_capacity;
  d.ts = ts;
  d.lts = (uint32_t)__builtin_ctz(ts);
  d.max_rounds = c.max_rounds;
  d.frontier_cap = c.frontier_capacity;
  d.spin_limit = gpq::spin_limit();
  // launch geometry
  const void* kern = c.tile_worker ? (const void*)astar_persistent_kernel<true> : (const void*)astar_persistent_kernel<false>;
  const size_t smem = astar_worker_smem_bytes(ts, c.frontier_capacity) * (c.tile_worker ? c.block_threads / 32 : 1);
  GPQ_CHECK_ARG(smem <= 227u * 1024u, "tile, frontier_capacity and workers need more than 227 KB of shared memory");
  GPQ_CUDA_TRY(gpq::raise_smem_limit(kern, (int)smem));
  int dev = 0, sms = 0, per_sm = 0;
  GPQ_CUDA_TRY(cudaGetDevice(&dev));
  GPQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GPQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)c.block_threads, smem));
  if (per_sm < 1) {
    set_last_error("astar: kernel does not fit on an SM (block %u, smem %zu)", c.block_threads, smem);
    return GPQ_ERR_INVALID;
  }
  if (c.ctas_per_sm) {
    per_sm = std::min<int>(per_sm, (int)c.ctas_per_sm);
  } else {
    // a search keeps about sqrt(tiles) tiles of an instance active at a time (its
    // frontier); tile workers beyond the active tiles only add grid-barrier work
    double active = 0.0;
    for (uint32_t i = 0; i < n; ++i) active += std::sqrt((double)a->h_inst[i].tiles_x * a->h_inst[i].tiles_y);
    const double workers = (double)sms * (c.tile_worker ? c.block_threads / 32 : 1);
    per_sm = std::min<int>(per_sm, std::max<int>(1, (int)std::ceil(active / workers)));
  }
  const uint32_t grid = (uint32_t)(per_sm * sms);
  a->grid = grid;
  a->block = c.block_threads;

  GPQ_CUDA_TRY(cudaMemcpyAsync(a->inst, a->h_inst.data(), n * sizeof(AstarInstDev), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(a->word0, a->h_word0.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaEventRecord(a->ev[0], st));
  GPQ_CUDA_TRY(cudaMemsetAsync(a->gcost, 0xff, cell0 * sizeof(uint32_t), st));
  GPQ_CUDA_TRY(cudaMemsetAsync(a->ctl, 0, sizeof(AstarCtl), st));
  const uint64_t words = cell0 / 32;
  astar_bitmap_kernel<<<(uint32_t)std::min<uint64_t>((words + 255) / 256, (uint64_t)sms * 64), 256, 0, st>>>(
      a->inst, n, a->word0, words, a->blk);
  astar_tiles_init_kernel<<<std::min<uint32_t>(n, 4096), 128, 0, st>>>(d, nullptr, n);
  astar_init_kernel<<<(n + 127) / 128, 128, 0, st>>>(d, nullptr, n, 0u);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaEventRecord(a->ev[1], st));
  uint32_t s0 = 0, step_rounds = 0;
  void* args[] = {&d, &s0, &step_rounds};
  GPQ_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(c.block_threads), args, smem, st));
  GPQ_CUDA_TRY(cudaEventRecord(a->ev[2], st));
  GPQ_CUDA_TRY(cudaMemsetAsync(a->fin, 0, 2ull * n * sizeof(unsigned long long), st));
  // about 16 blocks per SM over all instances, at least 64 per instance
  const uint32_t fx = (uint32_t)std::min<uint64_t>((max_cells + 255) / 256, std::max<uint64_t>(64, 16ull * sms / n));
  astar_finalize_kernel<<<dim3(fx, n), 256, 0, st>>>(d, nullptr, a->fin);
  if (max_cells >= kAstarPredBytesCells) astar_pred_kernel<<<dim3(fx, n), 256, 0, st>>>(d, nullptr);
  astar_path_kernel<<<n, kPathThreads, 0, st>>>(d, nullptr, n, a->pout, 0xFFFFFFFFu, nullptr, 0);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaEventRecord(a->ev[3], st));
  std::vector<unsigned long long> fin(2ull * n), pout(3ull * n);
  AstarCtl ctl{};
  GPQ_CUDA_TRY(cudaMemcpyAsync(fin.data(), a->fin, fin.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(pout.data(), a->pout, pout.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(a->h_inst.data(), a->inst, n * sizeof(AstarInstDev), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(&ctl, a->ctl, sizeof(AstarCtl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  GPQ_CUDA_TRY(cudaEventElapsedTime(&a->total_ms, a->ev[0], a->ev[3]));
  GPQ_CUDA_TRY(cudaEventElapsedTime(&a->search_ms, a->ev[1], a->ev[2]));
  a->rounds = ctl.rounds;
  a->visits = ctl.visits;
  a->solved = true;
  for (uint32_t i = 0; i < n; ++i) {
    const AstarInstDev& I = a->h_inst[i];
    gpq_astar_result& r = results[i];
    r.cost = I.ub;
    r.expanded = fin[2 * i];
    r.gsum = fin[2 * i + 1];
    r.path_len = (uint32_t)pout[3 * i];
    r.path_hash = pout[3 * i + 1];
    r.pops = I.pops;
    r.windows = I.windows;
    int32_t status = (int32_t)I.err;
    if (status == 0 && ctl.err) status = (int32_t)ctl.err;
    if (status == 0 && !I.done) status = GPQ_ERR_TIMEOUT;
    if (status == 0 && pout[3 * i + 2]) status = GPQ_ERR_INVALID;  // canonical walk found no predecessor
    r.status = status;
  }
  if (ctl.err) {
    set_last_error("astar: device error %u after %u rounds", ctl.err, ctl.rounds);
    return (gpq_status)ctl.err;
  }
  return GPQ_OK;
}

extern "C" {

// A batch in which some instance overflowed its tile buffers runs again with four times
// the capacities (at most twice); the capacities stay for later calls.
gpq_status gpq_astar_solve(gpq_astar* a, const gpq_astar_grid* grids, uint32_t n, gpq_astar_result* results,
                           void* stream) {
  GPQ_CHECK_ARG(a && grids && results, "NULL argument");
  GPQ_CHECK_ARG(n >= 1 && n <= 65535, "need 1 <= n <= 65535 instances per solve");
  const cudaStream_t st = gpq::as_stream(stream, a->own);
  float total = 0.f, search = 0.f;
  uint32_t rounds = 0;
  uint64_t visits = 0;
  for (int attempt = 0;; ++attempt) {
    const gpq_status s = astar_solve_pass(a, grids, n, results, st);
    total += a->total_ms;
    search += a->search_ms;
    rounds += a->rounds;
    visits += a->visits;
    if (s != GPQ_OK) return s;
    bool overflow = false;
    for (uint32_t i = 0; i < n; ++i)
      overflow |= results[i].status == GPQ_ERR_QUEUE_FULL || results[i].status == GPQ_ERR_INSERT_FULL;
    if (!overflow || attempt == 2) break;
    a->cfg.inbox_capacity *= 4;
    a->cfg.open_capacity *= 4;
    a->cap_tiles = 0;  // reallocate the tile buffers at the new capacities
  }
  a->total_ms = total;
  a->search_ms = search;
  a->rounds = rounds;
  a->visits = visits;
  return GPQ_OK;
}

gpq_status gpq_astar_last_stats(gpq_astar* a, float* total_ms, float* search_ms, uint32_t* rounds,
                                uint64_t* tile_visits, uint32_t* grid, uint32_t* block) {
  GPQ_CHECK_ARG(a, "NULL handle");
  if (!a->solved) return GPQ_ERR_NOT_READY;
  if (total_ms) *total_ms = a->total_ms;
  if (search_ms) *search_ms = a->search_ms;
  if (rounds) *rounds = a->rounds;
  if (tile_visits) *tile_visits = a->visits;
  if (grid) *grid = a->grid;
  if (block) *block = a->block;
  return GPQ_OK;
}

gpq_status gpq_astar_path(gpq_astar* a, uint32_t index, uint32_t* cells, uint32_t capacity, uint32_t* length,
                          void* stream) {
  GPQ_CHECK_ARG(a && length, "NULL argument");
  if (!a->solved) return GPQ_ERR_NOT_READY;
  GPQ_CHECK_ARG(index < a->n_inst, "index out of range");
  const cudaStream_t st = gpq::as_stream(stream, a->own);
  if (capacity > a->path_cap) {
    GPQ_TRY(grow(&a->path_buf, 0, capacity));
    a->path_cap = capacity;
  }
  AstarDev d{};
  d.inst = a->inst;
  d.gcost = a->gcost;
  d.blk = a->blk;
  d.pred = a->pred;
  d.n_inst = a->n_inst;
  astar_path_kernel<<<a->n_inst, kPathThreads, 0, st>>>(d, nullptr, a->n_inst, a->pout, index, a->path_buf,
                                                                   capacity);
  GPQ_CUDA_TRY(cudaGetLastError());
  unsigned long long po[3];
  GPQ_CUDA_TRY(cudaMemcpyAsync(po, a->pout + 3ull * index, sizeof(po), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  *length = (uint32_t)po[0];
  if (cells && capacity) {
    GPQ_CUDA_TRY(cudaMemcpyAsync(cells, a->path_buf, std::min<uint32_t>(capacity, *length) * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return *length > capacity ? GPQ_ERR_INVALID : GPQ_OK;
}

gpq_status gpq_astar_gcost(gpq_astar* a, uint32_t index, uint32_t* g, uint64_t capacity, void* stream) {
  GPQ_CHECK_ARG(a && g, "NULL argument");
  if (!a->solved) return GPQ_ERR_NOT_READY;
  GPQ_CHECK_ARG(index < a->n_inst, "index out of range");
  const AstarInstDev& I = a->h_inst[index];
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  GPQ_CHECK_ARG(capacity >= cells, "capacity below width * height");
  const cudaStream_t st = gpq::as_stream(stream, a->own);
  GPQ_CUDA_TRY(cudaMemcpyAsync(g, a->gcost + I.cell0, cells * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

// Headless image of instance `index` (the reference's dumpResult, src/a_star.cu:596-690,
// writes a P6 image of its agents' map; here one search is drawn): binary PPM, one pixel
// per cell, row 0 at the top.  Colours: free cell not reached black (0,0,0); blocked grey
// (90,90,90); reached but beyond the optimal cost dark blue (0,0,110); expanded
// (g + h <= C*) light blue (60,140,255); the canonical path red (255,40,40); start green
// (0,220,0); goal yellow (255,230,0).
gpq_status gpq_astar_write_ppm(gpq_astar* a, uint32_t index, const char* filename, void* stream) {
  GPQ_CHECK_ARG(a && filename, "NULL argument");
  if (!a->solved) return GPQ_ERR_NOT_READY;
  GPQ_CHECK_ARG(index < a->n_inst, "index out of range");
  const gpq_astar_grid G = a->h_inst[index].g;
  const uint64_t cells = (uint64_t)G.width * G.height;
  GPQ_CHECK_ARG(cells <= (1ull << 28), "grid above 2^28 cells");
  std::vector<uint32_t> g(cells);
  gpq_status st = gpq_astar_gcost(a, index, g.data(), cells, stream);
  if (st != GPQ_OK) return st;
  uint32_t len = 0;
  st = gpq_astar_path(a, index, nullptr, 0, &len, stream);
  if (st != GPQ_OK && st != GPQ_ERR_INVALID) return st;
  std::vector<uint32_t> path(len);
  if (len) {
    st = gpq_astar_path(a, index, path.data(), len, &len, stream);
    if (st != GPQ_OK) return st;
  }
  const uint32_t cs = g[G.goal];
  std::vector<unsigned char> px(cells * 3, 0);
  auto put = [&](uint64_t c, unsigned char r, unsigned char gg, unsigned char b) {
    px[3 * c] = r;
    px[3 * c + 1] = gg;
    px[3 * c + 2] = b;
  };
  for (uint64_t c = 0; c < cells; ++c) {
    const uint32_t cell = (uint32_t)c;
    if (gpq_astar_blocked(&G, cell)) {
      put(c, 90, 90, 90);
    } else if (g[c] != GPQ_ASTAR_INF) {
      const bool exp = cs == GPQ_ASTAR_INF || (uint64_t)g[c] + gpq_astar_h(G.conn, cell, G.goal, G.width) <= cs;
      if (exp) put(c, 60, 140, 255);
      else put(c, 0, 0, 110);
    }
  }
  for (uint32_t i = 0; i < len; ++i) put(path[i], 255, 40, 40);
  put(G.start, 0, 220, 0);
  put(G.goal, 255, 230, 0);
  FILE* f = std::fopen(filename, "wb");
  if (!f) {
    set_last_error("gpq_astar_write_ppm: cannot open %s", filename);
    return GPQ_ERR_INVALID;
  }
  const int hn = std::fprintf(f, "P6\n%u %u\n255\n", G.width, G.height);
  const size_t wn = std::fwrite(px.data(), 1, px.size(), f);
  const int cl = std::fclose(f);
  if (hn <= 0 || wn != px.size() || cl != 0) {
    set_last_error("gpq_astar_write_ppm: writing %s failed", filename);
    return GPQ_ERR_INVALID;
  }
  return GPQ_OK;
}

}  // extern "C"
