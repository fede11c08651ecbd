// Resident A* instances for serving (gpq_astar_session_*): instances are admitted into
// free ranges of one cell space (g values and blocked bits) and one tile space (tile
// records, inboxes, open arrays) reserved up front, stepped together by the persistent
// kernel for a bounded number of rounds per launch, and retired when their search ends.
// Between launches the queues stay in device memory.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "astar.cuh"
#include "host_common.h"
#include "range_alloc.h"

using gpq::set_last_error;

struct gpq_astar_session {
  gpq_astar_config cfg{};
  cudaStream_t own = nullptr;
  uint64_t max_cells = 0;
  uint32_t max_tiles = 0, max_inst = 0;
  // device state
  uint32_t* gcost = nullptr;
  uint8_t* pred = nullptr;  // [max_cells + kAstarPredSlack]
  uint32_t* blk = nullptr;
  AstarInstDev* inst = nullptr;
  AstarTileDev* tiles = nullptr;
  uint2* inbox = nullptr;
  uint2* open = nullptr;
  uint32_t* al = nullptr;
  AstarCtl* ctl = nullptr;
  uint8_t* on = nullptr;           // slot in use
  uint32_t* list = nullptr;        // [max_inst] scratch slot list
  uint32_t* list_n = nullptr;
  AstarInstDev* staged = nullptr;  // [max_inst] admitted records before the scatter
  unsigned long long* fin = nullptr;
  unsigned long long* pout = nullptr;
  // host state
  gpq::RangeAlloc cells, tile_space;
  std::vector<uint32_t> free_slots;
  std::vector<uint8_t> h_on;
  std::vector<gpq_astar_grid> h_grid;
  std::vector<AstarInstDev> pending;  // admitted, not yet initialized on the device
  std::vector<uint32_t> pending_slot;
  uint32_t high = 0;                  // slots [0, high) may be in use
  uint32_t active = 0;
  uint32_t next_round = 0;
  AstarInstDev* h_stage = nullptr;    // pinned
  uint32_t* h_list = nullptr;         // pinned
  int grid = 0;
  size_t smem = 0;
  const void* kern = nullptr;
};

namespace {

template <class T>
cudaError_t dmalloc(T** p, uint64_t n) {
  return cudaMalloc(p, std::max<uint64_t>(n, 1) * sizeof(T));
}

__global__ void astar_scatter_kernel(AstarInstDev* inst, const AstarInstDev* staged, const uint32_t* list, uint32_t n,
                                     uint8_t* on) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    inst[list[j]] = staged[j];
    on[list[j]] = 1;
  }
}

__global__ void astar_fill_g_kernel(const AstarInstDev* inst, const uint32_t* list, uint32_t* g) {
  const AstarInstDev& I = inst[list[blockIdx.y]];
  const uint64_t cells = (uint64_t)I.g.width * I.g.height;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < cells; c += (uint64_t)gridDim.x * blockDim.x)
    g[I.cell0 + c] = kAstarInf;
}

__global__ void astar_gather_kernel(const AstarInstDev* inst, const uint32_t* list, uint32_t n, AstarInstDev* out,
                                    uint8_t* on) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    out[j] = inst[list[j]];
    on[list[j]] = 0;
  }
}

AstarDev session_dev(const gpq_astar_session* s) {
  AstarDev d{};
  d.inst = s->inst;
  d.tiles = s->tiles;
  d.gcost = s->gcost;
  d.blk = s->blk;
  d.pred = s->pred;
  d.inbox = s->inbox;
  d.open = s->open;
  d.al = s->al;
  d.ctl = s->ctl;
  d.n_inst = s->high;
  d.n_tiles = s->max_tiles;
  d.in_cap = s->cfg.inbox_capacity;
  d.open_cap = s->cfg.open_capacity;
  d.ts = s->cfg.tile;
  d.lts = (uint32_t)__builtin_ctz(s->cfg.tile);
  d.max_rounds = 0;
  d.frontier_cap = s->cfg.frontier_capacity;
  d.spin_limit = gpq::spin_limit();
  return d;
}

// Device records of the admitted instances: scatter, g = inf, blocked bits, tiles, start.
gpq_status flush_pending(gpq_astar_session* s, cudaStream_t st) {
  const uint32_t n = (uint32_t)s->pending.size();
  if (n == 0) return GPQ_OK;
  std::copy(s->pending.begin(), s->pending.end(), s->h_stage);
  std::copy(s->pending_slot.begin(), s->pending_slot.end(), s->h_list);
  uint64_t max_cells = 0;
  for (const auto& I : s->pending) max_cells = std::max<uint64_t>(max_cells, (uint64_t)I.g.width * I.g.height);
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->staged, s->h_stage, n * sizeof(AstarInstDev), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->list, s->h_list, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  astar_scatter_kernel<<<(n + 127) / 128, 128, 0, st>>>(s->inst, s->staged, s->list, n, s->on);
  const AstarDev d = session_dev(s);
  for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
    const uint32_t nj = std::min<uint32_t>(65535, n - j0);
    const uint32_t gx = (uint32_t)std::min<uint64_t>((max_cells + 255) / 256, 256);
    astar_fill_g_kernel<<<dim3(gx, nj), 256, 0, st>>>(s->inst, s->list + j0, s->gcost);
    const uint32_t bx = (uint32_t)std::min<uint64_t>((max_cells / 32 + 256) / 256, 64);
    astar_bitmap_list_kernel<<<dim3(bx, nj), 256, 0, st>>>(s->inst, s->list + j0, s->blk);
  }
  astar_tiles_init_kernel<<<std::min<uint32_t>(n, 4096), 128, 0, st>>>(d, s->list, n);
  astar_init_kernel<<<(n + 127) / 128, 128, 0, st>>>(d, s->list, n, s->next_round & 1u);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));  // the staging buffers are reused
  s->pending.clear();
  s->pending_slot.clear();
  return GPQ_OK;
}

}  // namespace

extern "C" {

gpq_status gpq_astar_session_create(const gpq_astar_config* cfg, uint64_t max_cells, uint32_t max_tiles,
                                    uint32_t max_instances, gpq_astar_session** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  GPQ_CHECK_ARG(max_cells >= 32 && max_tiles >= 1 && max_instances >= 1 && max_instances <= (1u << 20),
                "need max_cells >= 32, max_tiles >= 1, 1 <= max_instances <= 2^20");
  gpq_astar_config c{};
  if (cfg) c = *cfg;
  const gpq_status st0 = gpq::astar_normalize(c);
  if (st0 != GPQ_OK) return st0;
  gpq_astar_session* s = new (std::nothrow) gpq_astar_session();
  if (!s) return GPQ_ERR_NOMEM;
  s->cfg = c;
  s->max_cells = (max_cells + 31) / 32 * 32;
  s->max_tiles = max_tiles;
  s->max_inst = max_instances;
  s->cells.reset(s->max_cells);
  s->tile_space.reset(max_tiles);
  s->h_on.assign(max_instances, 0);
  s->h_grid.assign(max_instances, gpq_astar_grid{});
  for (uint32_t i = max_instances; i-- > 0;) s->free_slots.push_back(i);
  cudaError_t e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = dmalloc(&s->gcost, s->max_cells);
  if (e == cudaSuccess) e = dmalloc(&s->blk, s->max_cells / 32 + 1);
  if (e == cudaSuccess) e = dmalloc(&s->pred, s->max_cells + kAstarPredSlack);
  if (e == cudaSuccess) e = dmalloc(&s->inst, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->tiles, max_tiles);
  if (e == cudaSuccess) e = dmalloc(&s->inbox, 2ull * max_tiles * c.inbox_capacity);
  if (e == cudaSuccess) e = dmalloc(&s->open, (uint64_t)max_tiles * c.open_capacity);
  if (e == cudaSuccess) e = dmalloc(&s->al, 2ull * max_tiles);
  if (e == cudaSuccess) e = dmalloc(&s->ctl, 1);
  if (e == cudaSuccess) e = dmalloc(&s->on, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->list, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->list_n, 1);
  if (e == cudaSuccess) e = dmalloc(&s->staged, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->fin, 2ull * max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->pout, 3ull * max_instances);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_stage, max_instances * sizeof(AstarInstDev));
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_list, max_instances * sizeof(uint32_t));
  if (e == cudaSuccess) {  // every slot starts (and ends) as a finished search
    std::vector<AstarInstDev> idle(max_instances);
    for (auto& I : idle) I.done = 1;
    e = cudaMemcpy(s->inst, idle.data(), idle.size() * sizeof(AstarInstDev), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(s->ctl, 0, sizeof(AstarCtl), s->own);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->on, 0, max_instances, s->own);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->tiles, 0, (size_t)max_tiles * sizeof(AstarTileDev), s->own);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->own);
  if (e != cudaSuccess) {
    set_last_error("gpq_astar_session_create: %s", cudaGetErrorString(e));
    gpq_astar_session_destroy(s);
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  }
  s->kern = c.tile_worker ? (const void*)astar_persistent_kernel<true> : (const void*)astar_persistent_kernel<false>;
  s->smem = astar_worker_smem_bytes(c.tile, c.frontier_capacity) * (c.tile_worker ? c.block_threads / 32 : 1);
  int dev = 0, sms = 0, per_sm = 0;
  GPQ_CUDA_TRY(gpq::raise_smem_limit(s->kern, (int)s->smem));
  GPQ_CUDA_TRY(cudaGetDevice(&dev));
  GPQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GPQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s->kern, (int)c.block_threads, s->smem));
  if (c.ctas_per_sm) per_sm = std::min<int>(per_sm, (int)c.ctas_per_sm);
  s->grid = per_sm * sms;
  *out = s;
  return GPQ_OK;
}

gpq_status gpq_astar_session_destroy(gpq_astar_session* s) {
  if (!s) return GPQ_OK;
  void* bufs[] = {s->gcost, s->pred, s->blk,    s->inst,   s->tiles, s->inbox, s->open, s->al,  s->ctl,
                  s->on,    s->list,   s->list_n, s->staged, s->fin,  s->pout};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (s->h_stage) cudaFreeHost(s->h_stage);
  if (s->h_list) cudaFreeHost(s->h_list);
  if (s->own) cudaStreamDestroy(s->own);
  delete s;
  return GPQ_OK;
}

gpq_status gpq_astar_session_admit(gpq_astar_session* s, const gpq_astar_grid* g, uint32_t* slot) {
  GPQ_CHECK_ARG(s && g && slot, "NULL argument");
  GPQ_CHECK_ARG(g->width >= 1 && g->height >= 1 && g->width <= 65535 && g->height <= 65535,
                "grid sides must be in [1, 65535]");
  GPQ_CHECK_ARG(g->conn == 4 || g->conn == 8, "conn must be 4 or 8");
  const uint64_t cells = (uint64_t)g->width * g->height;
  GPQ_CHECK_ARG(g->start < cells && g->goal < cells, "start and goal must be cells of the grid");
  const uint32_t ts = s->cfg.tile;
  const uint32_t tx = (g->width + ts - 1) / ts, ty = (g->height + ts - 1) / ts;
  const uint64_t need_cells = (cells + 31) / 32 * 32;
  if (s->free_slots.empty()) return GPQ_ERR_NOMEM;
  uint64_t c0 = 0, t0 = 0;
  if (!s->cells.alloc(need_cells, &c0)) return GPQ_ERR_NOMEM;
  if (!s->tile_space.alloc((uint64_t)tx * ty, &t0)) {
    s->cells.free(c0, need_cells);
    return GPQ_ERR_NOMEM;
  }
  const uint32_t i = s->free_slots.back();
  s->free_slots.pop_back();
  AstarInstDev I{};
  I.g = *g;
  I.cell0 = c0;
  I.tile0 = (uint32_t)t0;
  I.tiles_x = tx;
  I.tiles_y = ty;
  I.ub = (g->start == g->goal) ? 0u : kAstarInf;
  I.delta = s->cfg.window ? s->cfg.window : (g->conn == 4 ? 4u : 40u);
  I.gx = g->goal % g->width;
  I.gy = g->goal / g->width;
  const uint32_t h0 = gpq_astar_h(g->conn, g->start, g->goal, g->width);
  I.bound = (uint32_t)std::min<uint64_t>((uint64_t)h0 + I.delta, 0xFFFFFFFEull);
  s->pending.push_back(I);
  s->pending_slot.push_back(i);
  s->h_on[i] = 1;
  s->h_grid[i] = *g;
  s->high = std::max(s->high, i + 1);
  ++s->active;
  *slot = i;
  return GPQ_OK;
}

gpq_status gpq_astar_session_step(gpq_astar_session* s, uint32_t rounds, uint32_t* running, void* stream) {
  GPQ_CHECK_ARG(s, "NULL handle");
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  gpq_status r = flush_pending(s, st);
  if (r != GPQ_OK) return r;
  if (running) *running = s->active;
  if (s->active == 0) return GPQ_OK;
  AstarDev d = session_dev(s);
  uint32_t s0 = s->next_round, sr = rounds;
  void* args[] = {&d, &s0, &sr};
  GPQ_CUDA_TRY(cudaMemsetAsync(&s->ctl->bar, 0, sizeof(unsigned long long), st));
  GPQ_CUDA_TRY(cudaLaunchCooperativeKernel(s->kern, dim3(s->grid), dim3(s->cfg.block_threads), args, s->smem, st));
  AstarCtl ctl{};
  GPQ_CUDA_TRY(cudaMemcpyAsync(&ctl, s->ctl, sizeof(AstarCtl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (ctl.err) {
    set_last_error("astar session: device error %u at round %u", ctl.err, ctl.rounds);
    return (gpq_status)ctl.err;
  }
  s->next_round = ctl.rounds;
  return GPQ_OK;
}

gpq_status gpq_astar_session_collect(gpq_astar_session* s, uint32_t* slots, gpq_astar_result* results,
                                     uint32_t capacity, uint32_t* n_out, void* stream) {
  GPQ_CHECK_ARG(s && n_out, "NULL argument");
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  *n_out = 0;
  if (s->high == 0) return GPQ_OK;
  GPQ_CUDA_TRY(cudaMemsetAsync(s->list_n, 0, sizeof(uint32_t), st));
  astar_done_list_kernel<<<(s->high + 255) / 256, 256, 0, st>>>(s->inst, s->on, s->high, s->list, s->list_n);
  uint32_t n = 0;
  GPQ_CUDA_TRY(cudaMemcpyAsync(&n, s->list_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  n = std::min(n, capacity);
  if (n == 0) return GPQ_OK;
  const AstarDev d = session_dev(s);
  GPQ_CUDA_TRY(cudaMemsetAsync(s->fin, 0, 2ull * n * sizeof(unsigned long long), st));
  uint64_t max_cells = 0;
  // the list is on the device; size the finalize grid from the largest grid in the session
  for (uint32_t i = 0; i < s->high; ++i)
    if (s->h_on[i]) max_cells = std::max<uint64_t>(max_cells, (uint64_t)s->h_grid[i].width * s->h_grid[i].height);
  for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
    const uint32_t nj = std::min<uint32_t>(65535, n - j0);
    // a few blocks per resident search CTA over all instances, at least 64 per instance
    const uint32_t fx = (uint32_t)std::min<uint64_t>((max_cells + 255) / 256, std::max<uint64_t>(64, 4ull * s->grid / nj));
    astar_finalize_kernel<<<dim3(fx, nj), 256, 0, st>>>(d, s->list + j0, s->fin + 2ull * j0);
    if (max_cells >= kAstarPredBytesCells) astar_pred_kernel<<<dim3(fx, nj), 256, 0, st>>>(d, s->list + j0);
  }
  astar_path_kernel<<<n, kPathThreads, 0, st>>>(d, s->list, n, s->pout, 0xFFFFFFFFu, nullptr, 0);
  astar_gather_kernel<<<(n + 127) / 128, 128, 0, st>>>(s->inst, s->list, n, s->staged, s->on);
  GPQ_CUDA_TRY(cudaGetLastError());
  std::vector<unsigned long long> fin(2ull * n), pout(3ull * n);
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->h_list, s->list, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->h_stage, s->staged, n * sizeof(AstarInstDev), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(fin.data(), s->fin, fin.size() * 8, cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(pout.data(), s->pout, pout.size() * 8, cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (uint32_t j = 0; j < n; ++j) {
    const uint32_t i = s->h_list[j];
    const AstarInstDev& I = s->h_stage[j];
    gpq_astar_result r{};
    r.cost = I.ub;
    r.expanded = fin[2 * j];
    r.gsum = fin[2 * j + 1];
    r.path_len = (uint32_t)pout[3 * j];
    r.path_hash = pout[3 * j + 1];
    r.pops = I.pops;
    r.windows = I.windows;
    r.status = (int32_t)I.err;
    if (r.status == 0 && pout[3 * j + 2]) r.status = GPQ_ERR_INVALID;
    if (slots) slots[j] = i;
    if (results) results[j] = r;
    const uint64_t cells = (uint64_t)I.g.width * I.g.height;
    s->cells.free(I.cell0, (cells + 31) / 32 * 32);
    s->tile_space.free(I.tile0, (uint64_t)I.tiles_x * I.tiles_y);
    s->h_on[i] = 0;
    s->free_slots.push_back(i);
    --s->active;
  }
  while (s->high > 0 && !s->h_on[s->high - 1]) --s->high;
  *n_out = n;
  return GPQ_OK;
}

gpq_status gpq_astar_session_usage(gpq_astar_session* s, uint64_t* cells_used, uint64_t* tiles_used,
                                   uint32_t* instances) {
  GPQ_CHECK_ARG(s, "NULL handle");
  if (cells_used) *cells_used = s->cells.used();
  if (tiles_used) *tiles_used = s->tile_space.used();
  if (instances) *instances = s->active;
  return GPQ_OK;
}

uint64_t gpq_astar_session_bytes(const gpq_astar_config* cfg, uint64_t max_cells, uint32_t max_tiles,
                                 uint32_t max_instances) {
  gpq_astar_config c{};
  if (cfg) c = *cfg;
  const uint32_t tile = c.tile ? c.tile : 64;
  const uint64_t in_cap = c.inbox_capacity ? c.inbox_capacity : 8ull * tile;
  const uint64_t open_cap = c.open_capacity ? c.open_capacity : (uint64_t)tile * tile;
  return max_cells * 5 + kAstarPredSlack + max_cells / 8 + (uint64_t)max_tiles * (sizeof(AstarTileDev) + 8 * (2 * in_cap + open_cap) + 8) +
         (uint64_t)max_instances * (2 * sizeof(AstarInstDev) + 41);
}

}  // extern "C"
