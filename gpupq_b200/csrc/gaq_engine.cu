// Global array queue: host orchestration of the sorted-array window loop, and the radix
// sort / merge helpers (see gaq.cuh for the kernels and the reference mapping).
#include <algorithm>
#include <cstring>
#include <new>

#include "gaq.cuh"
#include "gaq_engine.h"
#include "host_common.h"
#include "phold_host.h"

namespace gpq {

size_t scan_scratch_words(uint64_t n) { return (size_t)((n + kScanChunk - 1) / kScanChunk) + 1; }

gpq_status scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, cudaStream_t st) {
  if (n == 0) return GPQ_OK;
  if (n <= 16 * kScanChunk) {  // one CTA: at most 64 entries a thread
    if (in != out) GPQ_CUDA_TRY(cudaMemcpyAsync(out, in, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    rs_scan_kernel<<<1, 1024, 0, st>>>(out, n);
  } else {
    const uint32_t chunks = (n + kScanChunk - 1) / kScanChunk;
    rs_chunk_sum_kernel<<<chunks, 1024, 0, st>>>(in, n, scratch);
    rs_scan_kernel<<<1, 1024, 0, st>>>(scratch, chunks);
    rs_chunk_scan_kernel<<<chunks, 1024, 0, st>>>(in, out, n, scratch);
  }
  GPQ_CUDA_TRY(cudaGetLastError());
  return GPQ_OK;
}

static uint32_t radix_tiles(uint32_t n) { return std::max<uint32_t>(1u, (n + kRsTile - 1) / kRsTile); }

// counts [256][tiles], their exclusive scan [256][tiles], scan scratch
size_t radix_hist_words(uint32_t n) {
  const size_t cells = (size_t)256 * radix_tiles(n);
  return 2 * cells + scan_scratch_words(cells);
}

gpq_status radix_sort_by_ts(gpq_item* a, gpq_item* b, uint32_t n, uint32_t kmin, uint32_t kmax, uint32_t* hist,
                            gpq_item** sorted, uint32_t* err, cudaStream_t st) {
  *sorted = a;
  if (n <= 1 || kmax <= kmin) return GPQ_OK;
  GPQ_CUDA_TRY(gpq::raise_smem_limit(rs_scatter_kernel, (int)(kRsTile * sizeof(gpq_item))));
  const uint32_t range = kmax - kmin;
  const uint32_t bits = 32 - __builtin_clz(range);
  const uint32_t passes = (bits + 7) / 8;
  const uint32_t ntiles = radix_tiles(n);
  const uint32_t cells = 256 * ntiles;
  uint32_t* cnt = hist;
  uint32_t* off = hist + cells;
  uint32_t* scratch = off + cells;
  gpq_item* src = a;
  gpq_item* dst = b;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = 8 * p;
    rs_hist_kernel<<<ntiles, kRsThreads, 0, st>>>(src, n, kmin, shift, cnt, ntiles);
    gpq_status s = scan_exclusive(cnt, off, cells, scratch, st);
    if (s != GPQ_OK) return s;
    rs_scatter_kernel<<<ntiles, kRsThreads, kRsTile * sizeof(gpq_item), st>>>(src, dst, n, kmin, shift, cnt, off,
                                                                              ntiles, err);
    GPQ_CUDA_TRY(cudaGetLastError());
    std::swap(src, dst);
  }
  *sorted = src;
  return GPQ_OK;
}

size_t merge_split_words(uint32_t total) { return (size_t)(total + kMpTile - 1) / kMpTile + 2; }

gpq_status merge_by_ts(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb, gpq_item* out, uint32_t* split,
                       uint32_t* err, cudaStream_t st) {
  const uint32_t total = na + nb;
  if (total == 0) return GPQ_OK;
  const uint32_t grid = (total + kMpTile - 1) / kMpTile;
  mp_splits_kernel<<<(grid + 1 + 255) / 256, 256, 0, st>>>(A, na, B, nb, split);
  mp_merge_kernel<<<grid, kMpThreads, 0, st>>>(A, na, B, nb, out, split, err);
  GPQ_CUDA_TRY(cudaGetLastError());
  return GPQ_OK;
}

// The engine's hist words serve the bulk sort and the window loop's smaller radix tiles.
static size_t engine_hist_words(uint32_t cap) {
  return std::max<size_t>(radix_hist_words(cap), (size_t)256 * std::max<uint32_t>(1u, (cap + kWinRsTile - 1) / kWinRsTile));
}

struct GaqEngine {
  gpq_phold_config c{};
  uint32_t cap = 0;  // array capacity (the population is conserved: num_lps * events_per_lp)
  gpq_item* arr[2] = {nullptr, nullptr};
  int cur = 0;
  uint32_t n = 0;
  gpq_item* ch = nullptr;
  gpq_item* ch_tmp = nullptr;
  gpq_item* stg = nullptr;
  uint32_t* stg_cnt = nullptr;
  uint32_t* info = nullptr;
  uint32_t* hist = nullptr;
  uint32_t* h_info = nullptr;  // pinned: [0..3] info, [4] head ts bits, [5] error
  unsigned long long* acc = nullptr;
  GaqWin* win = nullptr;        // device window state of the graph-replayed loop
  uint32_t* dig = nullptr;      // [256] digit totals / offsets of a radix pass
  uint32_t* split = nullptr;    // merge-path splits of the window's merge
  GaqWin* h_win = nullptr;      // pinned copy
  cudaGraph_t graph = nullptr;  // one window
  cudaGraphExec_t gexec = nullptr;
  uint32_t block = 256;
  static constexpr int G = 8;

  GaqDev dev() const { return GaqDev{stg, stg_cnt, ch, info, c.insert_capacity, cap}; }
  ~GaqEngine() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : {(void*)arr[0], (void*)arr[1], (void*)ch, (void*)ch_tmp, (void*)stg, (void*)stg_cnt, (void*)info,
                    (void*)hist, (void*)acc, (void*)win, (void*)dig, (void*)split})
      if (p) cudaFree(p);
    if (h_info) cudaFreeHost(h_info);
    if (h_win) cudaFreeHost(h_win);
  }
};

// Kernels of one window: begin, stage, process, sort set-up, 4 x (hist, row scan, digit
// scan, scatter), splits, merge, end.
uint32_t gaq_engine_launches_per_window() { return 4 + 4 * 4 + 3; }

gpq_status gaq_engine_create(const gpq_phold_config& c, GaqEngine** out) {
  *out = nullptr;
  GaqEngine* g = new (std::nothrow) GaqEngine();
  if (!g) return GPQ_ERR_NOMEM;
  g->c = c;
  const uint64_t cap = (uint64_t)c.num_lps * c.events_per_lp;
  if (cap > 0x7fffffffull) {
    delete g;
    set_last_error("global array queue: population too large");
    return GPQ_ERR_INVALID;
  }
  g->cap = (uint32_t)cap;
  auto fail = [&](cudaError_t e) {
    set_last_error("global array queue allocation: %s", cudaGetErrorString(e));
    delete g;
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&g->arr[0], cap * sizeof(gpq_item))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->arr[1], cap * sizeof(gpq_item))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->ch, cap * sizeof(gpq_item))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->ch_tmp, cap * sizeof(gpq_item))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->stg, (size_t)c.num_lps * c.insert_capacity * sizeof(gpq_item))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->stg_cnt, (size_t)c.num_lps * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->info, 8 * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  // the bulk sort's tiles (kRsTile) and the window loop's smaller ones (kWinRsTile)
  if ((e = cudaMalloc(&g->hist, engine_hist_words(g->cap) * sizeof(uint32_t))) != cudaSuccess)
    return fail(e);
  if ((e = gpq::raise_smem_limit(gaq_win_merge_kernel, (int)(kMpTile * sizeof(gpq_item)))) != cudaSuccess)
    return fail(e);
  if ((e = cudaMalloc(&g->acc, 8 * sizeof(unsigned long long))) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&g->h_info, 8 * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->win, sizeof(GaqWin))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->dig, 256 * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->split, ((g->cap + kMpTile - 1) / kMpTile + 2) * sizeof(uint32_t))) != cudaSuccess)
    return fail(e);
  if ((e = cudaMallocHost(&g->h_win, sizeof(GaqWin))) != cudaSuccess) return fail(e);
  const size_t smem = (size_t)(g->block / GaqEngine::G) * c.insert_capacity * sizeof(uint64_t);
  if ((e = gpq::raise_smem_limit(gaq_process_kernel<GaqEngine::G>, (int)smem)) != cudaSuccess)
    return fail(e);
  *out = g;
  return GPQ_OK;
}

void gaq_engine_destroy(GaqEngine* g) { delete g; }

void gaq_engine_state(GaqEngine* g, std::vector<std::pair<void*, size_t>>* dev,
                      std::vector<std::pair<void*, size_t>>* host) {
  const size_t cap = g->cap, L = g->c.num_lps;
  dev->push_back({g->arr[0], cap * sizeof(gpq_item)});
  dev->push_back({g->arr[1], cap * sizeof(gpq_item)});
  dev->push_back({g->ch, cap * sizeof(gpq_item)});
  dev->push_back({g->ch_tmp, cap * sizeof(gpq_item)});
  dev->push_back({g->stg, L * g->c.insert_capacity * sizeof(gpq_item)});
  dev->push_back({g->stg_cnt, L * sizeof(uint32_t)});
  dev->push_back({g->info, 8 * sizeof(uint32_t)});
  dev->push_back({g->hist, engine_hist_words(g->cap) * sizeof(uint32_t)});
  dev->push_back({g->acc, 8 * sizeof(unsigned long long)});
  dev->push_back({g->win, sizeof(GaqWin)});
  dev->push_back({g->dig, 256 * sizeof(uint32_t)});
  dev->push_back({g->split, ((g->cap + kMpTile - 1) / kMpTile + 2) * sizeof(uint32_t)});
  host->push_back({&g->cur, sizeof(g->cur)});
  host->push_back({&g->n, sizeof(g->n)});
  host->push_back({g->h_info, 8 * sizeof(uint32_t)});
  host->push_back({g->h_win, sizeof(GaqWin)});
}

gpq_status gaq_engine_populate(GaqEngine* g, const PholdDev& d, const gpq_item* dev_src, cudaStream_t st) {
  const gpq_phold_config& c = g->c;
  gaq_zero_stats_kernel<<<std::max(1u, std::min<uint32_t>((c.num_lps + 255) / 256, 4096)), 256, 0, st>>>(d);
  GPQ_CUDA_TRY(cudaMemsetAsync(g->stg_cnt, 0, (size_t)c.num_lps * sizeof(uint32_t), st));
  const uint32_t init_mm[2] = {0xffffffffu, 0u};
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->info, init_mm, sizeof(init_mm), cudaMemcpyHostToDevice, st));
  const uint32_t grid = std::max(1u, std::min<uint32_t>((g->cap + 255) / 256, 8192));
  gaq_initial_kernel<<<grid, 256, 0, st>>>(phold_params_of(c), c.num_lps, c.events_per_lp, dev_src, g->ch, g->info);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->h_info, g->info, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  gpq_item* sorted = nullptr;
  gpq_status s = radix_sort_by_ts(g->ch, g->ch_tmp, g->cap, g->h_info[0], g->h_info[1], g->hist, &sorted,
                                  &d.ctrl->err, st);
  if (s != GPQ_OK) return s;
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->arr[0], sorted, (size_t)g->cap * sizeof(gpq_item), cudaMemcpyDeviceToDevice, st));
  g->cur = 0;
  g->n = g->cap;
  *g->h_win = GaqWin{};
  g->h_win->n = g->cap;
  g->h_win->stop_at = 0xffffffffu;
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->win, g->h_win, sizeof(GaqWin), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

// Capture one window of the device-driven loop into a graph (once per engine).
static gpq_status gaq_capture(GaqEngine* g, const PholdDev& d, cudaStream_t st) {
  if (g->gexec) return GPQ_OK;
  const gpq_phold_config& c = g->c;
  GaqDev gd = g->dev();
  gd.info = reinterpret_cast<uint32_t*>(g->win);  // c, nc, kmin, kmax
  const uint32_t pgrid = std::max(1u, std::min<uint32_t>((c.num_lps + (g->block / GaqEngine::G) - 1) /
                                                             (g->block / GaqEngine::G), 8192));
  const size_t psmem = (size_t)(g->block / GaqEngine::G) * c.insert_capacity * sizeof(uint64_t);
  const uint32_t sgrid = std::max(1u, std::min<uint32_t>((g->cap + 255) / 256, 8192));
  const uint32_t max_tiles = std::max(1u, (g->cap + kWinRsTile - 1) / kWinRsTile);
  const uint32_t mgrid = std::max(1u, (g->cap + kMpTile - 1) / kMpTile);
  GPQ_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  gaq_win_begin_kernel<<<1, 1024, 0, st>>>(g->arr[0], g->arr[1], g->win, c.lookahead, c.end_time, &d.ctrl->err);
  gaq_win_stage_kernel<<<sgrid, 256, 0, st>>>(g->arr[0], g->arr[1], g->win, gd, c.num_lps, &d.ctrl->err);
  gaq_process_kernel<GaqEngine::G><<<pgrid, g->block, psmem, st>>>(d, gd, &d.ctrl->err, &g->win->gate);
  gaq_win_sort_setup_kernel<<<1, 32, 0, st>>>(g->win, g->cap, g->cap, &d.ctrl->err);
  for (uint32_t p = 0; p < 4; ++p) {
    gaq_win_hist_kernel<<<max_tiles, kRsThreads, 0, st>>>(g->ch, g->ch_tmp, g->win, p, g->hist);
    gaq_win_rowscan_kernel<<<256, 128, 0, st>>>(g->win, p, g->hist, g->dig);
    gaq_win_digscan_kernel<<<1, 256, 0, st>>>(g->win, p, g->dig);
    gaq_win_scatter_kernel<<<max_tiles, kRsThreads, 0, st>>>(g->ch, g->ch_tmp, g->win, p, g->hist, g->dig);
  }
  gaq_win_splits_kernel<<<(mgrid + 1 + 255) / 256, 256, 0, st>>>(g->arr[0], g->arr[1], g->ch, g->ch_tmp, g->win,
                                                                  g->split);
  gaq_win_merge_kernel<<<mgrid, kMpThreads, kMpTile * sizeof(gpq_item), st>>>(g->arr[0], g->arr[1], g->ch,
                                                                                  g->ch_tmp, g->win, g->split,
                                                                                  &d.ctrl->err);
  gaq_win_end_kernel<<<1, 32, 0, st>>>(g->win);
  const cudaError_t ce = cudaStreamEndCapture(st, &g->graph);
  if (ce != cudaSuccess) {
    set_last_error("global array queue: graph capture failed: %s", cudaGetErrorString(ce));
    return GPQ_ERR_CUDA;
  }
  GPQ_CUDA_TRY(cudaGraphInstantiate(&g->gexec, g->graph, 0));
  return GPQ_OK;
}

// des_run for the global array queue: replay the captured window in batches (16, 32, ...
// up to 256 windows) between host checks of the device window state.
gpq_status gaq_engine_run(GaqEngine* g, const PholdDev& d, uint32_t nsteps, int* done, uint64_t* windows,
                          cudaStream_t st) {
  const gpq_phold_config& c = g->c;
  if (done) *done = 0;
  gpq_status s = gaq_capture(g, d, st);
  if (s != GPQ_OK) return s;
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->h_win, g->win, sizeof(GaqWin), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  const uint32_t w0 = g->h_win->windows;
  uint64_t stop = nsteps ? (uint64_t)w0 + nsteps : 0xffffffffull;
  if (c.max_steps) stop = std::min<uint64_t>(stop, c.max_steps);
  g->h_win->stop_at = (uint32_t)std::min<uint64_t>(stop, 0xffffffffull);
  GPQ_CUDA_TRY(cudaMemcpyAsync(&g->win->stop_at, &g->h_win->stop_at, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  uint32_t batch = 16;
  for (;;) {
    for (uint32_t k = 0; k < batch; ++k) GPQ_CUDA_TRY(cudaGraphLaunch(g->gexec, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(g->h_win, g->win, sizeof(GaqWin), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&g->h_info[5], &d.ctrl->err, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    g->n = g->h_win->n;
    g->cur = (int)g->h_win->cur;
    if (g->h_info[5] != 0) {
      *windows += g->h_win->windows - w0;
      return (gpq_status)g->h_info[5];
    }
    if (g->h_win->done) {
      if (done) *done = 1;
      break;
    }
    if (g->h_win->windows >= g->h_win->stop_at) {
      if (c.max_steps && g->h_win->windows >= c.max_steps && done) *done = 1;
      break;
    }
    batch = std::min<uint32_t>(batch * 2, 256);
  }
  *windows += g->h_win->windows - w0;
  return GPQ_OK;
}

gpq_status gaq_engine_finalize(GaqEngine* g, const PholdDev& d, uint64_t out[4], uint32_t* pmin, cudaStream_t st) {
  GPQ_CUDA_TRY(cudaMemsetAsync(g->acc, 0, 4 * sizeof(unsigned long long), st));
  const uint32_t inf = kInfBits;
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->info + 6, &inf, 4, cudaMemcpyHostToDevice, st));
  const uint32_t grid = std::max(1u, std::min<uint32_t>((std::max(g->n, g->c.num_lps) + 255) / 256, 4096));
  gaq_finalize_kernel<<<grid, 256, 0, st>>>(d, g->arr[g->cur], g->n, g->acc, g->info + 6);
  GPQ_CUDA_TRY(cudaGetLastError());
  unsigned long long h[4];
  GPQ_CUDA_TRY(cudaMemcpyAsync(h, g->acc, sizeof(h), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(pmin, g->info + 6, 4, cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (int i = 0; i < 4; ++i) out[i] = h[i];
  return GPQ_OK;
}

}  // namespace gpq
