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

size_t radix_hist_words(uint32_t n) { return (size_t)256 * std::max<uint32_t>(1u, (n + kRsTile - 1) / kRsTile); }

gpq_status radix_sort_by_ts(gpq_item* a, gpq_item* b, uint32_t n, uint32_t kmin, uint32_t kmax, uint32_t* hist,
                            gpq_item** sorted, cudaStream_t st) {
  *sorted = a;
  if (n <= 1 || kmax <= kmin) return GPQ_OK;
  const uint32_t range = kmax - kmin;
  const uint32_t bits = 32 - __builtin_clz(range);
  const uint32_t passes = (bits + 7) / 8;
  const uint32_t ntiles = (n + kRsTile - 1) / kRsTile;
  gpq_item* src = a;
  gpq_item* dst = b;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = 8 * p;
    rs_hist_kernel<<<ntiles, kRsThreads, 0, st>>>(src, n, kmin, shift, hist, ntiles);
    rs_scan_kernel<<<1, 1024, 0, st>>>(hist, 256 * ntiles);
    rs_scatter_kernel<<<ntiles, kRsThreads, 0, st>>>(src, dst, n, kmin, shift, hist, ntiles);
    GPQ_CUDA_TRY(cudaGetLastError());
    std::swap(src, dst);
  }
  *sorted = src;
  return GPQ_OK;
}

gpq_status merge_by_ts(const gpq_item* A, uint32_t na, const gpq_item* B, uint32_t nb, gpq_item* out,
                       cudaStream_t st) {
  const uint32_t total = na + nb;
  if (total == 0) return GPQ_OK;
  const uint32_t grid = (total + kMpTile - 1) / kMpTile;
  mp_merge_kernel<<<grid, kMpThreads, 0, st>>>(A, na, B, nb, out);
  GPQ_CUDA_TRY(cudaGetLastError());
  return GPQ_OK;
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
  uint32_t block = 256;
  static constexpr int G = 8;

  GaqDev dev() const { return GaqDev{stg, stg_cnt, ch, info, c.insert_capacity, cap}; }
  ~GaqEngine() {
    for (void* p : {(void*)arr[0], (void*)arr[1], (void*)ch, (void*)ch_tmp, (void*)stg, (void*)stg_cnt, (void*)info,
                    (void*)hist, (void*)acc})
      if (p) cudaFree(p);
    if (h_info) cudaFreeHost(h_info);
  }
};

uint32_t gaq_engine_launches_per_window() { return 5 + 3 * 3; }

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
  if ((e = cudaMalloc(&g->hist, radix_hist_words(g->cap) * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&g->acc, 8 * sizeof(unsigned long long))) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&g->h_info, 8 * sizeof(uint32_t))) != cudaSuccess) return fail(e);
  const size_t smem = (size_t)(g->block / GaqEngine::G) * c.insert_capacity * sizeof(uint64_t);
  if ((e = cudaFuncSetAttribute(gaq_process_kernel<GaqEngine::G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem)) != cudaSuccess)
    return fail(e);
  *out = g;
  return GPQ_OK;
}

void gaq_engine_destroy(GaqEngine* g) { delete g; }

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
  gpq_status s = radix_sort_by_ts(g->ch, g->ch_tmp, g->cap, g->h_info[0], g->h_info[1], g->hist, &sorted, st);
  if (s != GPQ_OK) return s;
  GPQ_CUDA_TRY(cudaMemcpyAsync(g->arr[0], sorted, (size_t)g->cap * sizeof(gpq_item), cudaMemcpyDeviceToDevice, st));
  g->cur = 0;
  g->n = g->cap;
  return GPQ_OK;
}

gpq_status gaq_engine_run(GaqEngine* g, const PholdDev& d, uint32_t nsteps, int* done, uint64_t* windows,
                          cudaStream_t st) {
  const gpq_phold_config& c = g->c;
  if (done) *done = 0;
  const uint32_t pgrid = std::max(1u, std::min<uint32_t>((c.num_lps + (g->block / GaqEngine::G) - 1) /
                                                             (g->block / GaqEngine::G), 8192));
  const size_t psmem = (size_t)(g->block / GaqEngine::G) * c.insert_capacity * sizeof(uint64_t);
  uint32_t executed = 0;
  for (;;) {
    if (nsteps && executed >= nsteps) break;
    if (c.max_steps && *windows >= c.max_steps) { if (done) *done = 1; break; }
    // des_run: the window minimum is the array head (src/global_array_queue.cu:299-306)
    g->h_info[4] = kInfBits;
    if (g->n) GPQ_CUDA_TRY(cudaMemcpyAsync(&g->h_info[4], &g->arr[g->cur][0].ts, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&g->h_info[5], &d.ctrl->err, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const float m = gpq_u2f(g->h_info[4]);
    if (g->h_info[5] != 0) return (gpq_status)g->h_info[5];
    if (g->n == 0 || !(m < c.end_time)) { if (done) *done = 1; break; }
    const float bound = GPQ_FADD(m, c.lookahead);
    gpq_item* a = g->arr[g->cur];
    gaq_split_kernel<<<1, 32, 0, st>>>(a, g->n, bound, c.end_time, g->info);
    gaq_stage_kernel<<<std::max(1u, std::min<uint32_t>((g->n + 255) / 256, 8192)), 256, 0, st>>>(
        a, g->info, g->dev(), c.num_lps, &d.ctrl->err);
    gaq_process_kernel<GaqEngine::G><<<pgrid, g->block, psmem, st>>>(d, g->dev(), &d.ctrl->err);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(g->h_info, g->info, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t cpre = g->h_info[0], nc = std::min(g->h_info[1], g->cap);
    gpq_item* sorted = g->ch;
    gpq_status s = radix_sort_by_ts(g->ch, g->ch_tmp, nc, g->h_info[2], g->h_info[3], g->hist, &sorted, st);
    if (s != GPQ_OK) return s;
    if (g->n - cpre + nc > g->cap) {
      set_last_error("global array queue overflow");
      return GPQ_ERR_QUEUE_FULL;
    }
    s = merge_by_ts(a + cpre, g->n - cpre, sorted, nc, g->arr[g->cur ^ 1], st);
    if (s != GPQ_OK) return s;
    g->n = g->n - cpre + nc;
    g->cur ^= 1;
    ++*windows;
    ++executed;
  }
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
