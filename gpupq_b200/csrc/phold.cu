// PHOLD engine: C-ABI implementation (host side).
//
// Replaces the reference's DES driver and PHOLD model host code:
//   des_init / des_run / des_finish  src/des.cu:74-221
//   model_init / model_handle_next / model_get_events  src/phold.cu:124-192
// The host owns every device buffer through the handle (the reference keeps them in
// static __device__ globals, src/local_array_queue.cu:38-50).
#include <algorithm>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "host_common.h"
#include "phold_host.h"
#include "gaq.cuh"
#include "gaq_engine.h"
#include "hq_grid.cuh"
#include "hq_kernels.cuh"
#include "lab.cuh"
#include "phold_kernels.cuh"

namespace {

constexpr uint32_t kDefaultBlock = 256;

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

uint32_t ilog2(uint32_t x) { return gpq::ilog2_ceil(x); }

}  // namespace

struct gpq_phold {
  gpq_phold_config cfg{};
  int device = 0;
  int num_sms = 0;
  cudaStream_t own = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // device memory (one allocation per array)
  gpq_item* items = nullptr;  // per-LP queue items (ring / heap / node pool)
  uint32_t* qa = nullptr;     // per-LP queue words (see LpQueueDev)
  uint32_t* qb = nullptr;
  uint32_t* qc = nullptr;
  uint32_t* links = nullptr;  // splay links
  uint16_t* freestk = nullptr;
  gpq_item* ibuf = nullptr;
  uint32_t* icnt = nullptr;
  uint32_t* count = nullptr;
  unsigned long long* csum = nullptr;
  unsigned long long* ohash = nullptr;
  PholdCtrl* ctrl = nullptr;
  PholdAcc* acc = nullptr;
  gpq_item* staging = nullptr;  // host-provided initial events
  uint64_t staging_n = 0;

  // pinned host mirror of the control block (plain loop reads it every window)
  PholdCtrl* h_ctrl = nullptr;

  uint32_t cap_log2 = 0;
  uint32_t block = kDefaultBlock;
  uint32_t phase = 0;  // next window (host view; plain loop)
  // sharded runs (gpq_phold_shard_create): LPs [lp_begin, lp_end) of num_lps, outbox per
  // destination shard
  bool sharded = false;
  uint32_t rank = 0, world = 1, lp_begin = 0, lp_end = 0, shard_lps = 0, out_cap = 0;
  LabPeer* lab_peers = nullptr;  // connected bucketed shards: [world] bucket arrays (device)
  gpq_item* outbox = nullptr;   // [world][out_cap]
  uint32_t* out_n = nullptr;    // [world]
  gpq_item* inject_buf = nullptr;
  uint64_t inject_cap = 0;
  uint32_t last_grid = 0;  // CTAs of the last persistent launch
  bool populated = false;
  bool finalized = false;
  float elapsed_ms = 0.f;

  PholdDev dev() const {
    PholdDev d;
    d.p.seed = cfg.seed;
    d.p.num_lps = cfg.num_lps;
    d.p.dest_mode = cfg.dest_mode;
    d.p.ring_width = cfg.ring_width;
    d.p.ring_threshold = cfg.ring_threshold;
    d.p.lookahead = cfg.lookahead;
    d.p.end_time = cfg.end_time;
    d.L = cfg.num_lps;
    d.count = count;
    d.csum = csum;
    d.ohash = ohash;
    d.ctrl = ctrl;
    d.spin_limit = gpq::spin_limit();
    d.lp_begin = lp_begin;
    d.lp_end = sharded ? lp_end : cfg.num_lps;
    d.shard_lps = shard_lps;
    d.out_cap = out_cap;
    d.outbox = sharded ? outbox : nullptr;
    d.out_n = out_n;
    d.peers = sharded ? lab_peers : nullptr;
    return d;
  }
  LpQueueDev lq() const {
    LpQueueDev l;
    l.kind = cfg.queue_kind;
    l.cap_log2 = cap_log2;
    l.items = items;
    l.a = qa;
    l.b = qb;
    l.c = qc;
    l.links = links;
    l.freestk = freestk;
    return l;
  }
  InsDev ins() const { return InsDev{ibuf, icnt, cfg.insert_capacity}; }
  PholdKernelSet ks{};
  gpq::GaqEngine* gaq = nullptr;  // global array queue state (queue_kind == GPQ_QUEUE_GAQ)
  uint64_t gaq_windows = 0;
  // parallel heap (queue_kind == GPQ_QUEUE_HQ): one CTA runs the heap up to node size
  // kHqMaxR, the whole GPU (one cooperative launch) above it
  HqDev hq{};
  HqgDev hqg{};
  bool hq_grid = false;
  uint32_t hqg_blocks = 0;
  gpq_item* hq_sort[2] = {nullptr, nullptr};
  uint32_t* hq_hist = nullptr;
  uint32_t* hq_mm = nullptr;
  uint64_t hq_windows = 0;
  bool is_hq = false;
  // bucketed local array queue (queue_kind == GPQ_QUEUE_LAQ, laq_mode 2)
  LabDev lab{};
  LabKernelSet lks{};
  bool is_lab = false;
  size_t window_smem() const {
    return is_lab ? lab_cta_smem_bytes(block) : phold_window_smem_bytes(block, ks.group, ks.group_smem);
  }

  ~gpq_phold() {
    for (void* p : {(void*)items, (void*)qa, (void*)qb, (void*)qc, (void*)links, (void*)freestk, (void*)ibuf,
                    (void*)icnt, (void*)count, (void*)csum, (void*)ohash, (void*)ctrl, (void*)acc, (void*)staging,
                    (void*)outbox, (void*)out_n, (void*)inject_buf, (void*)lab_peers})
      if (p) cudaFree(p);
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (gaq) gpq::gaq_engine_destroy(gaq);
    for (void* p : {(void*)hq.nodes, (void*)hq.cnt, (void*)hq.meta, (void*)hq_sort[0], (void*)hq_sort[1],
                    (void*)hq_hist, (void*)hq_mm, (void*)lab.keys, (void*)lab.cnt, (void*)lab.spill,
                    (void*)lab.scnt, (void*)lab.wj, (void*)hqg.root2, (void*)hqg.t0, (void*)hqg.t1,
                    (void*)hqg.pa, (void*)hqg.pb, (void*)hqg.bref, (void*)hqg.k0, (void*)hqg.k1, (void*)hqg.rank,
                    (void*)hqg.addc, (void*)hqg.ovf, (void*)hqg.ilist, (void*)hqg.icnt, (void*)hqg.plist,
                    (void*)hqg.pcnt})
      if (p) cudaFree(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own) cudaStreamDestroy(own);
  }
};

namespace {

gpq_phold_params params_of(const gpq_phold_config& c) { return gpq::phold_params_of(c); }

gpq_status validate(const gpq_phold_config* c) { return gpq::validate_phold_config(c); }

}  // namespace

extern "C" {

gpq_status gpq_phold_create(const gpq_phold_config* cfg_in, gpq_phold** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  gpq_status st = validate(cfg_in);
  if (st != GPQ_OK) return st;
  gpq_phold_config c = *cfg_in;
  st = gpq::normalize_queue_config(&c);
  if (st != GPQ_OK) return st;

  gpq_phold* h = new (std::nothrow) gpq_phold();
  if (!h) return GPQ_ERR_NOMEM;
  h->cfg = c;
  h->cap_log2 = ilog2(c.capacity);
  h->block = c.block_threads;
  auto fail = [&](gpq_status s) { delete h; return s; };
#define TRY(expr)                                   \
  do {                                              \
    cudaError_t e_ = (expr);                        \
    if (e_ != cudaSuccess) {                        \
      gpq::set_last_error("%s -> %s", #expr, cudaGetErrorString(e_)); \
      return fail(e_ == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA); \
    }                                               \
  } while (0)
  TRY(cudaGetDevice(&h->device));
  TRY(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
  TRY(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  TRY(cudaEventCreate(&h->ev0));
  TRY(cudaEventCreate(&h->ev1));
  const size_t L = c.num_lps;
  // The global array queue as one sorted array in one launch: the heap kernel with a single
  // node that holds the population.
  const uint64_t pop = (uint64_t)c.num_lps * c.events_per_lp;
  const bool gaq_array = c.queue_kind == GPQ_QUEUE_GAQ && c.gaq_engine == 0 && pop <= kHqgMaxR;
  if (c.gaq_engine > 1) {
    gpq::set_last_error("gaq_engine must be 0 or 1");
    return fail(GPQ_ERR_INVALID);
  }
  if (c.queue_kind == GPQ_QUEUE_HQ || gaq_array) {
    // Default node size: the reference's 256 K root; a smaller population gets a root that
    // just holds it (a larger root changes nothing but its buffers' size).
    uint32_t r = gaq_array ? 0u : c.node_size;
    if (r == 0) {
      r = 2048;
      while (r < pop && r < (gaq_array ? kHqgMaxR : (256u << 10))) r <<= 1;
    }
    const bool grid = r > kHqMaxR;
    if (!gpq::is_pow2(r) || r < 2 || r > kHqgMaxR || (!grid && c.num_lps > (1u << 21))) {
      gpq::set_last_error("heap queue: node_size must be a power of two in [2, %u] (num_lps <= 2^21 up to node "
                          "size %u, where one CTA works the heap)", kHqgMaxR, kHqMaxR);
      return fail(GPQ_ERR_INVALID);
    }
    const uint64_t N = (uint64_t)c.num_lps * c.events_per_lp;
    h->is_hq = true;
    h->hq.r = r;
    h->hq.maxnodes = (uint32_t)((N + r - 1) / r + 2);
    TRY(cudaMalloc(&h->hq.nodes, (size_t)h->hq.maxnodes * r * sizeof(gpq_item)));
    TRY(cudaMalloc(&h->hq.cnt, (size_t)h->hq.maxnodes * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->hq.meta, 4 * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->hq_sort[0], N * sizeof(gpq_item)));
    TRY(cudaMalloc(&h->hq_sort[1], N * sizeof(gpq_item)));
    h->hq.ch = h->hq_sort[1];  // after populate: the children of a window
    TRY(cudaMalloc(&h->hq_hist, gpq::radix_hist_words((uint32_t)N) * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->hq_mm, 2 * sizeof(uint32_t)));
    if (grid) {
      HqgDev& g = h->hqg;
      h->hq_grid = true;
      TRY(cudaMalloc(&g.root2, (size_t)r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.t0, (size_t)2 * r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.t1, (size_t)3 * r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.pa, (size_t)r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.pb, (size_t)r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.bref, (size_t)r * sizeof(gpq_item)));
      TRY(cudaMalloc(&g.k0, (size_t)r * sizeof(unsigned long long)));
      TRY(cudaMalloc(&g.k1, (size_t)r * sizeof(unsigned long long)));
      TRY(cudaMalloc(&g.rank, (size_t)r * sizeof(uint32_t)));
      TRY(cudaMalloc(&g.addc, (size_t)r * sizeof(uint32_t)));
      TRY(cudaMalloc(&g.ovf, sizeof(uint32_t)));
      if ((uint64_t)c.num_lps * c.events_per_lp <= r) {  // the root holds every item: bucket lists
        TRY(cudaMalloc(&g.ilist, (size_t)kHqgMaxBuckets * kHqgListCapI * sizeof(gpq_item)));
        TRY(cudaMalloc(&g.icnt, 2 * kHqgMaxBuckets * sizeof(uint32_t)));
        TRY(cudaMalloc(&g.plist, (size_t)kHqgMaxBuckets * kHqgListCapP * sizeof(unsigned long long)));
        TRY(cudaMalloc(&g.pcnt, 2 * kHqgMaxBuckets * sizeof(uint32_t)));
      }
      g.e2 = h->hq_sort[0];  // after populate: the sort scratch of a window's children
      TRY(gpq::raise_smem_limit(hqg_phold_kernel, hqg_smem_bytes()));
      int per_sm = 0;
      TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hqg_phold_kernel, (int)kHqgThreads,
                                                        hqg_smem_bytes()));
      if (per_sm < 1) {
        gpq::set_last_error("heap queue: the grid kernel does not fit on an SM");
        return fail(GPQ_ERR_INVALID);
      }
      h->hqg_blocks = std::min<uint32_t>((uint32_t)h->num_sms, kHqgMaxBuckets);  // one CTA per SM
    } else {
      TRY(gpq::raise_smem_limit(hq_phold_kernel, (int)hq_smem_bytes(r)));
    }
  } else if (c.queue_kind == GPQ_QUEUE_LAQ && c.laq_mode == 2) {
    gpq::LabGeometry geo{};
    const gpq_status gs = gpq::lab_geometry(c, &geo);
    if (gs != GPQ_OK) return fail(gs);
    if (!lab_kernel_set(c.lanes_per_lp, &h->lks)) return fail(GPQ_ERR_INVALID);
    h->is_lab = true;
    LabDev& q = h->lab;
    q.nb_log2 = geo.nb_log2;
    q.c_log2 = geo.c_log2;
    q.F = geo.spill;
    q.inv_w = geo.inv_w;
    q.chunk = lab_chunk_lps(c.lookahead, q.inv_w, c.events_per_lp);
    TRY(cudaMalloc(&q.keys, (L << (q.nb_log2 + q.c_log2)) * sizeof(unsigned long long)));
    TRY(cudaMalloc(&q.cnt, (L << q.nb_log2) * sizeof(uint32_t)));
    TRY(cudaMalloc(&q.spill, 2 * L * q.F * sizeof(unsigned long long)));
    TRY(cudaMalloc(&q.scnt, 2 * L * sizeof(uint32_t)));
    TRY(cudaMalloc(&q.wj, 4 * sizeof(uint32_t)));
  } else if (c.queue_kind != GPQ_QUEUE_GAQ) {  // per-LP queues
    TRY(cudaMalloc(&h->items, (L << h->cap_log2) * sizeof(gpq_item)));
    TRY(cudaMalloc(&h->qa, L * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->qb, L * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->qc, L * sizeof(uint32_t)));
  }
  if (c.queue_kind == GPQ_QUEUE_LSQ) {
    TRY(cudaMalloc(&h->links, (L << h->cap_log2) * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->freestk, (L << h->cap_log2) * sizeof(uint16_t)));
  }
  if (!h->is_lab) {
    TRY(cudaMalloc(&h->ibuf, 2 * L * c.insert_capacity * sizeof(gpq_item)));
    TRY(cudaMalloc(&h->icnt, 2 * L * sizeof(uint32_t)));
  }
  TRY(cudaMalloc(&h->count, L * sizeof(uint32_t)));
  TRY(cudaMalloc(&h->csum, L * sizeof(unsigned long long)));
  TRY(cudaMalloc(&h->ohash, L * sizeof(unsigned long long)));
  TRY(cudaMalloc(&h->ctrl, sizeof(PholdCtrl)));
  TRY(cudaMalloc(&h->acc, sizeof(PholdAcc)));
  TRY(cudaMallocHost(&h->h_ctrl, sizeof(PholdCtrl)));
  if (h->is_hq) {
    *out = h;
    return GPQ_OK;
  }
  if (c.queue_kind == GPQ_QUEUE_GAQ) {
    gpq_status gs = gpq::gaq_engine_create(c, &h->gaq);
    if (gs != GPQ_OK) return fail(gs);
    *out = h;
    return GPQ_OK;
  }
  if (h->is_lab) {
    h->ks.group = c.lanes_per_lp;
    h->ks.group_smem = lab_group_smem_bytes();
    h->ks.window = h->lks.window;
    h->ks.persistent = h->lks.persistent;
  } else if (!phold_kernel_set(c.queue_kind, c.lanes_per_lp, c.insert_capacity, &h->ks, c.laq_mode)) {
    return fail(GPQ_ERR_INVALID);
  }
  if (!gpq::fit_block_to_smem(&h->block, h->ks.group, h->ks.group_smem + 24 * kStageRounds,
                              200 * 1024 - 2048 * 16 - 16)) {
    gpq::set_last_error("insert_capacity %u needs too much shared memory per lane group", c.insert_capacity);
    return fail(GPQ_ERR_INVALID);
  }
  h->cfg.block_threads = h->block;
  const size_t smem = h->window_smem();
  TRY(gpq::raise_smem_limit(h->ks.window, (int)smem));
  TRY(gpq::raise_smem_limit(h->ks.persistent, (int)smem));
#undef TRY
  *out = h;
  return GPQ_OK;
}

gpq_status gpq_phold_destroy(gpq_phold* h) {
  if (!h) return GPQ_ERR_INVALID;
  cudaStreamSynchronize(h->own);
  delete h;
  return GPQ_OK;
}

gpq_status gpq_phold_populate(gpq_phold* h, const gpq_item* initial, uint64_t n, void* stream) {
  GPQ_CHECK_ARG(h, "handle is NULL");
  cudaStream_t st = gpq::as_stream(stream, h->own);
  const gpq_phold_config& c = h->cfg;
  const size_t L = c.num_lps;
  const gpq_item* src = nullptr;
  if (initial) {
    GPQ_CHECK_ARG(n == (uint64_t)L * c.events_per_lp, "initial must hold num_lps * events_per_lp items");
    if (h->staging_n < n) {
      if (h->staging) cudaFree(h->staging);
      h->staging = nullptr;
      h->staging_n = 0;
      GPQ_CUDA_TRY(cudaMalloc(&h->staging, n * sizeof(gpq_item)));
      h->staging_n = n;
    }
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->staging, initial, n * sizeof(gpq_item), cudaMemcpyHostToDevice, st));
    src = h->staging;
  }
  PholdCtrl init{};
  for (int i = 0; i < 3; ++i) { init.mins[i] = kInfBits; init.errs[i] = 0; }
  *h->h_ctrl = init;
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->ctrl, h->h_ctrl, sizeof(PholdCtrl), cudaMemcpyHostToDevice, st));
  if (h->icnt) GPQ_CUDA_TRY(cudaMemsetAsync(h->icnt, 0, 2 * L * sizeof(uint32_t), st));
  h->phase = 0;
  h->gaq_windows = 0;
  h->hq_windows = 0;
  if (h->is_hq) {
    const uint32_t N = c.num_lps * c.events_per_lp;
    gaq_zero_stats_kernel<<<std::max(1u, std::min<uint32_t>((c.num_lps + 255) / 256, 4096)), 256, 0, st>>>(h->dev());
    const uint32_t mm[2] = {0xffffffffu, 0u};
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->hq_mm, mm, sizeof(mm), cudaMemcpyHostToDevice, st));
    gaq_initial_kernel<<<std::max(1u, std::min<uint32_t>((N + 255) / 256, 8192)), 256, 0, st>>>(
        params_of(c), c.num_lps, c.events_per_lp, src, h->hq_sort[0], h->hq_mm);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint32_t hmm[2];
    GPQ_CUDA_TRY(cudaMemcpyAsync(hmm, h->hq_mm, sizeof(hmm), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    gpq_item* sorted = nullptr;
    gpq_status ss = gpq::radix_sort_by_ts(h->hq_sort[0], h->hq_sort[1], N, hmm[0], hmm[1], h->hq_hist, &sorted,
                                          &h->ctrl->err, st);
    if (ss != GPQ_OK) return ss;
    // The sorted population laid out in level order is a valid heap of full nodes.
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->hq.nodes, sorted, (size_t)N * sizeof(gpq_item), cudaMemcpyDeviceToDevice, st));
    const uint32_t r = h->hq.r;
    const uint32_t nfull = N / r, rem = N % r;
    std::vector<uint32_t> cnt(h->hq.maxnodes, 0);
    for (uint32_t i = 0; i < nfull; ++i) cnt[i] = r;
    if (rem) cnt[nfull] = rem;
    const uint32_t last = (N == 0) ? 0 : (rem ? nfull : nfull - 1);
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->hq.cnt, cnt.data(), cnt.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    const uint32_t meta[4] = {last, 0, 0, 0};
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->hq.meta, meta, sizeof(meta), cudaMemcpyHostToDevice, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    h->populated = true;
    h->finalized = false;
    h->elapsed_ms = 0.f;
    return GPQ_OK;
  }
  if (h->gaq) {
    gpq_status gs = gpq::gaq_engine_populate(h->gaq, h->dev(), src, st);
    if (gs != GPQ_OK) return gs;
    h->populated = true;
    h->finalized = false;
    h->elapsed_ms = 0.f;
    return GPQ_OK;
  }
  if (h->is_lab) {
    // every key slot starts all ones (never written: not live)
    const LabDev& q = h->lab;
    GPQ_CUDA_TRY(cudaMemsetAsync(q.keys, 0xff, (L << (q.nb_log2 + q.c_log2)) * sizeof(unsigned long long), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(q.cnt, 0, (L << q.nb_log2) * sizeof(uint32_t), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(q.scnt, 0, 2 * L * sizeof(uint32_t), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(q.wj, 0, 4 * sizeof(uint32_t), st));
    const uint64_t n_ev = (uint64_t)L * c.events_per_lp;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n_ev + 255) / 256, 8192));
    lab_populate_kernel<<<grid, 256, 0, st>>>(h->dev(), q, c.events_per_lp, src);
    GPQ_CUDA_TRY(cudaGetLastError());
    h->phase = 0;
    h->populated = true;
    h->finalized = false;
    h->elapsed_ms = 0.f;
    return GPQ_OK;
  }
  // one warp per LP ranks its events in shared memory (24 B each): four warps per CTA up
  // to 2,048 events per LP, one beyond (8,192 events: 192 KiB)
  const uint32_t wpb = c.events_per_lp <= 2048 ? 4 : 1;
  const size_t smem = (size_t)wpb * c.events_per_lp * (sizeof(gpq_item) + sizeof(uint64_t));
  GPQ_CUDA_TRY(gpq::raise_smem_limit(phold_populate_kernel, (int)smem));
  const uint32_t grid = (uint32_t)((L + wpb - 1) / wpb);
  phold_populate_kernel<<<grid, wpb * 32, smem, st>>>(h->dev(), h->lq(), c.events_per_lp, src);
  GPQ_CUDA_TRY(cudaGetLastError());
  h->phase = 0;
  h->populated = true;
  h->finalized = false;
  h->elapsed_ms = 0.f;
  return GPQ_OK;
}

static gpq_status run_plain(gpq_phold* h, uint32_t nsteps, int* done, cudaStream_t st) {
  const gpq_phold_config& c = h->cfg;
  const uint32_t gpb = h->is_lab ? lab_plain_lps_per_cta(h->block, h->lab.chunk) : h->block / h->ks.group;  // LPs per CTA
  const uint32_t grid = (uint32_t)((c.num_lps + gpb - 1) / gpb);
  const size_t smem = h->window_smem();
  PholdDev d = h->dev();
  LpQueueDev q = h->lq();
  InsDev ib = h->ins();
  uint32_t executed = 0;
  if (done) *done = 0;
  // des_run loop: read the window minimum (D2H) -> run the window -> repeat.
  for (;;) {
    if (nsteps && executed >= nsteps) break;
    if (c.max_steps && h->phase >= c.max_steps) { if (done) *done = 1; break; }
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const float m = gpq_u2f(h->h_ctrl->mins[h->phase % 3]);
    if (h->h_ctrl->err != 0 || h->h_ctrl->errs[h->phase % 3] != 0 || !(m < c.end_time)) {
      if (done) *done = 1;
      break;
    }
    uint32_t phase = h->phase;
    void* args[] = {&d, &q, &ib, &phase};
    void* lab_args[] = {&d, &h->lab, &phase};
    GPQ_CUDA_TRY(cudaLaunchKernel(h->ks.window, dim3(grid), dim3(h->block), h->is_lab ? lab_args : args, smem, st));
    ++h->phase;
    ++executed;
  }
  return GPQ_OK;
}

// Parallel heap: up to nsteps windows (0 = all) of the heap -- one CTA for nodes up to
// kHqMaxR items, one cooperative launch over every SM for larger nodes.
static gpq_status run_hq(gpq_phold* h, uint32_t nsteps, int* done, cudaStream_t st) {
  if (h->hq_grid) {
    GPQ_CUDA_TRY(cudaMemsetAsync(&h->ctrl->bar, 0, sizeof(unsigned long long), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(h->hqg.ovf, 0, sizeof(uint32_t), st));
    if (h->hqg.icnt) {
      GPQ_CUDA_TRY(cudaMemsetAsync(h->hqg.icnt, 0, 2 * kHqgMaxBuckets * sizeof(uint32_t), st));
      GPQ_CUDA_TRY(cudaMemsetAsync(h->hqg.pcnt, 0, 2 * kHqgMaxBuckets * sizeof(uint32_t), st));
    }
    PholdDev d = h->dev();
    HqgDev g = h->hqg;
    g.h = h->hq;
    void* args[] = {&d, &g, &nsteps};
    GPQ_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)hqg_phold_kernel, dim3(h->hqg_blocks), dim3(kHqgThreads),
                                             args, hqg_smem_bytes(), st));
    h->last_grid = h->hqg_blocks;
  } else {
    hq_phold_kernel<<<1, 512, hq_smem_bytes(h->hq.r), st>>>(h->dev(), h->hq, nsteps);
    GPQ_CUDA_TRY(cudaGetLastError());
  }
  uint32_t meta[2];
  GPQ_CUDA_TRY(cudaMemcpyAsync(meta, h->hq.meta, sizeof(meta), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  h->hq_windows += meta[1];
  if (done) *done = (nsteps == 0 || meta[1] < nsteps) ? 1 : 0;
  return GPQ_OK;
}

static gpq_status run_persistent(gpq_phold* h, cudaStream_t st) {
  const gpq_phold_config& c = h->cfg;
  const size_t smem = h->window_smem();
  int per_sm = 0;
  GPQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, h->ks.persistent, (int)h->block, smem));
  if (per_sm <= 0) {
    gpq::set_last_error("persistent kernel does not fit on an SM (block %u, smem %zu)", h->block, smem);
    return GPQ_ERR_INVALID;
  }
  if (c.ctas_per_sm) per_sm = std::min<int>(per_sm, (int)c.ctas_per_sm);
  uint32_t grid = (uint32_t)(per_sm * h->num_sms);
  const uint32_t gpb = h->is_lab ? 1u : h->block / h->ks.group;  // LPs per CTA at least
  const uint32_t need = (uint32_t)((c.num_lps + gpb - 1) / gpb);
  grid = std::min(grid, std::max(need, 1u));
  GPQ_CUDA_TRY(cudaMemsetAsync(&h->ctrl->bar, 0, sizeof(unsigned long long), st));
  PholdDev d = h->dev();
  LpQueueDev q = h->lq();
  InsDev ib = h->ins();
  uint32_t s0 = h->phase;
  uint32_t maxs = c.max_steps ? (c.max_steps > s0 ? c.max_steps - s0 : 0) : 0;
  if (c.max_steps && maxs == 0) return GPQ_OK;
  void* args[] = {&d, &q, &ib, &s0, &maxs};
  void* lab_args[] = {&d, &h->lab, &s0, &maxs};
  GPQ_CUDA_TRY(cudaLaunchCooperativeKernel(h->ks.persistent, dim3(grid), dim3(h->block), h->is_lab ? lab_args : args,
                                           smem, st));
  h->last_grid = grid;
  return GPQ_OK;
}

// After a persistent launch: the device recorded the next window index in ctrl->phase.
static gpq_status sync_phase(gpq_phold* h, cudaStream_t st) {
  GPQ_CUDA_TRY(cudaMemcpyAsync(&h->h_ctrl->phase, &h->ctrl->phase, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  h->phase = h->h_ctrl->phase;
  return GPQ_OK;
}

gpq_status gpq_phold_run(gpq_phold* h, void* stream) {
  GPQ_CHECK_ARG(h, "handle is NULL");
  GPQ_CHECK_ARG(!h->sharded, "a shard handle runs window by window (gpq_phold_shard_window)");
  if (!h->populated) { gpq::set_last_error("gpq_phold_run before gpq_phold_populate"); return GPQ_ERR_NOT_READY; }
  cudaStream_t st = gpq::as_stream(stream, h->own);
  h->finalized = false;
  GPQ_CUDA_TRY(cudaEventRecord(h->ev0, st));
  gpq_status s;
  if (h->is_hq) {
    const uint64_t cap = h->cfg.max_steps;
    s = (cap && h->hq_windows >= cap) ? GPQ_OK : run_hq(h, cap ? (uint32_t)(cap - h->hq_windows) : 0u, nullptr, st);
  }
  else if (h->gaq) s = gpq::gaq_engine_run(h->gaq, h->dev(), 0, nullptr, &h->gaq_windows, st);
  else s = (h->cfg.loop_mode == GPQ_LOOP_PERSISTENT) ? run_persistent(h, st) : run_plain(h, 0, nullptr, st);
  if (s != GPQ_OK) return s;
  GPQ_CUDA_TRY(cudaEventRecord(h->ev1, st));
  if (!h->gaq && !h->is_hq && h->cfg.loop_mode == GPQ_LOOP_PERSISTENT) {
    s = sync_phase(h, st);
    if (s != GPQ_OK) return s;
  }
  GPQ_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  GPQ_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->elapsed_ms = ms;
  return GPQ_OK;
}

gpq_status gpq_phold_step(gpq_phold* h, uint32_t nsteps, int* done, void* stream) {
  GPQ_CHECK_ARG(h, "handle is NULL");
  GPQ_CHECK_ARG(!h->sharded, "a shard handle runs window by window (gpq_phold_shard_window)");
  if (!h->populated) return GPQ_ERR_NOT_READY;
  h->finalized = false;
  if (h->is_hq) {
    if (nsteps == 0) nsteps = 0xffffffffu;
    return run_hq(h, nsteps, done, gpq::as_stream(stream, h->own));
  }
  if (h->gaq) return gpq::gaq_engine_run(h->gaq, h->dev(), nsteps, done, &h->gaq_windows, gpq::as_stream(stream, h->own));
  return run_plain(h, nsteps, done, gpq::as_stream(stream, h->own));
}

gpq_status gpq_phold_result_get(gpq_phold* h, gpq_phold_result* out, void* stream) {
  GPQ_CHECK_ARG(h && out, "NULL argument");
  if (!h->populated) return GPQ_ERR_NOT_READY;
  cudaStream_t st = gpq::as_stream(stream, h->own);
  if (h->is_hq) {
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(h->acc);
    GPQ_CUDA_TRY(cudaMemsetAsync(acc, 0, 4 * sizeof(unsigned long long), st));
    const uint32_t inf = kInfBits;
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->hq_mm, &inf, 4, cudaMemcpyHostToDevice, st));
    hq_finalize_kernel<<<512, 256, 0, st>>>(h->dev(), h->hq, acc, h->hq_mm);
    GPQ_CUDA_TRY(cudaGetLastError());
    unsigned long long v[4];
    uint32_t pmin = kInfBits;
    GPQ_CUDA_TRY(cudaMemcpyAsync(v, acc, sizeof(v), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&pmin, h->hq_mm, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    std::memset(out, 0, sizeof(*out));
    out->committed = v[0];
    out->pending = v[1];
    out->pending_csum = v[2];
    out->digest = v[3];
    out->steps = h->hq_windows;
    out->final_min = gpq_u2f(pmin);
    out->elapsed_ms = h->elapsed_ms;
    out->status = (int32_t)h->h_ctrl->err;
    h->finalized = true;
    return (gpq_status)h->h_ctrl->err;
  }
  if (h->gaq) {
    uint64_t v[4];
    uint32_t pmin = kInfBits;
    gpq_status gs = gpq::gaq_engine_finalize(h->gaq, h->dev(), v, &pmin, st);
    if (gs != GPQ_OK) return gs;
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    std::memset(out, 0, sizeof(*out));
    out->committed = v[0];
    out->pending = v[1];
    out->pending_csum = v[2];
    out->digest = v[3];
    out->steps = h->gaq_windows;
    out->final_min = gpq_u2f(pmin);
    out->elapsed_ms = h->elapsed_ms;
    out->status = (int32_t)h->h_ctrl->err;
    h->finalized = true;
    return (gpq_status)h->h_ctrl->err;
  }
  PholdAcc a{};
  a.pending_min = kInfBits;
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->acc, &a, sizeof(PholdAcc), cudaMemcpyHostToDevice, st));
  const uint32_t wpb = 8;
  const uint32_t grid = std::max(1u, std::min<uint32_t>((h->cfg.num_lps + wpb - 1) / wpb, 4096u));
  if (h->is_lab) lab_finalize_kernel<<<grid, wpb * 32, 0, st>>>(h->dev(), h->lab, h->acc);
  else phold_finalize_kernel<<<grid, wpb * 32, 0, st>>>(h->dev(), h->lq(), h->ins(), h->acc);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaMemcpyAsync(&a, h->acc, sizeof(PholdAcc), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  std::memset(out, 0, sizeof(*out));
  out->committed = a.committed;
  out->steps = h->h_ctrl->steps;
  out->pending = a.pending;
  out->pending_csum = a.pending_csum;
  out->digest = a.digest;
  out->final_min = gpq_u2f(a.pending_min);
  out->elapsed_ms = h->elapsed_ms;
  out->status = (int32_t)h->h_ctrl->err;
  h->finalized = true;
  return (gpq_status)h->h_ctrl->err;
}

gpq_status gpq_phold_lp_stats(gpq_phold* h, uint32_t* count, uint64_t* csum, uint64_t* ohash, void* stream) {
  GPQ_CHECK_ARG(h, "handle is NULL");
  cudaStream_t st = gpq::as_stream(stream, h->own);
  const size_t L = h->cfg.num_lps;
  if (count) GPQ_CUDA_TRY(cudaMemcpyAsync(count, h->count, L * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (csum) GPQ_CUDA_TRY(cudaMemcpyAsync(csum, h->csum, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  if (ohash) GPQ_CUDA_TRY(cudaMemcpyAsync(ohash, h->ohash, L * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

gpq_status gpq_phold_launch_info(gpq_phold* h, uint32_t* grid, uint32_t* block, uint32_t* launches_per_run) {
  GPQ_CHECK_ARG(h, "handle is NULL");
  if (grid) *grid = h->last_grid;
  if (block) *block = h->hq_grid ? kHqgThreads : h->block;
  if (launches_per_run)
    *launches_per_run = h->is_hq ? 1u
                      : h->gaq ? (uint32_t)(h->gaq_windows * gpq::gaq_engine_launches_per_window())
                               : (h->cfg.loop_mode == GPQ_LOOP_PERSISTENT) ? 1u : h->phase;
  return GPQ_OK;
}

}  // extern "C"

namespace {

// Every device buffer the handle owns (pointer, bytes) and its host-side state words: the
// whole state of a run between windows.
void phold_state(gpq_phold* h, std::vector<std::pair<void*, size_t>>* dev,
                 std::vector<std::pair<void*, size_t>>* host) {
  const gpq_phold_config& c = h->cfg;
  const size_t L = c.num_lps;
  auto add = [&](void* p, size_t n) {
    if (p && n) dev->push_back({p, n});
  };
  add(h->items, (L << h->cap_log2) * sizeof(gpq_item));
  add(h->qa, L * sizeof(uint32_t));
  add(h->qb, L * sizeof(uint32_t));
  add(h->qc, L * sizeof(uint32_t));
  add(h->links, (L << h->cap_log2) * sizeof(uint32_t));
  add(h->freestk, (L << h->cap_log2) * sizeof(uint16_t));
  add(h->ibuf, 2 * L * c.insert_capacity * sizeof(gpq_item));
  add(h->icnt, 2 * L * sizeof(uint32_t));
  add(h->count, L * sizeof(uint32_t));
  add(h->csum, L * sizeof(unsigned long long));
  add(h->ohash, L * sizeof(unsigned long long));
  add(h->ctrl, sizeof(PholdCtrl));
  if (h->is_lab) {
    const LabDev& q = h->lab;
    add(q.keys, (L << (q.nb_log2 + q.c_log2)) * sizeof(unsigned long long));
    add(q.cnt, (L << q.nb_log2) * sizeof(uint32_t));
    add(q.spill, 2 * L * q.F * sizeof(unsigned long long));
    add(q.scnt, 2 * L * sizeof(uint32_t));
    add(q.wj, 4 * sizeof(uint32_t));
  }
  if (h->is_hq) {
    const uint64_t N = (uint64_t)c.num_lps * c.events_per_lp;
    add(h->hq.nodes, (size_t)h->hq.maxnodes * h->hq.r * sizeof(gpq_item));
    add(h->hq.cnt, (size_t)h->hq.maxnodes * sizeof(uint32_t));
    add(h->hq.meta, 4 * sizeof(uint32_t));
    add(h->hq_sort[0], N * sizeof(gpq_item));
    add(h->hq_sort[1], N * sizeof(gpq_item));
    add(h->hq_mm, 2 * sizeof(uint32_t));
  }
  if (h->gaq) gpq::gaq_engine_state(h->gaq, dev, host);
  host->push_back({&h->phase, sizeof(h->phase)});
  host->push_back({&h->gaq_windows, sizeof(h->gaq_windows)});
  host->push_back({&h->hq_windows, sizeof(h->hq_windows)});
  host->push_back({&h->populated, sizeof(h->populated)});
}

constexpr uint64_t kSnapMagic = 0x3150414e53515047ull;  // "GPQSNAP1"

}  // namespace

extern "C" {

gpq_status gpq_phold_snapshot(gpq_phold* h, void* buf, uint64_t capacity, uint64_t* size, void* stream) {
  GPQ_CHECK_ARG(h && size, "NULL argument");
  std::vector<std::pair<void*, size_t>> dev, host;
  phold_state(h, &dev, &host);
  uint64_t need = 8 + sizeof(gpq_phold_config) + 8;
  for (auto& r : dev) need += 8 + r.second;
  for (auto& r : host) need += 8 + r.second;
  *size = need;
  if (!buf) return GPQ_OK;
  GPQ_CHECK_ARG(capacity >= need, "capacity below the snapshot size");
  GPQ_CHECK_ARG(h->populated, "gpq_phold_snapshot before gpq_phold_populate");
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  unsigned char* p = static_cast<unsigned char*>(buf);
  auto put = [&](const void* src, size_t n) {
    std::memcpy(p, src, n);
    p += n;
  };
  put(&kSnapMagic, 8);
  put(&h->cfg, sizeof(gpq_phold_config));
  const uint32_t counts[2] = {(uint32_t)dev.size(), (uint32_t)host.size()};
  put(counts, 8);
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (auto& r : dev) {
    const uint64_t n = r.second;
    put(&n, 8);
    GPQ_CUDA_TRY(cudaMemcpyAsync(p, r.first, n, cudaMemcpyDeviceToHost, st));
    p += n;
  }
  for (auto& r : host) {
    const uint64_t n = r.second;
    put(&n, 8);
    put(r.first, n);
  }
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

gpq_status gpq_phold_restore(gpq_phold* h, const void* buf, uint64_t size, void* stream) {
  GPQ_CHECK_ARG(h && buf, "NULL argument");
  std::vector<std::pair<void*, size_t>> dev, host;
  phold_state(h, &dev, &host);
  const unsigned char* p = static_cast<const unsigned char*>(buf);
  const unsigned char* end = p + size;
  auto take = [&](void* dst, size_t n) -> bool {
    if ((uint64_t)(end - p) < n) return false;
    if (dst) std::memcpy(dst, p, n);
    p += n;
    return true;
  };
  uint64_t magic = 0;
  gpq_phold_config cfg{};
  uint32_t counts[2] = {0, 0};
  GPQ_CHECK_ARG(take(&magic, 8) && magic == kSnapMagic, "not a PHOLD snapshot");
  GPQ_CHECK_ARG(take(&cfg, sizeof(cfg)) && std::memcmp(&cfg, &h->cfg, sizeof(cfg)) == 0,
                "snapshot of a run with another configuration");
  GPQ_CHECK_ARG(take(counts, 8) && counts[0] == dev.size() && counts[1] == host.size(), "snapshot layout differs");
  // check every region's size before anything is overwritten
  const unsigned char* scan = p;
  for (size_t i = 0; i < dev.size() + host.size(); ++i) {
    const size_t want = i < dev.size() ? dev[i].second : host[i - dev.size()].second;
    uint64_t n = 0;
    GPQ_CHECK_ARG((uint64_t)(end - scan) >= 8, "snapshot truncated");
    std::memcpy(&n, scan, 8);
    GPQ_CHECK_ARG(n == want && (uint64_t)(end - scan - 8) >= n, "snapshot region differs or is truncated");
    scan += 8 + n;
  }
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (auto& r : dev) {
    p += 8;
    GPQ_CUDA_TRY(cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyHostToDevice, st));
    p += r.second;
  }
  for (auto& r : host) {
    p += 8;
    take(r.first, r.second);
  }
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  h->finalized = false;
  return GPQ_OK;
}

gpq_status gpq_phold_shard_create(const gpq_phold_config* cfg, uint32_t rank, uint32_t world,
                                  uint32_t outbox_capacity, gpq_phold** out) {
  GPQ_CHECK_ARG(cfg && out, "NULL argument");
  *out = nullptr;
  GPQ_CHECK_ARG(world >= 1 && rank < world, "need world >= 1 and rank < world");
  GPQ_CHECK_ARG(cfg->queue_kind == GPQ_QUEUE_LHQ || cfg->queue_kind == GPQ_QUEUE_LSQ || cfg->queue_kind == GPQ_QUEUE_LAQ,
                "sharded runs take the per-LP queue kinds (LAQ in any form, LHQ, LSQ)");
  GPQ_CHECK_ARG(cfg->num_lps >= world, "need at least one LP per shard");
  gpq_phold* h = nullptr;
  gpq_status r = gpq_phold_create(cfg, &h);
  if (r != GPQ_OK) return r;
  const uint32_t L = h->cfg.num_lps;
  h->sharded = true;
  h->rank = rank;
  h->world = world;
  if (h->is_lab) {  // the window that hands children of other shards' LPs over
    lab_kernel_set(h->cfg.lanes_per_lp, &h->lks, true);
    h->ks.window = h->lks.window;
    cudaError_t e = gpq::raise_smem_limit(h->ks.window, (int)h->window_smem());
    if (e != cudaSuccess) {
      gpq::set_last_error("gpq_phold_shard_create: %s", cudaGetErrorString(e));
      gpq_phold_destroy(h);
      return GPQ_ERR_CUDA;
    }
  }
  h->shard_lps = (uint32_t)(((uint64_t)L + world - 1) / world);
  h->lp_begin = std::min<uint32_t>(L, rank * h->shard_lps);
  h->lp_end = (uint32_t)std::min<uint64_t>(L, (uint64_t)h->lp_begin + h->shard_lps);
  // default: as many handed-over children per destination as this shard's insert buffers
  // hold (the bucketed form: as many as its LPs hold pending events)
  const uint64_t per_lp = h->is_lab ? h->cfg.events_per_lp : h->cfg.insert_capacity;
  h->out_cap = outbox_capacity ? outbox_capacity
                               : (uint32_t)std::min<uint64_t>((uint64_t)(h->lp_end - h->lp_begin) * per_lp, 1u << 26);
  cudaError_t e = cudaMalloc(&h->outbox, std::max<uint64_t>(1, (uint64_t)world * h->out_cap) * sizeof(gpq_item));
  if (e == cudaSuccess) e = cudaMalloc(&h->out_n, world * sizeof(uint32_t));
  if (e != cudaSuccess) {
    gpq::set_last_error("gpq_phold_shard_create: %s", cudaGetErrorString(e));
    gpq_phold_destroy(h);
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  }
  *out = h;
  return GPQ_OK;
}

gpq_status gpq_phold_shard_range(gpq_phold* h, uint32_t* lp_begin, uint32_t* lp_end, uint32_t* outbox_capacity) {
  GPQ_CHECK_ARG(h && h->sharded, "not a shard handle");
  if (lp_begin) *lp_begin = h->lp_begin;
  if (lp_end) *lp_end = h->lp_end;
  if (outbox_capacity) *outbox_capacity = h->out_cap;
  return GPQ_OK;
}

gpq_status gpq_phold_shard_populate(gpq_phold* h, float* local_min, void* stream) {
  GPQ_CHECK_ARG(h && h->sharded && local_min, "not a shard handle or NULL argument");
  gpq_status r = gpq_phold_populate(h, nullptr, 0, stream);
  if (r != GPQ_OK) return r;
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  *local_min = gpq_u2f(h->h_ctrl->mins[0]);
  return GPQ_OK;
}

gpq_status gpq_phold_shard_window(gpq_phold* h, float global_min, float* local_min, uint32_t* out_counts,
                                  void* stream) {
  GPQ_CHECK_ARG(h && h->sharded && local_min && out_counts, "not a shard handle or NULL argument");
  GPQ_CHECK_ARG(h->populated, "gpq_phold_shard_window before gpq_phold_shard_populate");
  GPQ_CHECK_ARG(global_min < h->cfg.end_time, "the run has ended: global_min >= end_time");
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  const uint32_t s = h->phase;
  const uint32_t mb = gpq_f2u(global_min);
  GPQ_CUDA_TRY(cudaMemcpyAsync(&h->ctrl->mins[s % 3], &mb, sizeof(mb), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemsetAsync(h->out_n, 0, h->world * sizeof(uint32_t), st));
  const uint32_t gpb = h->is_lab ? lab_plain_lps_per_cta(h->block, h->lab.chunk)
                                 : h->block / h->ks.group;  // LPs per CTA and round
  const uint32_t grid = std::max(1u, (h->lp_end - h->lp_begin + gpb - 1) / gpb);
  PholdDev d = h->dev();
  LpQueueDev q = h->lq();
  InsDev ib = h->ins();
  uint32_t phase = s;
  void* args[] = {&d, &q, &ib, &phase};
  void* lab_args[] = {&d, &h->lab, &phase};
  GPQ_CUDA_TRY(cudaLaunchKernel(h->ks.window, dim3(grid), dim3(h->block), h->is_lab ? lab_args : args,
                                h->window_smem(), st));
  ++h->phase;
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(out_counts, h->out_n, h->world * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  *local_min = gpq_u2f(h->h_ctrl->mins[(s + 1) % 3]);
  if (h->h_ctrl->err) {
    gpq::set_last_error("sharded PHOLD: device error %u in window %u", h->h_ctrl->err, s);
    return (gpq_status)h->h_ctrl->err;
  }
  return GPQ_OK;
}

gpq_status gpq_phold_shard_outbox(gpq_phold* h, gpq_item** items, uint32_t* capacity) {
  GPQ_CHECK_ARG(h && h->sharded && items, "not a shard handle or NULL argument");
  *items = h->outbox;
  if (capacity) *capacity = h->out_cap;
  return GPQ_OK;
}

gpq_status gpq_phold_shard_inject(gpq_phold* h, const gpq_item* items, uint64_t n, int on_device, void* stream) {
  GPQ_CHECK_ARG(h && h->sharded, "not a shard handle");
  GPQ_CHECK_ARG(h->phase > 0, "gpq_phold_shard_inject before the first window");
  if (n == 0) return GPQ_OK;
  GPQ_CHECK_ARG(items, "items is NULL");
  const cudaStream_t st = gpq::as_stream(stream, h->own);
  const gpq_item* src = items;
  if (!on_device) {
    if (h->inject_cap < n) {
      if (h->inject_buf) cudaFree(h->inject_buf);
      h->inject_buf = nullptr;
      h->inject_cap = 0;
      GPQ_CUDA_TRY(cudaMalloc(&h->inject_buf, n * sizeof(gpq_item)));
      h->inject_cap = n;
    }
    GPQ_CUDA_TRY(cudaMemcpyAsync(h->inject_buf, items, n * sizeof(gpq_item), cudaMemcpyHostToDevice, st));
    src = h->inject_buf;
  }
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 4096));
  if (h->is_lab)
    lab_inject_kernel<<<grid, 256, 0, st>>>(h->dev(), h->lab, src, n, h->phase - 1);
  else
    phold_inject_kernel<<<grid, 256, 0, st>>>(h->dev(), h->ins(), src, n, (h->phase - 1) & 1u);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(PholdCtrl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (h->h_ctrl->err) {
    gpq::set_last_error("sharded PHOLD: handed-over items rejected (error %u)", h->h_ctrl->err);
    return (gpq_status)h->h_ctrl->err;
  }
  return GPQ_OK;
}

gpq_status gpq_phold_shard_connect(gpq_phold* h, gpq_phold* const* shards, uint32_t world) {
  GPQ_CHECK_ARG(h && h->sharded && shards, "not a shard handle or NULL argument");
  GPQ_CHECK_ARG(h->is_lab, "direct hand-over connects the bucketed local array queue's shards (laq_mode 2)");
  GPQ_CHECK_ARG(world == h->world, "world differs from the shard's");
  std::vector<LabPeer> tab(world);
  for (uint32_t r = 0; r < world; ++r) {
    const gpq_phold* o = shards[r];
    GPQ_CHECK_ARG(o && o->sharded && o->is_lab && o->rank == r && o->world == world, "shards[r] must be shard r");
    GPQ_CHECK_ARG(std::memcmp(&o->cfg, &h->cfg, sizeof(h->cfg)) == 0, "every shard must run the same configuration");
    if (o->device != h->device) {  // another GPU: its memory through peer access
      int can = 0;
      GPQ_CUDA_TRY(cudaDeviceCanAccessPeer(&can, h->device, o->device));
      GPQ_CHECK_ARG(can, "no peer access between the shards' GPUs");
      const cudaError_t e = cudaDeviceEnablePeerAccess(o->device, 0);
      if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) GPQ_CUDA_TRY(e);
      (void)cudaGetLastError();
    }
    tab[r] = LabPeer{o->lab.keys, o->lab.cnt, o->lab.spill, o->lab.scnt};
  }
  if (h->lab_peers == nullptr) GPQ_CUDA_TRY(cudaMalloc(&h->lab_peers, world * sizeof(LabPeer)));
  GPQ_CUDA_TRY(cudaMemcpy(h->lab_peers, tab.data(), world * sizeof(LabPeer), cudaMemcpyHostToDevice));
  return GPQ_OK;
}

gpq_status gpq_host_alloc(uint64_t bytes, void** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  GPQ_CUDA_TRY(cudaMallocHost(out, bytes ? bytes : 1));
  return GPQ_OK;
}

gpq_status gpq_host_free(void* p) {
  if (p) GPQ_CUDA_TRY(cudaFreeHost(p));
  return GPQ_OK;
}

gpq_status gpq_phold_initial_events(const gpq_phold_config* cfg, gpq_item* out, uint64_t n) {
  gpq_status st = validate(cfg);
  if (st != GPQ_OK) return st;
  GPQ_CHECK_ARG(out, "out is NULL");
  GPQ_CHECK_ARG(n == (uint64_t)cfg->num_lps * cfg->events_per_lp, "n must be num_lps * events_per_lp");
  const gpq_phold_params p = params_of(*cfg);
  uint64_t i = 0;
  for (uint32_t lp = 0; lp < cfg->num_lps; ++lp)
    for (uint32_t k = 0; k < cfg->events_per_lp; ++k) out[i++] = gpq_phold_initial(p, lp, k, cfg->events_per_lp);
  return GPQ_OK;
}

gpq_status gpq_phold_children(const gpq_phold_config* cfg, const gpq_item* events, gpq_item* children, uint64_t n) {
  gpq_status st = validate(cfg);
  if (st != GPQ_OK) return st;
  GPQ_CHECK_ARG(events && children, "NULL array");
  if (n == 0) return GPQ_OK;
  gpq_item* d = nullptr;
  GPQ_CUDA_TRY(cudaMalloc(&d, 2 * n * sizeof(gpq_item)));
  cudaError_t e = cudaMemcpy(d, events, n * sizeof(gpq_item), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, 65535);
    phold_children_kernel<<<grid, 256>>>(params_of(*cfg), d, d + n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(children, d + n, n * sizeof(gpq_item), cudaMemcpyDeviceToHost);
  cudaFree(d);
  GPQ_CUDA_TRY(e);
  return GPQ_OK;
}

}  // extern "C"
