// Global array queue object (reference: src/global_array_queue.cu, host API
// :181-308): one array sorted by timestamp; queue_post sorts the buffered inserts with
// the project's radix sort and merges them in; the dequeue takes, per LP, the first
// max_per_lp items below the bound (the reference's mark_safe_events takes one per LP,
// :147-179) and compacts the rest back in order.
#include <algorithm>
#include <new>
#include <vector>

#include "gaq.cuh"
#include "gaq_engine.h"
#include "host_common.h"
#include "queue_impl.h"

namespace gpq {

namespace {

// Staged index lists per LP: idx[lp * ibc + slot] = array position.
__global__ void gq_stage_idx_kernel(const gpq_item* __restrict__ arr, uint32_t c, uint32_t L, uint32_t* idx,
                                    uint32_t* cnt, uint32_t ibc, uint32_t* err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const uint32_t lp = arr[i].lp;
    if (lp >= L) { gpq_set_error(err, GPQ_ERR_INVALID); continue; }
    const uint32_t slot = atomicAdd(&cnt[lp], 1u);
    if (slot < ibc) idx[(size_t)lp * ibc + slot] = i;
    else gpq_set_error(err, GPQ_ERR_INSERT_FULL);
  }
}

// Per LP: rank the staged items by key; the first `max_per_lp` (0 = all) are taken:
// flagged in `taken` and written to tmp[lp * ibc + rank].
__global__ void gq_take_kernel(const gpq_item* __restrict__ arr, uint32_t L, const uint32_t* idx, uint32_t* cnt,
                               uint32_t ibc, uint32_t max_per_lp, uint32_t* taken, gpq_item* tmp, uint32_t* out_cnt) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t k = min(cnt[lp], ibc);
    const uint32_t lim = max_per_lp ? min(k, max_per_lp) : k;
    const uint32_t* li = idx + (size_t)lp * ibc;
    for (uint32_t j = 0; j < k; ++j) {
      const gpq_item e = arr[li[j]];
      uint32_t r = 0;
      for (uint32_t i = 0; i < k; ++i) r += gpq_item_less(arr[li[i]], e) ? 1u : 0u;
      if (r < lim) {
        taken[li[j]] = 1u;
        tmp[(size_t)lp * ibc + r] = e;
      }
    }
    out_cnt[lp] = lim;
    cnt[lp] = 0;
  }
}

__global__ void gq_gather_kernel(uint32_t L, uint32_t ibc, const gpq_item* tmp, const uint32_t* out_cnt,
                                 const uint32_t* off, gpq_item* out) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x)
    for (uint32_t i = 0; i < out_cnt[lp]; ++i) out[off[lp] + i] = tmp[(size_t)lp * ibc + i];
}

// keep[i] = 1 - taken[i] (prefix part), then after an exclusive scan the kept items
// move to their compacted positions.
__global__ void gq_keep_kernel(const uint32_t* taken, uint32_t c, uint32_t* keep) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= c; i += gridDim.x * blockDim.x)
    keep[i] = (i < c) ? (1u - taken[i]) : 0u;
}

__global__ void gq_compact_kernel(const gpq_item* __restrict__ arr, uint32_t c, uint32_t n, const uint32_t* taken,
                                  const uint32_t* pos, gpq_item* out) {
  const uint32_t kept = pos[c];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < c) {
      if (!taken[i]) out[pos[i]] = arr[i];
    } else {
      out[kept + (i - c)] = arr[i];
    }
  }
}

__global__ void gq_clear_lp_kernel(const gpq_item* __restrict__ arr, uint32_t n, uint32_t lp, uint32_t* keep) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
    keep[i] = (i < n && arr[i].lp != lp) ? 1u : 0u;
}

__global__ void gq_select_kernel(const gpq_item* __restrict__ arr, uint32_t n, const uint32_t* keep, const uint32_t* pos,
                                 gpq_item* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (keep[i]) out[pos[i]] = arr[i];
}

__global__ void gq_minmax_kernel(const gpq_item* __restrict__ a, uint32_t n, uint32_t* mm) {
  uint32_t mn = 0xffffffffu, mx = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    mn = min(mn, gpq_f2u(a[i].ts));
    mx = max(mx, gpq_f2u(a[i].ts));
  }
  mn = warp_min_u32(mn);
  mx = __reduce_max_sync(GPQ_FULL_MASK, mx);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], mn);
    atomicMax(&mm[1], mx);
  }
}

__global__ void gq_count_lp_kernel(const gpq_item* __restrict__ arr, uint32_t n, uint32_t lp, uint32_t* out) {
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += arr[i].lp == lp;
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

class GaqQueue final : public QueueImpl {
 public:
  ~GaqQueue() override {
    for (void* p : {(void*)arr_[0], (void*)arr_[1], (void*)pend_, (void*)pend_tmp_, (void*)hist_, (void*)scan_tmp_, (void*)idx_,
                    (void*)cnt_, (void*)out_cnt_, (void*)off_, (void*)tmp_, (void*)taken_, (void*)keep_,
                    (void*)words_, (void*)out_, (void*)split_})
      if (p) cudaFree(p);
    if (h_words_) cudaFreeHost(h_words_);
    if (own_) cudaStreamDestroy(own_);
  }

  gpq_status init(const gpq_queue_config& c) {
    L_ = c.num_lps;
    const uint64_t cap = (uint64_t)(c.capacity ? c.capacity : 256) * L_;
    GPQ_CHECK_ARG(cap <= 0x3fffffffull, "global array queue capacity too large");
    cap_ = (uint32_t)cap;
    ibc_ = c.insert_capacity ? c.insert_capacity : 64;
    GPQ_CHECK_ARG(ibc_ <= 4096, "insert_capacity must be <= 4096");
    pend_cap_ = (uint32_t)std::min<uint64_t>((uint64_t)ibc_ * L_, cap_);
    lpcap_ = c.capacity ? c.capacity : 256;  // a dequeue may take every item of an LP
    GPQ_CUDA_TRY(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking));
    GPQ_CUDA_TRY(cudaMalloc(&arr_[0], (size_t)cap_ * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&arr_[1], (size_t)cap_ * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&pend_, (size_t)pend_cap_ * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&pend_tmp_, (size_t)pend_cap_ * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&hist_, radix_hist_words(pend_cap_) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&split_, merge_split_words(cap_) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&scan_tmp_, scan_scratch_words((uint64_t)std::max(cap_, L_) + 1) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&idx_, (size_t)L_ * lpcap_ * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&tmp_, (size_t)L_ * lpcap_ * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&cnt_, (size_t)L_ * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&out_cnt_, (size_t)(L_ + 1) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&off_, (size_t)(L_ + 1) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&taken_, (size_t)(cap_ + 1) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&keep_, (size_t)(cap_ + 1) * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&words_, 16 * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMallocHost(&h_words_, 16 * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMemsetAsync(cnt_, 0, (size_t)L_ * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaMemsetAsync(words_, 0, 16 * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaStreamSynchronize(own_));
    return GPQ_OK;
  }

  uint32_t num_lps() const override { return L_; }
  cudaStream_t stream() const override { return own_; }

  gpq_status insert(const gpq_item* items, uint64_t n, bool on_device, cudaStream_t st) override {
    if (npend_ + n > pend_cap_) {
      set_last_error("global array queue: more than %u inserts before post", pend_cap_);
      return GPQ_ERR_INSERT_FULL;
    }
    GPQ_CUDA_TRY(cudaMemcpyAsync(pend_ + npend_, items, n * sizeof(gpq_item),
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    npend_ += (uint32_t)n;
    enq_ += n;
    return GPQ_OK;
  }

  gpq_status post(cudaStream_t st) override {
    if (npend_ == 0) return GPQ_OK;
    if ((uint64_t)n_ + npend_ > cap_) {
      set_last_error("global array queue full");
      return GPQ_ERR_QUEUE_FULL;
    }
    const uint32_t mm0[2] = {0xffffffffu, 0u};
    GPQ_CUDA_TRY(cudaMemcpyAsync(words_, mm0, sizeof(mm0), cudaMemcpyHostToDevice, st));
    gq_minmax_kernel<<<grid(npend_), 256, 0, st>>>(pend_, npend_, words_);
    GPQ_CUDA_TRY(cudaMemcpyAsync(h_words_, words_, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    gpq_item* sorted = nullptr;
    gpq_status s = radix_sort_by_ts(pend_, pend_tmp_, npend_, h_words_[0], h_words_[1], hist_, &sorted,
                                    words_ + kBulkErrWord, st);
    if (s != GPQ_OK) return s;
    s = merge_by_ts(arr_[cur_], n_, sorted, npend_, arr_[cur_ ^ 1], split_, words_ + kBulkErrWord, st);
    if (s != GPQ_OK) return s;
    cur_ ^= 1;
    n_ += npend_;
    npend_ = 0;
    uint32_t berr = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&berr, words_ + kBulkErrWord, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (berr) {
      set_last_error("global array queue: a staged sort or merge tile did not arrive in time");
      return (gpq_status)berr;
    }
    return GPQ_OK;
  }

  gpq_status get_min(float* min_ts, cudaStream_t st) override {
    uint32_t b = kInfBits;
    if (n_) {
      GPQ_CUDA_TRY(cudaMemcpyAsync(&b, &arr_[cur_][0].ts, 4, cudaMemcpyDeviceToHost, st));
      GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    }
    *min_ts = gpq_u2f(b);
    return GPQ_OK;
  }

  gpq_status dequeue(float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                     cudaStream_t st) override {
    *n_out = 0;
    if (n_ == 0) return GPQ_OK;
    const gpq_item* a = arr_[cur_];
    gaq_split_kernel<<<1, 32, 0, st>>>(a, n_, bound, 3.0e38f, words_);
    GPQ_CUDA_TRY(cudaMemcpyAsync(h_words_, words_, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t c = h_words_[0];
    if (c == 0) return GPQ_OK;
    GPQ_CUDA_TRY(cudaMemsetAsync(taken_, 0, (size_t)(c + 1) * sizeof(uint32_t), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(&words_[8], 0, 4, st));
    gq_stage_idx_kernel<<<grid(c), 256, 0, st>>>(a, c, L_, idx_, cnt_, lpcap_, &words_[8]);
    gq_take_kernel<<<grid(L_), 256, 0, st>>>(a, L_, idx_, cnt_, lpcap_, max_per_lp, taken_, tmp_, out_cnt_);
    GPQ_CUDA_TRY(cudaMemsetAsync(out_cnt_ + L_, 0, 4, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(off_, out_cnt_, (size_t)(L_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    if (gpq_status s_ = scan_exclusive(off_, off_, L_ + 1, scan_tmp_, st)) return s_;
    uint32_t total = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&total, off_ + L_, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&h_words_[8], &words_[8], 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (h_words_[8]) return (gpq_status)h_words_[8];
    *n_out = total;
    if (total > out_capacity) {
      set_last_error("dequeue: %u items do not fit the output", total);
      return GPQ_ERR_INVALID;
    }
    if (!out_ || out_n_ < total) {
      if (out_) cudaFree(out_);
      out_ = nullptr;
      GPQ_CUDA_TRY(cudaMalloc(&out_, (size_t)std::max(total, 1u) * sizeof(gpq_item)));
      out_n_ = total;
    }
    gq_gather_kernel<<<grid(L_), 256, 0, st>>>(L_, lpcap_, tmp_, out_cnt_, off_, out_);
    // stable compaction of the untaken prefix, followed by the rest of the array
    gq_keep_kernel<<<grid(c + 1), 256, 0, st>>>(taken_, c, keep_);
    if (gpq_status s_ = scan_exclusive(keep_, keep_, c + 1, scan_tmp_, st)) return s_;
    gq_compact_kernel<<<grid(n_), 256, 0, st>>>(a, c, n_, taken_, keep_, arr_[cur_ ^ 1]);
    GPQ_CUDA_TRY(cudaGetLastError());
    if (total) GPQ_CUDA_TRY(cudaMemcpyAsync(out, out_, (size_t)total * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    cur_ ^= 1;
    n_ -= total;
    deq_ += total;
    return GPQ_OK;
  }

  gpq_status length(uint32_t lp, uint32_t* len, cudaStream_t st) override {
    GPQ_CUDA_TRY(cudaMemsetAsync(&words_[9], 0, 4, st));
    if (n_) gq_count_lp_kernel<<<grid(n_), 256, 0, st>>>(arr_[cur_], n_, lp, &words_[9]);
    GPQ_CUDA_TRY(cudaMemcpyAsync(len, &words_[9], 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  gpq_status clear(uint32_t lp, cudaStream_t st) override {
    if (n_ == 0) return GPQ_OK;
    gq_clear_lp_kernel<<<grid(n_ + 1), 256, 0, st>>>(arr_[cur_], n_, lp, keep_);
    GPQ_CUDA_TRY(cudaMemcpyAsync(taken_, keep_, (size_t)(n_ + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    if (gpq_status s_ = scan_exclusive(keep_, keep_, n_ + 1, scan_tmp_, st)) return s_;
    gq_select_kernel<<<grid(n_), 256, 0, st>>>(arr_[cur_], n_, taken_, keep_, arr_[cur_ ^ 1]);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint32_t kept = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&kept, keep_ + n_, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    deq_ += n_ - kept;
    n_ = kept;
    cur_ ^= 1;
    return GPQ_OK;
  }

  // queue_print as data: the LP's items, in key order (the selection and the final order
  // of equal timestamps are done on a host copy).
  gpq_status dump(uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out, cudaStream_t st) override {
    std::vector<gpq_item> h(n_);
    if (n_) GPQ_CUDA_TRY(cudaMemcpyAsync(h.data(), arr_[cur_], (size_t)n_ * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<gpq_item> sel;
    for (const gpq_item& e : h)
      if (e.lp == lp) sel.push_back(e);
    std::sort(sel.begin(), sel.end(), [](const gpq_item& a, const gpq_item& b) { return gpq_item_less(a, b); });
    *n_out = sel.size();
    if (sel.size() > out_capacity) return GPQ_ERR_INVALID;
    std::copy(sel.begin(), sel.end(), out);
    return GPQ_OK;
  }

  gpq_status counts(uint64_t* enqueued, uint64_t* dequeued, cudaStream_t) override {
    *enqueued = enq_;
    *dequeued = deq_;
    return GPQ_OK;
  }

 private:
  static uint32_t grid(uint32_t n) { return std::max(1u, std::min<uint32_t>((n + 255) / 256, 4096)); }
  uint32_t L_ = 0, cap_ = 0, ibc_ = 0, pend_cap_ = 0, lpcap_ = 0;
  cudaStream_t own_ = nullptr;
  gpq_item* arr_[2] = {nullptr, nullptr};
  int cur_ = 0;
  uint32_t n_ = 0, npend_ = 0;
  uint64_t enq_ = 0, deq_ = 0;
  gpq_item* pend_ = nullptr;
  gpq_item* pend_tmp_ = nullptr;
  uint32_t* hist_ = nullptr;
  uint32_t* scan_tmp_ = nullptr;  // scan_exclusive scratch
  uint32_t* idx_ = nullptr;
  uint32_t* cnt_ = nullptr;
  uint32_t* out_cnt_ = nullptr;
  uint32_t* off_ = nullptr;
  gpq_item* tmp_ = nullptr;
  uint32_t* taken_ = nullptr;
  uint32_t* keep_ = nullptr;
  uint32_t* words_ = nullptr;  // [16] scratch words; [kBulkErrWord] the sort/merge staging error
  static constexpr uint32_t kBulkErrWord = 15;
  uint32_t* split_ = nullptr;  // merge-path splits of the post's merge
  uint32_t* h_words_ = nullptr;
  gpq_item* out_ = nullptr;
  uint32_t out_n_ = 0;
};

}  // namespace

gpq_status make_gaq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out) {
  auto q = std::unique_ptr<GaqQueue>(new (std::nothrow) GaqQueue());
  if (!q) return GPQ_ERR_NOMEM;
  gpq_status s = q->init(cfg);
  if (s != GPQ_OK) return s;
  out = std::move(q);
  return GPQ_OK;
}

}  // namespace gpq
