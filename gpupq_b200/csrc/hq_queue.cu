// Parallel heap queue object (reference: src/heap_queue.cu host API, :1305-1906): the
// heap of sorted r-item nodes maintained by the single-CTA kernels of hq_kernels.cuh.
#include <algorithm>
#include <new>
#include <vector>

#include "host_common.h"
#include "hq_kernels.cuh"
#include "queue_impl.h"

namespace gpq {

namespace {

__global__ void hq_count_lp_kernel(HqDev h, uint32_t lp, uint32_t* out) {
  const uint32_t last = h.meta[0];
  uint32_t c = 0;
  const uint64_t total = (uint64_t)(last + 1) * h.r;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
    if ((i % h.r) < h.cnt[i / h.r] && h.nodes[i].lp == lp) ++c;
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// Gathers every item not of `lp` into out (order irrelevant) and empties the heap.
__global__ void hq_drain_except_kernel(HqDev h, uint32_t lp, gpq_item* out, uint32_t* n_out) {
  const uint32_t last = h.meta[0];
  const uint64_t total = (uint64_t)(last + 1) * h.r;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    if ((i % h.r) < h.cnt[i / h.r]) {
      const gpq_item e = h.nodes[i];
      if (e.lp != lp) out[atomicAdd(n_out, 1u)] = e;
    }
  }
}

class HqQueue final : public QueueImpl {
 public:
  ~HqQueue() override {
    for (void* p : {(void*)h_.nodes, (void*)h_.cnt, (void*)h_.meta, (void*)pend_, (void*)out_, (void*)words_})
      if (p) cudaFree(p);
    if (own_) cudaStreamDestroy(own_);
  }

  gpq_status init(const gpq_queue_config& c) {
    L_ = c.num_lps;
    const uint32_t r = c.node_size ? c.node_size : 1024;
    GPQ_CHECK_ARG(is_pow2(r) && r >= 2 && r <= kHqMaxR, "node_size must be a power of two in [2, 1024]");
    GPQ_CHECK_ARG(L_ <= (1u << 21), "heap queue supports at most 2^21 LPs");
    const uint64_t cap = (uint64_t)(c.capacity ? c.capacity : 256) * L_;
    GPQ_CHECK_ARG(cap <= 0x3fffffffull, "heap queue capacity too large");
    h_.r = r;
    h_.maxnodes = (uint32_t)((cap + r - 1) / r + 2);
    pend_cap_ = (uint32_t)std::min<uint64_t>((uint64_t)(c.insert_capacity ? c.insert_capacity : 64) * L_, cap);
    GPQ_CUDA_TRY(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking));
    GPQ_CUDA_TRY(cudaMalloc(&h_.nodes, (size_t)h_.maxnodes * r * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&h_.cnt, (size_t)h_.maxnodes * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&h_.meta, 4 * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&pend_, (size_t)std::max(pend_cap_, (uint32_t)((cap + 1))) * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&out_, (size_t)(r + 1) * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&words_, 8 * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMemsetAsync(h_.cnt, 0, (size_t)h_.maxnodes * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaMemsetAsync(h_.meta, 0, 4 * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaMemsetAsync(words_, 0, 8 * sizeof(uint32_t), own_));
    const int smem = (int)hq_smem_bytes(r);
    GPQ_CUDA_TRY(gpq::raise_smem_limit(hq_post_kernel, smem));
    GPQ_CUDA_TRY(gpq::raise_smem_limit(hq_dequeue_kernel, smem));
    GPQ_CUDA_TRY(cudaStreamSynchronize(own_));
    return GPQ_OK;
  }

  uint32_t num_lps() const override { return L_; }
  cudaStream_t stream() const override { return own_; }

  gpq_status insert(const gpq_item* items, uint64_t n, bool on_device, cudaStream_t st) override {
    if (npend_ + n > pend_cap_) {
      set_last_error("heap queue: more than %u inserts before post", pend_cap_);
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
    hq_post_kernel<<<1, 512, hq_smem_bytes(h_.r), st>>>(h_, pend_, npend_, words_);
    GPQ_CUDA_TRY(cudaGetLastError());
    npend_ = 0;
    return take_error(st);
  }

  gpq_status get_min(float* min_ts, cudaStream_t st) override {
    uint32_t n0 = 0, b = kInfBits;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&n0, h_.cnt, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (n0) {
      GPQ_CUDA_TRY(cudaMemcpyAsync(&b, &h_.nodes[0].ts, 4, cudaMemcpyDeviceToHost, st));
      GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    }
    *min_ts = gpq_u2f(b);
    return GPQ_OK;
  }

  gpq_status dequeue(float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                     cudaStream_t st) override {
    hq_dequeue_kernel<<<1, 512, hq_smem_bytes(h_.r), st>>>(h_, bound, max_per_lp, out_, words_ + 4);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint32_t n = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&n, words_ + 4, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    *n_out = n;
    if (n > out_capacity) return GPQ_ERR_INVALID;
    if (n) GPQ_CUDA_TRY(cudaMemcpyAsync(out, out_, n * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    deq_ += n;
    return GPQ_OK;
  }

  gpq_status length(uint32_t lp, uint32_t* len, cudaStream_t st) override {
    GPQ_CUDA_TRY(cudaMemsetAsync(words_ + 5, 0, 4, st));
    hq_count_lp_kernel<<<64, 256, 0, st>>>(h_, lp, words_ + 5);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(len, words_ + 5, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  // queue_clear(lp): the other LPs' items are re-inserted into an emptied heap.
  gpq_status clear(uint32_t lp, cudaStream_t st) override {
    if (npend_) {
      gpq_status s = post(st);
      if (s != GPQ_OK) return s;
    }
    uint32_t len = 0;
    gpq_status s = length(lp, &len, st);
    if (s != GPQ_OK) return s;
    GPQ_CUDA_TRY(cudaMemsetAsync(words_ + 6, 0, 4, st));
    hq_drain_except_kernel<<<64, 256, 0, st>>>(h_, lp, pend_, words_ + 6);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint32_t n = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&n, words_ + 6, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemsetAsync(h_.cnt, 0, (size_t)h_.maxnodes * sizeof(uint32_t), st));
    GPQ_CUDA_TRY(cudaMemsetAsync(h_.meta, 0, 4 * sizeof(uint32_t), st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (n) {
      hq_post_kernel<<<1, 512, hq_smem_bytes(h_.r), st>>>(h_, pend_, n, words_);
      GPQ_CUDA_TRY(cudaGetLastError());
    }
    deq_ += len;
    return take_error(st);
  }

  // queue_print as data: the LP's items from a host copy of the nodes, in key order.
  gpq_status dump(uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out, cudaStream_t st) override {
    uint32_t meta[2];
    GPQ_CUDA_TRY(cudaMemcpyAsync(meta, h_.meta, sizeof(meta), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t nn = meta[0] + 1;
    std::vector<uint32_t> cnt(nn);
    std::vector<gpq_item> it((size_t)nn * h_.r);
    GPQ_CUDA_TRY(cudaMemcpyAsync(cnt.data(), h_.cnt, nn * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(it.data(), h_.nodes, it.size() * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<gpq_item> sel;
    for (uint32_t i = 0; i < nn; ++i)
      for (uint32_t j = 0; j < cnt[i]; ++j)
        if (it[(size_t)i * h_.r + j].lp == lp) sel.push_back(it[(size_t)i * h_.r + j]);
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
  static bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }
  gpq_status take_error(cudaStream_t st) {
    uint32_t e = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&e, words_, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (e) {
      GPQ_CUDA_TRY(cudaMemsetAsync(words_, 0, 4, st));
      set_last_error("heap queue reported status %u", e);
    }
    return (gpq_status)e;
  }
  uint32_t L_ = 0, pend_cap_ = 0, npend_ = 0;
  uint64_t enq_ = 0, deq_ = 0;
  cudaStream_t own_ = nullptr;
  HqDev h_{};
  gpq_item* pend_ = nullptr;
  gpq_item* out_ = nullptr;
  uint32_t* words_ = nullptr;
};

}  // namespace

gpq_status make_hq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out) {
  auto q = std::unique_ptr<HqQueue>(new (std::nothrow) HqQueue());
  if (!q) return GPQ_ERR_NOMEM;
  gpq_status s = q->init(cfg);
  if (s != GPQ_OK) return s;
  out = std::move(q);
  return GPQ_OK;
}

}  // namespace gpq
