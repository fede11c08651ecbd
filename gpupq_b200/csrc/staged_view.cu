// Staged per-LP heads: device-side queue access for the global array, heap and local
// splay queues (see staged_view.h).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "host_common.h"
#include "queue_impl.h"
#include "staged_view.h"

namespace gpq {

namespace {

__global__ void staged_reset_kernel(gpq_item* head, uint32_t* taken, uint32_t* icnt, uint32_t L) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    gpq_item e;
    e.ts = gpq_u2f(kInfBits);
    e.lp = lp;
    e.id = 0xffffffffu;
    e.aux = 0;
    head[lp] = e;
    taken[lp] = 0;
    icnt[lp] = 0;
  }
}

// Gathers, for the queue's insert path, the items inserted by model kernels and every
// staged head that was not taken; clears the per-LP state.
__global__ void staged_gather_kernel(gpq_item* head, uint32_t* taken, gpq_item* ibuf, uint32_t* icnt, uint32_t ibc,
                                     uint32_t L, gpq_item* out, uint32_t* words) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t c = icnt[lp];
    if (c > ibc) gpq_set_error(&words[0], GPQ_ERR_INSERT_FULL);
    const uint32_t k = min(c, ibc);
    if (k) {
      const uint32_t pos = atomicAdd(&words[1], k);
      for (uint32_t j = 0; j < k; ++j) out[pos + j] = ibuf[(size_t)lp * ibc + j];
    }
    const gpq_item h = head[lp];
    if (gpq_f2u(h.ts) != kInfBits && !taken[lp]) {
      out[atomicAdd(&words[1], 1u)] = h;
      atomicAdd(&words[2], 1u);
    }
    gpq_item e = h;
    e.ts = gpq_u2f(kInfBits);
    head[lp] = e;
    taken[lp] = 0;
    icnt[lp] = 0;
  }
}

__global__ void staged_bound_kernel(float* bound, float b) { *bound = b; }

}  // namespace

StagedView::~StagedView() {
  for (void* p : {(void*)head_, (void*)taken_, (void*)ibuf_, (void*)icnt_, (void*)bound_, (void*)ctr_,
                  (void*)words_, (void*)out_})
    if (p) cudaFree(p);
  if (h_words_) cudaFreeHost(h_words_);
}

gpq_status StagedView::init(uint32_t num_lps, uint32_t insert_capacity, cudaStream_t st) {
  L_ = num_lps;
  ibc_ = insert_capacity ? insert_capacity : 64;
  GPQ_CHECK_ARG(ibc_ <= 1024, "insert_capacity must be <= 1024");
  GPQ_CUDA_TRY(cudaMalloc(&head_, (size_t)L_ * sizeof(gpq_item)));
  GPQ_CUDA_TRY(cudaMalloc(&taken_, (size_t)L_ * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&ibuf_, (size_t)L_ * ibc_ * sizeof(gpq_item)));
  GPQ_CUDA_TRY(cudaMalloc(&icnt_, (size_t)L_ * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&bound_, sizeof(float)));
  GPQ_CUDA_TRY(cudaMalloc(&ctr_, 2 * sizeof(unsigned long long)));
  GPQ_CUDA_TRY(cudaMalloc(&words_, 4 * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&out_, ((size_t)L_ * ibc_ + L_) * sizeof(gpq_item)));
  GPQ_CUDA_TRY(cudaMallocHost(&h_words_, 4 * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMemsetAsync(ctr_, 0, 2 * sizeof(unsigned long long), st));
  GPQ_CUDA_TRY(cudaMemsetAsync(words_, 0, 4 * sizeof(uint32_t), st));
  const uint32_t grid = std::max(1u, std::min<uint32_t>((L_ + 255) / 256, 4096));
  staged_reset_kernel<<<grid, 256, 0, st>>>(head_, taken_, icnt_, L_);
  staged_bound_kernel<<<1, 1, 0, st>>>(bound_, gpq_u2f(kInfBits));
  GPQ_CUDA_TRY(cudaGetLastError());
  h_out_.resize(L_);
  h_head_.resize(L_);
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

void StagedView::fill(gpq_device_queue* v, uint32_t kind) const {
  std::memset(v, 0, sizeof(*v));
  v->ibuf = ibuf_;
  v->icnt = icnt_;
  v->bound = bound_;
  v->enqueued = &ctr_[0];
  v->dequeued = &ctr_[1];
  v->err = &words_[0];
  v->num_lps = L_;
  v->ibc = ibc_;
  v->kind = kind;
  v->head = head_;
  v->taken = taken_;
  v->staged = 1u;
}

gpq_status StagedView::set_bound(QueueImpl* q, float bound, cudaStream_t st) {
  gpq_status s = flush(q, st);  // heads of an earlier bound go back first
  if (s != GPQ_OK) return s;
  s = q->post(st);
  if (s != GPQ_OK) return s;
  uint64_t n = 0;
  s = q->dequeue(bound, 1, h_out_.data(), h_out_.size(), &n, st);
  if (s != GPQ_OK) return s;
  gpq_item none;
  none.ts = gpq_u2f(kInfBits);
  none.id = 0xffffffffu;
  none.aux = 0;
  for (uint32_t lp = 0; lp < L_; ++lp) {
    none.lp = lp;
    h_head_[lp] = none;
  }
  for (uint64_t i = 0; i < n; ++i) h_head_[h_out_[i].lp] = h_out_[i];
  GPQ_CUDA_TRY(cudaMemcpyAsync(head_, h_head_.data(), (size_t)L_ * sizeof(gpq_item), cudaMemcpyHostToDevice, st));
  staged_bound_kernel<<<1, 1, 0, st>>>(bound_, bound);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));  // h_head_ is reused by the next call
  return GPQ_OK;
}

gpq_status StagedView::flush(QueueImpl* q, cudaStream_t st) {
  GPQ_CUDA_TRY(cudaMemsetAsync(&words_[1], 0, 2 * sizeof(uint32_t), st));
  const uint32_t grid = std::max(1u, std::min<uint32_t>((L_ + 255) / 256, 4096));
  staged_gather_kernel<<<grid, 256, 0, st>>>(head_, taken_, ibuf_, icnt_, ibc_, L_, out_, words_);
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaMemcpyAsync(h_words_, words_, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_words_[0] != 0) {
    const uint32_t e = h_words_[0];
    GPQ_CUDA_TRY(cudaMemsetAsync(&words_[0], 0, sizeof(uint32_t), st));
    set_last_error(e == GPQ_ERR_UNSUPPORTED
                       ? "a model kernel called queue_length, queue_is_empty or queue_clear, which this queue kind "
                         "does not offer on the device"
                       : "a model kernel inserted more items into one LP than insert_capacity between two posts");
    return (gpq_status)e;
  }
  restaged_ += h_words_[2];
  if (h_words_[1]) return q->insert(out_, h_words_[1], true, st);
  return GPQ_OK;
}

}  // namespace gpq
