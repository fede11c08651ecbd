// Local array queue object (reference: src/local_array_queue.cu): per-LP sorted ring,
// warp-per-LP merge on queue_post, head-of-ring dequeue inside the window.
#include <algorithm>
#include <new>

#include "laq.cuh"
#include "local_queue_base.h"

namespace gpq {

namespace {

__global__ void laq_post_kernel(LaqDev q, gpq_item* ibuf, uint32_t* icnt, uint32_t ibc, uint32_t L,
                                LocalQueueCounters* ctr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LaneGroup<32> g;
  const uint32_t wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const LaqGroupSmem sm = laq_group_smem(smem_raw + (size_t)wib * laq_group_smem_bytes(ibc, 32), ibc, 32);
  const uint32_t cap = 1u << q.cap_log2, mask = cap - 1u;
  for (uint32_t lp = blockIdx.x * wpb + wib; lp < L; lp += gridDim.x * wpb) {
    uint32_t k = min(icnt[lp], ibc);
    if (k == 0) continue;
    const uint32_t rd = q.rd[lp], wr = q.wr[lp];
    const uint32_t n = wr - rd;
    if (n + k > cap) {
      if (g.gl == 0) gpq_set_error(&ctr->err, GPQ_ERR_QUEUE_FULL);
      k = cap - n;
    }
    laq_merge<32>(q.ring + ((size_t)lp << q.cap_log2), mask, rd, n, ibuf + (size_t)lp * ibc, k, sm, g);
    if (g.gl == 0) {
      q.wr[lp] = wr + k;
      icnt[lp] = 0;
    }
  }
}

__global__ void laq_min_kernel(LaqDev q, uint32_t L, LocalQueueCounters* ctr) {
  __shared__ uint32_t red[32];
  const uint32_t mask = (1u << q.cap_log2) - 1u;
  uint32_t mn = kInfBits;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t rd = q.rd[lp], wr = q.wr[lp];
    if (rd != wr) mn = min(mn, gpq_f2u(q.ring[((size_t)lp << q.cap_log2) + (rd & mask)].ts));
  }
  mn = block_min_u32(mn, red);
  if (threadIdx.x == 0) atomicMin(&ctr->min_bits, mn);
}

// Pass 1 of the dequeue: number of items of each LP below the bound (<= max_per_lp).
__global__ void laq_count_safe_kernel(LaqDev q, uint32_t L, float bound, uint32_t max_per_lp, uint32_t* cnt) {
  const uint32_t mask = (1u << q.cap_log2) - 1u;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t rd = q.rd[lp], n = q.wr[lp] - rd;
    const gpq_item* ring = q.ring + ((size_t)lp << q.cap_log2);
    uint32_t c = 0;
    while (c < n && (max_per_lp == 0 || c < max_per_lp) && ring[(rd + c) & mask].ts < bound) ++c;
    cnt[lp] = c;
  }
}

// Pass 2: copy the counted items to their LP's output range and advance fel_read
// (queue_peek + queue_set_done, src/local_array_queue.cu:710-779).
__global__ void laq_take_kernel(LaqDev q, uint32_t L, const uint32_t* cnt, const unsigned long long* off,
                                gpq_item* out, LocalQueueCounters* ctr) {
  const uint32_t mask = (1u << q.cap_log2) - 1u;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t c = cnt[lp];
    if (!c) continue;
    const uint32_t rd = q.rd[lp];
    const gpq_item* ring = q.ring + ((size_t)lp << q.cap_log2);
    for (uint32_t i = 0; i < c; ++i) out[off[lp] + i] = ring[(rd + i) & mask];
    q.rd[lp] = rd + c;
    atomicAdd(&ctr->dequeued, (unsigned long long)c);
  }
}

__global__ void laq_set_bound_kernel(float* bound, float value) { *bound = value; }

__global__ void laq_clear_kernel(LaqDev q, uint32_t lp, LocalQueueCounters* ctr) {
  const uint32_t n = q.wr[lp] - q.rd[lp];
  q.rd[lp] = q.wr[lp];
  atomicAdd(&ctr->dequeued, (unsigned long long)n);
}

class LaqQueue final : public LocalQueueBase {
 public:
  ~LaqQueue() override {
    for (void* p : {(void*)ring_, (void*)rd_, (void*)wr_, (void*)bound_})
      if (p) cudaFree(p);
  }

  gpq_status device_view(gpq_device_queue* v) override {
    *v = gpq_device_queue{};
    v->ring = ring_;
    v->rd = rd_;
    v->wr = wr_;
    v->ibuf = ibuf_;
    v->icnt = icnt_;
    v->bound = bound_;
    v->enqueued = &ctr_->enqueued;
    v->dequeued = &ctr_->dequeued;
    v->err = &ctr_->err;
    v->num_lps = L_;
    v->cap_log2 = cap_log2_;
    v->ibc = ibc_;
    v->kind = GPQ_QUEUE_LAQ;
    v->size = nullptr;
    return GPQ_OK;
  }

  gpq_status set_bound(float b, cudaStream_t st) override {
    laq_set_bound_kernel<<<1, 1, 0, st>>>(bound_, b);
    GPQ_CUDA_TRY(cudaGetLastError());
    return GPQ_OK;
  }

  gpq_status init(const gpq_queue_config& c) {
    uint32_t cap = c.capacity ? c.capacity : 256;
    GPQ_CHECK_ARG(cap >= 2 && cap <= (1u << 20) && !(cap & (cap - 1)), "LAQ capacity must be a power of two");
    uint32_t ibc = c.insert_capacity ? c.insert_capacity : 64;
    GPQ_CHECK_ARG(ibc <= 1024, "insert_capacity must be <= 1024");
    cap_log2_ = 0;
    while ((1u << cap_log2_) < cap) ++cap_log2_;
    gpq_status s = init_base(c.num_lps, ibc);
    if (s != GPQ_OK) return s;
    GPQ_CUDA_TRY(cudaMalloc(&ring_, ((size_t)L_ << cap_log2_) * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&rd_, (size_t)L_ * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&wr_, (size_t)L_ * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMemsetAsync(rd_, 0, (size_t)L_ * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaMemsetAsync(wr_, 0, (size_t)L_ * sizeof(uint32_t), own_));
    GPQ_CUDA_TRY(cudaMalloc(&bound_, sizeof(float)));
    laq_set_bound_kernel<<<1, 1, 0, own_>>>(bound_, gpq_u2f(kInfBits));
    const size_t smem = 8 * laq_group_smem_bytes(ibc_, 32);
    GPQ_CUDA_TRY(gpq::raise_smem_limit(laq_post_kernel, (int)smem));
    GPQ_CUDA_TRY(cudaStreamSynchronize(own_));
    return GPQ_OK;
  }

  gpq_status post(cudaStream_t st) override {
    const uint32_t grid = std::max(1u, std::min<uint32_t>((L_ + 7) / 8, 8192));
    laq_post_kernel<<<grid, 256, 8 * laq_group_smem_bytes(ibc_, 32), st>>>(dev(), ibuf_, icnt_, ibc_, L_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    return take_error(st);
  }

  gpq_status get_min(float* min_ts, cudaStream_t st) override {
    const uint32_t inf = kInfBits;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&ctr_->min_bits, &inf, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    const uint32_t grid = std::max(1u, std::min<uint32_t>((L_ + 255) / 256, 1024));
    laq_min_kernel<<<grid, 256, 0, st>>>(dev(), L_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(&h_ctr_->min_bits, &ctr_->min_bits, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    *min_ts = gpq_u2f(h_ctr_->min_bits);
    return GPQ_OK;
  }

  gpq_status dequeue(float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                     cudaStream_t st) override {
    const uint32_t grid = std::max(1u, std::min<uint32_t>((L_ + 255) / 256, 1024));
    laq_count_safe_kernel<<<grid, 256, 0, st>>>(dev(), L_, bound, max_per_lp, dq_cnt_);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint64_t total = 0;
    gpq_status s = scan_counts(dq_cnt_, &total, st);
    if (s != GPQ_OK) return s;
    *n_out = total;
    if (total > out_capacity) {
      set_last_error("dequeue: %llu items do not fit the output (%llu)", (unsigned long long)total,
                     (unsigned long long)out_capacity);
      return GPQ_ERR_INVALID;
    }
    if (total == 0) return GPQ_OK;
    if (dq_out_n_ < total) {
      if (dq_out_) cudaFree(dq_out_);
      dq_out_ = nullptr;
      dq_out_n_ = 0;
      GPQ_CUDA_TRY(cudaMalloc(&dq_out_, total * sizeof(gpq_item)));
      dq_out_n_ = total;
    }
    laq_take_kernel<<<grid, 256, 0, st>>>(dev(), L_, dq_cnt_, dq_off_, dq_out_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(out, dq_out_, total * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  gpq_status length(uint32_t lp, uint32_t* len, cudaStream_t st) override {
    uint32_t rw[2];
    GPQ_CUDA_TRY(cudaMemcpyAsync(&rw[0], rd_ + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&rw[1], wr_ + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    *len = rw[1] - rw[0];
    return GPQ_OK;
  }

  gpq_status clear(uint32_t lp, cudaStream_t st) override {
    laq_clear_kernel<<<1, 1, 0, st>>>(dev(), lp, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    return GPQ_OK;
  }

  gpq_status dump(uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out, cudaStream_t st) override {
    uint32_t rw[2];
    GPQ_CUDA_TRY(cudaMemcpyAsync(&rw[0], rd_ + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&rw[1], wr_ + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t n = rw[1] - rw[0];
    *n_out = n;
    if (n > out_capacity) return GPQ_ERR_INVALID;
    const uint32_t cap = 1u << cap_log2_, mask = cap - 1u;
    const gpq_item* ring = ring_ + ((size_t)lp << cap_log2_);
    const uint32_t start = rw[0] & mask;
    const uint32_t first = std::min(n, cap - start);
    if (first) GPQ_CUDA_TRY(cudaMemcpyAsync(out, ring + start, first * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    if (n > first) GPQ_CUDA_TRY(cudaMemcpyAsync(out + first, ring, (n - first) * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  // Raw ring slots of one LP (for the reference's ring-position known-answer tests).
  LaqDev dev() const { return LaqDev{ring_, rd_, wr_, cap_log2_}; }

 private:
  gpq_item* ring_ = nullptr;
  float* bound_ = nullptr;  // window bound read by queue_peek on the device
  uint32_t* rd_ = nullptr;
  uint32_t* wr_ = nullptr;
  uint32_t cap_log2_ = 0;
};

}  // namespace

gpq_status make_laq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out) {
  auto q = std::unique_ptr<LaqQueue>(new (std::nothrow) LaqQueue());
  if (!q) return GPQ_ERR_NOMEM;
  gpq_status s = q->init(cfg);
  if (s != GPQ_OK) return s;
  out = std::move(q);
  return GPQ_OK;
}

}  // namespace gpq
