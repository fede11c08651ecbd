// Shared plumbing of the per-LP queue objects, and the queue-kind factory.
#include <algorithm>

#include "local_queue_base.h"

namespace gpq {

__global__ void lq_insert_kernel(const gpq_item* __restrict__ items, uint64_t n, uint32_t L, gpq_item* ibuf,
                                 uint32_t* icnt, uint32_t ibc, LocalQueueCounters* ctr) {
  uint32_t ok = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const gpq_item it = items[i];
    if (it.lp >= L) {
      gpq_set_error(&ctr->err, GPQ_ERR_INVALID);
      continue;
    }
    const uint32_t slot = atomicAdd(&icnt[it.lp], 1u);
    if (slot < ibc) {
      ibuf[(size_t)it.lp * ibc + slot] = it;
      ++ok;
    } else {
      gpq_set_error(&ctr->err, GPQ_ERR_INSERT_FULL);
    }
  }
  ok = warp_sum_u32(ok);
  if ((threadIdx.x & 31) == 0 && ok) atomicAdd(&ctr->enqueued, (unsigned long long)ok);
}

// One block of 1024 threads scans L counts in chunks (test/utility path).
__global__ void lq_exclusive_scan_kernel(const uint32_t* __restrict__ cnt, uint32_t L, unsigned long long* offs) {
  __shared__ unsigned long long part[1024];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < L; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const unsigned long long v = (i < L) ? cnt[i] : 0ull;
    part[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
      unsigned long long t = (threadIdx.x >= o) ? part[threadIdx.x - o] : 0ull;
      __syncthreads();
      part[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < L) offs[i] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += part[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) offs[L] = carry;
}

LocalQueueBase::~LocalQueueBase() {
  for (void* p : {(void*)ibuf_, (void*)icnt_, (void*)ctr_, (void*)staging_, (void*)dq_cnt_, (void*)dq_off_,
                  (void*)dq_out_})
    if (p) cudaFree(p);
  if (h_ctr_) cudaFreeHost(h_ctr_);
  if (own_) cudaStreamDestroy(own_);
}

gpq_status LocalQueueBase::init_base(uint32_t L, uint32_t ibc) {
  L_ = L;
  ibc_ = ibc;
  GPQ_CUDA_TRY(cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking));
  GPQ_CUDA_TRY(cudaMalloc(&ibuf_, (size_t)L * ibc * sizeof(gpq_item)));
  GPQ_CUDA_TRY(cudaMalloc(&icnt_, (size_t)L * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&ctr_, sizeof(LocalQueueCounters)));
  GPQ_CUDA_TRY(cudaMallocHost(&h_ctr_, sizeof(LocalQueueCounters)));
  GPQ_CUDA_TRY(cudaMalloc(&dq_cnt_, (size_t)L * sizeof(uint32_t)));
  GPQ_CUDA_TRY(cudaMalloc(&dq_off_, (size_t)(L + 1) * sizeof(unsigned long long)));
  GPQ_CUDA_TRY(cudaMemsetAsync(icnt_, 0, (size_t)L * sizeof(uint32_t), own_));
  GPQ_CUDA_TRY(cudaMemsetAsync(ctr_, 0, sizeof(LocalQueueCounters), own_));
  GPQ_CUDA_TRY(cudaStreamSynchronize(own_));
  return GPQ_OK;
}

gpq_status LocalQueueBase::insert(const gpq_item* items, uint64_t n, bool on_device, cudaStream_t st) {
  const gpq_item* src = items;
  if (!on_device) {
    if (staging_n_ < n) {
      if (staging_) cudaFree(staging_);
      staging_ = nullptr;
      staging_n_ = 0;
      GPQ_CUDA_TRY(cudaMalloc(&staging_, n * sizeof(gpq_item)));
      staging_n_ = n;
    }
    GPQ_CUDA_TRY(cudaMemcpyAsync(staging_, items, n * sizeof(gpq_item), cudaMemcpyHostToDevice, st));
    src = staging_;
  }
  const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, 4096);
  lq_insert_kernel<<<grid, 256, 0, st>>>(src, n, L_, ibuf_, icnt_, ibc_, ctr_);
  GPQ_CUDA_TRY(cudaGetLastError());
  if (!on_device) GPQ_CUDA_TRY(cudaStreamSynchronize(st));  // staging reuse
  return GPQ_OK;
}

gpq_status LocalQueueBase::counts(uint64_t* enqueued, uint64_t* dequeued, cudaStream_t st) {
  GPQ_CUDA_TRY(cudaMemcpyAsync(h_ctr_, ctr_, sizeof(LocalQueueCounters), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  *enqueued = h_ctr_->enqueued;
  *dequeued = h_ctr_->dequeued;
  return GPQ_OK;
}

gpq_status LocalQueueBase::take_error(cudaStream_t st) {
  GPQ_CUDA_TRY(cudaMemcpyAsync(&h_ctr_->err, &ctr_->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  const uint32_t e = h_ctr_->err;
  if (e) {
    GPQ_CUDA_TRY(cudaMemsetAsync(&ctr_->err, 0, sizeof(uint32_t), st));
    set_last_error("queue operation reported status %u", e);
  }
  return (gpq_status)e;
}

gpq_status LocalQueueBase::scan_counts(const uint32_t* cnt, uint64_t* total, cudaStream_t st) {
  lq_exclusive_scan_kernel<<<1, 1024, 0, st>>>(cnt, L_, dq_off_);
  GPQ_CUDA_TRY(cudaGetLastError());
  unsigned long long t = 0;
  GPQ_CUDA_TRY(cudaMemcpyAsync(&t, dq_off_ + L_, sizeof(t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  *total = t;
  return GPQ_OK;
}

gpq_status make_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out) {
  switch (cfg.kind) {
    case GPQ_QUEUE_LAQ: return make_laq_queue(cfg, out);
    case GPQ_QUEUE_LHQ:
    case GPQ_QUEUE_LSQ: return make_lpq_queue(cfg, out);
    case GPQ_QUEUE_GAQ: return make_gaq_queue(cfg, out);
    case GPQ_QUEUE_HQ: return make_hq_queue(cfg, out);
    default:
      set_last_error("queue kind %u is not available", cfg.kind);
      return GPQ_ERR_UNSUPPORTED;
  }
}

}  // namespace gpq
