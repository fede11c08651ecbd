// Queue objects for the local heap queue (src/local_heap_queue.cu) and the local splay
// queue (src/local_splay_queue.cu): the reference's host queue API over the same
// per-LP layouts and device operations the PHOLD engine uses (lhq.cuh, lsq.cuh), one
// thread per LP.
#include <algorithm>
#include <new>
#include <vector>

#include "lhq.cuh"
#include "local_queue_base.h"
#include "lsq.cuh"

namespace gpq {

namespace {

struct LpqDev {
  uint32_t kind;
  uint32_t cap_log2;
  gpq_item* items;
  uint32_t* size;
  uint32_t* root;      // LSQ
  uint32_t* freetop;   // LSQ
  uint32_t* links;     // LSQ
  uint16_t* freestk;   // LSQ
};

__global__ void lpq_init_kernel(LpqDev q, uint32_t L) {
  const uint32_t cap = 1u << q.cap_log2;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    q.size[lp] = 0;
    if (q.kind == GPQ_QUEUE_LSQ) {
      const size_t base = (size_t)lp << q.cap_log2;
      for (uint32_t j = 0; j < cap; ++j) {
        q.items[base + j].lp = 0xffffffffu;
        q.freestk[base + j] = (uint16_t)(cap - 1 - j);
      }
      q.root[lp] = kLsqNil;
      q.freetop[lp] = cap;
    }
  }
}

// queue_post: push / insert the buffered items of every LP.
__global__ void lpq_post_kernel(LpqDev q, gpq_item* ibuf, uint32_t* icnt, uint32_t ibc, uint32_t L,
                                LocalQueueCounters* ctr) {
  const uint32_t cap = 1u << q.cap_log2;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const uint32_t k = min(icnt[lp], ibc);
    if (k == 0) continue;
    const gpq_item* src = ibuf + (size_t)lp * ibc;
    const size_t base = (size_t)lp << q.cap_log2;
    uint32_t n = q.size[lp];
    if (q.kind == GPQ_QUEUE_LHQ) {
      for (uint32_t j = 0; j < k; ++j) {
        if (n == cap) { gpq_set_error(&ctr->err, GPQ_ERR_QUEUE_FULL); break; }
        lhq_push<4>(q.items + base, n, src[j]);
        ++n;
      }
    } else {
      const LsqView v{q.items + base, q.links + base};
      uint32_t root = q.root[lp], ftop = q.freetop[lp];
      for (uint32_t j = 0; j < k; ++j) {
        if (ftop == 0) { gpq_set_error(&ctr->err, GPQ_ERR_QUEUE_FULL); break; }
        const uint32_t x = q.freestk[base + --ftop];
        v.it[x] = src[j];
        root = lsq_insert(v, root, x);
        ++n;
      }
      q.root[lp] = root;
      q.freetop[lp] = ftop;
    }
    q.size[lp] = n;
    icnt[lp] = 0;
  }
}

__device__ __forceinline__ bool lpq_peek(const LpqDev& q, uint32_t lp, gpq_item* out) {
  const size_t base = (size_t)lp << q.cap_log2;
  if (q.size[lp] == 0) return false;
  if (q.kind == GPQ_QUEUE_LHQ) {
    *out = q.items[base];
    return true;
  }
  const LsqView v{q.items + base, q.links + base};
  const uint32_t r = lsq_splay(v, q.root[lp], 0ull);
  q.root[lp] = r;
  *out = v.it[r];
  return true;
}

__global__ void lpq_min_kernel(LpqDev q, uint32_t L, LocalQueueCounters* ctr) {
  __shared__ uint32_t red[32];
  uint32_t mn = kInfBits;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    gpq_item e;
    if (lpq_peek(q, lp, &e)) mn = min(mn, gpq_f2u(e.ts));
  }
  mn = block_min_u32(mn, red);
  if (threadIdx.x == 0) atomicMin(&ctr->min_bits, mn);
}

// queue_peek + queue_set_done repeated per LP: pop up to max_per_lp items below the
// bound into tmp[lp << cap_log2 ...] and count them.
__global__ void lpq_pop_kernel(LpqDev q, uint32_t L, float bound, uint32_t max_per_lp, gpq_item* tmp, uint32_t* cnt,
                               LocalQueueCounters* ctr) {
  const LaneGroup<1> g;
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const size_t base = (size_t)lp << q.cap_log2;
    uint32_t n = q.size[lp], c = 0;
    if (q.kind == GPQ_QUEUE_LHQ) {
      while (n > 0 && (max_per_lp == 0 || c < max_per_lp)) {
        const gpq_item top = q.items[base];
        if (!(top.ts < bound)) break;
        tmp[base + c++] = top;
        lhq_pop<1, 4>(q.items + base, n, g);
        --n;
      }
    } else {
      const LsqView v{q.items + base, q.links + base};
      uint32_t root = q.root[lp], ftop = q.freetop[lp];
      while (root != kLsqNil && (max_per_lp == 0 || c < max_per_lp)) {
        root = lsq_splay(v, root, 0ull);
        const gpq_item e = v.it[root];
        if (!(e.ts < bound)) break;
        tmp[base + c++] = e;
        const uint32_t x = root;
        root = v.right(x);
        v.it[x].lp = 0xffffffffu;
        q.freestk[base + ftop++] = (uint16_t)x;
        --n;
      }
      q.root[lp] = root;
      q.freetop[lp] = ftop;
    }
    q.size[lp] = n;
    cnt[lp] = c;
    if (c) atomicAdd(&ctr->dequeued, (unsigned long long)c);
  }
}

__global__ void lpq_gather_kernel(uint32_t cap_log2, uint32_t L, const gpq_item* tmp, const uint32_t* cnt,
                                  const unsigned long long* off, gpq_item* out) {
  for (uint32_t lp = blockIdx.x * blockDim.x + threadIdx.x; lp < L; lp += gridDim.x * blockDim.x) {
    const size_t base = (size_t)lp << cap_log2;
    for (uint32_t i = 0; i < cnt[lp]; ++i) out[off[lp] + i] = tmp[base + i];
  }
}

__global__ void lpq_clear_kernel(LpqDev q, uint32_t lp, LocalQueueCounters* ctr) {
  const uint32_t cap = 1u << q.cap_log2;
  const size_t base = (size_t)lp << q.cap_log2;
  atomicAdd(&ctr->dequeued, (unsigned long long)q.size[lp]);
  q.size[lp] = 0;
  if (q.kind == GPQ_QUEUE_LSQ) {
    for (uint32_t j = 0; j < cap; ++j) {
      q.items[base + j].lp = 0xffffffffu;
      q.freestk[base + j] = (uint16_t)(cap - 1 - j);
    }
    q.root[lp] = kLsqNil;
    q.freetop[lp] = cap;
  }
}

__global__ void lpq_set_bound_kernel(float* bound, float value) { *bound = value; }

class LpqQueue final : public LocalQueueBase {
 public:
  ~LpqQueue() override {
    for (void* p : {(void*)d_.items, (void*)d_.size, (void*)d_.root, (void*)d_.freetop, (void*)d_.links,
                    (void*)d_.freestk, (void*)tmp_, (void*)bound_})
      if (p) cudaFree(p);
  }

  // The local heap queue's device view for model kernels (include/gpq/queue.cuh); the
  // splay queue has none.
  gpq_status device_view(gpq_device_queue* v) override {
    if (d_.kind != GPQ_QUEUE_LHQ) return GPQ_ERR_UNSUPPORTED;
    *v = gpq_device_queue{};
    v->ring = d_.items;
    v->ibuf = ibuf_;
    v->icnt = icnt_;
    v->bound = bound_;
    v->enqueued = &ctr_->enqueued;
    v->dequeued = &ctr_->dequeued;
    v->err = &ctr_->err;
    v->num_lps = L_;
    v->cap_log2 = d_.cap_log2;
    v->ibc = ibc_;
    v->kind = GPQ_QUEUE_LHQ;
    v->size = d_.size;
    return GPQ_OK;
  }

  gpq_status set_bound(float b, cudaStream_t st) override {
    lpq_set_bound_kernel<<<1, 1, 0, st>>>(bound_, b);
    GPQ_CUDA_TRY(cudaGetLastError());
    return GPQ_OK;
  }

  gpq_status init(const gpq_queue_config& c) {
    uint32_t cap = c.capacity ? c.capacity : 256;
    GPQ_CHECK_ARG(cap >= 2 && cap <= (1u << 16) && !(cap & (cap - 1)), "capacity must be a power of two <= 65536");
    if (c.kind == GPQ_QUEUE_LSQ) GPQ_CHECK_ARG(cap <= 32768, "splay queue capacity must be <= 32768");
    uint32_t ibc = c.insert_capacity ? c.insert_capacity : 64;
    GPQ_CHECK_ARG(ibc <= 1024, "insert_capacity must be <= 1024");
    gpq_status s = init_base(c.num_lps, ibc);
    if (s != GPQ_OK) return s;
    d_.kind = c.kind;
    d_.cap_log2 = ilog2(cap);
    const size_t slots = (size_t)L_ << d_.cap_log2;
    GPQ_CUDA_TRY(cudaMalloc(&d_.items, slots * sizeof(gpq_item)));
    GPQ_CUDA_TRY(cudaMalloc(&d_.size, (size_t)L_ * sizeof(uint32_t)));
    GPQ_CUDA_TRY(cudaMalloc(&tmp_, slots * sizeof(gpq_item)));
    if (c.kind == GPQ_QUEUE_LSQ) {
      GPQ_CUDA_TRY(cudaMalloc(&d_.root, (size_t)L_ * sizeof(uint32_t)));
      GPQ_CUDA_TRY(cudaMalloc(&d_.freetop, (size_t)L_ * sizeof(uint32_t)));
      GPQ_CUDA_TRY(cudaMalloc(&d_.links, slots * sizeof(uint32_t)));
      GPQ_CUDA_TRY(cudaMalloc(&d_.freestk, slots * sizeof(uint16_t)));
    }
    lpq_init_kernel<<<grid(), 256, 0, own_>>>(d_, L_);
    GPQ_CUDA_TRY(cudaMalloc(&bound_, sizeof(float)));
    lpq_set_bound_kernel<<<1, 1, 0, own_>>>(bound_, gpq_u2f(kInfBits));
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaStreamSynchronize(own_));
    return GPQ_OK;
  }

  gpq_status post(cudaStream_t st) override {
    lpq_post_kernel<<<grid(), 256, 0, st>>>(d_, ibuf_, icnt_, ibc_, L_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    return take_error(st);
  }

  gpq_status get_min(float* min_ts, cudaStream_t st) override {
    const uint32_t inf = kInfBits;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&ctr_->min_bits, &inf, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    lpq_min_kernel<<<grid(), 256, 0, st>>>(d_, L_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(&h_ctr_->min_bits, &ctr_->min_bits, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    *min_ts = gpq_u2f(h_ctr_->min_bits);
    return GPQ_OK;
  }

  gpq_status dequeue(float bound, uint32_t max_per_lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out,
                     cudaStream_t st) override {
    lpq_pop_kernel<<<grid(), 256, 0, st>>>(d_, L_, bound, max_per_lp, tmp_, dq_cnt_, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    uint64_t total = 0;
    gpq_status s = scan_counts(dq_cnt_, &total, st);
    if (s != GPQ_OK) return s;
    *n_out = total;
    if (total > out_capacity) {
      set_last_error("dequeue: %llu items do not fit the output", (unsigned long long)total);
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
    lpq_gather_kernel<<<grid(), 256, 0, st>>>(d_.cap_log2, L_, tmp_, dq_cnt_, dq_off_, dq_out_);
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaMemcpyAsync(out, dq_out_, total * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  gpq_status length(uint32_t lp, uint32_t* len, cudaStream_t st) override {
    GPQ_CUDA_TRY(cudaMemcpyAsync(len, d_.size + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    return GPQ_OK;
  }

  gpq_status clear(uint32_t lp, cudaStream_t st) override {
    lpq_clear_kernel<<<1, 1, 0, st>>>(d_, lp, ctr_);
    GPQ_CUDA_TRY(cudaGetLastError());
    return GPQ_OK;
  }

  // The LP's items in key order: the heap array (sorted on the host) or an in-order walk
  // of the splay tree (on the host, over a copy of the LP's pool).
  gpq_status dump(uint32_t lp, gpq_item* out, uint64_t out_capacity, uint64_t* n_out, cudaStream_t st) override {
    const uint32_t cap = 1u << d_.cap_log2;
    const size_t base = (size_t)lp << d_.cap_log2;
    uint32_t n = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(&n, d_.size + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    *n_out = n;
    if (n > out_capacity) return GPQ_ERR_INVALID;
    if (d_.kind == GPQ_QUEUE_LHQ) {
      std::vector<gpq_item> h(n);
      if (n) GPQ_CUDA_TRY(cudaMemcpyAsync(h.data(), d_.items + base, n * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
      GPQ_CUDA_TRY(cudaStreamSynchronize(st));
      std::sort(h.begin(), h.end(), [](const gpq_item& a, const gpq_item& b) { return gpq_item_less(a, b); });
      std::copy(h.begin(), h.end(), out);
      return GPQ_OK;
    }
    std::vector<gpq_item> it(cap);
    std::vector<uint32_t> ln(cap);
    uint32_t root = 0;
    GPQ_CUDA_TRY(cudaMemcpyAsync(it.data(), d_.items + base, cap * sizeof(gpq_item), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(ln.data(), d_.links + base, cap * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaMemcpyAsync(&root, d_.root + lp, 4, cudaMemcpyDeviceToHost, st));
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<uint32_t> stack;
    uint32_t x = root, k = 0;
    while ((x != kLsqNil || !stack.empty()) && k <= n) {
      while (x != kLsqNil && stack.size() <= cap) { stack.push_back(x); x = ln[x] >> 16; }
      if (stack.empty()) break;
      x = stack.back();
      stack.pop_back();
      if (k < n) out[k] = it[x];
      ++k;
      x = ln[x] & 0xffffu;
    }
    if (k != n) {
      set_last_error("splay tree of LP %u holds %u nodes, expected %u", lp, k, n);
      return GPQ_ERR_INVALID;
    }
    return GPQ_OK;
  }

 private:
  static uint32_t ilog2(uint32_t x) { uint32_t r = 0; while ((1u << r) < x) ++r; return r; }
  uint32_t grid() const { return std::max(1u, std::min<uint32_t>((L_ + 255) / 256, 4096)); }
  LpqDev d_{};
  gpq_item* tmp_ = nullptr;
  float* bound_ = nullptr;  // window bound of the device view
};

}  // namespace

gpq_status make_lpq_queue(const gpq_queue_config& cfg, std::unique_ptr<QueueImpl>& out) {
  auto q = std::unique_ptr<LpqQueue>(new (std::nothrow) LpqQueue());
  if (!q) return GPQ_ERR_NOMEM;
  gpq_status s = q->init(cfg);
  if (s != GPQ_OK) return s;
  out = std::move(q);
  return GPQ_OK;
}

}  // namespace gpq
