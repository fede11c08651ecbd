// Resident PHOLD instances (gpq_phold_session_*): many runs in one persistent launch for
// batching and serving.  Instances take free ranges of one LP space reserved up front,
// advance together one window per grid barrier (each with its own window), and are
// collected when their minimum reaches their end time.  The LP space holds either sorted
// rings (phold_multi.cuh) or time buckets (phold_multi_lab.cuh, a bucketed session).
#include <algorithm>
#include <cstring>
#include <vector>

#include "host_common.h"
#include "phold_host.h"
#include "phold_multi.cuh"
#include "phold_multi_lab.cuh"
#include "range_alloc.h"

using gpq::set_last_error;

struct gpq_phold_session {
  cudaStream_t own = nullptr;
  uint32_t max_lps = 0, max_inst = 0, cap_log2 = 0, ibc = 0, group = 8, block = 256;
  // device
  PmInstDev* inst = nullptr;
  uint32_t* mins = nullptr;
  uint32_t* errs = nullptr;
  uint8_t* on = nullptr;
  uint32_t* lp_inst = nullptr;
  gpq_item* ring = nullptr;
  uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  gpq_item* ibuf = nullptr;
  uint32_t* icnt = nullptr;
  uint32_t* count = nullptr;
  unsigned long long* csum = nullptr;
  unsigned long long* ohash = nullptr;
  PmCtl* ctl = nullptr;
  uint32_t* list = nullptr;
  uint32_t* list_n = nullptr;
  PmAcc* acc = nullptr;
  PmInstDev* staged = nullptr;  // [max_inst] admission records / retired records
  // host
  gpq::RangeAlloc lps;
  std::vector<uint32_t> free_slots;
  std::vector<uint8_t> h_on;
  std::vector<PmInstDev> h_inst;
  std::vector<uint32_t> pending;
  uint32_t high = 0, lp_high = 0, active = 0, next_window = 0;
  uint32_t max_per_lp = 0;
  int grid = 0;
  size_t smem = 0;
  const void* kern = nullptr;
  // bucketed sessions
  bool bucketed = false;
  PmbDev b{};
};

namespace {

template <class T>
cudaError_t dmalloc(T** p, uint64_t n) {
  return cudaMalloc(p, std::max<uint64_t>(n, 1) * sizeof(T));
}

const void* pm_kernel(uint32_t group) {
  switch (group) {
    case 4: return (const void*)pm_persistent_kernel<4>;
    case 8: return (const void*)pm_persistent_kernel<8>;
    case 16: return (const void*)pm_persistent_kernel<16>;
    case 32: return (const void*)pm_persistent_kernel<32>;
  }
  return nullptr;
}

PmDev session_dev(const gpq_phold_session* s) {
  PmDev d{};
  d.inst = s->inst;
  d.mins = s->mins;
  d.errs = s->errs;
  d.on = s->on;
  d.n_inst = s->high;
  d.lp_inst = s->lp_inst;
  d.n_lps = s->lp_high;
  d.ring = s->ring;
  d.rd = s->rd;
  d.wr = s->wr;
  d.cap_log2 = s->cap_log2;
  d.ibuf = s->ibuf;
  d.icnt = s->icnt;
  d.ibc = s->ibc;
  d.max_lps = s->max_lps;
  d.count = s->count;
  d.csum = s->csum;
  d.ohash = s->ohash;
  d.ctl = s->ctl;
  d.spin_limit = gpq::spin_limit();
  return d;
}

__global__ void pm_admit_kernel(PmInstDev* inst, uint32_t* mins, uint32_t* errs, uint8_t* on, const PmInstDev* staged,
                                const uint32_t* list, uint32_t n) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = list[j];
  inst[i] = staged[j];
  for (int k = 0; k < 3; ++k) {
    mins[3 * i + k] = kInfBits;
    errs[3 * i + k] = 0;
  }
  on[i] = 1;
}

__global__ void pm_retire_kernel(uint8_t* on, const uint32_t* list, uint32_t n, PmInstDev* inst, PmInstDev* out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    out[j] = inst[list[j]];
    on[list[j]] = 0;
  }
}

// Device arrays and the persistent kernel's launch shape, once the per-LP queue arrays exist.
gpq_status finish_create(gpq_phold_session* s, uint32_t max_instances) {
  cudaError_t e = dmalloc(&s->inst, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->mins, 3ull * max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->errs, 3ull * max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->on, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->lp_inst, s->max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->count, s->max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->csum, s->max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->ohash, s->max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->ctl, 1);
  if (e == cudaSuccess) e = dmalloc(&s->list, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->list_n, 1);
  if (e == cudaSuccess) e = dmalloc(&s->acc, max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->staged, max_instances);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->on, 0, max_instances, s->own);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->lp_inst, 0xff, (size_t)s->max_lps * 4, s->own);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->ctl, 0, sizeof(PmCtl), s->own);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->own);
  if (e != cudaSuccess) {
    set_last_error("gpq_phold_session_create: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  }
  int dev = 0, sms = 0, per_sm = 0;
  GPQ_CUDA_TRY(gpq::raise_smem_limit(s->kern, (int)s->smem));
  GPQ_CUDA_TRY(cudaGetDevice(&dev));
  GPQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GPQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s->kern, (int)s->block, s->smem));
  if (per_sm < 1) {
    set_last_error("phold session: kernel does not fit on an SM");
    return GPQ_ERR_INVALID;
  }
  s->grid = per_sm * sms;
  return GPQ_OK;
}

gpq_status flush_pending(gpq_phold_session* s, cudaStream_t st) {
  const uint32_t n = (uint32_t)s->pending.size();
  if (n == 0) return GPQ_OK;
  std::vector<PmInstDev> staged(n);
  uint32_t max_lps = 0, max_p = 0;
  for (uint32_t j = 0; j < n; ++j) {
    s->h_inst[s->pending[j]].w0 = s->next_window;
    staged[j] = s->h_inst[s->pending[j]];
    max_lps = std::max(max_lps, staged[j].p.num_lps);
    max_p = std::max(max_p, staged[j].per_lp);
  }
  PmInstDev* dstaged = s->staged;
  GPQ_CUDA_TRY(cudaMemcpyAsync(dstaged, staged.data(), n * sizeof(PmInstDev), cudaMemcpyHostToDevice, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->list, s->pending.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  pm_admit_kernel<<<(n + 127) / 128, 128, 0, st>>>(s->inst, s->mins, s->errs, s->on, dstaged, s->list, n);
  const PmDev d = session_dev(s);
  if (s->bucketed) {
    for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
      const uint32_t nj = std::min<uint32_t>(65535, n - j0);
      const uint32_t gx = std::min<uint32_t>((max_lps + 7) / 8, 1024);
      pmb_populate_kernel<<<dim3(gx, nj), 256, 0, st>>>(d, s->b, s->list + j0, s->next_window);
    }
    GPQ_CUDA_TRY(cudaGetLastError());
    GPQ_CUDA_TRY(cudaStreamSynchronize(st));
    s->pending.clear();
    return GPQ_OK;
  }
  const uint32_t block = 256, wpb = block / 32;
  const size_t smem = (size_t)wpb * max_p * (sizeof(gpq_item) + sizeof(uint64_t));
  GPQ_CUDA_TRY(gpq::raise_smem_limit(pm_populate_kernel, (int)smem));
  for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
    const uint32_t nj = std::min<uint32_t>(65535, n - j0);
    const uint32_t gx = std::min<uint32_t>((max_lps + wpb - 1) / wpb, 1024);
    pm_populate_kernel<<<dim3(gx, nj), block, smem, st>>>(d, s->list + j0, s->next_window);
  }
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  s->pending.clear();
  return GPQ_OK;
}

constexpr uint64_t kSessionSnapMagic = 0x3153534553515047ull;  // "GPQSESS1"
constexpr uint32_t kSessionSnapHeader = 12;

// Device regions of a session's state for slots [0, high) and LPs [0, lp_high): the
// scratch buffers (list, acc, staged) are not state.  Parity-major arrays give one
// region per parity.
std::vector<std::pair<void*, size_t>> session_regions(const gpq_phold_session* s, uint64_t H, uint64_t L) {
  std::vector<std::pair<void*, size_t>> r;
  const uint64_t M = s->max_lps;
  auto add = [&](void* p, uint64_t n) { r.push_back({p, (size_t)n}); };
  add(s->inst, H * sizeof(PmInstDev));
  add(s->mins, 3 * H * sizeof(uint32_t));
  add(s->errs, 3 * H * sizeof(uint32_t));
  add(s->on, H);
  add(s->lp_inst, L * sizeof(uint32_t));
  add(s->count, L * sizeof(uint32_t));
  add(s->csum, L * sizeof(unsigned long long));
  add(s->ohash, L * sizeof(unsigned long long));
  add(s->ctl, sizeof(PmCtl));
  if (s->bucketed) {
    const LabDev& q = s->b.q;
    add(q.keys, (L << (q.nb_log2 + q.c_log2)) * sizeof(unsigned long long));
    add(q.cnt, (L << q.nb_log2) * sizeof(uint32_t));
    for (uint64_t par = 0; par < 2; ++par) {
      add(q.spill + par * M * q.F, L * q.F * sizeof(unsigned long long));
      add(q.scnt + par * M, L * sizeof(uint32_t));
    }
    add(s->b.wj, 4 * H * sizeof(uint32_t));
    add(s->b.fin, H * sizeof(uint32_t));
  } else {
    add(s->ring, (L << s->cap_log2) * sizeof(gpq_item));
    add(s->rd, L * sizeof(uint32_t));
    add(s->wr, L * sizeof(uint32_t));
    for (uint64_t par = 0; par < 2; ++par) {
      add(s->ibuf + par * M * s->ibc, L * s->ibc * sizeof(gpq_item));
      add(s->icnt + par * M, L * sizeof(uint32_t));
    }
  }
  return r;
}

void session_header(const gpq_phold_session* s, uint32_t h[kSessionSnapHeader]) {
  const uint32_t v[kSessionSnapHeader] = {s->bucketed ? 1u : 0u, s->max_lps, s->max_inst, s->cap_log2, s->ibc,
                                          s->group, s->block, s->b.q.nb_log2, s->b.q.c_log2, s->b.q.F,
                                          (uint32_t)sizeof(PmInstDev), 1u};
  std::memcpy(h, v, sizeof(v));
}

// Host state: counters, slot tables, free slots, the LP-range allocator.
std::vector<unsigned char> session_host_blob(const gpq_phold_session* s) {
  std::vector<unsigned char> b;
  auto put = [&](const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  };
  const uint32_t k[5] = {s->high, s->lp_high, s->active, s->next_window, s->max_per_lp};
  put(k, sizeof(k));
  put(s->h_on.data(), s->h_on.size());
  put(s->h_inst.data(), s->h_inst.size() * sizeof(PmInstDev));
  const uint64_t nf = s->free_slots.size();
  put(&nf, 8);
  put(s->free_slots.data(), nf * sizeof(uint32_t));
  const auto ranges = s->lps.free_ranges();
  const uint64_t a[3] = {s->lps.size(), s->lps.used(), ranges.size()};
  put(a, sizeof(a));
  for (const auto& r : ranges) {
    const uint64_t pr[2] = {r.first, r.second};
    put(pr, sizeof(pr));
  }
  return b;
}

}  // namespace

extern "C" {

gpq_status gpq_phold_session_snapshot(gpq_phold_session* s, void* buf, uint64_t capacity, uint64_t* size,
                                      void* stream) {
  GPQ_CHECK_ARG(s && size, "NULL argument");
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  if (buf) {
    const gpq_status r = flush_pending(s, st);
    if (r != GPQ_OK) return r;
  }
  const std::vector<unsigned char> blob = session_host_blob(s);
  const auto regions = session_regions(s, s->high, s->lp_high);
  uint64_t need = 8 + 4 * kSessionSnapHeader + 8 + blob.size() + 4;
  for (const auto& r : regions) need += 8 + r.second;
  *size = need;
  if (!buf) return GPQ_OK;
  GPQ_CHECK_ARG(capacity >= need, "capacity below the snapshot size");
  unsigned char* p = static_cast<unsigned char*>(buf);
  auto put = [&](const void* src, size_t n) {
    std::memcpy(p, src, n);
    p += n;
  };
  uint32_t hdr[kSessionSnapHeader];
  session_header(s, hdr);
  put(&kSessionSnapMagic, 8);
  put(hdr, sizeof(hdr));
  const uint64_t nb = blob.size();
  put(&nb, 8);
  put(blob.data(), nb);
  const uint32_t nr = (uint32_t)regions.size();
  put(&nr, 4);
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (const auto& r : regions) {
    const uint64_t n = r.second;
    put(&n, 8);
    if (n) GPQ_CUDA_TRY(cudaMemcpyAsync(p, r.first, n, cudaMemcpyDeviceToHost, st));
    p += n;
  }
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  return GPQ_OK;
}

gpq_status gpq_phold_session_restore(gpq_phold_session* s, const void* buf, uint64_t size, void* stream) {
  GPQ_CHECK_ARG(s && buf, "NULL argument");
  const unsigned char* p = static_cast<const unsigned char*>(buf);
  const unsigned char* end = p + size;
  auto take = [&](void* dst, size_t n) -> bool {
    if ((uint64_t)(end - p) < n) return false;
    if (dst) std::memcpy(dst, p, n);
    p += n;
    return true;
  };
  uint64_t magic = 0;
  uint32_t hdr[kSessionSnapHeader], mine[kSessionSnapHeader];
  session_header(s, mine);
  GPQ_CHECK_ARG(take(&magic, 8) && magic == kSessionSnapMagic, "not a PHOLD session snapshot");
  GPQ_CHECK_ARG(take(hdr, sizeof(hdr)) && std::memcmp(hdr, mine, sizeof(hdr)) == 0,
                "snapshot of a session with other parameters");
  // host state into temporaries; nothing changes until every part has been checked
  uint64_t nb = 0;
  GPQ_CHECK_ARG(take(&nb, 8) && (uint64_t)(end - p) >= nb, "snapshot truncated");
  const unsigned char* hb = p;
  p += nb;
  const unsigned char* hend = hb + nb;
  auto htake = [&](void* dst, size_t n) -> bool {
    if ((uint64_t)(hend - hb) < n) return false;
    std::memcpy(dst, hb, n);
    hb += n;
    return true;
  };
  uint32_t k[5];
  std::vector<uint8_t> h_on(s->max_inst);
  std::vector<PmInstDev> h_inst(s->max_inst);
  uint64_t nf = 0, a[3] = {0, 0, 0};
  bool ok = htake(k, sizeof(k)) && htake(h_on.data(), h_on.size()) &&
            htake(h_inst.data(), h_inst.size() * sizeof(PmInstDev)) && htake(&nf, 8) && nf <= s->max_inst;
  std::vector<uint32_t> free_slots(ok ? nf : 0);
  ok = ok && htake(free_slots.data(), nf * sizeof(uint32_t)) && htake(a, sizeof(a)) && a[0] == s->max_lps &&
       a[2] <= s->max_lps;
  std::vector<std::pair<uint64_t, uint64_t>> ranges(ok ? a[2] : 0);
  for (auto& r : ranges) {
    uint64_t pr[2];
    ok = ok && htake(pr, sizeof(pr)) && pr[0] + pr[1] <= s->max_lps;
    r = {pr[0], pr[1]};
  }
  GPQ_CHECK_ARG(ok && hb == hend && k[0] <= s->max_inst && k[1] <= s->max_lps, "snapshot host state is damaged");
  const auto regions = session_regions(s, k[0], k[1]);
  uint32_t nr = 0;
  GPQ_CHECK_ARG(take(&nr, 4) && nr == regions.size(), "snapshot layout differs");
  const unsigned char* scan = p;
  for (const auto& r : regions) {
    uint64_t n = 0;
    GPQ_CHECK_ARG((uint64_t)(end - scan) >= 8, "snapshot truncated");
    std::memcpy(&n, scan, 8);
    GPQ_CHECK_ARG(n == r.second && (uint64_t)(end - scan - 8) >= n, "snapshot region differs or is truncated");
    scan += 8 + n;
  }
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (const auto& r : regions) {
    p += 8;
    if (r.second) GPQ_CUDA_TRY(cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyHostToDevice, st));
    p += r.second;
  }
  // slots and LPs above the snapshot's highest ones are free
  if (k[0] < s->max_inst) GPQ_CUDA_TRY(cudaMemsetAsync(s->on + k[0], 0, s->max_inst - k[0], st));
  if (k[1] < s->max_lps)
    GPQ_CUDA_TRY(cudaMemsetAsync(s->lp_inst + k[1], 0xff, (size_t)(s->max_lps - k[1]) * sizeof(uint32_t), st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  s->high = k[0];
  s->lp_high = k[1];
  s->active = k[2];
  s->next_window = k[3];
  s->max_per_lp = k[4];
  s->h_on.swap(h_on);
  s->h_inst.swap(h_inst);
  s->free_slots.swap(free_slots);
  s->lps.assign(a[0], a[1], ranges);
  s->pending.clear();
  return GPQ_OK;
}

gpq_status gpq_phold_session_create(uint32_t max_lps, uint32_t capacity, uint32_t insert_capacity,
                                    uint32_t max_instances, uint32_t lanes_per_lp, gpq_phold_session** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  if (capacity == 0) capacity = 256;
  if (insert_capacity == 0) insert_capacity = 64;
  if (lanes_per_lp == 0) lanes_per_lp = 8;
  GPQ_CHECK_ARG(max_lps >= 1 && max_instances >= 1 && max_instances <= (1u << 20), "need max_lps >= 1, 1 <= max_instances <= 2^20");
  GPQ_CHECK_ARG(gpq::is_pow2(capacity) && capacity >= 8 && capacity <= (1u << 20), "capacity must be a power of two in [8, 2^20]");
  GPQ_CHECK_ARG(insert_capacity >= 1 && insert_capacity <= 4096, "insert_capacity in [1, 4096]");
  GPQ_CHECK_ARG(pm_kernel(lanes_per_lp) != nullptr, "lanes_per_lp must be 4, 8, 16 or 32");
  gpq_phold_session* s = new (std::nothrow) gpq_phold_session();
  if (!s) return GPQ_ERR_NOMEM;
  s->max_lps = max_lps;
  s->max_inst = max_instances;
  s->cap_log2 = gpq::ilog2_ceil(capacity);
  s->ibc = insert_capacity;
  s->group = lanes_per_lp;
  s->lps.reset(max_lps);
  s->h_on.assign(max_instances, 0);
  s->h_inst.assign(max_instances, PmInstDev{});
  for (uint32_t i = max_instances; i-- > 0;) s->free_slots.push_back(i);
  cudaError_t e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = dmalloc(&s->ring, (uint64_t)max_lps << s->cap_log2);
  if (e == cudaSuccess) e = dmalloc(&s->rd, max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->wr, max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->ibuf, 2ull * max_lps * insert_capacity);
  if (e == cudaSuccess) e = dmalloc(&s->icnt, 2ull * max_lps);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->icnt, 0, 2ull * max_lps * 4, s->own);
  if (e != cudaSuccess) {
    set_last_error("gpq_phold_session_create: %s", cudaGetErrorString(e));
    gpq_phold_session_destroy(s);
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  }
  s->kern = pm_kernel(s->group);
  s->smem = (size_t)(s->block / s->group) * laq_group_smem_bytes(s->ibc, s->group);
  const gpq_status fs = finish_create(s, max_instances);
  if (fs != GPQ_OK) {
    gpq_phold_session_destroy(s);
    return fs;
  }
  *out = s;
  return GPQ_OK;
}

gpq_status gpq_phold_session_create_bucketed(uint32_t max_lps, uint32_t buckets, uint32_t bucket_slots,
                                             uint32_t max_instances, gpq_phold_session** out) {
  GPQ_CHECK_ARG(out, "out is NULL");
  *out = nullptr;
  if (buckets == 0) buckets = 32;
  if (bucket_slots == 0) bucket_slots = 16;
  GPQ_CHECK_ARG(max_lps >= 1 && max_instances >= 1 && max_instances <= (1u << 20), "need max_lps >= 1, 1 <= max_instances <= 2^20");
  GPQ_CHECK_ARG(gpq::is_pow2(buckets) && buckets >= 8 && buckets <= 1024, "buckets must be a power of two in [8, 1024]");
  GPQ_CHECK_ARG(gpq::is_pow2(bucket_slots) && bucket_slots >= 8 && bucket_slots <= 1024,
                "bucket_slots must be a power of two in [8, 1024]");
  gpq_phold_session* s = new (std::nothrow) gpq_phold_session();
  if (!s) return GPQ_ERR_NOMEM;
  s->bucketed = true;
  s->max_lps = max_lps;
  s->max_inst = max_instances;
  s->block = 512;
  s->lps.reset(max_lps);
  s->h_on.assign(max_instances, 0);
  s->h_inst.assign(max_instances, PmInstDev{});
  for (uint32_t i = max_instances; i-- > 0;) s->free_slots.push_back(i);
  LabDev& q = s->b.q;
  q.nb_log2 = gpq::ilog2_ceil(buckets);
  q.c_log2 = gpq::ilog2_ceil(bucket_slots);
  q.F = std::max(64u, bucket_slots);
  cudaError_t e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = dmalloc(&q.keys, (uint64_t)max_lps << (q.nb_log2 + q.c_log2));
  if (e == cudaSuccess) e = dmalloc(&q.cnt, (uint64_t)max_lps << q.nb_log2);
  if (e == cudaSuccess) e = dmalloc(&q.spill, 2ull * max_lps * q.F);
  if (e == cudaSuccess) e = dmalloc(&q.scnt, 2ull * max_lps);
  if (e == cudaSuccess) e = dmalloc(&s->b.wj, 4ull * max_instances);
  if (e == cudaSuccess) e = dmalloc(&s->b.fin, max_instances);
  if (e != cudaSuccess) {
    set_last_error("gpq_phold_session_create_bucketed: %s", cudaGetErrorString(e));
    gpq_phold_session_destroy(s);
    return e == cudaErrorMemoryAllocation ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;
  }
  s->kern = (const void*)pmb_persistent_kernel;
  s->smem = lab_cta_smem_bytes(s->block);
  const gpq_status fs = finish_create(s, max_instances);
  if (fs != GPQ_OK) {
    gpq_phold_session_destroy(s);
    return fs;
  }
  *out = s;
  return GPQ_OK;
}

gpq_status gpq_phold_session_destroy(gpq_phold_session* s) {
  if (!s) return GPQ_OK;
  void* bufs[] = {s->inst,   s->mins,   s->errs,     s->on,       s->lp_inst,   s->ring,     s->rd,    s->wr,
                  s->ibuf,   s->icnt,   s->count,    s->csum,     s->ohash,     s->ctl,      s->list,  s->list_n,
                  s->acc,    s->staged, s->b.q.keys, s->b.q.cnt, s->b.q.spill, s->b.q.scnt, s->b.wj, s->b.fin};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (s->own) cudaStreamDestroy(s->own);
  delete s;
  return GPQ_OK;
}

gpq_status gpq_phold_session_admit(gpq_phold_session* s, const gpq_phold_config* cfg, uint32_t* slot) {
  GPQ_CHECK_ARG(s && cfg && slot, "NULL argument");
  gpq_phold_config c = *cfg;
  c.queue_kind = GPQ_QUEUE_LAQ;
  c.capacity = 1u << s->cap_log2;
  c.insert_capacity = s->ibc;
  {
    const gpq_status v = gpq::validate_phold_config(&c);
    if (v != GPQ_OK) return v;
  }
  if (!s->bucketed)
    GPQ_CHECK_ARG(c.events_per_lp <= (1u << s->cap_log2), "events_per_lp above the session's queue capacity");
  GPQ_CHECK_ARG(c.events_per_lp <= 1024, "events_per_lp above 1024");
  uint32_t inv_bits = 0;
  if (s->bucketed) {
    // the run's bucket width: about 6 events in an LP's front bucket, a window spanning at
    // most lookahead / 2.5 buckets, and the session's NB buckets covering lookahead + 7
    const double la = c.lookahead, E = c.events_per_lp, NB = (double)(1u << s->b.q.nb_log2);
    const double w = std::max(std::max(6.0 * (la + 1.0) / E, la / 2.5), (la + 7.0) / NB);
    const float inv = (float)(1.0 / w);
    GPQ_CHECK_ARG((double)c.lookahead * inv + 3.0 <= NB, "lookahead too wide for the session's buckets");
    GPQ_CHECK_ARG(((double)c.end_time + la + 20.0) * inv < 2147483648.0, "end_time too large for the bucket width");
    std::memcpy(&inv_bits, &inv, 4);
  }
  if (s->free_slots.empty()) return GPQ_ERR_NOMEM;
  uint64_t lp0 = 0;
  if (!s->lps.alloc(c.num_lps, &lp0)) return GPQ_ERR_NOMEM;
  const uint32_t i = s->free_slots.back();
  s->free_slots.pop_back();
  PmInstDev I{};
  I.p = gpq::phold_params_of(c);
  I.lp0 = (uint32_t)lp0;
  I.per_lp = c.events_per_lp;
  I.aux = inv_bits;
  s->h_inst[i] = I;
  s->h_on[i] = 1;
  s->pending.push_back(i);
  s->high = std::max(s->high, i + 1);
  s->lp_high = std::max<uint32_t>(s->lp_high, (uint32_t)lp0 + c.num_lps);
  ++s->active;
  *slot = i;
  return GPQ_OK;
}

gpq_status gpq_phold_session_step(gpq_phold_session* s, uint32_t windows, uint32_t* running, void* stream) {
  GPQ_CHECK_ARG(s, "NULL handle");
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  gpq_status r = flush_pending(s, st);
  if (r != GPQ_OK) return r;
  if (running) *running = s->active;
  if (s->active == 0) return GPQ_OK;
  PmDev d = session_dev(s);
  PmbDev b = s->b;
  uint32_t s0 = s->next_window, sw = windows;
  void* args[] = {&d, &s0, &sw};
  void* bargs[] = {&d, &b, &s0, &sw};
  GPQ_CUDA_TRY(cudaMemsetAsync(&s->ctl->bar, 0, sizeof(unsigned long long), st));
  GPQ_CUDA_TRY(cudaLaunchCooperativeKernel(s->kern, dim3(s->grid), dim3(s->block), s->bucketed ? bargs : args,
                                           s->smem, st));
  PmCtl ctl{};
  GPQ_CUDA_TRY(cudaMemcpyAsync(&ctl, s->ctl, sizeof(PmCtl), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (ctl.err) {
    set_last_error("phold session: device error %u at window %u", ctl.err, ctl.phase);
    return (gpq_status)ctl.err;
  }
  s->next_window = ctl.phase;
  return GPQ_OK;
}

gpq_status gpq_phold_session_collect(gpq_phold_session* s, uint32_t* slots, gpq_phold_result* results,
                                     uint32_t capacity, uint32_t* n_out, void* stream) {
  GPQ_CHECK_ARG(s && n_out, "NULL argument");
  const cudaStream_t st = gpq::as_stream(stream, s->own);
  *n_out = 0;
  if (s->high == 0) return GPQ_OK;
  const PmDev d = session_dev(s);
  GPQ_CUDA_TRY(cudaMemsetAsync(s->list_n, 0, sizeof(uint32_t), st));
  pm_done_list_kernel<<<(s->high + 255) / 256, 256, 0, st>>>(d, s->next_window, s->list, s->list_n);
  uint32_t n = 0;
  GPQ_CUDA_TRY(cudaMemcpyAsync(&n, s->list_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  n = std::min(n, capacity);
  if (n == 0) return GPQ_OK;
  uint32_t max_lps = 0;
  for (uint32_t i = 0; i < s->high; ++i)
    if (s->h_on[i]) max_lps = std::max(max_lps, s->h_inst[i].p.num_lps);
  std::vector<PmAcc> init(n);
  for (auto& a : init) a = PmAcc{0, 0, 0, 0, kInfBits, 0};
  GPQ_CUDA_TRY(cudaMemcpyAsync(s->acc, init.data(), n * sizeof(PmAcc), cudaMemcpyHostToDevice, st));
  for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
    const uint32_t nj = std::min<uint32_t>(65535, n - j0);
    const uint32_t gx = std::min<uint32_t>((max_lps + 7) / 8, 256);
    if (s->bucketed) pmb_finalize_kernel<<<dim3(gx, nj), 256, 0, st>>>(d, s->b, s->list + j0, s->acc + j0);
    else pm_finalize_kernel<<<dim3(gx, nj), 256, 0, st>>>(d, s->list + j0, s->acc + j0);
  }
  std::vector<uint32_t> list(n);
  std::vector<PmAcc> acc(n);
  std::vector<PmInstDev> fin(n);
  PmInstDev* dfin = s->staged;
  pm_retire_kernel<<<(n + 127) / 128, 128, 0, st>>>(s->on, s->list, n, s->inst, dfin);
  for (uint32_t j0 = 0; j0 < n; j0 += 65535) {
    const uint32_t nj = std::min<uint32_t>(65535, n - j0);
    const uint32_t gx = std::min<uint32_t>((max_lps + 255) / 256, 256);
    pm_release_kernel<<<dim3(gx, nj), 256, 0, st>>>(d, s->list + j0);
  }
  GPQ_CUDA_TRY(cudaGetLastError());
  GPQ_CUDA_TRY(cudaMemcpyAsync(list.data(), s->list, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(acc.data(), s->acc, n * sizeof(PmAcc), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaMemcpyAsync(fin.data(), dfin, n * sizeof(PmInstDev), cudaMemcpyDeviceToHost, st));
  GPQ_CUDA_TRY(cudaStreamSynchronize(st));
  for (uint32_t j = 0; j < n; ++j) {
    const uint32_t i = list[j];
    gpq_phold_result r{};
    r.committed = acc[j].committed;
    r.steps = fin[j].windows;
    r.pending = acc[j].pending;
    r.pending_csum = acc[j].pending_csum;
    r.digest = acc[j].digest;
    r.final_min = gpq_u2f(acc[j].pending_min);
    r.status = (int32_t)fin[j].err;
    if (slots) slots[j] = i;
    if (results) results[j] = r;
    s->lps.free(s->h_inst[i].lp0, s->h_inst[i].p.num_lps);
    s->h_on[i] = 0;
    s->free_slots.push_back(i);
    --s->active;
  }
  while (s->high > 0 && !s->h_on[s->high - 1]) --s->high;
  s->lp_high = 0;
  for (uint32_t i = 0; i < s->high; ++i)
    if (s->h_on[i]) s->lp_high = std::max(s->lp_high, s->h_inst[i].lp0 + s->h_inst[i].p.num_lps);
  *n_out = n;
  return GPQ_OK;
}

gpq_status gpq_phold_session_usage(gpq_phold_session* s, uint64_t* lps_used, uint32_t* instances) {
  GPQ_CHECK_ARG(s, "NULL handle");
  if (lps_used) *lps_used = s->lps.used();
  if (instances) *instances = s->active;
  return GPQ_OK;
}

uint64_t gpq_phold_session_bytes_bucketed(uint32_t max_lps, uint32_t buckets, uint32_t bucket_slots,
                                          uint32_t max_instances) {
  if (buckets == 0) buckets = 32;
  if (bucket_slots == 0) bucket_slots = 16;
  const uint64_t F = std::max(64u, bucket_slots);
  const uint64_t per_lp = 8ull * buckets * bucket_slots + 4ull * buckets + 16 * F + 8 + 4 * 2 + 8 * 2;
  return per_lp * max_lps + (uint64_t)max_instances * (sizeof(PmInstDev) + 24 + 1 + 4 + sizeof(PmAcc) + 20);
}

uint64_t gpq_phold_session_bytes(uint32_t max_lps, uint32_t capacity, uint32_t insert_capacity,
                                 uint32_t max_instances) {
  if (capacity == 0) capacity = 256;
  if (insert_capacity == 0) insert_capacity = 64;
  const uint64_t per_lp = 16ull * capacity + 32ull * insert_capacity + 4 * 6 + 8 * 2;
  return per_lp * max_lps + (uint64_t)max_instances * (sizeof(PmInstDev) + 24 + 1 + 4 + sizeof(PmAcc));
}

}  // extern "C"
