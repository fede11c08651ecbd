// PHOLD run without any device allocation (gpq_phold_run_static).
//
// Some callers cannot allocate device memory when they want to run: an application
// that embeds the simulator under a fixed memory plan (another allocator already owns
// the device memory, so a cudaMalloc would fail or break the plan), or a latency-bound
// loop that cannot afford cudaMalloc/cudaFree, which may synchronize the device.
// This entry point serves them: the caller passes the initial events (or none) and the
// per-LP output arrays; every other buffer the run needs -- the per-LP rings, the
// double-buffered insert buffers, the control block -- lives in one file-scope
// __device__ array of fixed size, GPQ_STATIC_SCRATCH_BYTES.  The array exists once per
// GPU that loads this library and stays allocated until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the array's
// device address with cudaGetSymbolAddress (host code only ever sees a host-side
// stand-in for the symbol, which must not be handed to a kernel) and caches it for that
// device.  Make that first call before any stream capture.  The cached address does not
// survive cudaDeviceReset: a process that resets a device must not call this entry point
// on it afterwards.  Every call raises (never lowers) the shared-memory limits of the
// kernels it launches to what this configuration needs, so it neither breaks nor is
// broken by handles created before or after it.
//
// Every call shares the one array and leaves its last contents there: each call clears
// the parts that must start at zero (control block, insert counters) itself.  Calls
// that overlap on the GPU (different streams or host threads, same device) race on the
// array and produce garbage; serialize them.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "host_common.h"
#include "phold_host.h"
#include "phold_kernels.cuh"

static __device__ __align__(256) unsigned char g_phold_static_scratch[GPQ_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_dev[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct StaticLayout {
  size_t ring, rd, wr, ibuf, icnt, ctrl, acc, total;
};

StaticLayout layout_for(const gpq_phold_config& c) {
  const size_t L = c.num_lps;
  StaticLayout s{};
  size_t off = 0;
  s.ring = off; off = align256(off + (L << gpq::ilog2_ceil(c.capacity)) * sizeof(gpq_item));
  s.rd = off; off = align256(off + L * sizeof(uint32_t));
  s.wr = off; off = align256(off + L * sizeof(uint32_t));
  s.ibuf = off; off = align256(off + 2 * L * c.insert_capacity * sizeof(gpq_item));
  s.icnt = off; off = align256(off + 2 * L * sizeof(uint32_t));
  s.ctrl = off; off = align256(off + sizeof(PholdCtrl));
  s.acc = off; off = align256(off + sizeof(PholdAcc));
  s.total = off;
  return s;
}

// Once per device: device address of the scratch array.
gpq_status scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  GPQ_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    gpq::set_last_error("device ordinal %d out of range", dev);
    return GPQ_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_phold_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      gpq::set_last_error("cudaGetSymbolAddress(scratch) -> %s", cudaGetErrorString(e));
      return GPQ_ERR_CUDA;
    }
    g_scratch_dev[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_dev[dev];
  return GPQ_OK;
}

__global__ void static_reset_kernel(PholdCtrl* ctrl, PholdAcc* acc, uint32_t* icnt, size_t n_icnt) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i == 0) {
    for (int k = 0; k < 3; ++k) { ctrl->mins[k] = kInfBits; ctrl->errs[k] = 0; }
    ctrl->err = 0;
    ctrl->phase = 0;
    ctrl->bar = 0;
    ctrl->steps = 0;
    acc->committed = acc->pending = acc->pending_csum = acc->digest = 0;
    acc->pending_min = kInfBits;
  }
  for (size_t j = i; j < n_icnt; j += (size_t)gridDim.x * blockDim.x) icnt[j] = 0;
}

}  // namespace

extern "C" gpq_status gpq_phold_run_static(const gpq_phold_config* cfg_in, const gpq_item* d_initial,
                                           uint32_t* d_count, uint64_t* d_csum, uint64_t* d_ohash,
                                           gpq_phold_result* out, void* stream) {
  gpq_status st = gpq::validate_phold_config(cfg_in);
  if (st != GPQ_OK) return st;
  GPQ_CHECK_ARG(d_count && d_csum && d_ohash && out, "output pointers must not be NULL");
  gpq_phold_config c = *cfg_in;
  if (c.queue_kind != GPQ_QUEUE_LAQ) {
    gpq::set_last_error("gpq_phold_run_static supports the local array queue only");
    return GPQ_ERR_UNSUPPORTED;
  }
  if (c.laq_mode != 0) {
    gpq::set_last_error("gpq_phold_run_static supports the sorted local array queue only (laq_mode 0, not %u)",
                        c.laq_mode);
    return GPQ_ERR_UNSUPPORTED;
  }
  st = gpq::normalize_laq_config(&c);
  if (st != GPQ_OK) return st;
  const StaticLayout lay = layout_for(c);
  if (lay.total > (size_t)GPQ_STATIC_SCRATCH_BYTES) {
    gpq::set_last_error("gpq_phold_run_static: this configuration needs %zu bytes of scratch; the static "
                        "array holds %zu (reduce num_lps, capacity or insert_capacity)",
                        lay.total, (size_t)GPQ_STATIC_SCRATCH_BYTES);
    return GPQ_ERR_INVALID;
  }
  const size_t pop_smem = (size_t)4 * c.events_per_lp * (sizeof(gpq_item) + sizeof(uint64_t));
  PholdKernelSet ks;
  if (!phold_kernel_set(GPQ_QUEUE_LAQ, c.lanes_per_lp, c.insert_capacity, &ks)) return GPQ_ERR_INVALID;
  gpq::fit_block_to_smem(&c.block_threads, c.lanes_per_lp, ks.group_smem + 24 * kStageRounds,
                         96 * 1024 - 2048 * 16 - 16);
  const size_t win_smem = phold_window_smem_bytes(c.block_threads, c.lanes_per_lp, ks.group_smem);
  if (pop_smem > 200 * 1024 || win_smem > 96 * 1024) {
    gpq::set_last_error("gpq_phold_run_static: events_per_lp or insert_capacity too large for shared memory");
    return GPQ_ERR_INVALID;
  }

  unsigned char* base = nullptr;
  st = scratch_for_current_device(&base);
  if (st != GPQ_OK) return st;
  GPQ_CUDA_TRY(gpq::raise_smem_limit(ks.persistent, win_smem));
  GPQ_CUDA_TRY(gpq::raise_smem_limit(phold_populate_kernel, pop_smem));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  GPQ_CUDA_TRY(cudaGetDevice(&dev));
  GPQ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  PholdDev d{};  // unsharded: all LPs, no outbox
  d.p = gpq::phold_params_of(c);
  d.L = c.num_lps;
  d.lp_end = c.num_lps;
  d.count = d_count;
  d.csum = reinterpret_cast<unsigned long long*>(d_csum);
  d.ohash = reinterpret_cast<unsigned long long*>(d_ohash);
  d.ctrl = reinterpret_cast<PholdCtrl*>(base + lay.ctrl);
  d.spin_limit = gpq::spin_limit();
  LpQueueDev q{};
  q.kind = GPQ_QUEUE_LAQ;
  q.cap_log2 = gpq::ilog2_ceil(c.capacity);
  q.items = reinterpret_cast<gpq_item*>(base + lay.ring);
  q.a = reinterpret_cast<uint32_t*>(base + lay.rd);
  q.b = reinterpret_cast<uint32_t*>(base + lay.wr);
  InsDev ib{reinterpret_cast<gpq_item*>(base + lay.ibuf), reinterpret_cast<uint32_t*>(base + lay.icnt),
            c.insert_capacity};
  PholdAcc* acc = reinterpret_cast<PholdAcc*>(base + lay.acc);

  const size_t n_icnt = 2 * (size_t)c.num_lps;
  static_reset_kernel<<<(unsigned)std::min<size_t>((n_icnt + 255) / 256, 1024), 256, 0, s>>>(d.ctrl, acc, ib.cnt, n_icnt);
  GPQ_CUDA_TRY(cudaGetLastError());
  const uint32_t pwpb = 4;
  phold_populate_kernel<<<(c.num_lps + pwpb - 1) / pwpb, pwpb * 32, pop_smem, s>>>(d, q, c.events_per_lp, d_initial);
  GPQ_CUDA_TRY(cudaGetLastError());

  int per_sm = 0;
  GPQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ks.persistent, (int)c.block_threads, win_smem));
  if (per_sm <= 0) {
    gpq::set_last_error("gpq_phold_run_static: window kernel does not fit on an SM");
    return GPQ_ERR_INVALID;
  }
  if (c.ctas_per_sm) per_sm = std::min<int>(per_sm, (int)c.ctas_per_sm);
  const uint32_t gpb = c.block_threads / c.lanes_per_lp;
  uint32_t grid = std::min<uint32_t>((uint32_t)(per_sm * sms), std::max(1u, (c.num_lps + gpb - 1) / gpb));
  uint32_t s0 = 0, maxs = c.max_steps;
  void* args[] = {&d, &q, &ib, &s0, &maxs};
  GPQ_CUDA_TRY(cudaLaunchCooperativeKernel(ks.persistent, dim3(grid), dim3(c.block_threads), args,
                                           win_smem, s));
  const uint32_t fwpb = 8;
  phold_finalize_kernel<<<std::max(1u, std::min<uint32_t>((c.num_lps + fwpb - 1) / fwpb, 4096u)), fwpb * 32, 0, s>>>(
      d, q, ib, acc);
  GPQ_CUDA_TRY(cudaGetLastError());

  PholdAcc ha;
  PholdCtrl hc;
  GPQ_CUDA_TRY(cudaMemcpyAsync(&ha, acc, sizeof(ha), cudaMemcpyDeviceToHost, s));
  GPQ_CUDA_TRY(cudaMemcpyAsync(&hc, d.ctrl, sizeof(hc), cudaMemcpyDeviceToHost, s));
  GPQ_CUDA_TRY(cudaStreamSynchronize(s));
  std::memset(out, 0, sizeof(*out));
  out->committed = ha.committed;
  out->steps = hc.steps;
  out->pending = ha.pending;
  out->pending_csum = ha.pending_csum;
  out->digest = ha.digest;
  out->final_min = gpq_u2f(ha.pending_min);
  out->elapsed_ms = 0.f;
  out->status = (int32_t)hc.err;
  if (hc.err != 0)
    gpq::set_last_error("gpq_phold_run_static: the device reported %s (status %u) at window %u",
                        gpq_status_string((gpq_status)hc.err), hc.err, hc.steps);
  return (gpq_status)hc.err;
}
