// Utilities of the C ABI: status strings, version, last error, spin limit.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "host_common.h"

namespace gpq {

static thread_local char g_last_error[512] = "";
static std::atomic<uint64_t> g_spin_limit{1ull << 24};

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

uint64_t spin_limit() { return g_spin_limit.load(); }

cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex m;
  std::lock_guard<std::mutex> lock(m);
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace gpq

extern "C" {

const char* gpq_status_string(gpq_status s) {
  switch (s) {
    case GPQ_OK: return "ok";
    case GPQ_ERR_INVALID: return "invalid argument";
    case GPQ_ERR_CUDA: return "CUDA error";
    case GPQ_ERR_QUEUE_FULL: return "queue full";
    case GPQ_ERR_INSERT_FULL: return "insert buffer full";
    case GPQ_ERR_TIMEOUT: return "device wait timed out";
    case GPQ_ERR_NOMEM: return "out of device memory";
    case GPQ_ERR_UNSUPPORTED: return "unsupported";
    case GPQ_ERR_NOT_READY: return "not ready";
  }
  return "unknown status";
}

const char* gpq_version(void) { return "gpupq_b200 0.1.0 (sm_100a)"; }

const char* gpq_last_error(void) { return gpq::g_last_error; }

gpq_status gpq_set_spin_limit(uint64_t iterations) {
  if (iterations == 0) return GPQ_ERR_INVALID;
  gpq::g_spin_limit.store(iterations);
  return GPQ_OK;
}

}  // extern "C"
