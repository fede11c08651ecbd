// Host-side helpers shared by the C-ABI implementation files.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "gpq.h"

namespace gpq {

void set_last_error(const char* fmt, ...);
uint64_t spin_limit();

// Raises `kernel`'s dynamic shared-memory limit on the current device to at least
// `bytes`; never lowers it.  Several handles (and the allocation-free run) launch the
// same kernel instantiations with different shared-memory sizes, so a limit set to one
// caller's exact size would make another caller's larger launch fail.  Serialized by a
// process-wide mutex; reads the current limit from the driver, so it holds after a
// cudaDeviceReset too.
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);
template <class K>
inline cudaError_t raise_smem_limit(K* kernel, size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

inline cudaStream_t as_stream(void* s, cudaStream_t fallback) {
  return s ? reinterpret_cast<cudaStream_t>(s) : fallback;
}

}  // namespace gpq

#define GPQ_CUDA_TRY(expr)                                                                      \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      gpq::set_last_error("%s:%d: %s -> %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_)); \
      return (e_ == cudaErrorMemoryAllocation) ? GPQ_ERR_NOMEM : GPQ_ERR_CUDA;                 \
    }                                                                                           \
  } while (0)

#define GPQ_CHECK_ARG(cond, msg)             \
  do {                                       \
    if (!(cond)) {                           \
      gpq::set_last_error("invalid: %s", msg); \
      return GPQ_ERR_INVALID;                \
    }                                        \
  } while (0)
