// errors.hpp -- CUDA error -> aak_status mapping shared by the C-ABI units,
// remembering the CUDA error text of the calling thread for aak_last_error_detail().
#pragma once

#include <cuda_runtime.h>

#include <cstdio>

#include "aak.h"

namespace aak {

inline char *last_error_buffer() {
  static thread_local char buf[256] = {0};
  return buf;
}

inline int cuda_status_of(cudaError_t e) {
  if (e == cudaSuccess) return AAK_OK;
  std::snprintf(last_error_buffer(), 256, "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? AAK_ERR_NO_MEMORY : AAK_ERR_CUDA;
}

}  // namespace aak
