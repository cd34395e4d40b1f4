// Shared host-side helpers of libhrdaya_b200: error state and CUDA checks.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "../../include/hrdaya_b200.h"

namespace hp {

// Per-thread message of the last failure (hp_last_error()).
void set_error(const char* fmt, ...);

#define HP_CUDA_TRY(expr)                                                         \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      hp::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e),       \
                    __FILE__, __LINE__);                                          \
      return _e == cudaErrorMemoryAllocation ? HP_ERR_OOM : HP_ERR_CUDA;          \
    }                                                                             \
  } while (0)

#define HP_REQUIRE(cond, ...)        \
  do {                               \
    if (!(cond)) {                   \
      hp::set_error(__VA_ARGS__);    \
      return HP_ERR_INVALID;         \
    }                                \
  } while (0)

template <typename T>
static hp_status dev_upload(T** dst, const T* src, size_t n, cudaStream_t s) {
  *dst = nullptr;
  if (n == 0) return HP_OK;
  HP_CUDA_TRY(cudaMalloc((void**)dst, n * sizeof(T)));
  if (src) HP_CUDA_TRY(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return HP_OK;
}

template <typename T>
static hp_status dev_alloc(T** dst, size_t n) {
  *dst = nullptr;
  if (n == 0) return HP_OK;
  HP_CUDA_TRY(cudaMalloc((void**)dst, n * sizeof(T)));
  return HP_OK;
}

}  // namespace hp
