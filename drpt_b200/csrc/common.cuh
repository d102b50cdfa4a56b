// Shared definitions of libdrpt_gpu.so (B200, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>

#include "drpt_gpu.h"

namespace drpt {

// Last error text of the calling host thread (drpt_last_error).
void set_error(const char *fmt, ...);

// Streaming multiprocessors of the current device (grid-stride launches are
// sized in multiples of it); 148 if the query fails.
int device_sm_count();

#define DRPT_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      ::drpt::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? DRPT_ERR_OOM : DRPT_ERR_CUDA;              \
    }                                                                                     \
  } while (0)

#define DRPT_LAUNCH_CHECK() DRPT_CUDA(cudaGetLastError())

#define DRPT_TRY(expr)               \
  do {                               \
    drpt_status s_ = (expr);         \
    if (s_ != DRPT_OK) return s_;    \
  } while (0)

constexpr int kBins = 16;       // histogram slots per node (dist_length, math_operations.cpp:236)
constexpr int kMaxK = 64;       // largest nn the leaf kernels accept
constexpr unsigned kFull = 0xffffffffu;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

}  // namespace drpt
