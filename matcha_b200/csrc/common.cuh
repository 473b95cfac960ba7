// Shared helpers for the matcha_b200 CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/matcha_b200.h"

#define MTB_CUDA_TRY(expr)                                                     \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      mtb_set_last_error(cudaGetErrorString(_e), __FILE__, __LINE__);          \
      return (_e == cudaErrorMemoryAllocation) ? MTB_ERR_OOM : MTB_ERR_CUDA;   \
    }                                                                          \
  } while (0)

#define MTB_ARG_CHECK(cond, msg)                                               \
  do {                                                                         \
    if (!(cond)) {                                                             \
      mtb_set_last_error(msg, __FILE__, __LINE__);                             \
      return MTB_ERR_ARG;                                                      \
    }                                                                          \
  } while (0)

// Records the launch error of the kernel just issued (no device sync).
#define MTB_LAUNCH_CHECK() MTB_CUDA_TRY(cudaGetLastError())

void mtb_set_last_error(const char* msg, const char* file, int line);

__host__ __device__ inline int mtb_dsize(int L) {
  // entries of D for degrees 0..L: (L+1)(2L+1)(2L+3)/3
  return L < 0 ? 0 : (L + 1) * (2 * L + 1) * (2 * L + 3) / 3;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
