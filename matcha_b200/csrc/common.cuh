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

// Launch timing (mtb_profile_start): an event before and one after a kernel launch on its
// stream, a no-op while recording is off.
void mtb_prof_begin(cudaStream_t st);
void mtb_prof_end(cudaStream_t st, const char* kernel);

__host__ __device__ inline int mtb_dsize(int L) {
  // entries of D for degrees 0..L: (L+1)(2L+1)(2L+3)/3
  return L < 0 ? 0 : (L + 1) * (2 * L + 1) * (2 * L + 3) / 3;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Round a finite float to the nearest bf16 (ties to even) with integer operations, which keeps
// the split below off the conversion unit; the bf16 bits are returned in the low half.
__device__ __forceinline__ uint32_t bf16_bits_rne(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
}

// BF16 hi + lo split of x: hi = bf16(x), lo = bf16(x - hi).
__device__ __forceinline__ void split_bf16(float x, uint32_t& hi, uint32_t& lo) {
  hi = bf16_bits_rne(x);
  lo = bf16_bits_rne(x - __uint_as_float(hi << 16));
}

// The same for a complex value, packed as bf16 pairs (real part in the low half), with the
// paired round-to-nearest-even conversion (cvt.rn.bf16x2.f32).
__device__ __forceinline__ void split_bf16x2(float re, float im, uint32_t& hi, uint32_t& lo) {
  uint32_t h, l;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(im), "f"(re));
  const float rr = re - __uint_as_float(h << 16), ri = im - __uint_as_float(h & 0xFFFF0000u);
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l) : "f"(ri), "f"(rr));
  hi = h;
  lo = l;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
