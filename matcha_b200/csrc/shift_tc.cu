// Tensor-core path of the shift match's local upsampled DFT (tcgen05, BF16 hi+lo split).
//
// The refined correlation of src/matcha/core/ShiftMatcher.py:46-91, 241-272,
//   V[u0,u1,u2] = Re sum_{m0,m1,m2} P[m0,m1,m2] E0[u0,m0] E0[u1,m1] E2[u2,m2],
// E[u,m] = exp(+2 pi i (u - dftshift) fftfreq(n, uf)[m]), is computed as three GEMMs whose
// complex products are real GEMMs on interleaved (re, im) K axes:
//   pass 1  rows (b, m2, m1),  K = (m0, re/im) = 2N,    N-tile = (u0, re/im) = 2U
//   pass 2  rows (b, u0, m2),  K = (m1, re/im) = 2N,    N-tile = (u1, re/im) = 2U
//   pass 3  rows (b, u0, u1),  K = (m2, re/im) = 2H -> padded to 2N, N-tile = u2 (real part)
// Each pass's epilogue writes the next pass's A operand directly in its K-major bf16 hi/lo
// layout (no transpose kernel), and pass 3 keeps a running argmax per subtomogram in a
// 64-bit key (ordered value, inverted flat index), so the U^3 grid never reaches memory.
// Operands are split A = A_hi + A_lo, B = B_hi + B_lo; A B ~ A_hi B_hi + A_lo B_hi + A_hi B_lo
// is one GEMM over three K segments.  All device waits are bounded.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>
#include "common.cuh"
#include "shift_tc.cuh"
#include "tc_common.cuh"

namespace {

using namespace tc;

constexpr int TM = 128, TK = 64;
constexpr int kStages = 2;
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 256;

struct UParams {
  int KB;         // 64-element K blocks of A and B
  int KBo;        // 64-element K blocks of the output operand (passes 1, 2)
  int R;          // rows per part of A (padded)
  int rows;       // valid rows (B * rows per subtomogram)
  int rpb;        // rows per subtomogram
  int N, H, U;
  int R_out;      // rows per part of the output operand (passes 1, 2)
  int rpb_out;    // rows per subtomogram of the output operand
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo_elem, float hi_elem) {
  // first element in the low half
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat16 rh = __float2bfloat16_rn(re), ih = __float2bfloat16_rn(im);
  hi = pack_bf16x2(__bfloat162float(rh), __bfloat162float(ih));
  lo = pack_bf16x2(re - __bfloat162float(rh), im - __bfloat162float(ih));
}

__device__ __forceinline__ unsigned long long argmax_key(float v, int flat) {
  uint32_t b = __float_as_uint(v);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // order-preserving
  return ((unsigned long long)b << 32) | (unsigned long long)(0xFFFFFFFFu - (uint32_t)flat);
}

template <int NT>
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* out) {
  uint32_t v[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) out[i] = __uint_as_float(v[i]);
}

// MODE 1: pass 1 -> A2; MODE 2: pass 2 -> A3; MODE 3: pass 3 -> argmax keys.
template <int NT, int MODE>
__global__ void __launch_bounds__(kThreads, 1)
updft_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, UParams P,
                uint32_t* __restrict__ out, unsigned long long* __restrict__ best, int* __restrict__ err) {
  constexpr int A_TILE = TM * TK * 2;
  constexpr int B_TILE = NT * TK * 2;
  constexpr int STAGE = A_TILE + B_TILE;
  const int KB = P.KB;
  const int KB3 = 3 * KB;  // with the hi/lo split
  constexpr uint32_t IDESC = idesc_bf16(TM, NT);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;

  const int row0 = blockIdx.x * TM;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  if (warp == 0 && lane == 0) {
    for (int j = 0; j < KB3; ++j) {
      const int s = j % kStages;
      const uint32_t use = j / kStages;
      if (j >= kStages && !mbar_wait(&empty_bar[s], (use - 1) & 1)) {
        atomicExch(err, 11);
        abort_flag = 1;
        break;
      }
      if (abort_flag) break;
      const int part = j / KB, kb = j - part * KB;
      const int ap = (part == 1) ? 1 : 0, bp = (part == 2) ? 1 : 0;
      uint8_t* sa = smem + s * STAGE;
      mbar_expect_tx(&full_bar[s], STAGE);
      tma_load_2d(sa, &mapA, kb * TK, ap * P.R + row0, &full_bar[s]);
      tma_load_2d(sa + A_TILE, &mapB, kb * TK, bp * NT, &full_bar[s]);
    }
  } else if (warp == 1 && lane == 0) {
    bool ok = true;
    for (int j = 0; j < KB3; ++j) {
      const int s = j % kStages;
      const uint32_t use = j / kStages;
      if (!mbar_wait(&full_bar[s], use & 1)) {
        atomicExch(err, 12);
        abort_flag = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint8_t* sa = smem + s * STAGE;
      const uint64_t ad = smem_desc(sa), bd = smem_desc(sa + A_TILE);
#pragma unroll
      for (int kk = 0; kk < TK / 16; ++kk)
        mma_bf16_id(tmem, ad + (uint64_t)(kk * 2), bd + (uint64_t)(kk * 2), IDESC, (j > 0 || kk > 0) ? 1u : 0u);
      mma_commit_to(&empty_bar[s]);
    }
    if (ok) mma_commit_to(&done_bar);
  } else if (warp >= 2) {
    const bool ok = mbar_wait(&done_bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
      atomicExch(err, 13);
    } else {
      const int q = warp & 3;
      const int g = row0 + q * 32 + lane;  // global row
      const bool valid = g < P.rows;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16);
      const int b = valid ? g / P.rpb : 0;
      const int rem = valid ? g - b * P.rpb : 0;
      if (MODE == 1) {
        // row (b, m2, m1): write A2[part][b, u0, m2][2 m1 + c]
        const int m2 = rem / P.N, m1 = rem - m2 * P.N;
        const size_t base_row = (size_t)b * P.rpb_out + m2;  // + u0 * H
        const size_t ws = (size_t)P.KBo * (TK / 2);           // row stride in bf16 pairs
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += 16) {
          float v[16];
          tmem_ld16<NT>(taddr + (uint32_t)cb, v);
          if (valid) {
#pragma unroll
            for (int t = 0; t < 8; ++t) {
              const int u0 = cb / 2 + t;
              if (u0 >= P.U) break;
              uint32_t hi, lo;
              split2(v[2 * t], v[2 * t + 1], hi, lo);
              const size_t row = base_row + (size_t)u0 * P.H;
              out[row * ws + m1] = hi;
              out[((size_t)P.R_out + row) * ws + m1] = lo;
            }
          }
        }
      } else if (MODE == 2) {
        // row (b, u0, m2): write A3[part][b, u0, u1][2 m2 + c]
        const int u0 = rem / P.H, m2 = rem - u0 * P.H;
        const size_t base_row = (size_t)b * P.rpb_out + (size_t)u0 * P.U;  // + u1
        const size_t ws = (size_t)P.KBo * (TK / 2);
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += 16) {
          float v[16];
          tmem_ld16<NT>(taddr + (uint32_t)cb, v);
          if (valid) {
#pragma unroll
            for (int t = 0; t < 8; ++t) {
              const int u1 = cb / 2 + t;
              if (u1 >= P.U) break;
              uint32_t hi, lo;
              split2(v[2 * t], v[2 * t + 1], hi, lo);
              const size_t row = base_row + u1;
              out[row * ws + m2] = hi;
              out[((size_t)P.R_out + row) * ws + m2] = lo;
            }
          }
        }
      } else {
        // row (b, u0, u1): running argmax over u2 < U, flat = rem * U + u2
        float bv = -INFINITY;
        int bi = 0x7fffffff;
        bool have = false;
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += 16) {
          float v[16];
          tmem_ld16<NT>(taddr + (uint32_t)cb, v);
#pragma unroll
          for (int t = 0; t < 16; ++t) {
            const int u2 = cb + t;
            if (u2 < P.U) {
              const float x = v[t];
              const bool nan_x = isnan(x);
              if (!have || (nan_x && !isnan(bv)) || (!isnan(bv) && x > bv)) {
                bv = x;
                bi = u2;
                have = true;
              }
            }
          }
        }
        unsigned long long key = valid ? argmax_key(bv, rem * P.U + bi) : 0ull;
        // combine lanes of the same subtomogram before the atomic
        const int b0 = __shfl_sync(0xffffffffu, b, 0);
        const bool uniform = __all_sync(0xffffffffu, !valid || b == b0);
        if (uniform) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
            key = k2 > key ? k2 : key;
          }
          if (lane == 0 && key) atomicMax(&best[b0], key);
        } else if (valid) {
          atomicMax(&best[b], key);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_map(void* map, void* base, uint64_t inner, uint64_t rows, uint32_t box_rows) {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return MTB_ERR_CUDA;
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  const cuuint64_t dims[2] = {inner, rows};
  const cuuint64_t strides[1] = {inner * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MTB_OK : MTB_ERR_CUDA;
}

uint16_t f2bf(float f) {  // round to nearest even
  uint32_t u;
  memcpy(&u, &f, 4);
  const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}
float bf2f(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

template <int NT, int MODE>
int launch_pass(const ShiftTc* t, const void* mapA, const void* mapB, const UParams& P, uint32_t* out,
                cudaStream_t st) {
  // at least 100 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
  size_t smem = (size_t)kStages * (TM * TK * 2 + NT * TK * 2) + 1024;
  if (smem < 100 * 1024) smem = 100 * 1024;
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft_tc_kernel<NT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (P.rows + TM - 1) / TM;
  updft_tc_kernel<NT, MODE><<<grid, kThreads, smem, st>>>(*reinterpret_cast<const CUtensorMap*>(mapA),
                                                          *reinterpret_cast<const CUtensorMap*>(mapB), P, out,
                                                          t->best, t->err);
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

}  // namespace

int shift_tc_prepare(ShiftTc* t, int N, int H, int U, int uf, float dftshift, int max_batch) {
  memset(t, 0, sizeof(*t));
  // N-tile of passes 1, 2 is round_up(2U, 16) <= 256; of pass 3 round_up(U, 16)
  if (U < 1 || 2 * U > 256 || N < 2) return MTB_ERR_ARG;
  t->N = N;
  t->H = H;
  t->U = U;
  t->NT12 = (2 * U + 15) / 16 * 16;
  t->NT3 = (U + 15) / 16 * 16;
  t->KB12 = (2 * N + TK - 1) / TK;
  t->KB3 = (2 * H + TK - 1) / TK;
  t->Bmax = max_batch;
  auto pad = [](size_t r) { return (r + TM - 1) / TM * TM; };
  t->R1 = (int)pad((size_t)max_batch * N * H);
  t->R2 = (int)pad((size_t)max_batch * U * H);
  t->R3 = (int)pad((size_t)max_batch * U * U);
  const size_t k12 = (size_t)t->KB12 * TK, k3 = (size_t)t->KB3 * TK;
  const size_t a1 = (size_t)2 * t->R1 * k12 * 2, a2 = (size_t)2 * t->R2 * k12 * 2, a3 = (size_t)2 * t->R3 * k3 * 2;
  if (cudaMalloc(&t->A1, a1) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->A2, a2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->A3, a3) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->E1, (size_t)2 * t->NT12 * k12 * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->E3, (size_t)2 * t->NT3 * k3 * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->best, (size_t)max_batch * 8) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->err, 4) != cudaSuccess) return MTB_ERR_OOM;
  // K columns past 2N (A1, A2) and 2H (A3) stay zero; the rest is rewritten by every call
  if (cudaMemset(t->A1, 0, a1) != cudaSuccess || cudaMemset(t->A2, 0, a2) != cudaSuccess ||
      cudaMemset(t->A3, 0, a3) != cudaSuccess || cudaMemset(t->err, 0, 4) != cudaSuccess)
    return MTB_ERR_CUDA;
  // B operands: E1 rows (u, re/im), K (m, re/im); E3 rows u2, K (m2, re/im) -> real part
  auto E = [&](int n, int u, int m, double* re, double* im) {
    const int mm = (m < (n + 1) / 2) ? m : m - n;
    const double f = (double)mm / ((double)uf * n);
    const double ph = 2.0 * M_PI * ((double)u - dftshift) * f;
    *re = cos(ph);
    *im = sin(ph);
  };
  std::vector<uint16_t> e1((size_t)2 * t->NT12 * k12, 0), e3((size_t)2 * t->NT3 * k3, 0);
  auto put = [&](std::vector<uint16_t>& dst, size_t k, int rows, int r, int kk, double v) {
    const uint16_t hi = f2bf((float)v);
    const uint16_t lo = f2bf((float)(v - (double)bf2f(hi)));
    dst[(size_t)r * k + kk] = hi;
    dst[((size_t)rows + r) * k + kk] = lo;
  };
  for (int u = 0; u < U; ++u)
    for (int m = 0; m < N; ++m) {
      double er, ei;
      E(N, u, m, &er, &ei);
      put(e1, k12, t->NT12, 2 * u + 0, 2 * m + 0, er);
      put(e1, k12, t->NT12, 2 * u + 0, 2 * m + 1, -ei);
      put(e1, k12, t->NT12, 2 * u + 1, 2 * m + 0, ei);
      put(e1, k12, t->NT12, 2 * u + 1, 2 * m + 1, er);
    }
  for (int u = 0; u < U; ++u)
    for (int m = 0; m < H; ++m) {
      double er, ei;
      E(H, u, m, &er, &ei);
      put(e3, k3, t->NT3, u, 2 * m + 0, er);
      put(e3, k3, t->NT3, u, 2 * m + 1, -ei);
    }
  if (cudaMemcpy(t->E1, e1.data(), e1.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t->E3, e3.data(), e3.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess)
    return MTB_ERR_CUDA;
  int rc = make_map(t->mapA1, t->A1, k12, (uint64_t)2 * t->R1, TM);
  if (!rc) rc = make_map(t->mapA2, t->A2, k12, (uint64_t)2 * t->R2, TM);
  if (!rc) rc = make_map(t->mapA3, t->A3, k3, (uint64_t)2 * t->R3, TM);
  if (!rc) rc = make_map(t->mapE1, t->E1, k12, (uint64_t)2 * t->NT12, t->NT12);
  if (!rc) rc = make_map(t->mapE3, t->E3, k3, (uint64_t)2 * t->NT3, t->NT3);
  return rc;
}

void shift_tc_release(ShiftTc* t) {
  void* ptrs[] = {t->A1, t->A2, t->A3, t->E1, t->E3, t->best, t->err};
  for (void* p : ptrs) if (p) cudaFree(p);
  memset(t, 0, sizeof(*t));
}

template <int MODE>
int dispatch(const ShiftTc* t, int nt, const void* mapA, const void* mapB, const UParams& P, uint32_t* out,
             cudaStream_t st) {
  switch (nt) {
    case 16: return launch_pass<16, MODE>(t, mapA, mapB, P, out, st);
    case 32: return launch_pass<32, MODE>(t, mapA, mapB, P, out, st);
    case 48: return launch_pass<48, MODE>(t, mapA, mapB, P, out, st);
    case 64: return launch_pass<64, MODE>(t, mapA, mapB, P, out, st);
    case 80: return launch_pass<80, MODE>(t, mapA, mapB, P, out, st);
    case 96: return launch_pass<96, MODE>(t, mapA, mapB, P, out, st);
    case 112: return launch_pass<112, MODE>(t, mapA, mapB, P, out, st);
    case 128: return launch_pass<128, MODE>(t, mapA, mapB, P, out, st);
    case 144: return launch_pass<144, MODE>(t, mapA, mapB, P, out, st);
    case 160: return launch_pass<160, MODE>(t, mapA, mapB, P, out, st);
    case 176: return launch_pass<176, MODE>(t, mapA, mapB, P, out, st);
    case 192: return launch_pass<192, MODE>(t, mapA, mapB, P, out, st);
    case 208: return launch_pass<208, MODE>(t, mapA, mapB, P, out, st);
    case 224: return launch_pass<224, MODE>(t, mapA, mapB, P, out, st);
    case 240: return launch_pass<240, MODE>(t, mapA, mapB, P, out, st);
    case 256: return launch_pass<256, MODE>(t, mapA, mapB, P, out, st);
    default: return MTB_ERR_ARG;
  }
}

int shift_tc_passes(ShiftTc* t, int B, cudaStream_t st) {
  MTB_CUDA_TRY(cudaMemsetAsync(t->best, 0, (size_t)B * 8, st));
  const int N = t->N, H = t->H, U = t->U;
  UParams P;
  P.N = N;
  P.H = H;
  P.U = U;
  // pass 1: rows (b, m2, m1) -> A2 rows (b, u0, m2)
  P.KB = t->KB12;
  P.KBo = t->KB12;
  P.R = t->R1;
  P.rpb = N * H;
  P.rows = B * P.rpb;
  P.R_out = t->R2;
  P.rpb_out = U * H;
  int rc = dispatch<1>(t, t->NT12, t->mapA1, t->mapE1, P, (uint32_t*)t->A2, st);
  if (rc) return rc;
  // pass 2: rows (b, u0, m2) -> A3 rows (b, u0, u1)
  P.KB = t->KB12;
  P.KBo = t->KB3;
  P.R = t->R2;
  P.rpb = U * H;
  P.rows = B * P.rpb;
  P.R_out = t->R3;
  P.rpb_out = U * U;
  rc = dispatch<2>(t, t->NT12, t->mapA2, t->mapE1, P, (uint32_t*)t->A3, st);
  if (rc) return rc;
  // pass 3: rows (b, u0, u1) -> argmax keys
  P.KB = t->KB3;
  P.KBo = 0;
  P.R = t->R3;
  P.rpb = U * U;
  P.rows = B * P.rpb;
  P.R_out = 0;
  P.rpb_out = 0;
  return dispatch<3>(t, t->NT3, t->mapA3, t->mapE3, P, nullptr, st);
}

int shift_tc_check(ShiftTc* t, cudaStream_t st) {
  int h = 0;
  MTB_CUDA_TRY(cudaMemcpyAsync(&h, t->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MTB_CUDA_TRY(cudaStreamSynchronize(st));
  return h ? MTB_ERR_TIMEOUT : MTB_OK;
}
