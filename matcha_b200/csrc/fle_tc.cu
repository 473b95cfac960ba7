// Tensor-core path of the ball expansion: BF16 hi+lo split GEMM on tcgen05 (sm_100a).
//
// The 8 octant-parity GEMMs of fle.cu, C_p = A_p * B_p (A: folded volumes, B: basis
// columns), run here as BF16 x BF16 -> FP32 products with a split correction:
//     A B ~= A_hi B_hi + A_lo B_hi + A_hi B_lo,   A_hi = bf16(A), A_lo = bf16(A - A_hi)
// (the dropped A_lo B_lo term is ~2^-16 relative).  The three products are one GEMM over
// a K axis three times as long: k-block j of [0, 3 KB) selects (A_hi, B_hi), (A_lo, B_hi)
// or (A_hi, B_lo), so every pipeline stage moves one A tile and one B tile.  (Staging the
// hi and lo tiles of both operands per K block, 96 KB, leaves room for two stages only,
// which measured 2.2x slower: the loads are no longer hidden.)
//
// Accumulation: the tensor core adds each K=16 product into the FP32 accumulator with a
// truncating alignment, an error of about one unit in the last place of the accumulator per
// instruction.  Over the full K (15 216 octant representatives at 64^3, 2 856 instructions)
// that biases coefficients whose terms share a sign (the low degrees of a positive-mean
// volume) by ~2e-4 relative.  So the K axis is cut into chunks of kChunkKB blocks (240
// instructions, ~2e-5): each chunk accumulates into one of two tensor-memory buffers, and the
// epilogue warps add the finished buffer into running sums in registers (FP32 round-to-nearest,
// chunks in order, so the result is deterministic) while the MMAs of the next chunk run into
// the other buffer; C is written once at the end.  (Adding each chunk into C in global memory
// instead measured 2.4x slower: one row per lane makes every access a 32-way scatter.)
//
// Layout: both operands K-major bf16, 128-byte swizzled tiles staged by TMA
// (cp.async.bulk.tensor.2d), tile M = 128 (a batch block), N = 256 (basis columns),
// K = 64 per stage, 4 stages of 48 KB.  One thread issues tcgen05.mma (kind::f16, M128 N256
// K16); eight warps read the accumulators back with tcgen05.ld, two per 32-lane quarter of
// tensor memory, each keeping 128 columns of its row.  A and B of all classes and
// both parts share two tensor maps: rows (class * 2 + part) * Mpad + m of A,
// (class * 2 + part) * Npad + n of B.
//
// Every mbarrier wait is bounded; on expiry the kernel records an error code, stops
// issuing, waits (bounded) for the MMAs it issued, and frees its tensor memory before
// returning.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>
#include "common.cuh"
#include "fle_tc.cuh"
#include "tc_common.cuh"

namespace {

using namespace tc;

constexpr int TM = 128, TN = 256, TK = 64;
constexpr int STAGES = 4;
constexpr int A_TILE = TM * TK * 2;  // 16 KB
constexpr int B_TILE = TN * TK * 2;  // 32 KB
constexpr int STAGE_BYTES = A_TILE + B_TILE;
constexpr int kThreads = 320;        // warp 0: TMA, warp 1: MMA, warps 2-9: epilogue
constexpr int kEpiThreads = 256;
constexpr uint32_t kTmemCols = 512;  // two 256-column FP32 accumulators
constexpr int kChunkKB = 60;         // K blocks per accumulator chunk: 60 x 4 = 240 MMAs

struct TcParams {
  int Mpad, Npad, KB;   // padded batch rows per (class, part), padded columns, K blocks of 64
  int M;                // valid batch rows
  int ncols[8];         // valid columns per class
  int coff[8];          // column offset of the class inside C
  int ldc;              // row stride of C (floats)
  int stall;            // test hook: no loads are issued, and waits give up after kStallPolls
  int ntn;              // N tiles per class
  const int* split;     // (8, ntn): 1 = hi+lo split (three K segments), 0 = plain BF16 (one)
};

// Poll limit of every wait while the stall hook is on: at most kStallPolls x kSuspendNs (20 ms).
constexpr long long kStallPolls = 1 << 10;

// Instruction descriptor, kind::f16: D f32, A/B bf16, both K-major, M=128, N=256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_cta(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kThreads, 1)
gemm_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcParams P,
               float* __restrict__ C, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2], drain_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;

  const int cls = blockIdx.z;
  // M tiles vary fastest: the CTAs of one basis N-tile run together and read its B slab from
  // L2 rather than once per M tile from DRAM
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  if (n0 >= P.ncols[cls]) return;  // uniform per CTA
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // K blocks: the three hi/lo segments, or the (hi, hi) segment alone for a plain BF16 tile
  const int KB3 = (__ldg(&P.split[cls * P.ntn + blockIdx.y]) ? 3 : 1) * P.KB;
  const int nchunks = (KB3 + kChunkKB - 1) / kChunkKB;
  const long long polls = P.stall ? kStallPolls : kSpinLimit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiThreads);
    }
    mbar_init(&drain_bar, 1);
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
    // ---- TMA producer (the stall hook issues nothing, so the MMA thread's first wait runs out)
    for (int j = 0; j < KB3 && !abort_flag && !P.stall; ++j) {
      const int s = j % STAGES;
      const uint32_t use = j / STAGES;
      if (j >= STAGES && !mbar_wait_n(&empty_bar[s], (use - 1) & 1, polls)) {
        atomicCAS(err, 0, 1);
        abort_flag = 1;
        break;
      }
      const int part = j / P.KB;           // 0: (hi, hi), 1: (lo, hi), 2: (hi, lo)
      const int kb = j - part * P.KB;
      const int apart = (part == 1) ? 1 : 0, bpart = (part == 2) ? 1 : 0;
      uint8_t* sa = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full_bar[s], STAGE_BYTES);
      tma_load_2d(sa, &mapA, kb * TK, (cls * 2 + apart) * P.Mpad + m0, &full_bar[s]);
      tma_load_2d(sa + A_TILE, &mapB, kb * TK, (cls * 2 + bpart) * P.Npad + n0, &full_bar[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: chunk c of kChunkKB K blocks into accumulator c & 1
    bool ok = true;
    int issued = 0;
    for (int c = 0; c < nchunks && ok; ++c) {
      const int buf = c & 1;
      if (c >= 2 && !mbar_wait_n(&acc_empty[buf], ((c >> 1) - 1) & 1, polls)) {
        atomicCAS(err, 0, 4);
        abort_flag = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(buf * TN);
      const int j1 = (c + 1) * kChunkKB < KB3 ? (c + 1) * kChunkKB : KB3;
      for (int j = c * kChunkKB; j < j1; ++j) {
        const int s = j % STAGES;
        const uint32_t use = j / STAGES;
        if (abort_flag || !mbar_wait_n(&full_bar[s], use & 1, polls)) {
          atomicCAS(err, 0, 2);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* sa = smem + s * STAGE_BYTES;
        const uint64_t ad = smem_desc(sa), bd = smem_desc(sa + A_TILE);
#pragma unroll
        for (int kk = 0; kk < TK / 16; ++kk) {
          // 16 bf16 = 32 bytes further along K inside the swizzle atom: +2 in the >>4 address field
          mma_bf16(d, ad + (uint64_t)(kk * 2), bd + (uint64_t)(kk * 2), (j > c * kChunkKB || kk > 0) ? 1u : 0u);
        }
        mma_commit(&empty_bar[s]);
        ++issued;
      }
      if (ok) mma_commit(&acc_full[buf]);
    }
    if (!ok && issued > 0) {
      // let the MMAs already issued finish before the tensor memory is freed
      mma_commit(&drain_bar);
      mbar_wait_n(&drain_bar, 0, polls);
    }
  } else if (warp >= 2) {
    // ---- epilogue: warp w reads TMEM lanes 32*(w%4) .. +31 (rows m0 + that range), columns
    // h*128 .. +127 with h = (w-2)/4, and keeps their running sums over the chunks
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int row = m0 + q * 32 + lane;
    float acc[TN / 2];
#pragma unroll
    for (int t = 0; t < TN / 2; ++t) acc[t] = 0.f;
    bool done = true;
    for (int c = 0; c < nchunks; ++c) {
      const int buf = c & 1;
      if (abort_flag || !mbar_wait_n(&acc_full[buf], (c >> 1) & 1, polls)) {
        atomicCAS(err, 0, 3);
        abort_flag = 1;
        done = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * TN + h * (TN / 2));
#pragma unroll
      for (int cb = 0; cb < TN / 2; cb += 32) {
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr + (uint32_t)cb));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int t = 0; t < 32; ++t) acc[cb + t] += __uint_as_float(v[t]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive_cta(&acc_empty[buf]);
    }
    if (done && row < P.M) {
      float* crow = C + (int64_t)row * P.ldc + P.coff[cls];
      const int nc = P.ncols[cls];
      const int nb = n0 + h * (TN / 2);
#pragma unroll
      for (int t = 0; t < TN / 2; ++t)
        if (nb + t < nc) crow[nb + t] = acc[t];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---------------------------------------------------------------- operand preparation
// Folded channels, split into bf16 hi/lo: Aall[((cls*2 + part) * Mpad + b) * Kpad + rep].
__global__ void fold_split_kernel(const float* __restrict__ vol, int64_t vol_stride, int B, int n_rep, int Mpad,
                                  int Kpad, const int* __restrict__ rep_img, __nv_bfloat16* __restrict__ A) {
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (rep >= Kpad || b >= B) return;
  float f[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int idx = rep < n_rep ? __ldg(&rep_img[rep * 8 + s]) : -1;
    f[s] = idx >= 0 ? __ldg(&vol[(int64_t)b * vol_stride + idx]) : 0.f;
  }
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int s = 0; s < 8; ++s)
      if (!(s & bit)) {
        const float u = f[s], w = f[s | bit];
        f[s] = u + w;
        f[s | bit] = u - w;
      }
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    uint32_t hi, lo;
    split_bf16(f[p], hi, lo);
    A[((int64_t)(p * 2 + 0) * Mpad + b) * Kpad + rep] = __ushort_as_bfloat16((unsigned short)hi);
    A[((int64_t)(p * 2 + 1) * Mpad + b) * Kpad + rep] = __ushort_as_bfloat16((unsigned short)lo);
  }
}

// Basis (K x n_p, row-major FP32 per class) -> Ball[((cls*2 + part) * Npad + n) * Kpad + k], K-major bf16.
__global__ void basis_split_kernel(const float* __restrict__ basis, int n_rep, int ncls, int cls, int Npad, int Kpad,
                                   __nv_bfloat16* __restrict__ Bm) {
  __shared__ float tile[32][33];
  const int k0 = blockIdx.x * 32, n0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int k = k0 + i, n = n0 + threadIdx.x;
    tile[i][threadIdx.x] = (k < n_rep && n < ncls) ? basis[(int64_t)k * ncls + n] : 0.f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int n = n0 + i, k = k0 + threadIdx.x;
    if (n >= Npad || k >= Kpad) continue;
    const float v = tile[threadIdx.x][i];
    uint32_t hi, lo;
    split_bf16(v, hi, lo);
    Bm[((int64_t)(cls * 2 + 0) * Npad + n) * Kpad + k] = __ushort_as_bfloat16((unsigned short)hi);
    Bm[((int64_t)(cls * 2 + 1) * Npad + n) * Kpad + k] = __ushort_as_bfloat16((unsigned short)lo);
  }
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_map(CUtensorMap* map, void* base, uint64_t inner, uint64_t rows, uint32_t box_rows) {
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
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MTB_OK : MTB_ERR_CUDA;
}

}  // namespace

size_t fle_tc_a_elems(int max_batch, int n_rep) {
  const int Mpad = (max_batch + TM - 1) / TM * TM;
  const int Kpad = (n_rep + TK - 1) / TK * TK;
  return (size_t)16 * Mpad * Kpad;
}

int fle_tc_prepare(FleTc* t, float* const* basis, const int* class_cols, const int* class_off, int n_rep,
                   int max_batch, int n_cols, const std::vector<std::vector<int>>& col_deg, int split_degree) {
  memset(t, 0, sizeof(*t));
  t->Mpad = (max_batch + TM - 1) / TM * TM;
  t->Kpad = (n_rep + TK - 1) / TK * TK;
  int maxc = 0;
  for (int k = 0; k < 8; ++k) maxc = class_cols[k] > maxc ? class_cols[k] : maxc;
  t->Npad = (maxc + TN - 1) / TN * TN;
  t->n_rep = n_rep;
  t->n_cols = n_cols;
  for (int k = 0; k < 8; ++k) {
    t->ncols[k] = class_cols[k];
    t->coff[k] = class_off[k];
  }
  const size_t asz = (size_t)16 * t->Mpad * t->Kpad, bsz = (size_t)16 * t->Npad * t->Kpad;
  if (cudaMalloc(&t->A, asz * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->B, bsz * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->err, sizeof(int)) != cudaSuccess) return MTB_ERR_OOM;
  // which tiles take the split: those holding a column of degree above split_degree
  t->ntn = t->Npad / TN;
  {
    std::vector<int> flags((size_t)8 * t->ntn, 1);
    for (int k = 0; k < 8; ++k)
      for (int n = 0; n < t->ntn; ++n) {
        const int c0 = n * TN;
        if (c0 >= class_cols[k]) continue;
        const int c1 = (c0 + TN < class_cols[k] ? c0 + TN : class_cols[k]) - 1;
        const int top = (size_t)k < col_deg.size() && (size_t)c1 < col_deg[k].size() ? col_deg[k][c1] : 1 << 30;
        flags[(size_t)k * t->ntn + n] = (split_degree < 0 || top > split_degree) ? 1 : 0;
        t->n_tiles += 1;
        t->n_split_tiles += flags[(size_t)k * t->ntn + n];
      }
    if (cudaMalloc(&t->split, flags.size() * sizeof(int)) != cudaSuccess) return MTB_ERR_OOM;
    if (cudaMemcpy(t->split, flags.data(), flags.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      return MTB_ERR_CUDA;
  }
  if (cudaMemset(t->B, 0, bsz * 2) != cudaSuccess || cudaMemset(t->A, 0, asz * 2) != cudaSuccess ||
      cudaMemset(t->err, 0, sizeof(int)) != cudaSuccess)
    return MTB_ERR_CUDA;
  for (int k = 0; k < 8; ++k) {
    if (!class_cols[k]) continue;
    dim3 g((t->Kpad + 31) / 32, (t->Npad + 31) / 32);
    basis_split_kernel<<<g, dim3(32, 8)>>>(basis[k], n_rep, class_cols[k], k, t->Npad, t->Kpad,
                                           reinterpret_cast<__nv_bfloat16*>(t->B));
    if (cudaGetLastError() != cudaSuccess) return MTB_ERR_CUDA;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return MTB_ERR_CUDA;
  int rc = make_map(reinterpret_cast<CUtensorMap*>(t->mapA), t->A, (uint64_t)t->Kpad, (uint64_t)16 * t->Mpad, TM);
  if (!rc) rc = make_map(reinterpret_cast<CUtensorMap*>(t->mapB), t->B, (uint64_t)t->Kpad, (uint64_t)16 * t->Npad, TN);
  return rc;
}

void fle_tc_release(FleTc* t) {
  if (t->A) cudaFree(t->A);
  if (t->B) cudaFree(t->B);
  if (t->err) cudaFree(t->err);
  if (t->split) cudaFree(t->split);
  memset(t, 0, sizeof(*t));
}

int fle_tc_forward(FleTc* t, const float* vol, int64_t vol_stride, int B, const int* rep_img, float* C,
                   cudaStream_t st) {
  dim3 fg((t->Kpad + 255) / 256, B);
  mtb_prof_begin(st);
  fold_split_kernel<<<fg, 256, 0, st>>>(vol, vol_stride, B, t->n_rep, t->Mpad, t->Kpad, rep_img,
                                        reinterpret_cast<__nv_bfloat16*>(t->A));
  mtb_prof_end(st, "fold_split_kernel");
  MTB_LAUNCH_CHECK();
  TcParams P;
  P.Mpad = t->Mpad;
  P.Npad = t->Npad;
  P.KB = t->Kpad / TK;
  P.M = B;
  for (int k = 0; k < 8; ++k) {
    P.ncols[k] = t->ncols[k];
    P.coff[k] = t->coff[k];
  }
  P.ldc = t->n_cols;
  P.stall = t->stall;
  P.ntn = t->ntn;
  P.split = t->split;
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 1024;
  MTB_CUDA_TRY(cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 gg((B + TM - 1) / TM, t->Npad / TN, 8);
  mtb_prof_begin(st);
  gemm_tc_kernel<<<gg, kThreads, smem, st>>>(*reinterpret_cast<const CUtensorMap*>(t->mapA),
                                             *reinterpret_cast<const CUtensorMap*>(t->mapB), P, C, t->err);
  mtb_prof_end(st, "gemm_tc_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

int fle_tc_check(FleTc* t, cudaStream_t st) {
  int h = 0;
  MTB_CUDA_TRY(cudaMemcpyAsync(&h, t->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MTB_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) MTB_CUDA_TRY(cudaMemsetAsync(t->err, 0, sizeof(int), st));  // reported once
  return h ? MTB_ERR_TIMEOUT : MTB_OK;
}
