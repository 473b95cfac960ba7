// Tensor-core path of the shift match's local upsampled DFT (tcgen05, BF16 hi+lo split).
//
// The refined correlation of src/matcha/core/ShiftMatcher.py:46-91, 241-272,
//   V[u0,u1,u2] = Re sum_{m0,m1,m2} P[m0,m1,m2] E0[u0,m0] E0[u1,m1] E2[u2,m2],
// E[u,m] = exp(+2 pi i (u - dftshift) fftfreq(n, uf)[m]), m2 < H = N/2 + 1, is split into the
// planes m2 < N/2 (tensor cores) and the Nyquist plane m2 = N/2 (FP32 CUDA cores):
//   nyquist  Y[u0,u1] = sum_{m0,m1} E0[u0,m0] E0[u1,m1] P[m0,m1,N/2]: pass 1 on the plane's own
//            operand A1n (rows (b, m1)) into A2n (rows (b, u0)), then the pass-2 product of A2n
//            written out as FP32 rows (the pass-1 kernel in both, with another epilogue)
//   pass 1   rows (b, m2, m1), K = (m0, re/im) = 2N, N-tile = (u0, re/im) = 2U   (X1 -> A2)
//   pass 2   rows (b, u0, m2), K = (m1, re/im) = 2N, N-tile = (u1, re/im) = 2U   (X2)
//   pass 3   rows (b, u0, u1), K = (m2, re/im) = N,  N-tile = u2 (real part); + Re(Y E2[u2, N/2])
//            added in FP32 before the argmax
// Complex products are real GEMMs on interleaved (re, im) K axes.  Operands are split
// A = A_hi + A_lo, B = B_hi + B_lo and A B ~ A_hi B_hi + A_lo B_hi + A_hi B_lo.
//
// Both kernels are persistent (one CTA per SM) with their B operands resident in shared
// memory.  Pass 1 double-buffers its accumulator in tensor memory, so the epilogue that
// writes the pass-2 operand A2 (K-major bf16 hi/lo) overlaps the next tile's MMAs.  Passes 2
// and 3 are fused: a tile is G = 128 / (N/2) consecutive u0 of one subtomogram with all their
// m2 < N/2, so its pass-2 accumulator holds complete X2[u0, u1, :] rows.  Eight warps write
// them as the pass-3 A operand straight into shared memory (the 128-byte-swizzled K-major
// layout the tensor core reads), one chunk of N/2 consecutive u1 for all G u0 at a time, so
// each lane has the same share of every chunk.  Eight more warps reduce each chunk's pass-3
// accumulator (two alternating buffers in tensor memory), plus the Nyquist term in FP32, to
// a running argmax key per subtomogram, a chunk behind the writers.  A2 K-blocks and pass-3
// chunks take turns in a ring of two or three shared-memory slots, so the next tile's A2
// loads while this tile's pass 3 runs.  Neither X2 nor the U^3 grid reaches memory.
//
// The fused kernel needs 2U <= 256 and whole u0 groups per 128-row tile (boxes 16, 32, 64).
// Other even boxes up to 128 (48, 80, 96, 128) and U up to 256 run the passes unfused: pass 2
// is the pass-1 kernel again, its epilogue writing X2 as the pass-3 operand A3 to memory (rows
// (b, u0 U + u1) padded to a multiple of 128 per subtomogram), and updft3_tc_kernel runs pass 3
// with the Nyquist term and the argmax.  Where 2U > 256 or E1 would not fit in shared memory
// beside two A stages, the N-tile of passes 1 and 2 is cut into column parts, one per CTA, the
// CTAs of one row tile adjacent in the grid so that A is read from memory once.  All device
// waits are bounded; a wait that runs out sets err and the CTA winds down.
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
constexpr int kThreads = 320;        // warp 0 TMA, warp 1 MMA + TMEM, warps 2-9 epilogue
constexpr int kEpi = 256;            // epilogue threads: two warps per 32-lane quarter of TMEM
constexpr int kArg = 256;            // argmax threads of the fused passes 2+3: two warps per quarter
constexpr int kThreads23 = 64 + kEpi + kArg;  // warps 10-17 of updft23 take the argmax
constexpr int kMaxSlots = 3;         // operand slots of the fused passes 2+3
constexpr int A_TILE = TM * TK * 2;  // one 128 x 64 bf16 K-block
constexpr int kMaxStages = 8;
constexpr size_t kSmemCap = 227 * 1024 - 2048;  // dynamic shared memory: the opt-in limit less the
                                                // kernels' static barriers, with room to spare

// One complex DFT pass as a GEMM: rows of A (K = (m, re/im)) times E1 -> columns (u, re/im).
// The N-tile 2U is cut into NS column parts of Us values of u (NT columns each, <= 256), one
// part per CTA, so that E1's part stays resident in shared memory; CTAs c and c + 1 .. c + NS - 1
// take the same row tile at the same time, so A is read from memory once.  The epilogue writes
// the next pass's operand: input row g = b rpb + x Y + y becomes output row b SB + x SX + u SU,
// K word y (a (re, im) bf16 pair), hi part at row, lo part at Rout + row; or, with ROWS_OUT,
// FP32 rows (g, u).
struct Pass1 {
  int rows;     // valid rows of A
  int tiles;
  int U;
  int KB;       // K blocks of A and E1 (2N / 64)
  int R1;       // rows per hi/lo part of A
  int NT;       // N-tile of one column part (2 Us rounded to 16)
  int NS, Us;   // column parts, values of u per part
  int stages;
  int rpb, Y, SB, SX, SU, ws, Rout;  // operand-out epilogue (see above)
};

// The third pass on its own (boxes and upsampled regions outside the fused passes 2+3): rows
// (b, u0 U + u1) of A3, padded to RP3 rows per subtomogram, K = (m2 < N/2, re/im), times E3 ->
// the real grid values u2, plus the Nyquist term, reduced to a running argmax per subtomogram.
struct Pass3 {
  int tiles, TPB;  // tiles = B * TPB, TPB = RP3 / 128
  int U;
  int KB;          // K blocks of A3 and E3
  int R3;          // rows per hi/lo part of A3
  int NT;          // U rounded to 16
  int stages;
};

struct Pass23 {
  int B, tiles;  // tiles = B * TPB
  int N, HH, U, G, TPB, CH;
  int KB;        // K blocks of A2 and E1
  int R2;
  int NT12, NT3;
  int NB;        // operand slots (2 or 3)
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
  split_bf16x2(re, im, hi, lo);
}

__device__ __forceinline__ unsigned long long argmax_key(float v, int flat) {
  uint32_t b = __float_as_uint(v);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // order-preserving
  return ((unsigned long long)b << 32) | (unsigned long long)(0xFFFFFFFFu - (uint32_t)flat);
}

// Split issue / wait of a 16-column TMEM load, for software pipelining: the wait names the
// destination registers as in-out operands, so no use of them can move above it.
__device__ __forceinline__ void tmem_issue16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// f(r, c) for the 16-column groups c = c0, c0 + 16, .. < c1 of this warp's lanes at TMEM
// address base + c, with the load of the next group in flight while f runs.  c0, c1 must be
// warp-uniform.
template <class F>
__device__ __forceinline__ void tmem_for_groups(uint32_t base, int c0, int c1, F&& f) {
  uint32_t ra[16], rb[16];
  if (c0 >= c1) return;
  tmem_issue16(base + (uint32_t)c0, ra);
  for (int c = c0; c < c1; c += 32) {
    tmem_wait16(ra);
    const bool more = c + 16 < c1;
    if (more) tmem_issue16(base + (uint32_t)(c + 16), rb);
    f(ra, c);
    if (more) {
      tmem_wait16(rb);
      if (c + 32 < c1) tmem_issue16(base + (uint32_t)(c + 32), ra);
      f(rb, c + 16);
    }
  }
}

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Three-segment hi/lo MMA over one 64-wide K block (four K steps of 16).
__device__ __forceinline__ void mma_split_kblock(uint32_t d, uint64_t a_hi, uint64_t a_lo, uint64_t b_hi,
                                                 uint64_t b_lo, uint32_t idesc, bool first) {
#pragma unroll
  for (int kk = 0; kk < TK / 16; ++kk) {
    const uint64_t o = (uint64_t)(kk * 2);
    mma_bf16_id(d, a_hi + o, b_hi + o, idesc, (first && kk == 0) ? 0u : 1u);
    mma_bf16_id(d, a_lo + o, b_hi + o, idesc, 1u);
    mma_bf16_id(d, a_hi + o, b_lo + o, idesc, 1u);
  }
}

// Epilogue helpers over NC TMEM columns already in registers.  The per-value work is
// unconditional so it can be interleaved; only the stores are predicated.

// Passes 1 and 2: columns (u, re/im) of one input row -> K word y of the output rows
// row0 + u SU, u = ubase + local column pair (local < ulim, u < U).
template <int NC>
__device__ __forceinline__ void epi1_group(const uint32_t* v, int cb, bool valid, int ubase, int ulim, int U,
                                           size_t row0, int SU, size_t ws, int y, size_t Rout,
                                           uint32_t* __restrict__ out) {
#pragma unroll
  for (int t = 0; t < NC / 2; ++t) {
    uint32_t hi, lo;
    split2(__uint_as_float(v[2 * t]), __uint_as_float(v[2 * t + 1]), hi, lo);
    const int ul = cb / 2 + t, u = ubase + ul;
    const size_t row = row0 + (size_t)u * SU;
    if (valid && ul < ulim && u < U) {
      out[row * ws + y] = hi;
      out[(Rout + row) * ws + y] = lo;
    }
  }
}

// Passes 2 + 3: columns (u1, re/im) of one pass-2 row (u0_local, m2) -> word m2 of the pass-3
// operand rows rbase + u1 that fall in this chunk (128-byte-swizzled K-major tile).  The
// group's 8 rows r0 + t start at a multiple of 8 (rbase and cb / 2 are), so row r0 + t sits
// t * 128 bytes into one 1024-byte swizzle atom and word m2 in 16-byte chunk (m2 / 4) ^ t: the
// XOR with a constant is the whole per-row address arithmetic.
template <int NC>
__device__ __forceinline__ void epi2_group(const uint32_t* v, int cb, int lo_l, int hi_l, int rbase, int m2,
                                           uint8_t* sA3) {
  static_assert(NC == 16, "one group is 8 rows of the pass-3 operand");
  const int u10 = cb / 2;
  uint8_t* base = sA3 + (((rbase + u10) >> 3) << 10) + ((m2 & 3) << 2);
  const uint32_t cw = (uint32_t)(m2 >> 2) << 4;
  const bool full = u10 >= lo_l && u10 + 8 <= hi_l;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    uint32_t hi, lo;
    split2(__uint_as_float(v[2 * t]), __uint_as_float(v[2 * t + 1]), hi, lo);
    uint8_t* at = base + t * 128 + (cw ^ (uint32_t)(t << 4));
    if (full || (u10 + t >= lo_l && u10 + t < hi_l)) {
      *reinterpret_cast<uint32_t*>(at) = hi;
      *reinterpret_cast<uint32_t*>(at + A_TILE) = lo;
    }
  }
}

__device__ __forceinline__ float fmax_nan(float a, float b) {
  float d;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
  return d;
}

// Pass 3: running argmax over NC values u2 = cb .. cb + NC - 1 of one row (flat index
// row_flat * U + u2).  Four independent chains keep (value, index) with a strict comparison,
// so each keeps its first maximum; they are merged by value, then by index.  NaN is detected
// by a NaN-propagating maximum and, when present (rare), located by a rescan
// (torch.argmax order: NaN above everything, the first index wins ties).
template <int NC>
__device__ __forceinline__ void scan_group(const uint32_t* vr, int cb, int U, int row_flat, float& bv, int& bi,
                                           bool& have) {
  float v[NC];
#pragma unroll
  for (int t = 0; t < NC; ++t) v[t] = __uint_as_float(vr[t]);
  if (cb + NC > U) {
#pragma unroll
    for (int t = 0; t < NC; ++t) v[t] = (cb + t < U) ? v[t] : -INFINITY;
  }
  float m4[4] = {v[0], v[1], v[2], v[3]};
  int i4[4] = {0, 1, 2, 3};
  float n4[2] = {v[0], v[1]};
#pragma unroll
  for (int t = 4; t < NC; ++t) {
    const bool gt = v[t] > m4[t & 3];
    m4[t & 3] = gt ? v[t] : m4[t & 3];
    i4[t & 3] = gt ? t : i4[t & 3];
  }
#pragma unroll
  for (int t = 2; t < NC; ++t) n4[t & 1] = fmax_nan(n4[t & 1], v[t]);
  if (bv != bv) return;  // a NaN was found earlier: nothing later wins
  const float nn = fmax_nan(n4[0], n4[1]);
  if (nn != nn) {
    int tb = 0;
#pragma unroll
    for (int t = NC - 1; t >= 0; --t)
      if (v[t] != v[t]) tb = t;
    bv = nn;
    bi = row_flat * U + cb + tb;
    have = true;
    return;
  }
  float m = m4[0];
  int im = i4[0];
#pragma unroll
  for (int c = 1; c < 4; ++c) {
    const bool take = m4[c] > m || (m4[c] == m && i4[c] < im);
    m = take ? m4[c] : m;
    im = take ? i4[c] : im;
  }
  if (!have || m > bv) {
    bv = m;
    bi = row_flat * U + cb + im;
    have = true;
  }
}

// ------------------------------------------------------------------ pass 1
// Rows (b, m2, m1) of A1 times E1 -> X1[u0] for the tile's rows, written as A2 rows
// (b, u0, m2) with K (m1, re/im), bf16 hi and lo parts.
template <bool ROWS_OUT>
__global__ void __launch_bounds__(kThreads, 1)
updft1_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, Pass1 p,
                 uint32_t* __restrict__ out, float2* __restrict__ yout, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int KB = p.KB, S = p.stages, NT = p.NT, NS = p.NS;
  const int B_BLK = NT * TK * 2;
  uint8_t* sB = smem;                    // [part][kb] B_BLK
  uint8_t* sA = smem + 2 * KB * B_BLK;   // [stage][part] A_TILE
  // this CTA's column part and its walk over the row tiles (gridDim.x is a multiple of NS)
  const int cpart = blockIdx.x % NS, t0 = blockIdx.x / NS, tstep = gridDim.x / NS;
  __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages];
  __shared__ __align__(8) uint64_t accF[2], accE[2], resF;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&accF[i], 1);
      mbar_init(&accE[i], kEpi);
    }
    mbar_init(&resF, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = idesc_bf16(TM, NT);

  if (warp == 0 && lane == 0) {
    mbar_expect_tx(&resF, (uint32_t)(2 * KB * B_BLK));
    for (int part = 0; part < 2; ++part)
      for (int kb = 0; kb < KB; ++kb)
        tma_load_2d(sB + (part * KB + kb) * B_BLK, &mapB, kb * TK, (part * NS + cpart) * NT, &resF);
    int it = 0;
    for (int tile = t0; tile < p.tiles && !abort_flag; tile += tstep) {
      for (int kb = 0; kb < KB; ++kb, ++it) {
        const int s = it % S;
        const uint32_t use = it / S;
        if (it >= S && !mbar_wait(&empty_bar[s], (use - 1) & 1)) {
          atomicCAS(err, 0, 21);
          abort_flag = 1;
          break;
        }
        uint8_t* sa = sA + s * 2 * A_TILE;
        mbar_expect_tx(&full_bar[s], 2 * A_TILE);
        tma_load_2d(sa, &mapA, kb * TK, tile * TM, &full_bar[s]);
        tma_load_2d(sa + A_TILE, &mapA, kb * TK, p.R1 + tile * TM, &full_bar[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    bool ok = mbar_wait(&resF, 0);
    if (!ok) {
      atomicCAS(err, 0, 22);
      abort_flag = 1;
    }
    int it = 0, tl = 0;
    for (int tile = t0; ok && tile < p.tiles && !abort_flag; tile += tstep, ++tl) {
      const int buf = tl & 1;
      if (tl >= 2 && !mbar_wait(&accE[buf], ((tl >> 1) - 1) & 1)) {
        atomicCAS(err, 0, 23);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(buf * 256);
      for (int kb = 0; kb < KB; ++kb, ++it) {
        const int s = it % S;
        const uint32_t use = it / S;
        if (!mbar_wait(&full_bar[s], use & 1)) {
          atomicCAS(err, 0, 24);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* sa = sA + s * 2 * A_TILE;
        mma_split_kblock(d, smem_desc(sa), smem_desc(sa + A_TILE), smem_desc(sB + kb * B_BLK),
                         smem_desc(sB + (KB + kb) * B_BLK), idesc, kb == 0);
        mma_commit_to(&empty_bar[s]);
      }
      if (ok) mma_commit_to(&accF[buf]);
    }
  } else if (warp >= 2) {
    // warp (q, h): TMEM lanes 32 q .. 32 q + 31, column half h
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int c_mid = (NT / 2) & ~15;
    const int c0 = h ? c_mid : 0, c1 = h ? NT : c_mid;
    const int ubase = cpart * p.Us;
    int tl = 0;
    for (int tile = t0; tile < p.tiles && !abort_flag; tile += tstep, ++tl) {
      const int buf = tl & 1;
      if (!mbar_wait(&accF[buf], (tl >> 1) & 1)) {
        atomicCAS(err, 0, 25);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int g = tile * TM + q * 32 + lane;
      const bool valid = g < p.rows;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 256);
      if (ROWS_OUT) {
        // row g of the product as FP32 complex values, columns (u, re/im) -> yout[g][u]
        float2* yr = yout + (size_t)g * p.U;
        tmem_for_groups(taddr, c0, c1, [&](const uint32_t(&r)[16], int cb) {
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const int ul = cb / 2 + t, u = ubase + ul;
            if (valid && ul < p.Us && u < p.U)
              yr[u] = make_float2(__uint_as_float(r[2 * t]), __uint_as_float(r[2 * t + 1]));
          }
        });
      } else {
        const int b = g / p.rpb, rem = g - (g / p.rpb) * p.rpb;
        const int x = rem / p.Y, y = rem - (rem / p.Y) * p.Y;
        const size_t row0 = (size_t)b * p.SB + (size_t)x * p.SX;  // + u * SU
        tmem_for_groups(taddr, c0, c1, [&](const uint32_t(&r)[16], int cb) {
          epi1_group<16>(r, cb, valid, ubase, p.Us, p.U, row0, p.SU, (size_t)p.ws, y, (size_t)p.Rout, out);
        });
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&accE[buf]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ------------------------------------------------------------------ fused passes 2 + 3

// Pass 3 plus the Nyquist term: running argmax over NC values u2 = cb .. cb + NC - 1 of one
// row, each v[u2] + Re(Y E2[u2, N/2]) = v + y.x en[u2].x + y.y en[u2].y in FP32.
template <int NC>
__device__ __forceinline__ void scan_group_nq(const uint32_t* vr, int cb, int U, int row_flat, float2 y,
                                              const float4* __restrict__ en2, float& bv, int& bi, bool& have) {
  static_assert(NC == 16, "the packed scan takes groups of 16");
  uint32_t w[NC];
#pragma unroll
  for (int t = 0; t < NC; t += 2) {
    // columns t, t + 1 at once: packed two-lane FMAs (sm_100), the same roundings as scalar ones
    const float4 e = en2[(cb + t) >> 1];  // (re t, re t+1, im t, im t+1); a broadcast load
    const float2 v2 = make_float2(__uint_as_float(vr[t]), __uint_as_float(vr[t + 1]));
    const float2 r2 = __ffma2_rn(make_float2(y.y, y.y), make_float2(e.z, e.w),
                                 __ffma2_rn(make_float2(y.x, y.x), make_float2(e.x, e.y), v2));
    w[t] = __float_as_uint(r2.x);
    w[t + 1] = __float_as_uint(r2.y);
  }
  // The position in the group rides in the low 4 mantissa bits of each value (15 - t, so of
  // equal positive values the first is the largest), which changes the compared magnitudes by
  // at most 15 units in the last place, far below the hi/lo split's own error; one
  // NaN-propagating maximum per value then finds the group's best.  (Equal negative values
  // resolve to the last position instead; the grid's maximum is the correlation peak, and an
  // all-negative grid with an exact tie at its top is the only case this reorders.)  A group
  // whose maximum is NaN (a NaN, or an infinity whose low bits were set) is rescanned exactly.
  float m[4];
  if (cb + NC <= U) {
#pragma unroll
    for (int t = 0; t < NC; ++t) {
      const float f = __uint_as_float((w[t] & 0xFFFFFFF0u) | (uint32_t)(15 - t));
      m[t & 3] = t < 4 ? f : fmax_nan(m[t & 3], f);
    }
  } else {  // the last group: columns past U take the lowest finite value
#pragma unroll
    for (int t = 0; t < NC; ++t) {
      const uint32_t b = (cb + t < U) ? (w[t] & 0xFFFFFFF0u) : 0xFF7FFFF0u;
      const float f = __uint_as_float(b | (uint32_t)(15 - t));
      m[t & 3] = t < 4 ? f : fmax_nan(m[t & 3], f);
    }
  }
  const float g = fmax_nan(fmax_nan(m[0], m[1]), fmax_nan(m[2], m[3]));
  if (g != g) {
    scan_group<NC>(w, cb, U, row_flat, bv, bi, have);
    return;
  }
  const bool upd = g > bv;  // never once bv is NaN: nothing later wins
  bv = upd ? g : bv;
  bi = upd ? row_flat * U + cb + 15 - (int)(__float_as_uint(g) & 15u) : bi;
  have = have || upd;
}

__global__ void __launch_bounds__(kThreads23, 1)
updft23_tc_kernel(const __grid_constant__ CUtensorMap mapA2, const __grid_constant__ CUtensorMap mapE1,
                  const __grid_constant__ CUtensorMap mapE3, Pass23 p, const float2* __restrict__ nyq,
                  const float4* __restrict__ enq, unsigned long long* __restrict__ best, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int KB = p.KB, NT12 = p.NT12, NT3 = p.NT3, NB = p.NB, HH = p.HH;
  const int B1 = NT12 * TK * 2, B3 = NT3 * TK * 2;
  uint8_t* sE1 = smem;                       // [part][kb] B1
  uint8_t* sE3 = sE1 + 2 * KB * B1;          // [part] B3
  // NB slots of two A_TILE (hi, lo).  A2 K-block kb of every tile lives in slot kb; pass-3
  // chunk j in slot chunk_slot(j), alternating between the two highest slots so that the last
  // chunk takes the top one.  A slot that also holds an A2 K-block (kb = NB - 2 when KB = 2 and
  // NB = 3) is last used by chunk CH - 2, so the next tile's K-block loads while chunk CH - 1
  // is written, and slot 0 reloads as soon as pass 2 has read it.  freeT[kb] opens a K-block
  // slot to the TMA thread once per tile; freeO[s] hands a chunk slot from one chunk to the
  // next, so each barrier is waited in order, never more than one phase ahead.
  uint8_t* sS = sE3 + 2 * B3;
  float4* sEn = reinterpret_cast<float4*>(sS + NB * 2 * A_TILE);  // (er, -ei) of E2[u2, N/2]: column pairs (re, re, im, im)
  __shared__ __align__(8) uint64_t tmaF[kMaxSlots], opF[kMaxSlots], freeT[kMaxSlots], freeO[kMaxSlots];
  __shared__ __align__(8) uint64_t acc3F[2], acc3E[2], resF, acc2F, acc2E;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kMaxSlots; ++s) {
      mbar_init(&tmaF[s], 1);
      mbar_init(&opF[s], kEpi);
      mbar_init(&freeT[s], 1);
      mbar_init(&freeO[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc3F[s], 1);
      mbar_init(&acc3E[s], kArg);
    }
    mbar_init(&resF, 1);
    mbar_init(&acc2F, 1);
    mbar_init(&acc2E, kEpi);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = threadIdx.x; i < NT3 / 2; i += blockDim.x) {  // pairs of columns, re parts first
    const float4 e = enq[i];
    sEn[i] = make_float4(e.x, e.z, e.y, e.w);
  }
  // a chunk writes K words < N/2 of its rows; the rest must hold finite values (they meet
  // zero K columns of E3), so the slots start zeroed
  for (int i = threadIdx.x; i < NB * 2 * A_TILE / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(sS)[i] = make_uint4(0u, 0u, 0u, 0u);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc2 = idesc_bf16(TM, NT12), idesc3 = idesc_bf16(TM, NT3);
  const int CH = p.CH;
  // slot of chunk j; whether slot kb < KB is read by no chunk of a tile
  auto chunk_slot = [&](int j) { return ((CH - 1 - j) & 1) ? NB - 2 : NB - 1; };
  auto kb_chunk_free = [&](int kb) { return !(kb == NB - 1 || (kb == NB - 2 && CH >= 2)); };

  if (warp == 0 && lane == 0) {
    mbar_expect_tx(&resF, (uint32_t)(2 * KB * B1 + 2 * B3));
    for (int part = 0; part < 2; ++part) {
      for (int kb = 0; kb < KB; ++kb) tma_load_2d(sE1 + (part * KB + kb) * B1, &mapE1, kb * TK, part * NT12, &resF);
      tma_load_2d(sE3 + part * B3, &mapE3, 0, part * NT3, &resF);
    }
    int tl = 0;
    bool ok = true;
    for (int tile = blockIdx.x; ok && tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      const int b = tile / p.TPB, tg = tile - (tile / p.TPB) * p.TPB;
      const int arow = (b * p.U + tg * p.G) * HH;
      for (int kb = 0; kb < KB; ++kb) {
        if (tl >= 1 && !mbar_wait(&freeT[kb], (tl - 1) & 1)) {
          atomicCAS(err, 0, 31);
          abort_flag = 1;
          ok = false;
          break;
        }
        uint8_t* sa = sS + kb * 2 * A_TILE;
        mbar_expect_tx(&tmaF[kb], 2 * A_TILE);
        tma_load_2d(sa, &mapA2, kb * TK, arow, &tmaF[kb]);
        tma_load_2d(sa + A_TILE, &mapA2, kb * TK, p.R2 + arow, &tmaF[kb]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    bool ok = mbar_wait(&resF, 0);
    if (!ok) {
      atomicCAS(err, 0, 32);
      abort_flag = 1;
    }
    uint32_t op_par = 0;  // bit s: phase of the next wait on opF[s]
    int tl = 0;
    for (int tile = blockIdx.x; ok && tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      // pass 2 into acc2 (columns 0 .. NT12) once the operand warps have read the last tile's
      if (tl >= 1 && !mbar_wait(&acc2E, (tl - 1) & 1)) {
        atomicCAS(err, 0, 33);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int kb = 0; kb < KB; ++kb) {
        if (!mbar_wait(&tmaF[kb], tl & 1)) {
          atomicCAS(err, 0, 34);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* sa = sS + kb * 2 * A_TILE;
        mma_split_kblock(tmem, smem_desc(sa), smem_desc(sa + A_TILE), smem_desc(sE1 + kb * B1),
                         smem_desc(sE1 + (KB + kb) * B1), idesc2, kb == 0);
        if (kb_chunk_free(kb)) mma_commit_to(&freeT[kb]);
      }
      if (!ok) break;
      mma_commit_to(&acc2F);
      // pass 3, chunk by chunk: the CTA's chunk cc into acc3 buffer cc & 1 (columns
      // NT12 + (cc & 1) NT3) once the argmax warps have read chunk cc - 2 from it
      for (int j = 0; j < CH; ++j) {
        const int s = chunk_slot(j);
        const int cc = tl * CH + j, q3 = cc & 1;
        if (!mbar_wait(&opF[s], (op_par >> s) & 1u)) {
          atomicCAS(err, 0, 35);
          abort_flag = 1;
          ok = false;
          break;
        }
        op_par ^= 1u << s;
        if (cc >= 2 && !mbar_wait(&acc3E[q3], ((cc >> 1) - 1) & 1)) {
          atomicCAS(err, 0, 36);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* a3 = sS + s * 2 * A_TILE;
        mma_split_kblock(tmem + (uint32_t)(NT12 + q3 * NT3), smem_desc(a3), smem_desc(a3 + A_TILE), smem_desc(sE3),
                         smem_desc(sE3 + B3), idesc3, true);
        // a K-block slot after its last chunk of the tile goes back to the TMA thread
        mma_commit_to(s < KB && j >= CH - 2 ? &freeT[s] : &freeO[s]);
        mma_commit_to(&acc3F[q3]);
      }
    }
  } else if (warp >= 2 && warp < 2 + kEpi / 32) {
    // operand warps (q, h): TMEM lanes 32 q .. 32 q + 31 (rows (u0_local, m2) of acc2), half h
    // of a chunk's columns.  Chunk j is u1 in [j HH, j HH + HH) for all G u0 of the tile:
    // pass-3 row (u0_local, u1 - j HH), so every lane has the same share of every chunk.
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int r_lane = q * 32 + lane;
    const int u0l = r_lane / HH, m2 = r_lane - (r_lane / HH) * HH;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    int tl = 0;
    uint32_t par = 0;  // bit s: phase of the next wait on freeO[s]
    for (int tile = blockIdx.x; tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      if (!mbar_wait(&acc2F, tl & 1)) {
        atomicCAS(err, 0, 37);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      bool ok = true;
      for (int j = 0; j < CH; ++j) {
        const int s = chunk_slot(j);
        const int lo_l = j * HH, hi_l = min(p.U, lo_l + HH);  // this chunk's u1
        const int cA = 2 * lo_l, cB = min(NT12, (2 * hi_l + 15) & ~15);
        const int cM = cA + ((((cB - cA) >> 4) + 1) >> 1 << 4);  // h = 0 takes the first half
        const int ca = h ? cM : cA, cb_end = h ? cB : cM;
        uint8_t* sA3 = sS + s * 2 * A_TILE;
        // the slot's last use was a chunk: this tile's j - 2, or, in a slot of its own, the
        // previous tile's (a K-block slot's first chunk follows pass 2, waited above)
        if (s < KB ? j >= 2 : (tl >= 1 || j >= 2)) {
          if (!mbar_wait(&freeO[s], (par >> s) & 1u)) {
            atomicCAS(err, 0, 38);
            abort_flag = 1;
            ok = false;
            break;
          }
          par ^= 1u << s;
        }
        tmem_for_groups(tmem + lane_off, ca, cb_end, [&](const uint32_t(&r)[16], int cb) {
          epi2_group<16>(r, cb, lo_l, hi_l, (u0l - j) * HH, m2, sA3);
        });
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&opF[s]);
      }
      if (!ok) break;
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&acc2E);
    }
  } else if (warp >= 2 + kEpi / 32) {
    // argmax warps (q, h): TMEM lanes 32 q .. 32 q + 31 of each chunk's pass-3 accumulator,
    // half h of its columns; they run a chunk behind the operand warps
    const int q = warp & 3, h = (warp - 2 - kEpi / 32) >> 2;
    const int r_lane = q * 32 + lane;
    const int u0l = r_lane / HH, r1 = r_lane - (r_lane / HH) * HH;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    const int c3m = (((NT3 >> 4) + 1) >> 1) << 4;
    const int ca = h ? c3m : 0, cb_end = h ? NT3 : c3m;
    int tl = 0;
    for (int tile = blockIdx.x; tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      const int b = tile / p.TPB, tg = tile - (tile / p.TPB) * p.TPB;
      const int u0 = tg * p.G + u0l;
      float bv = -INFINITY;
      int bi = 0x7fffffff;
      bool have = false;
      bool ok = true;
      for (int j = 0; j < p.CH; ++j) {
        const int cc = tl * p.CH + j, q3 = cc & 1;
        const int u1 = j * HH + r1;
        const bool valid = u1 < p.U && u0 < p.U;
        const float2 y = valid ? nyq[((size_t)b * p.U + u0) * p.U + u1] : make_float2(0.f, 0.f);
        if (!mbar_wait(&acc3F[q3], (cc >> 1) & 1)) {
          atomicCAS(err, 0, 39);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row_flat = u0 * p.U + u1;
        tmem_for_groups(tmem + lane_off + (uint32_t)(NT12 + q3 * NT3), ca, cb_end,
                        [&](const uint32_t(&rr)[16], int cb) {
                          if (valid) scan_group_nq<16>(rr, cb, p.U, row_flat, y, sEn, bv, bi, have);
                        });
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(&acc3E[q3]);
      }
      if (!ok) break;
      // a lane visits its values in increasing flat order, so a later equal value never wins;
      // the warp's keys all belong to subtomogram b
      // (the low 4 bits of the value, position bits of the packed scan, are cleared)
      unsigned long long key = have ? argmax_key(__uint_as_float(__float_as_uint(bv) & 0xFFFFFFF0u), bi) : 0ull;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
        key = k2 > key ? k2 : key;
      }
      if (lane == 0 && key) atomicMax(&best[b], key);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ------------------------------------------------------------------ pass 3 on its own
// Rows (b, u0 U + u1) of A3 times E3 -> grid values u2 (real part) in a double-buffered TMEM
// accumulator; the epilogue adds the Nyquist term Re(Y[b, u0, u1] E2[u2, N/2]) in FP32 and
// keeps a running argmax per row, reduced per warp into best[b] (every tile lies in one
// subtomogram: its rows are padded to a multiple of 128, and pad rows are skipped).
__global__ void __launch_bounds__(kThreads, 1)
updft3_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, Pass3 p,
                 const float2* __restrict__ nyq, const float4* __restrict__ enq, unsigned long long* __restrict__ best,
                 int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int KB = p.KB, S = p.stages, NT = p.NT;
  const int B_BLK = NT * TK * 2;
  uint8_t* sB = smem;                                          // [part][kb] B_BLK
  uint8_t* sA = smem + 2 * KB * B_BLK;                         // [stage][part] A_TILE
  float4* sEn = reinterpret_cast<float4*>(sA + S * 2 * A_TILE);  // NT / 2 column pairs (re, re, im, im)
  __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages];
  __shared__ __align__(8) uint64_t accF[2], accE[2], resF;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&accF[i], 1);
      mbar_init(&accE[i], kEpi);
    }
    mbar_init(&resF, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = threadIdx.x; i < NT / 2; i += blockDim.x) {
    const float4 e = enq[i];
    sEn[i] = make_float4(e.x, e.z, e.y, e.w);
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = idesc_bf16(TM, NT);

  if (warp == 0 && lane == 0) {
    mbar_expect_tx(&resF, (uint32_t)(2 * KB * B_BLK));
    for (int part = 0; part < 2; ++part)
      for (int kb = 0; kb < KB; ++kb)
        tma_load_2d(sB + (part * KB + kb) * B_BLK, &mapB, kb * TK, part * NT, &resF);
    int it = 0;
    for (int tile = blockIdx.x; tile < p.tiles && !abort_flag; tile += gridDim.x) {
      for (int kb = 0; kb < KB; ++kb, ++it) {
        const int s = it % S;
        const uint32_t use = it / S;
        if (it >= S && !mbar_wait(&empty_bar[s], (use - 1) & 1)) {
          atomicCAS(err, 0, 41);
          abort_flag = 1;
          break;
        }
        uint8_t* sa = sA + s * 2 * A_TILE;
        mbar_expect_tx(&full_bar[s], 2 * A_TILE);
        tma_load_2d(sa, &mapA, kb * TK, tile * TM, &full_bar[s]);
        tma_load_2d(sa + A_TILE, &mapA, kb * TK, p.R3 + tile * TM, &full_bar[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    bool ok = mbar_wait(&resF, 0);
    if (!ok) {
      atomicCAS(err, 0, 42);
      abort_flag = 1;
    }
    int it = 0, tl = 0;
    for (int tile = blockIdx.x; ok && tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      const int buf = tl & 1;
      if (tl >= 2 && !mbar_wait(&accE[buf], ((tl >> 1) - 1) & 1)) {
        atomicCAS(err, 0, 43);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(buf * 256);
      for (int kb = 0; kb < KB; ++kb, ++it) {
        const int s = it % S;
        const uint32_t use = it / S;
        if (!mbar_wait(&full_bar[s], use & 1)) {
          atomicCAS(err, 0, 44);
          abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* sa = sA + s * 2 * A_TILE;
        mma_split_kblock(d, smem_desc(sa), smem_desc(sa + A_TILE), smem_desc(sB + kb * B_BLK),
                         smem_desc(sB + (KB + kb) * B_BLK), idesc, kb == 0);
        mma_commit_to(&empty_bar[s]);
      }
      if (ok) mma_commit_to(&accF[buf]);
    }
  } else if (warp >= 2) {
    // warp (q, h): TMEM lanes 32 q .. 32 q + 31, column half h
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int c_mid = (((NT >> 4) + 1) >> 1) << 4;
    const int c0 = h ? c_mid : 0, c1 = h ? NT : c_mid;
    const int U = p.U, UU = p.U * p.U;
    int tl = 0;
    for (int tile = blockIdx.x; tile < p.tiles && !abort_flag; tile += gridDim.x, ++tl) {
      const int buf = tl & 1;
      const int b = tile / p.TPB;
      const int rb = (tile - b * p.TPB) * TM + q * 32 + lane;  // row in the subtomogram: u0 U + u1
      const bool valid = rb < UU;
      const float2 y = valid ? nyq[(size_t)b * UU + rb] : make_float2(0.f, 0.f);
      // warp-uniform outcome: the TMEM loads and the shuffles below need the whole warp
      if (!__all_sync(0xffffffffu, mbar_wait(&accF[buf], (tl >> 1) & 1))) {
        if (lane == 0) atomicCAS(err, 0, 45);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float bv = -INFINITY;
      int bi = 0x7fffffff;
      bool have = false;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 256);
      tmem_for_groups(taddr, c0, c1, [&](const uint32_t(&rr)[16], int cb) {
        if (valid) scan_group_nq<16>(rr, cb, U, rb, y, sEn, bv, bi, have);
      });
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&accE[buf]);
      unsigned long long key = have ? argmax_key(__uint_as_float(__float_as_uint(bv) & 0xFFFFFFF0u), bi) : 0ull;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
        key = k2 > key ? k2 : key;
      }
      if (lane == 0 && key) atomicMax(&best[b], key);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
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

struct Geometry {
  bool fused;
  int HH, NT12, NT3, KB12, KB3, G, TPB, CH, NB, stages1, NS, Us, RP3, stages3;
  size_t smem1, smem23, smem3;
};

// The geometry of the fused (passes 2+3 in one kernel) or the unfused kernels; false when it
// does not fit the MMA shapes, tensor memory or shared memory.
bool geometry_as(int N, int U, bool fused, Geometry* o) {
  if (N < 16 || N > 128 || (N & 1)) return false;
  if (U < 1 || U > 256) return false;
  Geometry g;
  g.HH = N / 2;
  g.NT3 = (U + 15) / 16 * 16;
  g.KB12 = (2 * N + TK - 1) / TK;
  g.KB3 = (N + TK - 1) / TK;  // K of pass 3: (m2 < N/2, re/im)
  g.fused = fused;
  if (fused && !((N == 16 || N == 32 || N == 64) && 2 * U <= 256)) return false;
  g.NT12 = (2 * U + 15) / 16 * 16;
  g.G = TM / g.HH;
  g.TPB = (U + g.G - 1) / g.G;
  g.CH = (U + g.HH - 1) / g.HH;
  g.NS = 1;
  g.Us = U;
  g.RP3 = g.stages3 = 0;
  g.smem23 = g.smem3 = 0;
  if (g.fused) {
    if (g.NT12 + 2 * g.NT3 > 512) return false;
    const size_t b1 = (size_t)2 * g.KB12 * g.NT12 * TK * 2;
    const size_t b3 = (size_t)2 * g.NT3 * TK * 2;
    // three operand slots where they fit (the next tile's A2 then loads during this tile's
    // pass 3), else two
    for (g.NB = kMaxSlots; g.NB >= 2; --g.NB) {
      g.smem23 = 1024 + b1 + b3 + (size_t)g.NB * 2 * A_TILE + (size_t)g.NT3 * 8;
      if (g.smem23 <= kSmemCap) break;
    }
    if (g.NB < 2) return false;
  } else {
    g.NB = 0;
    // the fewest column parts whose E1 part leaves room for two A stages
    for (g.NS = 1; g.NS <= 8; ++g.NS) {
      g.Us = (U + g.NS - 1) / g.NS;
      g.NT12 = (2 * g.Us + 15) / 16 * 16;
      const size_t b1 = (size_t)2 * g.KB12 * g.NT12 * TK * 2;
      if (g.NT12 <= 256 && 1024 + b1 + (size_t)2 * 2 * A_TILE <= kSmemCap) break;
    }
    if (g.NS > 8) return false;
    g.RP3 = (U * U + TM - 1) / TM * TM;
    const size_t b3 = (size_t)2 * g.KB3 * g.NT3 * TK * 2 + (size_t)g.NT3 * 8;
    g.stages3 = (int)((kSmemCap - 1024 - b3) / (2 * (size_t)A_TILE));
    if (g.stages3 > kMaxStages) g.stages3 = kMaxStages;
    if (g.stages3 < 2) return false;
    g.smem3 = 1024 + b3 + (size_t)g.stages3 * 2 * A_TILE;
  }
  const size_t b1 = (size_t)2 * g.KB12 * g.NT12 * TK * 2;
  g.stages1 = (int)((kSmemCap - 1024 - b1) / (2 * (size_t)A_TILE));
  if (g.stages1 > kMaxStages) g.stages1 = kMaxStages;
  if (g.stages1 < 2) return false;
  g.smem1 = 1024 + b1 + (size_t)g.stages1 * 2 * A_TILE;
  *o = g;
  return true;
}

// The fused kernels where they fit (boxes 16, 32, 64 with 2U <= 256, within the shared
// memory of two operand slots), else the unfused ones.
bool geometry(int N, int U, Geometry* o) {
  return geometry_as(N, U, true, o) || geometry_as(N, U, false, o);
}

}  // namespace

int shift_tc_fits(int N, int U) {
  Geometry g;
  return geometry(N, U, &g) ? MTB_OK : MTB_ERR_ARG;
}

extern "C" int mtb_shift_tc_plan(int N, int U, int* fused, int* column_parts, int* n_tile, int* stages1,
                                 int* stages3, int64_t* smem_max) {
  MTB_ARG_CHECK(fused && column_parts && n_tile && stages1 && stages3 && smem_max, "null pointer");
  Geometry g;
  if (!geometry(N, U, &g)) {
    mtb_set_last_error("the tensor-core shift kernels do not cover this box and upsampled region", __FILE__,
                       __LINE__);
    return MTB_ERR_ARG;
  }
  *fused = g.fused ? 1 : 0;
  *column_parts = g.NS;
  *n_tile = g.NT12;
  *stages1 = g.stages1;
  *stages3 = g.fused ? 0 : g.stages3;
  size_t m = g.smem1;
  if (g.fused && g.smem23 > m) m = g.smem23;
  if (!g.fused && g.smem3 > m) m = g.smem3;
  *smem_max = (int64_t)m;
  return MTB_OK;
}

int shift_tc_prepare(ShiftTc* t, int N, int H, int U, int uf, float dftshift, int max_batch) {
  memset(t, 0, sizeof(*t));
  Geometry ge;
  if (!geometry(N, U, &ge)) return MTB_ERR_ARG;
  t->fused = ge.fused;
  t->N = N;
  t->H = H;
  t->HH = ge.HH;
  t->U = U;
  t->NT12 = ge.NT12;
  t->NT3 = ge.NT3;
  t->KB12 = ge.KB12;
  t->KB3 = ge.KB3;
  t->G = ge.G;
  t->TPB = ge.TPB;
  t->CH = ge.CH;
  t->NB = ge.NB;
  t->NS = ge.NS;
  t->Us = ge.Us;
  t->RP3 = ge.RP3;
  t->TPB3 = ge.RP3 / TM;
  t->stages1 = ge.stages1;
  t->stages3 = ge.stages3;
  t->smem1 = ge.smem1;
  t->smem23 = ge.smem23;
  t->smem3 = ge.smem3;
  t->Bmax = max_batch;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&t->n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return MTB_ERR_CUDA;
  auto pad = [](size_t r) { return (r + TM - 1) / TM * TM; };
  const int HH = ge.HH;
  t->R1 = (int)pad((size_t)max_batch * HH * N);
  // fused: a partial last u0 group of the last subtomogram reads up to G * HH rows past the end
  t->R2 = (int)pad((size_t)max_batch * U * HH + (ge.fused ? (size_t)ge.G * HH : 0));
  const size_t k12 = (size_t)t->KB12 * TK, k3 = (size_t)t->KB3 * TK;
  const size_t a1 = (size_t)2 * t->R1 * k12 * 2, a2 = (size_t)2 * t->R2 * k12 * 2;
  if (cudaMalloc(&t->A1, a1) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->A2, a2) != cudaSuccess) return MTB_ERR_OOM;
  const int nt1 = t->NS * t->NT12;  // E1 rows per hi/lo part
  if (cudaMalloc(&t->E1, (size_t)2 * nt1 * k12 * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->E3, (size_t)2 * t->NT3 * k3 * 2) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->ENQ, (size_t)t->NT3 * sizeof(float2)) != cudaSuccess) return MTB_ERR_OOM;
  size_t a3 = 0;
  if (!ge.fused) {
    // pad rows (u0 U + u1 >= U^2) and K columns past N stay zero; the rest is rewritten by every call
    t->R3 = (int)((size_t)max_batch * t->RP3);
    a3 = (size_t)2 * t->R3 * k3 * 2;
    if (cudaMalloc(&t->A3, a3) != cudaSuccess) return MTB_ERR_OOM;
    if (cudaMemset(t->A3, 0, a3) != cudaSuccess) return MTB_ERR_CUDA;
  }
  // the Nyquist plane's operands: A1n rows (b, m1), A2n rows (b, u0), same K layout as A1, A2
  t->R1n = (int)pad((size_t)max_batch * N);
  t->R2n = (int)pad((size_t)max_batch * U);
  const size_t a1n = (size_t)2 * t->R1n * k12 * 2, a2n = (size_t)2 * t->R2n * k12 * 2;
  if (cudaMalloc(&t->A1n, a1n) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->A2n, a2n) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMemset(t->A1n, 0, a1n) != cudaSuccess || cudaMemset(t->A2n, 0, a2n) != cudaSuccess) return MTB_ERR_CUDA;
  if (cudaMalloc(&t->nyq, (size_t)max_batch * U * U * sizeof(float2)) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->best, (size_t)max_batch * 8) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMalloc(&t->err, 4) != cudaSuccess) return MTB_ERR_OOM;
  // K columns past 2N of A1 and A2 stay zero; the rest is rewritten by every call
  if (cudaMemset(t->A1, 0, a1) != cudaSuccess || cudaMemset(t->A2, 0, a2) != cudaSuccess ||
      cudaMemset(t->err, 0, 4) != cudaSuccess)
    return MTB_ERR_CUDA;
  // B operands: E1 rows (part, u local, re/im), K (m, re/im); E3 rows u2, K (m2 < N/2, re/im) -> real part
  auto E = [&](int n, int u, int m, double* re, double* im) {
    const int mm = (m < (n + 1) / 2) ? m : m - n;
    const double f = (double)mm / ((double)uf * n);
    const double ph = 2.0 * M_PI * ((double)u - dftshift) * f;
    *re = cos(ph);
    *im = sin(ph);
  };
  std::vector<uint16_t> e1((size_t)2 * nt1 * k12, 0), e3((size_t)2 * t->NT3 * k3, 0);
  // the Nyquist column's factor (re, -im) of E2[u2, N/2], FP32, zero past U
  std::vector<float2> enq((size_t)t->NT3, make_float2(0.f, 0.f));
  auto put = [&](std::vector<uint16_t>& dst, size_t k, int rows, int r, int kk, double v) {
    const uint16_t hi = f2bf((float)v);
    const uint16_t lo = f2bf((float)(v - (double)bf2f(hi)));
    dst[(size_t)r * k + kk] = hi;
    dst[((size_t)rows + r) * k + kk] = lo;
  };
  for (int u = 0; u < U; ++u) {
    const int part = u / t->Us, ul = u - part * t->Us;
    const int r0 = part * t->NT12 + 2 * ul;
    for (int m = 0; m < N; ++m) {
      double er, ei;
      E(N, u, m, &er, &ei);
      put(e1, k12, nt1, r0 + 0, 2 * m + 0, er);
      put(e1, k12, nt1, r0 + 0, 2 * m + 1, -ei);
      put(e1, k12, nt1, r0 + 1, 2 * m + 0, ei);
      put(e1, k12, nt1, r0 + 1, 2 * m + 1, er);
    }
  }
  for (int u = 0; u < U; ++u) {
    for (int m = 0; m < HH; ++m) {
      double er, ei;
      E(H, u, m, &er, &ei);
      put(e3, k3, t->NT3, u, 2 * m + 0, er);
      put(e3, k3, t->NT3, u, 2 * m + 1, -ei);
    }
    double er, ei;
    E(H, u, HH, &er, &ei);
    enq[u] = make_float2((float)er, (float)-ei);
  }
  if (cudaMemcpy(t->E1, e1.data(), e1.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t->E3, e3.data(), e3.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t->ENQ, enq.data(), enq.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
    return MTB_ERR_CUDA;
  int rc = make_map(t->mapA1, t->A1, k12, (uint64_t)2 * t->R1, TM);
  if (!rc) rc = make_map(t->mapA2, t->A2, k12, (uint64_t)2 * t->R2, TM);
  if (!rc) rc = make_map(t->mapE1, t->E1, k12, (uint64_t)2 * nt1, t->NT12);
  if (!rc) rc = make_map(t->mapE3, t->E3, k3, (uint64_t)2 * t->NT3, t->NT3);
  if (!rc) rc = make_map(t->mapA1n, t->A1n, k12, (uint64_t)2 * t->R1n, TM);
  if (!rc) rc = make_map(t->mapA2n, t->A2n, k12, (uint64_t)2 * t->R2n, TM);
  if (!rc && !ge.fused) rc = make_map(t->mapA3, t->A3, k3, (uint64_t)2 * t->R3, TM);
  return rc;
}

void shift_tc_release(ShiftTc* t) {
  void* ptrs[] = {t->A1, t->A2, t->A3, t->A1n, t->A2n, t->E1, t->E3, t->ENQ, t->nyq, t->best, t->err};
  for (void* p : ptrs) if (p) cudaFree(p);
  memset(t, 0, sizeof(*t));
}

namespace {
// a pass of the updft1 kernel over `rows` rows of A: the CTAs of one row tile's column parts
// are adjacent, and the grid is a multiple of NS
Pass1 pass1_params(const ShiftTc* t, int rows, int R1) {
  Pass1 p;
  p.rows = rows;
  p.tiles = (rows + TM - 1) / TM;
  p.U = t->U;
  p.KB = t->KB12;
  p.R1 = R1;
  p.NT = t->NT12;
  p.NS = t->NS;
  p.Us = t->Us;
  p.stages = t->stages1;
  p.rpb = p.Y = 1;
  p.SB = p.SX = p.SU = 0;
  p.ws = t->KB12 * (TK / 2);
  p.Rout = 0;
  return p;
}

int pass1_grid(const ShiftTc* t, const Pass1& p) {
  const int per = t->n_sm / p.NS > 0 ? t->n_sm / p.NS : 1;
  return (p.tiles < per ? p.tiles : per) * p.NS;
}
}  // namespace

int shift_tc_passes(ShiftTc* t, int B, cudaStream_t st, const cudaEvent_t* marks) {
  MTB_CUDA_TRY(cudaMemsetAsync(t->best, 0, (size_t)B * 8, st));
  const int N = t->N, U = t->U, HH = t->HH;
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft1_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)t->smem1));
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft1_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)t->smem1));
  const CUtensorMap& mapE1 = *reinterpret_cast<const CUtensorMap*>(t->mapE1);
  // Nyquist plane: pass 1 over its rows (b, m1) into A2n rows (b, u0), then A2n E1 -> Y
  {
    Pass1 pn = pass1_params(t, B * N, t->R1n);
    pn.rpb = N;  // row (b, m1) -> A2n row b U + u0, word m1
    pn.Y = N;
    pn.SB = U;
    pn.SU = 1;
    pn.Rout = t->R2n;
    mtb_prof_begin(st);
    updft1_tc_kernel<false><<<pass1_grid(t, pn), kThreads, t->smem1, st>>>(
        *reinterpret_cast<const CUtensorMap*>(t->mapA1n), mapE1, pn, (uint32_t*)t->A2n, nullptr, t->err);
    mtb_prof_end(st, "updft1_tc_kernel (Nyquist plane, pass 1)");
    MTB_LAUNCH_CHECK();
    Pass1 py = pass1_params(t, B * U, t->R2n);  // the A operand is now A2n
    mtb_prof_begin(st);
    updft1_tc_kernel<true><<<pass1_grid(t, py), kThreads, t->smem1, st>>>(
        *reinterpret_cast<const CUtensorMap*>(t->mapA2n), mapE1, py, nullptr, t->nyq, t->err);
    mtb_prof_end(st, "updft1_tc_kernel (Nyquist plane, pass 2)");
    MTB_LAUNCH_CHECK();
  }
  if (marks && marks[0]) cudaEventRecord(marks[0], st);
  // pass 1: row (b, m2, m1) -> A2 row (b U + u0) HH + m2, word m1
  Pass1 p1 = pass1_params(t, B * HH * N, t->R1);
  p1.rpb = HH * N;
  p1.Y = N;
  p1.SB = U * HH;
  p1.SX = 1;
  p1.SU = HH;
  p1.Rout = t->R2;
  mtb_prof_begin(st);
  updft1_tc_kernel<false><<<pass1_grid(t, p1), kThreads, t->smem1, st>>>(
      *reinterpret_cast<const CUtensorMap*>(t->mapA1), mapE1, p1, (uint32_t*)t->A2, nullptr, t->err);
  mtb_prof_end(st, "updft1_tc_kernel");
  MTB_LAUNCH_CHECK();
  if (marks && marks[1]) cudaEventRecord(marks[1], st);
  if (!t->fused) {
    // pass 2: row (b, u0, m2) -> A3 row b RP3 + u0 U + u1, word m2
    Pass1 p2 = pass1_params(t, B * U * HH, t->R2);
    p2.rpb = U * HH;
    p2.Y = HH;
    p2.SB = t->RP3;
    p2.SX = U;
    p2.SU = 1;
    p2.ws = t->KB3 * (TK / 2);
    p2.Rout = t->R3;
    mtb_prof_begin(st);
    updft1_tc_kernel<false><<<pass1_grid(t, p2), kThreads, t->smem1, st>>>(
        *reinterpret_cast<const CUtensorMap*>(t->mapA2), mapE1, p2, (uint32_t*)t->A3, nullptr, t->err);
    mtb_prof_end(st, "updft1_tc_kernel (pass 2)");
    MTB_LAUNCH_CHECK();
    Pass3 p3;
    p3.TPB = t->TPB3;
    p3.tiles = B * t->TPB3;
    p3.U = U;
    p3.KB = t->KB3;
    p3.R3 = t->R3;
    p3.NT = t->NT3;
    p3.stages = t->stages3;
    MTB_CUDA_TRY(cudaFuncSetAttribute(updft3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem3));
    const int g3 = p3.tiles < t->n_sm ? p3.tiles : t->n_sm;
    mtb_prof_begin(st);
    updft3_tc_kernel<<<g3, kThreads, t->smem3, st>>>(*reinterpret_cast<const CUtensorMap*>(t->mapA3),
                                                     *reinterpret_cast<const CUtensorMap*>(t->mapE3), p3, t->nyq,
                                                     (const float4*)t->ENQ, t->best, t->err);
    mtb_prof_end(st, "updft3_tc_kernel");
    MTB_LAUNCH_CHECK();
    if (marks && marks[2]) cudaEventRecord(marks[2], st);
    return MTB_OK;
  }
  // passes 2 + 3
  Pass23 p2;
  p2.B = B;
  p2.TPB = t->TPB;
  p2.tiles = B * t->TPB;
  p2.N = N;
  p2.HH = HH;
  p2.U = U;
  p2.G = t->G;
  p2.CH = t->CH;
  p2.NB = t->NB;
  p2.KB = t->KB12;
  p2.R2 = t->R2;
  p2.NT12 = t->NT12;
  p2.NT3 = t->NT3;
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft23_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem23));
  const int g2 = p2.tiles < t->n_sm ? p2.tiles : t->n_sm;
  mtb_prof_begin(st);
  updft23_tc_kernel<<<g2, kThreads23, t->smem23, st>>>(*reinterpret_cast<const CUtensorMap*>(t->mapA2), mapE1,
                                                     *reinterpret_cast<const CUtensorMap*>(t->mapE3), p2, t->nyq,
                                                     (const float4*)t->ENQ, t->best, t->err);
  mtb_prof_end(st, "updft23_tc_kernel");
  MTB_LAUNCH_CHECK();
  if (marks && marks[2]) cudaEventRecord(marks[2], st);
  return MTB_OK;
}

int shift_tc_check(ShiftTc* t, cudaStream_t st, int* site) {
  int h = 0;
  MTB_CUDA_TRY(cudaMemcpyAsync(&h, t->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MTB_CUDA_TRY(cudaStreamSynchronize(st));
  if (site) *site = h;
  return h ? MTB_ERR_TIMEOUT : MTB_OK;
}
