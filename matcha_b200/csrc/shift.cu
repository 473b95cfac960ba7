// RELION-style FFT shift match on sm_100a.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   estimate_shift_like_relion   src/matcha/core/ShiftMatcher.py:619-674
//   rotate_complex_volume        :491-537   (trilinear, align_corners=True, zero padding)
//   extract_shifted_patch_batch  :558-616   (set_coords_to_zero=True, normalize=False)
//   apply_cosine_mask            :540-555   masks: src/matcha/utils/setup_utils.py:239-270
//   compute_shift (local)        :94-282    with _upsampled_dft :46-91
//
// Design (B200): per subtomogram the pipeline is
//   xy      patch sampled from two input planes staged in shared memory, zero planes,
//           roll, 1/N^3, the real FFT along the last axis and the FFT along the middle
//           axis in one pass (one CTA per (b, plane)); the background fill enters linearly
//           (see patch_fft_xy_kernel), its weighted sum is accumulated on the way
//   z       background fill term, FFT along the first axis, fused with the rotated,
//           ifftshifted, masked Fourier reference (sampled on the fly), the product
//           conj(S) T and both norms
//   updft1  first pass of the local upsampled DFT (contract the first axis)
//   updft23 second and third passes (middle axis, then the half axis, real part only)
//           with a fused argmax: the U^3 refined correlation never reaches memory.
// Contracting the half axis (N/2+1) last needs 51M instead of 87M complex MACs per
// subtomogram at N=64, U=88; the separable sum is the same.
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <vector>
#include <cuda_bf16.h>
#include "common.cuh"
#include "shift_tc.cuh"

namespace {

constexpr int kT = 256;

struct ShiftGeom {
  int N, H, U, h;        // box, half width N/2+1, upsampled region, N/2
  float inv_n3;          // rfftn(norm="forward")
  int r2_inner, r2_outer;// cosine band: r2 >= r2_inner (not inner), r2 > r2_outer (outer)
  float rp, width;       // raised cosine: 0.5 + 0.5 cos(pi (rp - r) / width)
  float wsum;            // number of outer voxels + sum of raised cosine weights
  int mask_r2;           // mask_full: kp^2 + ip^2 + jp^2 <= (N/2)^2
  float dftshift;        // floor(U / 2)
  float uf;
};

__device__ __forceinline__ float2 trilinear_c(const float2* __restrict__ v, int N, float z, float y, float x) {
  const float z0 = floorf(z), y0 = floorf(y), x0 = floorf(x);
  const int iz = (int)z0, iy = (int)y0, ix = (int)x0;
  const float fz = z - z0, fy = y - y0, fx = x - x0;
  float ar = 0.f, ai = 0.f;
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const int zz = iz + dz, yy = iy + dy, xx = ix + dx;
        if (zz < 0 || zz >= N || yy < 0 || yy >= N || xx < 0 || xx >= N) continue;
        const float w = (dz ? fz : 1.f - fz) * (dy ? fy : 1.f - fy) * (dx ? fx : 1.f - fx);
        const float2 q = __ldg(&v[((int64_t)zz * N + yy) * N + xx]);
        ar += w * q.x;
        ai += w * q.y;
      }
  return make_float2(ar, ai);
}

// Corner quads of the Fourier reference for the gathers of the box-64 path: entry
// (zi, yi, xi), 0 <= zi <= N + 1, 0 <= yi, xi <= N, holds the four values at z = zi - 1,
// y = yi - 1 + {0, 1}, x = xi - 1 + {0, 1} (zero outside the box), so one trilinear sample is
// two aligned 32-byte entries.
__global__ void ref_quad_kernel(const float2* __restrict__ ref, int N, float4* __restrict__ q) {
  const int n1 = N + 1;
  const int64_t n = (int64_t)(N + 2) * n1 * n1;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int xi = (int)(t % n1), yi = (int)((t / n1) % n1), zi = (int)(t / ((int64_t)n1 * n1));
    const int z = zi - 1;
    float2 c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int y = yi - 1 + (k >> 1), x = xi - 1 + (k & 1);
      c[k] = (z >= 0 && z < N && y >= 0 && y < N && x >= 0 && x < N) ? ref[((int64_t)z * N + y) * N + x]
                                                                      : make_float2(0.f, 0.f);
    }
    q[2 * t] = make_float4(c[0].x, c[0].y, c[1].x, c[1].y);
    q[2 * t + 1] = make_float4(c[2].x, c[2].y, c[3].x, c[3].y);
  }
}

// One 32-byte corner quad in a single 256-bit load (the quads are 32-byte aligned): half the
// load instructions, and each sector is looked up once instead of twice.
__device__ __forceinline__ void ldg_quad(const float4* __restrict__ p, float4& lo, float4& hi) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z), "=f"(hi.w)
      : "l"(p));
}

// trilinear_c from the corner quads (same weights and summation order).
__device__ __forceinline__ float2 trilinear_quad(const float4* __restrict__ q, int N, float z, float y, float x) {
  const float z0 = floorf(z), y0 = floorf(y), x0 = floorf(x);
  const int iz = (int)z0, iy = (int)y0, ix = (int)x0;
  const float fz = z - z0, fy = y - y0, fx = x - x0;
  const bool in = iz >= -1 && iz < N && iy >= -1 && iy < N && ix >= -1 && ix < N;
  const int n1 = N + 1;
  const int64_t e0 = in ? ((int64_t)(iz + 1) * n1 + (iy + 1)) * n1 + (ix + 1) : 0;
  const int64_t e1 = e0 + (int64_t)n1 * n1;
  float4 a0, a1, b0, b1;
  ldg_quad(q + 2 * e0, a0, a1);
  ldg_quad(q + 2 * e1, b0, b1);
  const float2 v[8] = {make_float2(a0.x, a0.y), make_float2(a0.z, a0.w), make_float2(a1.x, a1.y),
                       make_float2(a1.z, a1.w), make_float2(b0.x, b0.y), make_float2(b0.z, b0.w),
                       make_float2(b1.x, b1.y), make_float2(b1.z, b1.w)};
  float ar = 0.f, ai = 0.f;
  if (in) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const float w = (dz ? fz : 1.f - fz) * (dy ? fy : 1.f - fy) * (dx ? fx : 1.f - fx);
      ar += w * v[c].x;
      ai += w * v[c].y;
    }
  }
  return make_float2(ar, ai);
}

// Per-subtomogram shift parameters: f = flip(shift_zyx) and the zeroed planes.
struct PatchShift {
  float f[3];
  int zp[3];
};

__device__ __forceinline__ PatchShift patch_shift(const float* __restrict__ shift_zyx, int b, int N) {
  PatchShift p;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float s = shift_zyx[b * 3 + (2 - d)];
    p.f[d] = s;
    const float a = fabsf(s);
    const float fl = floorf(a);
    if (a - fl > 0.f) {
      p.zp[d] = (s < 0.f) ? (int)fl : N - (int)ceilf(a);
    } else {
      p.zp[d] = -1;
    }
  }
  return p;
}

__device__ __forceinline__ float block_sum(float v, float* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

// ------------------------------------------------------------------ radix-2 FFT in shared memory
__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

template <int N>
__device__ __forceinline__ int brev(int k) {
  constexpr int kShift = 32 - ilog2c(N);
  return (int)(__brev((unsigned)k) >> kShift);
}

__device__ void load_twiddles(float2* tw, int L, int count) {
  for (int k = threadIdx.x; k < count; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * k / L, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}


// Boxes that are not powers of two (48, 80, 96) take the same kernels with the radix-2 FFTs
// replaced by direct DFTs (O(N^2) per line, natural-order output) and the index rolls done by
// comparison instead of a mask.
template <int N>
__host__ __device__ constexpr bool is_pow2() {
  return (N & (N - 1)) == 0;
}

template <int N>
__device__ __forceinline__ int wrap_n(int x) {  // x in [0, 2N) -> x mod N
  if constexpr (is_pow2<N>()) return x & (N - 1);
  return x >= N ? x - N : x;
}

// Twiddles a kernel loads: N/2 for the radix-2 FFT, N for the direct DFT.
template <int N>
__host__ __device__ constexpr int n_twiddles() {
  return is_pow2<N>() ? N / 2 : N;
}

// In-place decimation-in-frequency forward FFT (e^{-2 pi i k n / N}) of `lines` sequences,
// element t of line q at buf[q * ls + t * es]; the output of line q is left in bit-reversed
// order (frequency k at position brev<N>(k)).  tw[k] = e^{-2 pi i k / N}, k < N/2.  Ends
// with a barrier.
template <int N>
__device__ __forceinline__ void fft_dif(float2* buf, int lines, int ls, int es, const float2* __restrict__ tw) {
  constexpr int HALF = N / 2;
#pragma unroll
  for (int span = HALF; span >= 1; span >>= 1) {
    const int tstride = HALF / span;
    for (int e = threadIdx.x; e < lines * HALF; e += blockDim.x) {
      const int q = e / HALF, t = e % HALF;
      const int pos = t & (span - 1);
      const int i0 = 2 * t - pos, i1 = i0 + span;
      float2* p0 = buf + q * ls + i0 * es;
      float2* p1 = buf + q * ls + i1 * es;
      const float2 u = *p0, c = *p1;
      *p0 = make_float2(u.x + c.x, u.y + c.y);
      *p1 = cmul(make_float2(u.x - c.x, u.y - c.y), tw[pos * tstride]);
    }
    __syncthreads();
  }
}

// Position of frequency k in a transformed line: bit-reversed after fft_dif, natural after
// the direct DFT.
template <int N>
__device__ __forceinline__ int fpos(int k) {
  if constexpr (is_pow2<N>()) return brev<N>(k);
  return k;
}

// Forward transform of `lines` sequences in place (layout as fft_dif).  Powers of two: fft_dif
// (scratch unused); otherwise a direct DFT through scratch (lines x N elements at the same
// strides), tw[j] = e^{-2 pi i j / N} for j < N.  Ends with a barrier.
template <int N>
__device__ __forceinline__ void transform_lines(float2* buf, float2* scratch, int lines, int ls, int es,
                                                const float2* __restrict__ tw) {
  if constexpr (is_pow2<N>()) {
    fft_dif<N>(buf, lines, ls, es, tw);
  } else {
    for (int e = threadIdx.x; e < lines * N; e += blockDim.x) {
      const int q = e / N, t = e % N;
      scratch[q * ls + t * es] = buf[q * ls + t * es];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < lines * N; e += blockDim.x) {
      const int q = e / N, k = e % N;
      const float2* src = scratch + q * ls;
      float re = 0.f, im = 0.f;
      int j = 0;
      for (int n = 0; n < N; ++n) {
        const float2 x = src[n * es], w = tw[j];
        re += x.x * w.x - x.y * w.y;
        im += x.x * w.y + x.y * w.x;
        j += k;
        if (j >= N) j -= N;
      }
      buf[q * ls + k * es] = make_float2(re, im);
    }
    __syncthreads();
  }
}

// Raised-cosine fill weight of the band between the mask radius and rp (integer squared
// radius r2 >= r2_inner, <= r2_outer); 1 outside, 0 inside.
__device__ __forceinline__ float fill_weight(int r2, const ShiftGeom& g) {
  if (r2 > g.r2_outer) return 1.f;
  if (r2 < g.r2_inner) return 0.f;
  const float r = sqrtf((float)r2);
  return 0.5f + 0.5f * cospif((g.rp - r) / g.width);
}

// ------------------------------------------------------------------ patch -> 2-D rfft of a plane
// One CTA per (b, rolled plane i').  The patch of a plane (trilinear at a constant shift, so
// two input planes staged in shared memory cover it), its zeroed planes, the background
// weights and 1/N^3 are applied, then the real FFT along x (two rows per complex FFT) and the
// FFT along y; T[b][i'][j'][m2], m2 < N/2+1.
//
// The background fill is linear: the reference's filled patch is (1 - W) p + W avg with W the
// outer/raised-cosine weight, and avg (the W-weighted mean of the patch) is known only after
// every plane is done.  This kernel therefore transforms (1 - W) p / N^3 and accumulates the
// weighted background sum into bg[b]; the z pass adds avg times the transform of W / N^3
// (PATTERN = true computes that transform, once per geometry).
template <int N, bool PATTERN>
__global__ void __launch_bounds__(kT)
patch_fft_xy_kernel(const float* __restrict__ vol, const float* __restrict__ shift_zyx,
                    const float* __restrict__ bgw_tab, ShiftGeom g, float2* __restrict__ T,
                    float* __restrict__ bg) {
  constexpr int HN = N / 2, H = N / 2 + 1;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  constexpr int NTW = n_twiddles<N>();
  // the zb region holds N x H entries (HN x N used) so that it can serve as the y
  // transform's scratch in the direct-DFT case
  constexpr int ZB = is_pow2<N>() ? HN * N : N * H;
  float2* tw = sm2;                                       // NTW
  float2* zb = sm2 + NTW;                                 // HN x N: rows q (re) and q + HN (im)
  float* planes = reinterpret_cast<float*>(zb + ZB);      // 2 x N x N input planes
  float2* yb = reinterpret_cast<float2*>(planes);         // N x H, after the patch is built
  const int ip = blockIdx.x, b = blockIdx.y;
  const int i = wrap_n<N>(ip + HN);
  const int di = i - HN;
  load_twiddles(tw, N, NTW);
  auto put = [&](int jp, int kp, float val) {
    reinterpret_cast<float*>(zb + (jp < HN ? jp : jp - HN) * N + kp)[jp >= HN ? 1 : 0] = val;
  };
  float part = 0.f;
  if (PATTERN) {
    for (int e = threadIdx.x; e < N * N; e += kT) {
      const int jp = e / N, kp = e % N;
      const int dj = wrap_n<N>(jp + HN) - HN, dk = wrap_n<N>(kp + HN) - HN;
      put(jp, kp, fill_weight(di * di + dj * dj + dk * dk, g) * g.inv_n3);
    }
  } else {
    const float* v = vol + (int64_t)b * N * N * N;
    const PatchShift ps = patch_shift(shift_zyx, b, N);
    const float z = (float)i + ps.f[0];
    const float z0 = floorf(z);
    const int iz = (int)z0;
    const float fz = z - z0;
    // planes iz and iz + 1 (zero outside the box, which is what skipping them gives)
    constexpr int P4 = N * N / 4;
    float4* pl4 = reinterpret_cast<float4*>(planes);
    for (int e = threadIdx.x; e < 2 * P4; e += kT) {
      const int hi = e >= P4 ? 1 : 0;
      const int zz = iz + hi;
      pl4[e] = (zz >= 0 && zz < N) ? __ldg(reinterpret_cast<const float4*>(v + (int64_t)zz * N * N) + (e - hi * P4))
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    const bool zplane = (i == ps.zp[0]);
    for (int e = threadIdx.x; e < N * N; e += kT) {
      const int jp = e / N, kp = e % N;
      const int j = wrap_n<N>(jp + HN), k = wrap_n<N>(kp + HN);
      float p = 0.f;
      if (!zplane && j != ps.zp[1] && k != ps.zp[2]) {
        const float y = (float)j + ps.f[1], x = (float)k + ps.f[2];
        const float y0 = floorf(y), x0 = floorf(x);
        const int iy = (int)y0, ix = (int)x0;
        const float fy = y - y0, fx = x - x0;
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
          for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
              const int yy = iy + dy, xx = ix + dx;
              if (yy < 0 || yy >= N || xx < 0 || xx >= N) continue;
              const float w = (dz ? fz : 1.f - fz) * (dy ? fy : 1.f - fy) * (dx ? fx : 1.f - fx);
              p += w * planes[(dz * N + yy) * N + xx];
            }
      }
      const int dj = j - HN, dk = k - HN;
      const int r2 = di * di + dj * dj + dk * dk;
      part += __ldg(bgw_tab + r2) * p;
      put(jp, kp, (1.f - fill_weight(r2, g)) * p * g.inv_n3);
    }
  }
  __syncthreads();
  // (the direct DFT's scratch for zb is the planes region, free once the patch is built)
  transform_lines<N>(zb, reinterpret_cast<float2*>(planes), HN, N, 1, tw);
  // split the packed transforms: Z = A + i B with A, B the transforms of rows q and q + HN
  for (int e = threadIdx.x; e < HN * H; e += kT) {
    const int q = e / H, k = e % H;
    const float2 zk = zb[q * N + fpos<N>(k)];
    const float2 zm = zb[q * N + fpos<N>(k == 0 ? 0 : N - k)];
    yb[q * H + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    yb[(q + HN) * H + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
  }
  __syncthreads();
  transform_lines<N>(yb, zb, H, 1, H, tw);
  float2* out = T + ((int64_t)b * N + ip) * N * H;
  for (int e = threadIdx.x; e < N * H; e += kT) {
    const int jp = e / H, m2 = e % H;
    out[e] = yb[fpos<N>(jp) * H + m2];
  }
  if (!PATTERN) {
    part = block_sum(part, red);
    if (threadIdx.x == 0) atomicAdd(&bg[b], part);
  }
}

template <int N>
constexpr size_t xy_smem_bytes() {
  return (size_t)(n_twiddles<N>() + (is_pow2<N>() ? (N / 2) * N : N * (N / 2 + 1))) * sizeof(float2) +
         (size_t)2 * N * N * sizeof(float);
}

// ------------------------------------------------------------------ FFT along z + product
// One CTA per (b, j').  Adds avg_b times the plane transforms of W / N^3 (what), the FFT
// along z, then P = conj(S) T with the rotated, ifftshifted, masked Fourier reference S
// sampled on the fly, and the norms |T|^2, |S|^2 per subtomogram.  Without SPLIT P overwrites
// T; with SPLIT the pass-1 operand of the tensor-core upsampled DFT is written instead,
// A1[part][(b, m2, m1)][2 m0 + c] for m2 < N/2 as bf16 hi/lo pairs (a1_ws pairs per row, a1_R
// rows per part), and the Nyquist plane m2 = N/2 to a1n in the same format (rows (b, m1)).
template <int N, bool SPLIT>
__global__ void __launch_bounds__(kT)
fft_z_kernel(ShiftGeom g, float2* __restrict__ T, const float2* __restrict__ what, const float* __restrict__ bg,
             const float2* __restrict__ ref, const float* __restrict__ rot, const float* __restrict__ ctf,
             float* __restrict__ nrm, uint32_t* __restrict__ a1, int a1_ws, int a1_R, uint32_t* __restrict__ a1n,
             int a1n_R) {
  constexpr int HN = N / 2, H = N / 2 + 1;
  constexpr int NTW = n_twiddles<N>();
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  float2* tw = sm2;
  float2* buf = sm2 + NTW;   // N (i') x H
  float2* scr = buf + N * H; // the direct DFT's scratch (boxes that are not powers of two)
  const int jp = blockIdx.x, b = blockIdx.y;
  float2* base = T + (int64_t)b * N * N * H + (int64_t)jp * H;
  const float2* wb = what + (int64_t)jp * H;
  const float avg = g.wsum > 0.f ? __ldg(&bg[b]) / g.wsum : 0.f;
  load_twiddles(tw, N, NTW);
  for (int e = threadIdx.x; e < N * H; e += kT) {
    const int ip = e / H, m2 = e % H;
    const float2 t = base[(int64_t)ip * N * H + m2];
    const float2 w = __ldg(&wb[(int64_t)ip * N * H + m2]);
    buf[e] = make_float2(fmaf(avg, w.x, t.x), fmaf(avg, w.y, t.y));
  }
  __syncthreads();
  transform_lines<N>(buf, scr, H, 1, H, tw);
  float R[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) R[q] = __ldg(&rot[b * 9 + q]);
  const float c = (float)g.h;  // centre of the odd-padded grid, (N+1-1)/2
  float st = 0.f, ss = 0.f;
  for (int e = threadIdx.x; e < N * H; e += kT) {
    // SPLIT walks m0 fastest so the bf16 rows are written contiguously
    const int ip = SPLIT ? e % N : e / H, m2 = SPLIT ? e / N : e % H;
    const float2 t = buf[fpos<N>(ip) * H + m2];
    // mask_full on the (N, N, N/2+1) index grid (setup_utils.py:239-249)
    const int kp = ip < HN ? ip : ip - N;
    const int jq = jp < HN ? jp : jp - N;
    const int xq = m2 < HN ? m2 : m2 - H;
    float2 s = make_float2(0.f, 0.f);
    if (kp * kp + jq * jq + xq * xq <= g.mask_r2) {
      // ifftshift over (z, y) of the slice [..., N/2:] of the rotated reference
      const int zo = wrap_n<N>(ip + HN), yo = wrap_n<N>(jp + HN), xw = m2 + HN;
      const float bx = (float)xw - c, by = (float)yo - c, bz = (float)zo - c;
      const float rx = R[0] * bx + R[1] * by + R[2] * bz + c;
      const float ry = R[3] * bx + R[4] * by + R[5] * bz + c;
      const float rz = R[6] * bx + R[7] * by + R[8] * bz + c;
      s = trilinear_c(ref, N, rz, ry, rx);
      if (ctf) {
        const float cv = __ldg(&ctf[(((int64_t)b * N + ip) * N + jp) * H + m2]);
        s.x *= cv;
        s.y *= cv;
      }
    }
    st += t.x * t.x + t.y * t.y;
    ss += s.x * s.x + s.y * s.y;
    // conj(s) * t
    const float2 p = make_float2(s.x * t.x + s.y * t.y, s.x * t.y - s.y * t.x);
    if (SPLIT) {
      if (m2 < HN) {
        uint32_t hi, lo;
        split_bf16x2(p.x, p.y, hi, lo);
        const size_t row = ((size_t)b * HN + m2) * N + jp;
        a1[row * a1_ws + ip] = hi;
        a1[((size_t)a1_R + row) * a1_ws + ip] = lo;
      } else {
        // the Nyquist plane m2 = N/2: its own pass-1 operand, rows (b, m1), K (m0, re/im)
        uint32_t hi, lo;
        split_bf16x2(p.x, p.y, hi, lo);
        const size_t row = (size_t)b * N + jp;
        a1n[row * a1_ws + ip] = hi;
        a1n[((size_t)a1n_R + row) * a1_ws + ip] = lo;
      }
    } else {
      base[(int64_t)ip * N * H + m2] = p;
    }
  }
  st = block_sum(st, red);
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    atomicAdd(&nrm[2 * b], st);
    atomicAdd(&nrm[2 * b + 1], ss);
  }
}

template <int N>
constexpr size_t z_smem_bytes() {
  return (size_t)(n_twiddles<N>() + (is_pow2<N>() ? 1 : 2) * N * (N / 2 + 1)) * sizeof(float2);
}

// ------------------------------------------------------------------ box 64: radix-8 x 8 path
// The same two passes for N = 64 with the FFTs done by groups of 8 threads: a 64-point line
// is x[r + 8 s] (thread r, register s), an 8-point DFT in registers, the twiddles W64^(r k1),
// one transpose through the line's shared scratch (warp-synchronous: a line's 8 threads share
// a warp) and a second 8-point DFT, which leaves X[r + 8 k2] in thread r.  The patch is built
// by three separable linear interpolations (z, then x, then y) from the two staged planes.
constexpr int kT64 = 288;  // 36 groups of 8: 33 lines for the (N/2+1)-column passes
constexpr int kXS = 72;    // per-line scratch (float2): transpose slot (k1, r) at 9 k1 + r
constexpr int kYS = 34;    // row stride (float2) of the 64 x 33 y-FFT output of the patch pass
constexpr int kZS = 33;    // row stride (float2) of the 64 x 33 buffer of the z pass

// Complex add and subtract as one packed two-lane FP32 instruction each (sm_100): the same
// IEEE results as two scalar ones (a - b is a + (-1) b with one rounding).
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 c_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

// 8-point forward DFT, natural order in and out (radix-2 decimation in frequency).
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
  const float c = 0.70710678118654752f;
  const float2 a0 = c_add(v[0], v[4]), a4 = c_sub(v[0], v[4]);
  const float2 a1 = c_add(v[1], v[5]), d1 = c_sub(v[1], v[5]);
  const float2 a2 = c_add(v[2], v[6]), d2 = c_sub(v[2], v[6]);
  const float2 a3 = c_add(v[3], v[7]), d3 = c_sub(v[3], v[7]);
  const float2 a5 = make_float2(c * (d1.x + d1.y), c * (d1.y - d1.x));  // d1 W8
  const float2 a6 = c_mi(d2);                                           // d2 W8^2
  const float2 a7 = make_float2(c * (d3.y - d3.x), -c * (d3.x + d3.y)); // d3 W8^3
  const float2 b0 = c_add(a0, a2), b2 = c_sub(a0, a2);
  const float2 b1 = c_add(a1, a3), b3 = c_mi(c_sub(a1, a3));
  const float2 b4 = c_add(a4, a6), b6 = c_sub(a4, a6);
  const float2 b5 = c_add(a5, a7), b7 = c_mi(c_sub(a5, a7));
  v[0] = c_add(b0, b1); v[4] = c_sub(b0, b1);
  v[2] = c_add(b2, b3); v[6] = c_sub(b2, b3);
  v[1] = c_add(b4, b5); v[5] = c_sub(b4, b5);
  v[3] = c_add(b6, b7); v[7] = c_sub(b6, b7);
}

// 64-point forward FFT of one line by its 8 threads (r = lane % 8): v[s] = x[r + 8 s] on
// entry, v[k2] = X[r + 8 k2] on exit.  xs is the line's scratch (kXS float2); tw[m] = W64^m.
__device__ __forceinline__ void fft64_group(float2 (&v)[8], int r, float2* xs, const float2* tw) {
  dft8(v);
#pragma unroll
  for (int k1 = 1; k1 < 8; ++k1) v[k1] = cmul(v[k1], tw[r * k1]);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 8; ++k1) xs[9 * k1 + r] = v[k1];
  __syncwarp();
#pragma unroll
  for (int t = 0; t < 8; ++t) v[t] = xs[9 * r + t];
  dft8(v);
}

// FFT along the rows of a 64 x 33 column buffer (element (n, col) at buf[n * kZS + col], a
// dense row stride of 33) in place, one column per group of 8 threads; xs: 36 line scratches.
// The two groups of a half-warp take columns 8 apart (group 2 i + h: column (i & 7) + 16 (i / 8)
// + 8 h), so their 8-byte accesses r + 8 s, (r + 8 s) * 33 + col fill the 16 bank pairs once;
// the row-wise readers of the buffer, 16 consecutive rows per half-warp, do so too.
__device__ __forceinline__ void fft64_columns(float2* buf, float2* xs, const float2* tw) {
  const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
  // groups 33..35 shadow column 32 inside its own warp
  const int col = L < 32 ? ((L >> 1) & 7) + 16 * (L >> 4) + 8 * (L & 1) : 32;
  float2 v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) v[s] = buf[(r + 8 * s) * kZS + col];
  fft64_group(v, r, xs + L * kXS, tw);
  __syncwarp();
  if (L < 33) {
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) buf[(r + 8 * k2) * kZS + col] = v[k2];
  }
}

__device__ void load_twiddles64(float2* tw) {
  for (int k = threadIdx.x; k < 64; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * k / 64, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

// Element (q, c) of the 32 x 64 x-FFT output of the box-64 path: row q, column c ^ f(q) with
// f(q) = 8 (q & 1) + 2 (q / 2 & 3).  The x FFT stores rows q, q + 1 (one per group of 8
// lanes, 8 consecutive c) and the y FFT loads columns c, c + 1 (8 rows q = r + 8 s): both fill
// the 16 bank pairs of a half-warp's 8-byte accesses once.
__device__ __forceinline__ int z_at(int q, int c) { return q * 64 + (c ^ (((q & 1) << 3) | ((q << 1) & 6))); }

// patch_fft_xy_kernel<64, false> with the radix-8 x 8 FFTs; fill_tab[r2] is fill_weight(r2).
__global__ void __launch_bounds__(kT64, 4)
patch_fft_xy64_kernel(const float* __restrict__ vol, const float* __restrict__ shift_zyx,
                      const float* __restrict__ bgw_tab, const float* __restrict__ fill_tab, ShiftGeom g,
                      float2* __restrict__ T, float* __restrict__ bg) {
  constexpr int N = 64, HN = 32, H = 33;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  __shared__ int s_c[2][2][N];      // [y/x][tap] clamped source index
  __shared__ float s_w[2][2][N];    // [y/x][tap] weight (0 for taps outside the box or zeroed)
  __shared__ int4 s_ty[N];          // row j's y taps packed (c0, c1, w0, w1): one broadcast load
  float2* tw = sm2;                                     // 64
  float* P0 = reinterpret_cast<float*>(sm2 + 64);       // the z-interpolated plane
  float2* Z = reinterpret_cast<float2*>(P0 + N * N);    // 32 x 64 x FFT output, swizzled (z_at)
  float2* yb = reinterpret_cast<float2*>(P0);           // 64 x kYS, after the patch is built
  float2* zb = Z + HN * N;                              // 36 x kXS: packed rows, then scratch
  const int ip = blockIdx.x, b = blockIdx.y;
  const int i = (ip + HN) & (N - 1);
  const int di = i - HN;
  const float* v = vol + (int64_t)b * N * N * N;
  const PatchShift ps = patch_shift(shift_zyx, b, N);
  const float z = (float)i + ps.f[0];
  const float z0 = floorf(z);
  const int iz = (int)z0;
  const float fz = z - z0;
  load_twiddles64(tw);
  if (threadIdx.x < 2 * N) {
    const int ax = threadIdx.x / N, j = threadIdx.x % N;  // ax 0: y (index j), 1: x (index k)
    const float y = (float)j + ps.f[1 + ax];
    const float y0 = floorf(y);
    const int iy = (int)y0;
    const float fy = y - y0;
    const bool zero = (j == ps.zp[1 + ax]);
    s_c[ax][0][j] = min(max(iy, 0), N - 1);
    s_c[ax][1][j] = min(max(iy + 1, 0), N - 1);
    s_w[ax][0][j] = (zero || iy < 0 || iy >= N) ? 0.f : 1.f - fy;
    s_w[ax][1][j] = (zero || iy + 1 < 0 || iy + 1 >= N) ? 0.f : fy;
    if (ax == 0)
      s_ty[j] = make_int4(s_c[0][0][j], s_c[0][1][j], __float_as_int(s_w[0][0][j]), __float_as_int(s_w[0][1][j]));
  }
  // z, on the way in: P0 <- (1 - fz) plane(iz) + fz plane(iz + 1), straight from global memory
  // (a plane outside the box, or a zeroed plane, contributes zero)
  {
    constexpr int P4 = N * N / 4;
    const bool zplane = (i == ps.zp[0]);
    const bool in0 = iz >= 0 && iz < N, in1 = iz + 1 >= 0 && iz + 1 < N;
    const float w0 = (zplane || !in0) ? 0.f : 1.f - fz, w1 = (zplane || !in1) ? 0.f : fz;
    const float4* g0 = reinterpret_cast<const float4*>(v + (int64_t)(in0 ? iz : 0) * N * N);
    const float4* g1 = reinterpret_cast<const float4*>(v + (int64_t)(in1 ? iz + 1 : 0) * N * N);
    float4* pl4 = reinterpret_cast<float4*>(P0);
#pragma unroll 4
    for (int e = threadIdx.x; e < P4; e += kT64) {
      const float4 a = in0 ? __ldg(g0 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 c = in1 ? __ldg(g1 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      pl4[e] = make_float4(w0 * a.x + w1 * c.x, w0 * a.y + w1 * c.y, w0 * a.z + w1 * c.z, w0 * a.w + w1 * c.w);
    }
  }
  __syncthreads();
  // x and y in one pass from the z-interpolated plane: p(j, k) = wy0(j) (wx0(k) P0[cy0][cx0] +
  // wx1(k) P0[cy0][cx1]) + wy1(j) (..cy1..) (the x taps in registers, the y taps of a row one
  // broadcast load); then background, fill weight, 1/N^3, roll, and rows j and j + 32 (rolled
  // to j + 32 and j) packed into one complex line with one 8-byte store
  float part = 0.f;
  if (threadIdx.x < 256) {
    const int k = threadIdx.x & (N - 1), j0 = threadIdx.x >> 6;
    const float wx0 = s_w[1][0][k], wx1 = s_w[1][1][k];
    const int cx0 = s_c[1][0][k], cx1 = s_c[1][1][k];
    const int dk = k - HN, kp = (k + HN) & (N - 1);
    const int rk = di * di + dk * dk;
    auto sample = [&](int j) -> float {
      const int4 ty = s_ty[j];
      const int cy0 = ty.x, cy1 = ty.y;
      const float wy0 = __int_as_float(ty.z), wy1 = __int_as_float(ty.w);
      const float a = wx0 * P0[cy0 * N + cx0] + wx1 * P0[cy0 * N + cx1];
      const float c = wx0 * P0[cy1 * N + cx0] + wx1 * P0[cy1 * N + cx1];
      const float p = wy0 * a + wy1 * c;
      const int dj = j - HN;
      const int r2 = rk + dj * dj;
      float keep = 1.f;  // 1 - W
      if (r2 > g.r2_outer) {
        part += p;
        keep = 0.f;
      } else if (r2 >= g.r2_inner) {
        part += __ldg(bgw_tab + r2) * p;
        keep = 1.f - __ldg(fill_tab + r2);
      }
      return keep * p * g.inv_n3;
    };
#pragma unroll 2
    for (int j = j0; j < HN; j += 4) {
      const float lo = sample(j), hi = sample(j + HN);  // rolled to rows j + 32 and j
      zb[j * kXS + kp] = make_float2(hi, lo);
    }
  }
  __syncthreads();
  // x FFT of the 32 packed lines (groups 32..35 work on their own scratch lines and are
  // dropped), out to Z
  {
    const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
    float2* line = zb + L * kXS;
    float2 w[8];
#pragma unroll
    for (int s8 = 0; s8 < 8; ++s8) w[s8] = line[r + 8 * s8];
    fft64_group(w, r, line, tw);
    if (L < HN) {
#pragma unroll
      for (int k2 = 0; k2 < 8; ++k2) Z[z_at(L, r + 8 * k2)] = w[k2];
    }
  }
  __syncthreads();
  // y FFT of the columns m2 < 33, its input split on the way in: Z = A + i B holds the
  // transforms of rows q and q + 32, so a group's rows r + 8 s' and r + 8 s' + 32 (s' < 4)
  // come from the same two entries Z[q][m2], Z[q][-m2]
  {
    const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
    const int col = L < H ? L : H - 1;  // groups 33..35 shadow column 32 inside its own warp
    float2 w[8];
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4) {
      const int q = r + 8 * s4;
      const float2 zk = Z[z_at(q, col)];
      const float2 zm = Z[z_at(q, (N - col) & (N - 1))];
      w[s4] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      w[s4 + 4] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    __syncthreads();  // Z is read: yb may overwrite its first rows, zb is the transpose scratch
    fft64_group(w, r, zb + L * kXS, tw);
    if (L < H) {
#pragma unroll
      for (int k2 = 0; k2 < 8; ++k2) yb[(r + 8 * k2) * kYS + col] = w[k2];
    }
  }
  __syncthreads();
  float2* out = T + ((int64_t)b * N + ip) * N * H;
  for (int e = threadIdx.x; e < N * H; e += kT64) {
    const int jq = e / H, m2 = e - (e / H) * H;
    out[e] = yb[jq * kYS + m2];
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) atomicAdd(&bg[b], part);
}

constexpr size_t xy64_smem_bytes() {
  return (size_t)64 * sizeof(float2) + (size_t)64 * 64 * sizeof(float) + (size_t)32 * 64 * sizeof(float2) +
         (size_t)36 * kXS * sizeof(float2);
}

// fft_z_kernel<64, SPLIT> with the radix-8 x 8 FFT.
template <bool SPLIT>
__global__ void __launch_bounds__(kT64, 4)
fft_z64_kernel(ShiftGeom g, float2* __restrict__ T, const float2* __restrict__ what, const float* __restrict__ bg,
               const float4* __restrict__ refq, const float* __restrict__ rot, const float* __restrict__ ctf,
               float* __restrict__ nrm, uint32_t* __restrict__ a1, int a1_ws, int a1_R, uint32_t* __restrict__ a1n,
               int a1n_R) {
  constexpr int N = 64, HN = 32, H = 33;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  float2* tw = sm2;              // 64
  float2* buf = sm2 + 64;        // 64 (i') x kZS
  float2* xs = buf + N * kZS;    // 36 x kXS
  const int jp = blockIdx.x, b = blockIdx.y;
  float2* base = T + (int64_t)b * N * N * H + (int64_t)jp * H;
  const float2* wb = what + (int64_t)jp * H;
  const float avg = g.wsum > 0.f ? __ldg(&bg[b]) / g.wsum : 0.f;
  load_twiddles64(tw);
#pragma unroll 4
  for (int e = threadIdx.x; e < N * H; e += kT64) {
    const int ip = e / H, m2 = e - (e / H) * H;
    const float2 t = base[(int64_t)ip * N * H + m2];
    const float2 w = __ldg(&wb[(int64_t)ip * N * H + m2]);
    buf[ip * kZS + m2] = make_float2(fmaf(avg, w.x, t.x), fmaf(avg, w.y, t.y));
  }
  __syncthreads();
  fft64_columns(buf, xs, tw);
  __syncthreads();
  float R[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) R[q] = __ldg(&rot[b * 9 + q]);
  const float c = (float)g.h;
  float st = 0.f, ss = 0.f;
#pragma unroll 2
  for (int e = threadIdx.x; e < N * H; e += kT64) {
    const int ip = SPLIT ? e & (N - 1) : e / H, m2 = SPLIT ? e >> 6 : e - (e / H) * H;
    const float2 t = buf[ip * kZS + m2];
    const int kp = ip < HN ? ip : ip - N;
    const int jq = jp < HN ? jp : jp - N;
    const int xq = m2 < HN ? m2 : m2 - H;
    // outside the mask the sample is taken far outside the box, which reads zero (entry 0)
    const bool in_mask = kp * kp + jq * jq + xq * xq <= g.mask_r2;
    float2 s;
    {
      const int zo = (ip + HN) & (N - 1), yo = (jp + HN) & (N - 1), xw = m2 + HN;
      const float bx = (float)xw - c, by = (float)yo - c, bz = (float)zo - c;
      const float rx = R[0] * bx + R[1] * by + R[2] * bz + c;
      const float ry = R[3] * bx + R[4] * by + R[5] * bz + c;
      const float rz = in_mask ? R[6] * bx + R[7] * by + R[8] * bz + c : -4.f;
      s = trilinear_quad(refq, N, rz, ry, rx);
    }
    if (in_mask) {
      if (ctf) {
        const float cv = __ldg(&ctf[(((int64_t)b * N + ip) * N + jp) * H + m2]);
        s.x *= cv;
        s.y *= cv;
      }
    }
    st += t.x * t.x + t.y * t.y;
    ss += s.x * s.x + s.y * s.y;
    const float2 p = make_float2(s.x * t.x + s.y * t.y, s.x * t.y - s.y * t.x);
    if (SPLIT) {
      if (m2 < HN) {
        uint32_t hi, lo;
        split_bf16x2(p.x, p.y, hi, lo);
        const size_t row = ((size_t)b * HN + m2) * N + jp;
        a1[row * a1_ws + ip] = hi;
        a1[((size_t)a1_R + row) * a1_ws + ip] = lo;
      } else {
        // the Nyquist plane m2 = N/2: its own pass-1 operand, rows (b, m1), K (m0, re/im)
        uint32_t hi, lo;
        split_bf16x2(p.x, p.y, hi, lo);
        const size_t row = (size_t)b * N + jp;
        a1n[row * a1_ws + ip] = hi;
        a1n[((size_t)a1n_R + row) * a1_ws + ip] = lo;
      }
    } else {
      base[(int64_t)ip * N * H + m2] = p;
    }
  }
  st = block_sum(st, red);
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    atomicAdd(&nrm[2 * b], st);
    atomicAdd(&nrm[2 * b + 1], ss);
  }
}

constexpr size_t z64_smem_bytes() {
  return (size_t)64 * sizeof(float2) + (size_t)64 * kZS * sizeof(float2) + (size_t)36 * kXS * sizeof(float2);
}

// ------------------------------------------------------------------ box 128: radix-16 x 8 path
// The box-64 design at N = 128: a 128-point line is x[r + 8 s] (thread r of a group of 8,
// register s < 16); a 16-point DFT in registers (two 8-point DFTs and the W16 butterflies), the
// twiddles W128^(r k1), one transpose through the group's scratch, and two 8-point DFTs (for
// k1 = r and r + 8) leave X[r + 8 s] in thread r again.  36 groups take the 64 packed x lines
// and the 65 y / z columns in two rounds.  The x-FFT output overlays the z-interpolated plane
// once every sample is in registers, so a CTA holds about 113 KB and two fit on an SM.
constexpr int kT128 = 288;   // 36 groups of 8
constexpr int kG128 = 36;
constexpr int kXS128 = 152;  // per-group scratch (float2): slot (k1, r) at 9 k1 + r; 152 = 8 (mod 16)
                             // puts the two groups of a half-warp on disjoint bank pairs
constexpr int kZS128 = 65;   // row stride (float2) of the 128 x 65 buffer of the z pass

// 16-point forward DFT, natural order in and out: the even and odd halves by dft8, then the
// radix-2 butterflies with W16^k.
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
  float2 e[8], o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft8(e);
  dft8(o);
  // W16^k = (cos(pi k / 8), -sin(pi k / 8))
  const float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, c2 = 0.70710678118654752f;
  const float2 w16[8] = {make_float2(1.f, 0.f),  make_float2(c1, -s1),  make_float2(c2, -c2), make_float2(s1, -c1),
                         make_float2(0.f, -1.f), make_float2(-s1, -c1), make_float2(-c2, -c2), make_float2(-c1, -s1)};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float2 t = k == 0 ? o[0] : (k == 4 ? c_mi(o[4]) : cmul(o[k], w16[k]));
    v[k] = c_add(e[k], t);
    v[k + 8] = c_sub(e[k], t);
  }
}

// 128-point forward FFT of one line by its 8 threads (r = lane % 8): v[s] = x[r + 8 s] on
// entry and v[s] = X[r + 8 s] on exit.  xs is the group's scratch (kXS128 float2); tw[m] = W128^m.
__device__ __forceinline__ void fft128_group(float2 (&v)[16], int r, float2* xs, const float2* tw) {
  dft16(v);  // V_r[k1] = sum_s x[r + 8 s] W16^(s k1)
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1) v[k1] = cmul(v[k1], tw[r * k1]);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) xs[9 * k1 + r] = v[k1];
  __syncwarp();
  float2 a[8], b[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    a[t] = xs[9 * r + t];        // V_t[r]
    b[t] = xs[9 * (r + 8) + t];  // V_t[r + 8]
  }
  dft8(a);  // X[r + 16 k2]
  dft8(b);  // X[r + 8 + 16 k2]
#pragma unroll
  for (int k2 = 0; k2 < 8; ++k2) {
    v[2 * k2] = a[k2];
    v[2 * k2 + 1] = b[k2];
  }
}

__device__ void load_twiddles128(float2* tw) {
  for (int k = threadIdx.x; k < 128; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * k / 128, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

// Element (q, c) of the 64 x 128 x-FFT output: the box-64 swizzle (c ^ f(q), f(q) = 8 (q & 1)
// + 2 (q / 2 & 3)), so that the x FFT's row stores and the y FFT's column loads of a
// half-warp fill the 16 bank pairs once.
__device__ __forceinline__ int z_at128(int q, int c) { return q * 128 + (c ^ (((q & 1) << 3) | ((q << 1) & 6))); }

// Column of round idx (group L + 36 round): 0 .. 63 in an order that puts the two groups of
// a half-warp 8 columns apart, then the Nyquist column 64; idx > 64 shadows column 64.
__device__ __forceinline__ int col128(int idx) {
  return idx < 64 ? ((idx >> 1) & 7) + 16 * (idx >> 4) + 8 * (idx & 1) : 64;
}

// patch_fft_xy_kernel<128, false> with the radix-16 x 8 FFTs; fill_tab[r2] is fill_weight(r2).
__global__ void __launch_bounds__(kT128, 2)
patch_fft_xy128_kernel(const float* __restrict__ vol, const float* __restrict__ shift_zyx,
                       const float* __restrict__ bgw_tab, const float* __restrict__ fill_tab, ShiftGeom g,
                       float2* __restrict__ T, float* __restrict__ bg) {
  constexpr int N = 128, HN = 64, H = 65;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  __shared__ int s_cx[2][N];        // [tap] clamped source column
  __shared__ float s_wx[2][N];      // [tap] weight (0 for taps outside the box or zeroed)
  __shared__ int4 s_ty[N];          // row j's y taps packed (c0, c1, w0, w1)
  float2* tw = sm2;                                     // 128
  float* P0 = reinterpret_cast<float*>(sm2 + 128);      // the z-interpolated plane (128 x 128)
  float2* Z = reinterpret_cast<float2*>(P0);            // then the 64 x 128 x-FFT output (z_at128)
  float2* xs = reinterpret_cast<float2*>(P0 + N * N);   // 36 x kXS128 group scratch
  const int ip = blockIdx.x, b = blockIdx.y;
  const int i = (ip + HN) & (N - 1);
  const int di = i - HN;
  const float* v = vol + (int64_t)b * N * N * N;
  const PatchShift ps = patch_shift(shift_zyx, b, N);
  const float z = (float)i + ps.f[0];
  const float z0 = floorf(z);
  const int iz = (int)z0;
  const float fz = z - z0;
  load_twiddles128(tw);
  if (threadIdx.x < 2 * N) {
    const int ax = threadIdx.x / N, j = threadIdx.x % N;  // ax 0: y (index j), 1: x (index k)
    const float y = (float)j + ps.f[1 + ax];
    const float y0 = floorf(y);
    const int iy = (int)y0;
    const float fy = y - y0;
    const bool zero = (j == ps.zp[1 + ax]);
    const int c0 = min(max(iy, 0), N - 1), c1 = min(max(iy + 1, 0), N - 1);
    const float w0 = (zero || iy < 0 || iy >= N) ? 0.f : 1.f - fy;
    const float w1 = (zero || iy + 1 < 0 || iy + 1 >= N) ? 0.f : fy;
    if (ax == 0) {
      s_ty[j] = make_int4(c0, c1, __float_as_int(w0), __float_as_int(w1));
    } else {
      s_cx[0][j] = c0;
      s_cx[1][j] = c1;
      s_wx[0][j] = w0;
      s_wx[1][j] = w1;
    }
  }
  {
    constexpr int P4 = N * N / 4;
    const bool zplane = (i == ps.zp[0]);
    const bool in0 = iz >= 0 && iz < N, in1 = iz + 1 >= 0 && iz + 1 < N;
    const float w0 = (zplane || !in0) ? 0.f : 1.f - fz, w1 = (zplane || !in1) ? 0.f : fz;
    const float4* g0 = reinterpret_cast<const float4*>(v + (int64_t)(in0 ? iz : 0) * N * N);
    const float4* g1 = reinterpret_cast<const float4*>(v + (int64_t)(in1 ? iz + 1 : 0) * N * N);
    float4* pl4 = reinterpret_cast<float4*>(P0);
#pragma unroll 4
    for (int e = threadIdx.x; e < P4; e += kT128) {
      const float4 a = in0 ? __ldg(g0 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 c = in1 ? __ldg(g1 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      const int row = e >> 5;  // 32 float4 per row; the swizzle moves whole float4
      pl4[(row << 5) | ((e & 31) ^ ((row & 3) << 1))] =
          make_float4(w0 * a.x + w1 * c.x, w0 * a.y + w1 * c.y, w0 * a.z + w1 * c.z, w0 * a.w + w1 * c.w);
    }
  }
  __syncthreads();
  const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
  float part = 0.f;
  auto sample = [&](int j, int k) -> float {
    const int4 ty = s_ty[j];
    const int cy0 = ty.x, cy1 = ty.y;
    const float wy0 = __int_as_float(ty.z), wy1 = __int_as_float(ty.w);
    const float wx0 = s_wx[0][k], wx1 = s_wx[1][k];
    const int cx0 = s_cx[0][k], cx1 = s_cx[1][k];
    // plane row y holds column x at x ^ 8 (y & 3): the four groups of a warp read four
    // consecutive rows at the same columns, which then fall in four different 8-bank windows
    const int sy0 = (cy0 & 3) << 3, sy1 = (cy1 & 3) << 3;
    const float a = wx0 * P0[cy0 * N + (cx0 ^ sy0)] + wx1 * P0[cy0 * N + (cx1 ^ sy0)];
    const float c = wx0 * P0[cy1 * N + (cx0 ^ sy1)] + wx1 * P0[cy1 * N + (cx1 ^ sy1)];
    const float p = wy0 * a + wy1 * c;
    const int dj = j - HN, dk = k - HN;
    const int r2 = di * di + dj * dj + dk * dk;
    float keep = 1.f;  // 1 - W
    if (r2 > g.r2_outer) {
      part += p;
      keep = 0.f;
    } else if (r2 >= g.r2_inner) {
      part += __ldg(bgw_tab + r2) * p;
      keep = 1.f - __ldg(fill_tab + r2);
    }
    return keep * p * g.inv_n3;
  };
  // x FFT: packed line q (rolled rows q and q + 64 as real and imaginary parts) of group L in
  // rounds q = L and L + 36; all samples are taken before the plane is overwritten by Z
  float2 w0[16], w1[16];
  const bool second = L + kG128 < HN;  // warp-uniform (groups 28..35 are warps 7 and 8)
#pragma unroll
  for (int s8 = 0; s8 < 16; ++s8) {
    const int kp = r + 8 * s8, k = (kp + HN) & (N - 1);
    w0[s8] = make_float2(sample(L + HN, k), sample(L, k));
    if (second) w1[s8] = make_float2(sample(L + kG128 + HN, k), sample(L + kG128, k));
  }
  __syncthreads();  // the plane is read: Z may overwrite it
  float2* gx = xs + L * kXS128;
  fft128_group(w0, r, gx, tw);
#pragma unroll
  for (int k2 = 0; k2 < 16; ++k2) Z[z_at128(L, r + 8 * k2)] = w0[k2];
  if (second) {
    fft128_group(w1, r, gx, tw);
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) Z[z_at128(L + kG128, r + 8 * k2)] = w1[k2];
  }
  __syncthreads();
  // y FFT of the columns m2 < 65, its input split on the way in (Z = A + i B holds the
  // transforms of rows q and q + 64), each result stored straight to T
  float2* out = T + ((int64_t)b * N + ip) * N * H;
#pragma unroll 1
  for (int round = 0; round < 2; ++round) {
    const int idx = L + kG128 * round;
    if (idx >= 72) break;
    const int col = col128(idx);
    float2 w[16];
#pragma unroll
    for (int s8 = 0; s8 < 8; ++s8) {
      const int q = r + 8 * s8;
      const float2 zk = Z[z_at128(q, col)];
      const float2 zm = Z[z_at128(q, (N - col) & (N - 1))];
      w[s8] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      w[s8 + 8] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    fft128_group(w, r, gx, tw);
    if (idx <= 64) {
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) out[(r + 8 * k2) * H + col] = w[k2];
    }
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) atomicAdd(&bg[b], part);
}

constexpr size_t xy128_smem_bytes() {
  return (size_t)128 * sizeof(float2) + (size_t)128 * 128 * sizeof(float) + (size_t)kG128 * kXS128 * sizeof(float2);
}

// fft_z_kernel<128, SPLIT> with the radix-16 x 8 FFT.
template <bool SPLIT>
__global__ void __launch_bounds__(kT128, 2)
fft_z128_kernel(ShiftGeom g, float2* __restrict__ T, const float2* __restrict__ what, const float* __restrict__ bg,
                const float4* __restrict__ refq, const float* __restrict__ rot, const float* __restrict__ ctf,
                float* __restrict__ nrm, uint32_t* __restrict__ a1, int a1_ws, int a1_R, uint32_t* __restrict__ a1n,
                int a1n_R) {
  constexpr int N = 128, HN = 64, H = 65;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  float2* tw = sm2;                // 128
  float2* buf = sm2 + 128;         // 128 (i') x kZS128
  float2* xs = buf + N * kZS128;   // 36 x kXS128
  const int jp = blockIdx.x, b = blockIdx.y;
  float2* base = T + (int64_t)b * N * N * H + (int64_t)jp * H;
  const float2* wb = what + (int64_t)jp * H;
  const float avg = g.wsum > 0.f ? __ldg(&bg[b]) / g.wsum : 0.f;
  load_twiddles128(tw);
#pragma unroll 4
  for (int e = threadIdx.x; e < N * H; e += kT128) {
    const int ip = e / H, m2 = e - (e / H) * H;
    const float2 t = base[(int64_t)ip * N * H + m2];
    const float2 w = __ldg(&wb[(int64_t)ip * N * H + m2]);
    buf[ip * kZS128 + m2] = make_float2(fmaf(avg, w.x, t.x), fmaf(avg, w.y, t.y));
  }
  __syncthreads();
  {
    const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
    float2* gx = xs + L * kXS128;
#pragma unroll 1
    for (int round = 0; round < 2; ++round) {
      const int idx = L + kG128 * round;
      if (idx >= 72) break;
      const int col = col128(idx);
      float2 v[16];
#pragma unroll
      for (int s8 = 0; s8 < 16; ++s8) v[s8] = buf[(r + 8 * s8) * kZS128 + col];
      fft128_group(v, r, gx, tw);
      __syncwarp();
      if (idx <= 64) {
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) buf[(r + 8 * k2) * kZS128 + col] = v[k2];
      }
    }
  }
  __syncthreads();
  float R[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) R[q] = __ldg(&rot[b * 9 + q]);
  const float c = (float)g.h;
  float st = 0.f, ss = 0.f;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * H; e += kT128) {
    const int ip = SPLIT ? e & (N - 1) : e / H, m2 = SPLIT ? e >> 7 : e - (e / H) * H;
    const float2 t = buf[ip * kZS128 + m2];
    const int kp = ip < HN ? ip : ip - N;
    const int jq = jp < HN ? jp : jp - N;
    const int xq = m2 < HN ? m2 : m2 - H;
    // outside the mask the sample is taken far outside the box, which reads zero (entry 0)
    const bool in_mask = kp * kp + jq * jq + xq * xq <= g.mask_r2;
    float2 s;
    {
      const int zo = (ip + HN) & (N - 1), yo = (jp + HN) & (N - 1), xw = m2 + HN;
      const float bx = (float)xw - c, by = (float)yo - c, bz = (float)zo - c;
      const float rx = R[0] * bx + R[1] * by + R[2] * bz + c;
      const float ry = R[3] * bx + R[4] * by + R[5] * bz + c;
      const float rz = in_mask ? R[6] * bx + R[7] * by + R[8] * bz + c : -4.f;
      s = trilinear_quad(refq, N, rz, ry, rx);
    }
    if (in_mask && ctf) {
      const float cv = __ldg(&ctf[(((int64_t)b * N + ip) * N + jp) * H + m2]);
      s.x *= cv;
      s.y *= cv;
    }
    st += t.x * t.x + t.y * t.y;
    ss += s.x * s.x + s.y * s.y;
    const float2 p = make_float2(s.x * t.x + s.y * t.y, s.x * t.y - s.y * t.x);
    if (SPLIT) {
      uint32_t hi, lo;
      split_bf16x2(p.x, p.y, hi, lo);
      if (m2 < HN) {
        const size_t row = ((size_t)b * HN + m2) * N + jp;
        a1[row * a1_ws + ip] = hi;
        a1[((size_t)a1_R + row) * a1_ws + ip] = lo;
      } else {
        // the Nyquist plane m2 = N/2: its own pass-1 operand, rows (b, m1), K (m0, re/im)
        const size_t row = (size_t)b * N + jp;
        a1n[row * a1_ws + ip] = hi;
        a1n[((size_t)a1n_R + row) * a1_ws + ip] = lo;
      }
    } else {
      base[(int64_t)ip * N * H + m2] = p;
    }
  }
  st = block_sum(st, red);
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    atomicAdd(&nrm[2 * b], st);
    atomicAdd(&nrm[2 * b + 1], ss);
  }
}

constexpr size_t z128_smem_bytes() {
  return (size_t)128 * sizeof(float2) + (size_t)128 * kZS128 * sizeof(float2) + (size_t)kG128 * kXS128 * sizeof(float2);
}

// ------------------------------------------------------------------ boxes 48 and 96: radix-S x 8 path
// A line of N = 8 S points (S = 6 or 12) is x[r + 8 s] (thread r of a group of 8, register
// s < S): an S-point DFT in registers (Cooley-Tukey over 3 and 2 or 4), the twiddles W_N^(r k1),
// a transpose through the group's scratch, and 8-point DFTs over r for the k1 = r + 8 j < S the
// thread owns, which give X[k1 + S k2], k2 < 8.  The group synchronises on its own 8 lanes, so
// groups without work in a round simply skip it.  Same passes as the box-128 kernels.
constexpr int kTG = 288;  // 36 groups of 8
constexpr int kGG = 36;

// 3-point forward DFT in place.
__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c) {
  const float h = 0.86602540378443865f;  // sqrt(3) / 2
  const float2 t1 = c_add(b, c);
  const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
  const float2 d = c_sub(b, c);
  const float2 t3 = make_float2(h * d.y, -h * d.x);  // -i (sqrt(3)/2) (b - c)
  a = c_add(a, t1);
  b = c_add(t2, t3);
  c = c_sub(t2, t3);
}

// S-point forward DFT, natural order in and out, S = 6 (2 x 3) or 12 (4 x 3): for each residue
// s2 of s mod n2 a 3-point DFT over s1 (s = s2 + n2 s1), the twiddles W_S^(s2 k1), then an
// n2-point DFT over s2 for each k1: X[k1 + 3 k2].
template <int S>
__device__ __forceinline__ void dft_small(float2 (&v)[S]) {
  static_assert(S == 6 || S == 12, "dft_small covers S = 6 and 12");
  constexpr int n2 = S / 3;
  float2 y[n2][3];
#pragma unroll
  for (int s2 = 0; s2 < n2; ++s2) {
    y[s2][0] = v[s2];
    y[s2][1] = v[s2 + n2];
    y[s2][2] = v[s2 + 2 * n2];
    dft3(y[s2][0], y[s2][1], y[s2][2]);
  }
  const float h = 0.86602540378443865f;
  if constexpr (S == 6) {
    // W6^1 = (1/2, -h), W6^2 = (-1/2, -h)
    y[1][1] = cmul(y[1][1], make_float2(0.5f, -h));
    y[1][2] = cmul(y[1][2], make_float2(-0.5f, -h));
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      v[k1] = c_add(y[0][k1], y[1][k1]);
      v[k1 + 3] = c_sub(y[0][k1], y[1][k1]);
    }
  } else {
    // W12^m, m = s2 k1 <= 6: (cos(pi m / 6), -sin(pi m / 6))
    const float2 w12[7] = {make_float2(1.f, 0.f),  make_float2(h, -0.5f),   make_float2(0.5f, -h),
                           make_float2(0.f, -1.f), make_float2(-0.5f, -h),  make_float2(-h, -0.5f),
                           make_float2(-1.f, 0.f)};
#pragma unroll
    for (int s2 = 1; s2 < 4; ++s2)
#pragma unroll
      for (int k1 = 1; k1 < 3; ++k1) y[s2][k1] = cmul(y[s2][k1], w12[s2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      // 4-point DFT over s2: X[k1 + 3 k2]
      const float2 a = y[0][k1], b = y[1][k1], c = y[2][k1], d = y[3][k1];
      const float2 p0 = c_add(a, c), p1 = c_sub(a, c), q0 = c_add(b, d), q1 = c_mi(c_sub(b, d));
      v[k1] = c_add(p0, q0);
      v[k1 + 3] = c_add(p1, q1);
      v[k1 + 6] = c_sub(p0, q0);
      v[k1 + 9] = c_sub(p1, q1);
    }
  }
}

template <int S>
__host__ __device__ constexpr int grp_xs() {  // per-group scratch: 9 S entries, stride = 8 (mod 16)
  return ((9 * S + 7) / 16) * 16 + 8;
}

// N-point forward FFT (N = 8 S) of one line by its 8 threads; v[s] = x[r + 8 s] on entry; on
// exit o[j][k2] = X[(r + 8 j) + S k2] for the j with r + 8 j < S.  gmask: the group's lanes.
template <int S>
__device__ __forceinline__ void fft_grp(float2 (&v)[S], int r, unsigned gmask, float2* xs, const float2* tw,
                                        float2 (&o)[2][8]) {
  dft_small<S>(v);  // V_r[k1]
#pragma unroll
  for (int k1 = 1; k1 < S; ++k1) v[k1] = cmul(v[k1], tw[r * k1]);
  __syncwarp(gmask);
#pragma unroll
  for (int k1 = 0; k1 < S; ++k1) xs[9 * k1 + r] = v[k1];
  __syncwarp(gmask);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int k1 = r + 8 * j;
    if (k1 < S) {
#pragma unroll
      for (int t = 0; t < 8; ++t) o[j][t] = xs[9 * k1 + t];  // V_t[k1]
      dft8(o[j]);
    }
  }
}

// patch_fft_xy_kernel<N, false> for N = 48, 96 with the radix-S x 8 FFTs.
template <int N>
__global__ void __launch_bounds__(kTG, 2)
patch_fft_xy_grp_kernel(const float* __restrict__ vol, const float* __restrict__ shift_zyx,
                        const float* __restrict__ bgw_tab, const float* __restrict__ fill_tab, ShiftGeom g,
                        float2* __restrict__ T, float* __restrict__ bg) {
  constexpr int S = N / 8, HN = N / 2, H = N / 2 + 1;
  constexpr int PR = N + 8;  // plane row stride (floats): four consecutive rows fall on different banks
  constexpr int ZR = N + 1;  // x-FFT output row stride (float2)
  constexpr int XS = grp_xs<S>();
  constexpr size_t kRegion = (size_t)N * PR * 4 > (size_t)HN * ZR * 8 ? (size_t)N * PR * 4 : (size_t)HN * ZR * 8;
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  __shared__ int s_cx[2][N];
  __shared__ float s_wx[2][N];
  __shared__ int4 s_ty[N];
  float2* tw = sm2;                                       // N
  float* P0 = reinterpret_cast<float*>(sm2 + N);          // the z-interpolated plane (N x PR)
  float2* Z = reinterpret_cast<float2*>(P0);              // then the HN x ZR x-FFT output
  float2* xs = reinterpret_cast<float2*>(reinterpret_cast<char*>(P0) + kRegion);  // kGG x XS
  const int ip = blockIdx.x, b = blockIdx.y;
  const int i = wrap_n<N>(ip + HN);
  const int di = i - HN;
  const float* v = vol + (int64_t)b * N * N * N;
  const PatchShift ps = patch_shift(shift_zyx, b, N);
  const float z = (float)i + ps.f[0];
  const float z0 = floorf(z);
  const int iz = (int)z0;
  const float fz = z - z0;
  load_twiddles(tw, N, N);
  if (threadIdx.x < 2 * N) {
    const int ax = threadIdx.x / N, j = threadIdx.x % N;
    const float y = (float)j + ps.f[1 + ax];
    const float y0 = floorf(y);
    const int iy = (int)y0;
    const float fy = y - y0;
    const bool zero = (j == ps.zp[1 + ax]);
    const int c0 = min(max(iy, 0), N - 1), c1 = min(max(iy + 1, 0), N - 1);
    const float w0 = (zero || iy < 0 || iy >= N) ? 0.f : 1.f - fy;
    const float w1 = (zero || iy + 1 < 0 || iy + 1 >= N) ? 0.f : fy;
    if (ax == 0) {
      s_ty[j] = make_int4(c0, c1, __float_as_int(w0), __float_as_int(w1));
    } else {
      s_cx[0][j] = c0;
      s_cx[1][j] = c1;
      s_wx[0][j] = w0;
      s_wx[1][j] = w1;
    }
  }
  {
    constexpr int R4 = N / 4, P4 = N * R4;
    const bool zplane = (i == ps.zp[0]);
    const bool in0 = iz >= 0 && iz < N, in1 = iz + 1 >= 0 && iz + 1 < N;
    const float w0 = (zplane || !in0) ? 0.f : 1.f - fz, w1 = (zplane || !in1) ? 0.f : fz;
    const float4* g0 = reinterpret_cast<const float4*>(v + (int64_t)(in0 ? iz : 0) * N * N);
    const float4* g1 = reinterpret_cast<const float4*>(v + (int64_t)(in1 ? iz + 1 : 0) * N * N);
    float4* pl4 = reinterpret_cast<float4*>(P0);
#pragma unroll 4
    for (int e = threadIdx.x; e < P4; e += kTG) {
      const float4 a = in0 ? __ldg(g0 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 c = in1 ? __ldg(g1 + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      const int row = e / R4;
      pl4[row * (PR / 4) + (e - row * R4)] =
          make_float4(w0 * a.x + w1 * c.x, w0 * a.y + w1 * c.y, w0 * a.z + w1 * c.z, w0 * a.w + w1 * c.w);
    }
  }
  __syncthreads();
  const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
  const unsigned gmask = 0xFFu << (threadIdx.x & 24);
  float2* gx = xs + L * XS;
  float part = 0.f;
  auto sample = [&](int j, int k) -> float {
    const int4 ty = s_ty[j];
    const int cy0 = ty.x, cy1 = ty.y;
    const float wy0 = __int_as_float(ty.z), wy1 = __int_as_float(ty.w);
    const float wx0 = s_wx[0][k], wx1 = s_wx[1][k];
    const int cx0 = s_cx[0][k], cx1 = s_cx[1][k];
    const float a = wx0 * P0[cy0 * PR + cx0] + wx1 * P0[cy0 * PR + cx1];
    const float c = wx0 * P0[cy1 * PR + cx0] + wx1 * P0[cy1 * PR + cx1];
    const float p = wy0 * a + wy1 * c;
    const int dj = j - HN, dk = k - HN;
    const int r2 = di * di + dj * dj + dk * dk;
    float keep = 1.f;  // 1 - W
    if (r2 > g.r2_outer) {
      part += p;
      keep = 0.f;
    } else if (r2 >= g.r2_inner) {
      part += __ldg(bgw_tab + r2) * p;
      keep = 1.f - __ldg(fill_tab + r2);
    }
    return keep * p * g.inv_n3;
  };
  // x FFT: packed lines q = L and L + 36 (rolled rows q and q + HN as real and imaginary
  // parts), all samples taken before the plane is overwritten by Z
  constexpr int kRounds = (HN + kGG - 1) / kGG;
  static_assert(kRounds <= 2, "two rounds of lines at most");
  float2 w[2][S];
#pragma unroll
  for (int round = 0; round < kRounds; ++round) {
    const int q = L + kGG * round;
    if (q < HN) {
#pragma unroll
      for (int s8 = 0; s8 < S; ++s8) {
        const int kp = r + 8 * s8, k = wrap_n<N>(kp + HN);
        w[round][s8] = make_float2(sample(q + HN, k), sample(q, k));
      }
    }
  }
  __syncthreads();  // the plane is read: Z may overwrite it
#pragma unroll
  for (int round = 0; round < kRounds; ++round) {
    const int q = L + kGG * round;
    if (q < HN) {
      float2 o[2][8];
      fft_grp<S>(w[round], r, gmask, gx, tw, o);
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (r + 8 * j < S) {
#pragma unroll
          for (int k2 = 0; k2 < 8; ++k2) Z[q * ZR + r + 8 * j + S * k2] = o[j][k2];
        }
    }
  }
  __syncthreads();
  // y FFT of the columns m2 < H, its input split on the way in (Z = A + i B holds the
  // transforms of rows q and q + HN), each result stored straight to T
  float2* out = T + ((int64_t)b * N + ip) * N * H;
#pragma unroll 1
  for (int col = L; col < H; col += kGG) {
    float2 x[S];
    const int cm = col == 0 ? 0 : N - col;
#pragma unroll
    for (int s8 = 0; s8 < S / 2; ++s8) {
      const int q = r + 8 * s8;
      const float2 zk = Z[q * ZR + col];
      const float2 zm = Z[q * ZR + cm];
      x[s8] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      x[s8 + S / 2] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
    float2 o[2][8];
    fft_grp<S>(x, r, gmask, gx, tw, o);
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (r + 8 * j < S) {
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) out[(r + 8 * j + S * k2) * H + col] = o[j][k2];
      }
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) atomicAdd(&bg[b], part);
}

template <int N>
constexpr size_t xy_grp_smem_bytes() {
  constexpr int HN = N / 2;
  constexpr size_t plane = (size_t)N * (N + 8) * 4, zb = (size_t)HN * (N + 1) * 8;
  return (size_t)N * sizeof(float2) + (plane > zb ? plane : zb) + (size_t)kGG * grp_xs<N / 8>() * sizeof(float2);
}

// fft_z_kernel<N, SPLIT> for N = 48, 96 with the radix-S x 8 FFT.
template <int N, bool SPLIT>
__global__ void __launch_bounds__(kTG, 2)
fft_z_grp_kernel(ShiftGeom g, float2* __restrict__ T, const float2* __restrict__ what, const float* __restrict__ bg,
                 const float4* __restrict__ refq, const float* __restrict__ rot, const float* __restrict__ ctf,
                 float* __restrict__ nrm, uint32_t* __restrict__ a1, int a1_ws, int a1_R, uint32_t* __restrict__ a1n,
                 int a1n_R) {
  constexpr int S = N / 8, HN = N / 2, H = N / 2 + 1;
  constexpr int XS = grp_xs<S>();
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float red[32];
  float2* tw = sm2;            // N
  float2* buf = sm2 + N;       // N (i') x H
  float2* xs = buf + N * H;    // kGG x XS
  const int jp = blockIdx.x, b = blockIdx.y;
  float2* base = T + (int64_t)b * N * N * H + (int64_t)jp * H;
  const float2* wb = what + (int64_t)jp * H;
  const float avg = g.wsum > 0.f ? __ldg(&bg[b]) / g.wsum : 0.f;
  load_twiddles(tw, N, N);
#pragma unroll 4
  for (int e = threadIdx.x; e < N * H; e += kTG) {
    const int ip = e / H, m2 = e - (e / H) * H;
    const float2 t = base[(int64_t)ip * N * H + m2];
    const float2 w = __ldg(&wb[(int64_t)ip * N * H + m2]);
    buf[ip * H + m2] = make_float2(fmaf(avg, w.x, t.x), fmaf(avg, w.y, t.y));
  }
  __syncthreads();
  {
    const int L = threadIdx.x >> 3, r = threadIdx.x & 7;
    const unsigned gmask = 0xFFu << (threadIdx.x & 24);
    float2* gx = xs + L * XS;
#pragma unroll 1
    for (int col = L; col < H; col += kGG) {
      float2 x[S];
#pragma unroll
      for (int s8 = 0; s8 < S; ++s8) x[s8] = buf[(r + 8 * s8) * H + col];
      float2 o[2][8];
      fft_grp<S>(x, r, gmask, gx, tw, o);
      __syncwarp(gmask);  // the group has read its column: write the transform back
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (r + 8 * j < S) {
#pragma unroll
          for (int k2 = 0; k2 < 8; ++k2) buf[(r + 8 * j + S * k2) * H + col] = o[j][k2];
        }
    }
  }
  __syncthreads();
  float R[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) R[q] = __ldg(&rot[b * 9 + q]);
  const float c = (float)g.h;
  float st = 0.f, ss = 0.f;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * H; e += kTG) {
    const int ip = SPLIT ? e % N : e / H, m2 = SPLIT ? e / N : e % H;
    const float2 t = buf[ip * H + m2];
    const int kp = ip < HN ? ip : ip - N;
    const int jq = jp < HN ? jp : jp - N;
    const int xq = m2 < HN ? m2 : m2 - H;
    // outside the mask the sample is taken far outside the box, which reads zero (entry 0)
    const bool in_mask = kp * kp + jq * jq + xq * xq <= g.mask_r2;
    float2 s;
    {
      const int zo = wrap_n<N>(ip + HN), yo = wrap_n<N>(jp + HN), xw = m2 + HN;
      const float bx = (float)xw - c, by = (float)yo - c, bz = (float)zo - c;
      const float rx = R[0] * bx + R[1] * by + R[2] * bz + c;
      const float ry = R[3] * bx + R[4] * by + R[5] * bz + c;
      const float rz = in_mask ? R[6] * bx + R[7] * by + R[8] * bz + c : -4.f;
      s = trilinear_quad(refq, N, rz, ry, rx);
    }
    if (in_mask && ctf) {
      const float cv = __ldg(&ctf[(((int64_t)b * N + ip) * N + jp) * H + m2]);
      s.x *= cv;
      s.y *= cv;
    }
    st += t.x * t.x + t.y * t.y;
    ss += s.x * s.x + s.y * s.y;
    const float2 p = make_float2(s.x * t.x + s.y * t.y, s.x * t.y - s.y * t.x);
    if (SPLIT) {
      uint32_t hi, lo;
      split_bf16x2(p.x, p.y, hi, lo);
      if (m2 < HN) {
        const size_t row = ((size_t)b * HN + m2) * N + jp;
        a1[row * a1_ws + ip] = hi;
        a1[((size_t)a1_R + row) * a1_ws + ip] = lo;
      } else {
        const size_t row = (size_t)b * N + jp;
        a1n[row * a1_ws + ip] = hi;
        a1n[((size_t)a1n_R + row) * a1_ws + ip] = lo;
      }
    } else {
      base[(int64_t)ip * N * H + m2] = p;
    }
  }
  st = block_sum(st, red);
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    atomicAdd(&nrm[2 * b], st);
    atomicAdd(&nrm[2 * b + 1], ss);
  }
}

template <int N>
constexpr size_t z_grp_smem_bytes() {
  return (size_t)N * sizeof(float2) + (size_t)N * (N / 2 + 1) * sizeof(float2) +
         (size_t)kGG * grp_xs<N / 8>() * sizeof(float2);
}

__global__ void fill_table_kernel(ShiftGeom g, int n, float* __restrict__ tab) {
  const int r2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (r2 < n) tab[r2] = fill_weight(r2, g);
}

// ------------------------------------------------------------------ upsampled DFT, pass 1
// X1[b][u0][m1][m2] = sum_{m0} E0[u0][m0] P[b][m0][m1][m2].  CTA: (column tile of 64, b).
constexpr int kColTile = 64;

__global__ void __launch_bounds__(kT)
updft1_kernel(ShiftGeom g, const float2* __restrict__ P, const float2* __restrict__ E0, float2* __restrict__ X1) {
  extern __shared__ __align__(16) float2 sm2[];
  const int N = g.N, H = g.H, U = g.U;
  const int NC = N * H;
  float2* e0 = sm2;             // U x N
  float2* pt = e0 + U * N;      // N x kColTile
  const int c0 = blockIdx.x * kColTile, b = blockIdx.y;
  const float2* Pb = P + (int64_t)b * N * NC;
  for (int e = threadIdx.x; e < U * N; e += blockDim.x) e0[e] = E0[e];
  for (int e = threadIdx.x; e < N * kColTile; e += blockDim.x) {
    const int m0 = e / kColTile, cc = e % kColTile;
    pt[e] = (c0 + cc < NC) ? Pb[(int64_t)m0 * NC + c0 + cc] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  // thread: column cc = tid % 64, rows u0 = tid / 64 + 4 q
  const int cc = threadIdx.x % kColTile;
  const int r0 = threadIdx.x / kColTile;
  const int nr = blockDim.x / kColTile;
  float2* Xb = X1 + (int64_t)b * U * NC;
  for (int u0 = r0; u0 < U; u0 += nr) {
    float re = 0.f, im = 0.f;
    const float2* er = e0 + u0 * N;
    for (int m0 = 0; m0 < N; ++m0) {
      const float2 w = er[m0], x = pt[m0 * kColTile + cc];
      re += w.x * x.x - w.y * x.y;
      im += w.x * x.y + w.y * x.x;
    }
    if (c0 + cc < NC) Xb[(int64_t)u0 * NC + c0 + cc] = make_float2(re, im);
  }
}

// ------------------------------------------------------------------ passes 2 and 3 + argmax
// For each u0: X2[u1][m2] = sum_{m1} E1[u1][m1] X1[u0][m1][m2];
//              V[u1][u2]  = Re sum_{m2} E2[u2][m2] X2[u1][m2];   running argmax.
__device__ __forceinline__ bool better(float v1, int i1, float v2, int i2) {
  // torch.argmax order: NaN is the largest value, the first index wins ties
  if (isnan(v1) || isnan(v2)) return isnan(v1) && (!isnan(v2) || i1 < i2);
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

// stage_e: the twiddle tables E1, E2 are copied to shared memory; without it (large boxes or
// upsampled regions, whose tables do not fit beside the X1 and X2 slices) they are read from
// global memory through L1.
__global__ void __launch_bounds__(kT)
updft23_kernel(ShiftGeom g, const float2* __restrict__ X1, const float2* __restrict__ E1,
               const float2* __restrict__ E2, int rows_per_cta, int stage_e, float* __restrict__ pval,
               int* __restrict__ pidx) {
  extern __shared__ __align__(16) float2 sm2[];
  __shared__ float rv[32];
  __shared__ int ri[32];
  const int N = g.N, H = g.H, U = g.U;
  const float2* e1 = E1;       // U x N
  const float2* e2 = E2;       // U x H
  float2* x1 = sm2;            // N x H
  if (stage_e) {
    float2* s1 = sm2;
    float2* s2 = s1 + U * N;
    for (int e = threadIdx.x; e < U * N; e += blockDim.x) s1[e] = E1[e];
    for (int e = threadIdx.x; e < U * H; e += blockDim.x) s2[e] = E2[e];
    e1 = s1;
    e2 = s2;
    x1 = s2 + U * H;
  }
  float2* x2 = x1 + N * H;     // U x H
  const int grp = blockIdx.x, b = blockIdx.y;
  float bv = -INFINITY;
  int bi = 0x7fffffff;
  const int u0a = grp * rows_per_cta;
  const int u0b = min(U, u0a + rows_per_cta);
  for (int u0 = u0a; u0 < u0b; ++u0) {
    __syncthreads();
    const float2* src = X1 + ((int64_t)b * U + u0) * N * H;
    for (int e = threadIdx.x; e < N * H; e += blockDim.x) x1[e] = src[e];
    __syncthreads();
    for (int e = threadIdx.x; e < U * H; e += blockDim.x) {
      const int u1 = e / H, m2 = e % H;
      float re = 0.f, im = 0.f;
      const float2* er = e1 + u1 * N;
      for (int m1 = 0; m1 < N; ++m1) {
        const float2 w = er[m1], x = x1[m1 * H + m2];
        re += w.x * x.x - w.y * x.y;
        im += w.x * x.y + w.y * x.x;
      }
      x2[e] = make_float2(re, im);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < U * U; e += blockDim.x) {
      const int u1 = e / U, u2 = e % U;
      float re = 0.f;
      const float2* er = e2 + u2 * H;
      const float2* xr = x2 + u1 * H;
      for (int m2 = 0; m2 < H; ++m2) {
        const float2 w = er[m2], x = xr[m2];
        re += w.x * x.x - w.y * x.y;
      }
      const int flat = (u0 * U + u1) * U + u2;
      if (better(re, flat, bv, bi)) { bv = re; bi = flat; }
    }
  }
  // block argmax
  for (int o = 16; o > 0; o >>= 1) {
    const float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
    if (better(v2, i2, bv, bi)) { bv = v2; bi = i2; }
  }
  if ((threadIdx.x & 31) == 0) { rv[threadIdx.x >> 5] = bv; ri[threadIdx.x >> 5] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float v = rv[0];
    int i = ri[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
      if (better(rv[q], ri[q], v, i)) { v = rv[q]; i = ri[q]; }
    pval[b * gridDim.x + grp] = v;
    pidx[b * gridDim.x + grp] = i;
  }
}

__global__ void finalize_kernel(ShiftGeom g, int B, int ngrp, const float* __restrict__ pval,
                                const int* __restrict__ pidx, const float* __restrict__ nrm,
                                float* __restrict__ shift_xyz, float* __restrict__ score) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float bv = pval[b * ngrp];
  int bi = pidx[b * ngrp];
  for (int q = 1; q < ngrp; ++q)
    if (better(pval[b * ngrp + q], pidx[b * ngrp + q], bv, bi)) { bv = pval[b * ngrp + q]; bi = pidx[b * ngrp + q]; }
  const int U = g.U;
  const int u2 = bi % U, u1 = (bi / U) % U, u0 = bi / (U * U);
  // (dim1, dim2, dim3) = (u0, u1, u2) - dftshift, / uf; returned flipped to (x, y, z)
  shift_xyz[b * 3 + 0] = ((float)u2 - g.dftshift) / g.uf;
  shift_xyz[b * 3 + 1] = ((float)u1 - g.dftshift) / g.uf;
  shift_xyz[b * 3 + 2] = ((float)u0 - g.dftshift) / g.uf;
  const float den = sqrtf(nrm[2 * b]) * sqrtf(nrm[2 * b + 1]);
  score[b] = bv / den;
}

// The shift match's correlation at a continuous shift s and its gradient, from the FP32
// product P = conj(S) T (data axes (z, y, x) = (m0, m1, m2), the last of length N/2+1):
//   c(s) = Re sum_m P[m] exp(2 pi i s . f(m)) / (|T| |S|),  f = (fftfreq(N)[m0],
//   fftfreq(N)[m1], fftfreq(N/2+1)[m2]),
// the function whose values on the grid s = (u - dftshift) / uf the upsampled DFT evaluates
// (ShiftMatcher.py:46-91, with the half axis taken as a full period as there), and
// dc/ds_d = -2 pi sum_m f_d(m) Im(P[m] exp(2 pi i s . f(m))) / (|T| |S|).  One CTA per
// subtomogram; s and the gradient in (x, y, z) order like the shifts the search returns.
__device__ __forceinline__ float fftfreq_of(int m, int n) { return (float)(m <= (n - 1) / 2 ? m : m - n) / (float)n; }

__global__ void __launch_bounds__(256)
shift_score_grad_kernel(ShiftGeom g, const float2* __restrict__ P, const float* __restrict__ nrm,
                        const float* __restrict__ s_xyz, float* __restrict__ score, float* __restrict__ grad_xyz) {
  const int b = blockIdx.x;
  const int N = g.N, H = g.H;
  const int64_t per = (int64_t)N * N * H;
  const float2* p = P + (int64_t)b * per;
  const float sx = s_xyz[3 * b + 0], sy = s_xyz[3 * b + 1], sz = s_xyz[3 * b + 2];
  double v = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  for (int64_t e = threadIdx.x; e < per; e += blockDim.x) {
    const int m0 = (int)(e / ((int64_t)N * H)), m1 = (int)((e / H) % N), m2 = (int)(e % H);
    const float fz = fftfreq_of(m0, N), fy = fftfreq_of(m1, N), fx = fftfreq_of(m2, H);
    float sn, cs;
    sincospif(2.f * (sz * fz + sy * fy + sx * fx), &sn, &cs);
    const float2 q = p[e];
    const float re = q.x * cs - q.y * sn, im = q.x * sn + q.y * cs;
    v += re;
    gx += (double)(fx * im);
    gy += (double)(fy * im);
    gz += (double)(fz * im);
  }
  __shared__ double red[4][256];
  red[0][threadIdx.x] = v;
  red[1][threadIdx.x] = gx;
  red[2][threadIdx.x] = gy;
  red[3][threadIdx.x] = gz;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double den = sqrt((double)nrm[2 * b]) * sqrt((double)nrm[2 * b + 1]);
    const double tp = -2.0 * 3.14159265358979323846 / den;
    score[b] = (float)(red[0][0] / den);
    grad_xyz[3 * b + 0] = (float)(tp * red[1][0]);
    grad_xyz[3 * b + 1] = (float)(tp * red[2][0]);
    grad_xyz[3 * b + 2] = (float)(tp * red[3][0]);
  }
}

// Tensor-core path: decode the per-subtomogram argmax key of the third pass.
__global__ void finalize_tc_kernel(ShiftGeom g, int B, const unsigned long long* __restrict__ best,
                                   const float* __restrict__ nrm, float* __restrict__ shift_xyz,
                                   float* __restrict__ score) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const unsigned long long key = best[b];
  uint32_t vb = (uint32_t)(key >> 32);
  vb = (vb & 0x80000000u) ? (vb & 0x7FFFFFFFu) : ~vb;
  const float bv = __uint_as_float(vb);
  const int bi = (int)(0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFull));
  const int U = g.U;
  const int u2 = bi % U, u1 = (bi / U) % U, u0 = bi / (U * U);
  shift_xyz[b * 3 + 0] = ((float)u2 - g.dftshift) / g.uf;
  shift_xyz[b * 3 + 1] = ((float)u1 - g.dftshift) / g.uf;
  shift_xyz[b * 3 + 2] = ((float)u0 - g.dftshift) / g.uf;
  score[b] = bv / (sqrtf(nrm[2 * b]) * sqrtf(nrm[2 * b + 1]));
}

}  // namespace

struct mtb_shift {
  mtb_shift_config cfg;
  ShiftGeom g;
  float* bgw_tab;  // background weight by integer squared radius, 0 .. 3 (N/2)^2
  float* fill_tab; // fill weight W by integer squared radius (device formula)
  float2* what;    // (N, N, N/2+1) plane transforms of the fill weight W / N^3
  float2* ref;     // (N, N, N) Fourier reference, fftshifted and masked
  float4* refq;    // boxes 48, 64, 96, 128: corner quads of ref, (N + 2) (N + 1)^2 x 32 bytes
  float2* E0;      // (U, N)
  float2* E1;      // (U, N)
  float2* E2;      // (U, H)
  float* bg;       // (max_batch)
  float* nrm;      // (max_batch, 2)
  float2* T;       // (max_batch, N, N, H)
  float2* X1;      // (max_batch, U, N, H)
  float* pval;     // (max_batch, ngrp)
  int* pidx;
  int ngrp, rows_per_cta;
  bool has_ref;
  ShiftTc tc;
  bool use_tc;
  // launch profile: kProfMarks events per call in a ring of prof_cap calls
  int prof_cap, prof_n;
  std::vector<cudaEvent_t>* prof_ev;
};

namespace {
constexpr int kProfMarks = 7;  // start, after xy, after z, after Nyquist, after pass 1, after passes 2+3, end

void prof_mark(mtb_shift* h, int k, cudaStream_t st) {
  if (h->prof_cap > 0) cudaEventRecord((*h->prof_ev)[(h->prof_n % h->prof_cap) * kProfMarks + k], st);
}
}  // namespace

// The front of the pipeline for box size N: with B > 0 the patch / xy-FFT and the z-FFT +
// product of B subtomograms (into T, or into the tensor-core operand A1); with B == 0 the
// plane transforms of the background fill weight, once per geometry, into h->what.
template <int N>
int shift_front_n(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot, const float* ctf,
                  int B, cudaStream_t st, bool split, int phases = 3) {
  const ShiftGeom& g = h->g;
  const int sxy = (int)xy_smem_bytes<N>(), sz = (int)z_smem_bytes<N>();
  if (B == 0) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(patch_fft_xy_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sxy));
    patch_fft_xy_kernel<N, true><<<dim3(N, 1), kT, sxy, st>>>(nullptr, nullptr, nullptr, g, h->what, nullptr);
    MTB_LAUNCH_CHECK();
    return MTB_OK;
  }
  if (phases & 1) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(patch_fft_xy_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sxy));
    mtb_prof_begin(st);
    patch_fft_xy_kernel<N, false><<<dim3(N, B), kT, sxy, st>>>(subtomos, shift_zyx, h->bgw_tab, g, h->T, h->bg);
    mtb_prof_end(st, "patch_fft_xy_kernel");
    MTB_LAUNCH_CHECK();
    prof_mark(h, 1, st);
  }
  if (phases & 2) {
    if (split) {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z_kernel<N, true><<<dim3(N, B), kT, sz, st>>>(g, h->T, h->what, h->bg, h->ref, rot, ctf, h->nrm,
                                                         (uint32_t*)h->tc.A1, h->tc.KB12 * 32, h->tc.R1, (uint32_t*)h->tc.A1n,
          h->tc.R1n);
      mtb_prof_end(st, "fft_z_kernel");
    } else {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z_kernel<N, false><<<dim3(N, B), kT, sz, st>>>(g, h->T, h->what, h->bg, h->ref, rot, ctf, h->nrm, nullptr,
                                                          0, 0, nullptr, 0);
      mtb_prof_end(st, "fft_z_kernel");
    }
    MTB_LAUNCH_CHECK();
  }
  return MTB_OK;
}

int shift_front_64(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot, const float* ctf,
                   int B, cudaStream_t st, bool split, int phases = 3) {
  const ShiftGeom& g = h->g;
  const int sxy = (int)xy64_smem_bytes(), sz = (int)z64_smem_bytes();
  if (phases & 1) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(patch_fft_xy64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sxy));
    mtb_prof_begin(st);
    patch_fft_xy64_kernel<<<dim3(64, B), kT64, sxy, st>>>(subtomos, shift_zyx, h->bgw_tab, h->fill_tab, g, h->T, h->bg);
    mtb_prof_end(st, "patch_fft_xy64_kernel");
    MTB_LAUNCH_CHECK();
    prof_mark(h, 1, st);
  }
  if (phases & 2) {
    if (split) {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z64_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z64_kernel<true><<<dim3(64, B), kT64, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm,
                                                           (uint32_t*)h->tc.A1, h->tc.KB12 * 32, h->tc.R1, (uint32_t*)h->tc.A1n,
          h->tc.R1n);
      mtb_prof_end(st, "fft_z64_kernel");
    } else {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z64_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z64_kernel<false><<<dim3(64, B), kT64, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm, nullptr,
                                                            0, 0, nullptr, 0);
      mtb_prof_end(st, "fft_z64_kernel");
    }
    MTB_LAUNCH_CHECK();
  }
  return MTB_OK;
}

int shift_front_128(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot, const float* ctf,
                    int B, cudaStream_t st, bool split, int phases = 3) {
  const ShiftGeom& g = h->g;
  const int sxy = (int)xy128_smem_bytes(), sz = (int)z128_smem_bytes();
  if (phases & 1) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(patch_fft_xy128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sxy));
    mtb_prof_begin(st);
    patch_fft_xy128_kernel<<<dim3(128, B), kT128, sxy, st>>>(subtomos, shift_zyx, h->bgw_tab, h->fill_tab, g, h->T,
                                                              h->bg);
    mtb_prof_end(st, "patch_fft_xy128_kernel");
    MTB_LAUNCH_CHECK();
    prof_mark(h, 1, st);
  }
  if (phases & 2) {
    if (split) {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z128_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z128_kernel<true><<<dim3(128, B), kT128, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm,
                                                              (uint32_t*)h->tc.A1, h->tc.KB12 * 32, h->tc.R1,
                                                              (uint32_t*)h->tc.A1n, h->tc.R1n);
      mtb_prof_end(st, "fft_z128_kernel");
    } else {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z128_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z128_kernel<false><<<dim3(128, B), kT128, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm,
                                                               nullptr, 0, 0, nullptr, 0);
      mtb_prof_end(st, "fft_z128_kernel");
    }
    MTB_LAUNCH_CHECK();
  }
  return MTB_OK;
}

template <int N>
int shift_front_grp(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot, const float* ctf,
                    int B, cudaStream_t st, bool split, int phases = 3) {
  const ShiftGeom& g = h->g;
  const int sxy = (int)xy_grp_smem_bytes<N>(), sz = (int)z_grp_smem_bytes<N>();
  if (phases & 1) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(patch_fft_xy_grp_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, sxy));
    mtb_prof_begin(st);
    patch_fft_xy_grp_kernel<N><<<dim3(N, B), kTG, sxy, st>>>(subtomos, shift_zyx, h->bgw_tab, h->fill_tab, g, h->T,
                                                              h->bg);
    mtb_prof_end(st, "patch_fft_xy_grp_kernel");
    MTB_LAUNCH_CHECK();
    prof_mark(h, 1, st);
  }
  if (phases & 2) {
    if (split) {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z_grp_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z_grp_kernel<N, true><<<dim3(N, B), kTG, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm,
                                                              (uint32_t*)h->tc.A1, h->tc.KB12 * 32, h->tc.R1,
                                                              (uint32_t*)h->tc.A1n, h->tc.R1n);
      mtb_prof_end(st, "fft_z_grp_kernel");
    } else {
      MTB_CUDA_TRY(cudaFuncSetAttribute(fft_z_grp_kernel<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
      mtb_prof_begin(st);
      fft_z_grp_kernel<N, false><<<dim3(N, B), kTG, sz, st>>>(g, h->T, h->what, h->bg, h->refq, rot, ctf, h->nrm,
                                                               nullptr, 0, 0, nullptr, 0);
      mtb_prof_end(st, "fft_z_grp_kernel");
    }
    MTB_LAUNCH_CHECK();
  }
  return MTB_OK;
}

// split: the z pass writes the tensor-core pass-1 operand (A1) instead of the FP32 product in T.
// phases: bit 0 the patch and x/y transforms (independent of the orientation), bit 1 the z
// pass with the rotated reference (B > 0; B == 0 computes the fill weight's transforms).
int shift_front(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot, const float* ctf,
                int B, cudaStream_t st, bool split, int phases = 3) {
  switch (h->g.N) {
    case 4: return shift_front_n<4>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 8: return shift_front_n<8>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 16: return shift_front_n<16>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 32: return shift_front_n<32>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 64: return B > 0 ? shift_front_64(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases)
                          : shift_front_n<64>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 128: return B > 0 ? shift_front_128(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases)
                           : shift_front_n<128>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 48: return B > 0 ? shift_front_grp<48>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases)
                          : shift_front_n<48>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 80: return shift_front_n<80>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    case 96: return B > 0 ? shift_front_grp<96>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases)
                          : shift_front_n<96>(h, subtomos, shift_zyx, rot, ctf, B, st, split, phases);
    default: MTB_ARG_CHECK(false, "N must be a power of two in [4, 128] or 48, 80, 96");
  }
}

extern "C" int mtb_shift_create(const mtb_shift_config* cfg, mtb_shift** out) {
  MTB_ARG_CHECK(cfg && out, "null argument");
  *out = nullptr;
  const int N = cfg->N;
  MTB_ARG_CHECK((N >= 4 && N <= 128 && (N & (N - 1)) == 0) || N == 48 || N == 80 || N == 96,
                "N must be a power of two in [4, 128] or 48, 80, 96");
  MTB_ARG_CHECK(cfg->max_batch >= 1 && cfg->max_batch <= 65535, "max_batch out of range");
  MTB_ARG_CHECK(cfg->upsample_factor >= 2 && cfg->search_radius >= 0, "upsample_factor must be > 1");
  MTB_ARG_CHECK(cfg->cosine_width > 0.f, "cosine_width must be positive");
  MTB_ARG_CHECK(cfg->tile_rows >= 0 && cfg->tile_rows <= 32, "tile_rows must be in [0, 32]");
  MTB_ARG_CHECK(cfg->precision == MTB_SHIFT_FP32 || cfg->precision == MTB_SHIFT_BF16X3 ||
                    cfg->precision == MTB_SHIFT_AUTO,
                "precision must be MTB_SHIFT_FP32, MTB_SHIFT_BF16X3 or MTB_SHIFT_AUTO");
  {
    const int U = (int)ceil((double)cfg->upsample_factor * (2 * cfg->search_radius + 1));
    MTB_ARG_CHECK(cfg->precision != MTB_SHIFT_BF16X3 || shift_tc_fits(N, U) == MTB_OK,
                  "MTB_SHIFT_BF16X3: the tensor-core kernels do not cover this box and upsampled region "
                  "(MTB_SHIFT_AUTO falls back to FP32 there)");
  }
  mtb_shift* h = new mtb_shift();
  memset(h, 0, sizeof(*h));
  h->cfg = *cfg;
  ShiftGeom& g = h->g;
  g.N = N;
  g.H = N / 2 + 1;
  g.h = N / 2;
  const int window = 2 * cfg->search_radius + 1;
  g.U = (int)ceil((double)cfg->upsample_factor * window);
  g.uf = (float)cfg->upsample_factor;
  g.dftshift = floorf(g.U / 2.f);
  g.inv_n3 = 1.f / ((float)N * N * N);
  double radius = cfg->mask_radius;
  if (radius < 0) radius = N / 2.0;
  const double rp = radius + cfg->cosine_width;
  g.rp = (float)rp;
  g.width = cfg->cosine_width;
  g.mask_r2 = (N / 2) * (N / 2);
  // background voxels: r > rp (weight 1) and radius <= r <= rp (raised cosine); the weight
  // depends on the integer squared radius only
  const int r2max = 3 * (N / 2) * (N / 2);
  std::vector<float> wtab(r2max + 1, 0.f);
  for (int r2 = 0; r2 <= r2max; ++r2) {
    const double r = sqrt((double)r2);
    if (r > rp) wtab[r2] = 1.f;
    else if (!(r < radius)) wtab[r2] = (float)(0.5 + 0.5 * cos(M_PI * (rp - r) / cfg->cosine_width));
  }
  double wsum = 0.0;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const int di = i - N / 2, dj = j - N / 2, dk = k - N / 2;
        wsum += wtab[di * di + dj * dj + dk * dk];
      }
  // same sets by integer squared radius: outer r2 > floor(rp^2); band r2 >= ceil(radius^2)
  const int r2_outer = (int)floor(rp * rp);
  const int r2_inner = (int)ceil(radius * radius);
  g.r2_inner = r2_inner;
  g.r2_outer = r2_outer;
  g.wsum = (float)wsum;
  // DFT kernels exp(+2 pi i (u - dftshift) f_m), f = fftfreq(n, d=uf)
  auto kern = [&](int n, std::vector<float2>& E) {
    E.resize((size_t)g.U * n);
    for (int u = 0; u < g.U; ++u)
      for (int m = 0; m < n; ++m) {
        const int mm = (m < (n + 1) / 2) ? m : m - n;
        const double f = (double)mm / ((double)cfg->upsample_factor * n);
        const double ph = 2.0 * M_PI * ((double)u - g.dftshift) * f;
        E[(size_t)u * n + m] = make_float2((float)cos(ph), (float)sin(ph));
      }
  };
  std::vector<float2> e0, e2;
  kern(N, e0);
  kern(g.H, e2);
  h->rows_per_cta = cfg->tile_rows > 0 ? cfg->tile_rows : 2;
  h->ngrp = (g.U + h->rows_per_cta - 1) / h->rows_per_cta;
  const size_t B = cfg->max_batch;
  // MTB_SHIFT_BF16X3 was checked to fit the tensor-core kernels above; MTB_SHIFT_AUTO uses them
  // where they fit and the FP32 CUDA-core kernels elsewhere
  const bool want_tc = cfg->precision != MTB_SHIFT_FP32 && shift_tc_fits(N, g.U) == MTB_OK;
  auto fail = [&](int code) { mtb_shift_destroy(h); return code; };
  auto alloc = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes > 0 ? bytes : 4) == cudaSuccess; };
  if (!alloc((void**)&h->bgw_tab, wtab.size() * 4) || !alloc((void**)&h->fill_tab, wtab.size() * 4) || !alloc((void**)&h->what, (size_t)N * N * g.H * 8) ||
      !alloc((void**)&h->ref, (size_t)N * N * N * 8) || !alloc((void**)&h->E0, e0.size() * 8) ||
      !alloc((void**)&h->E1, e0.size() * 8) || !alloc((void**)&h->E2, e2.size() * 8) ||
      !alloc((void**)&h->bg, B * 4) || !alloc((void**)&h->nrm, B * 8) ||
      !alloc((void**)&h->T, B * N * N * g.H * 8))
    return fail(MTB_ERR_OOM);
  // the FP32 upsampled DFT's pass-1 output and per-group maxima (its kernels only)
  if (!want_tc && (!alloc((void**)&h->X1, B * g.U * N * g.H * 8) || !alloc((void**)&h->pval, B * h->ngrp * 4) ||
                   !alloc((void**)&h->pidx, B * h->ngrp * 4)))
    return fail(MTB_ERR_OOM);
  if ((N == 48 || N == 64 || N == 96 || N == 128) &&
      !alloc((void**)&h->refq, (size_t)(N + 2) * (N + 1) * (N + 1) * 32))
    return fail(MTB_ERR_OOM);
  if (cudaMemcpy(h->bgw_tab, wtab.data(), wtab.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->E0, e0.data(), e0.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->E1, e0.data(), e0.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->E2, e2.data(), e2.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(MTB_ERR_CUDA);
  fill_table_kernel<<<(r2max + 256) / 256, 256>>>(g, r2max + 1, h->fill_tab);
  if (cudaGetLastError() != cudaSuccess) return fail(MTB_ERR_CUDA);
  if (shift_front(h, nullptr, nullptr, nullptr, nullptr, 0, 0, false) != MTB_OK) return fail(MTB_ERR_CUDA);
  if (cudaStreamSynchronize(0) != cudaSuccess) return fail(MTB_ERR_CUDA);
  if (want_tc) {
    const int rc = shift_tc_prepare(&h->tc, N, g.H, g.U, cfg->upsample_factor, g.dftshift, cfg->max_batch);
    if (rc) return fail(rc);
    h->use_tc = true;
  }
  *out = h;
  return MTB_OK;
}

extern "C" void mtb_shift_destroy(mtb_shift* h) {
  if (!h) return;
  mtb_shift_profile(h, 0);
  shift_tc_release(&h->tc);
  void* ptrs[] = {h->bgw_tab, h->fill_tab, h->what, h->refq, h->ref, h->E0, h->E1, h->E2, h->bg, h->nrm, h->T, h->X1, h->pval, h->pidx};
  for (void* p : ptrs) if (p) cudaFree(p);
  delete h;
}

extern "C" int mtb_shift_precision(const mtb_shift* h, int* precision) {
  MTB_ARG_CHECK(h && precision, "null argument");
  *precision = h->use_tc ? MTB_SHIFT_BF16X3 : MTB_SHIFT_FP32;
  return MTB_OK;
}

extern "C" int mtb_shift_status(mtb_shift* h, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  if (!h->use_tc) {
    MTB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return MTB_OK;
  }
  int site = 0;
  const int rc = shift_tc_check(&h->tc, (cudaStream_t)stream, &site);
  if (rc == MTB_ERR_TIMEOUT) {
    char msg[96];
    snprintf(msg, sizeof(msg), "tensor-core shift DFT: a bounded wait ran out (wait site %d)", site);
    mtb_set_last_error(msg, __FILE__, __LINE__);
  }
  return rc;
}

extern "C" int mtb_shift_set_reference(mtb_shift* h, const float* ref_fourier, mtb_stream_t stream) {
  MTB_ARG_CHECK(h && ref_fourier, "null argument");
  const size_t n = (size_t)h->g.N * h->g.N * h->g.N;
  MTB_CUDA_TRY(cudaMemcpyAsync(h->ref, ref_fourier, n * 8, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  if (h->refq) {
    ref_quad_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(h->ref, h->g.N, h->refq);
    MTB_LAUNCH_CHECK();
  }
  h->has_ref = true;
  return MTB_OK;
}

extern "C" int mtb_shift_search(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot,
                                const float* ctf, int B, float* shift_xyz, float* score, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(h->has_ref, "shift reference is not set");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(subtomos && shift_zyx && rot && shift_xyz && score, "null pointer");
  int rc = mtb_shift_begin(h, subtomos, shift_zyx, B, stream);
  if (rc) return rc;
  return mtb_shift_finish(h, rot, ctf, B, shift_xyz, score, stream);
}

extern "C" int mtb_shift_begin(mtb_shift* h, const float* subtomos, const float* shift_zyx, int B,
                               mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(subtomos && shift_zyx, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  MTB_CUDA_TRY(cudaMemsetAsync(h->bg, 0, (size_t)B * 4, st));
  MTB_CUDA_TRY(cudaMemsetAsync(h->nrm, 0, (size_t)B * 8, st));
  prof_mark(h, 0, st);
  return shift_front(h, subtomos, shift_zyx, nullptr, nullptr, B, st, h->use_tc, 1);
}

extern "C" int mtb_shift_finish(mtb_shift* h, const float* rot, const float* ctf, int B, float* shift_xyz,
                                float* score, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(h->has_ref, "shift reference is not set");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(rot && shift_xyz && score, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const ShiftGeom& g = h->g;
  const int N = g.N, H = g.H, U = g.U;
  int rc = shift_front(h, nullptr, nullptr, rot, ctf, B, st, h->use_tc, 2);
  if (rc) return rc;
  prof_mark(h, 2, st);
  if (h->use_tc) {
    cudaEvent_t marks[3] = {nullptr, nullptr, nullptr};
    if (h->prof_cap > 0)
      for (int k = 0; k < 3; ++k) marks[k] = (*h->prof_ev)[(h->prof_n % h->prof_cap) * kProfMarks + 3 + k];
    rc = shift_tc_passes(&h->tc, B, st, marks);
    if (rc) return rc;
    mtb_prof_begin(st);
    finalize_tc_kernel<<<(B + 127) / 128, 128, 0, st>>>(g, B, h->tc.best, h->nrm, shift_xyz, score);
    mtb_prof_end(st, "finalize_tc_kernel");
    MTB_LAUNCH_CHECK();
    prof_mark(h, 6, st);
    if (h->prof_cap > 0) ++h->prof_n;
    return MTB_OK;
  }
  const size_t sm1 = (size_t)(U * N + N * kColTile) * 8;
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
  prof_mark(h, 3, st);
  mtb_prof_begin(st);
  updft1_kernel<<<dim3((N * H + kColTile - 1) / kColTile, B), kT, sm1, st>>>(g, h->T, h->E0, h->X1);
  mtb_prof_end(st, "updft1_kernel");
  MTB_LAUNCH_CHECK();
  prof_mark(h, 4, st);
  const size_t sm2_staged = (size_t)(U * N + U * H + N * H + U * H) * 8;
  const int stage_e = sm2_staged <= 220 * 1024;
  const size_t sm2 = stage_e ? sm2_staged : (size_t)(N * H + U * H) * 8;
  MTB_ARG_CHECK(sm2 <= 220 * 1024 && sm1 <= 220 * 1024, "upsampled region too large for shared memory");
  MTB_CUDA_TRY(cudaFuncSetAttribute(updft23_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
  mtb_prof_begin(st);
  updft23_kernel<<<dim3(h->ngrp, B), kT, sm2, st>>>(g, h->X1, h->E1, h->E2, h->rows_per_cta, stage_e, h->pval,
                                                    h->pidx);
  mtb_prof_end(st, "updft23_kernel");
  MTB_LAUNCH_CHECK();
  prof_mark(h, 5, st);
  mtb_prof_begin(st);
  finalize_kernel<<<(B + 127) / 128, 128, 0, st>>>(g, B, h->ngrp, h->pval, h->pidx, h->nrm, shift_xyz, score);
  mtb_prof_end(st, "finalize_kernel");
  MTB_LAUNCH_CHECK();
  prof_mark(h, 6, st);
  if (h->prof_cap > 0) ++h->prof_n;
  return MTB_OK;
}

extern "C" int mtb_shift_score_grad(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot,
                                    const float* ctf, int B, const float* query_xyz, float* score, float* grad_xyz,
                                    mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(h->has_ref, "shift reference is not set");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(subtomos && shift_zyx && rot && query_xyz && score && grad_xyz, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  MTB_CUDA_TRY(cudaMemsetAsync(h->bg, 0, (size_t)B * 4, st));
  MTB_CUDA_TRY(cudaMemsetAsync(h->nrm, 0, (size_t)B * 8, st));
  // the FP32 product in T, whatever the handle's precision
  if (int rc = shift_front(h, subtomos, shift_zyx, rot, ctf, B, st, false)) return rc;
  mtb_prof_begin(st);
  shift_score_grad_kernel<<<B, 256, 0, st>>>(h->g, reinterpret_cast<const float2*>(h->T), h->nrm, query_xyz, score,
                                             grad_xyz);
  mtb_prof_end(st, "shift_score_grad_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

extern "C" int mtb_shift_profile(mtb_shift* h, int n_calls) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(n_calls >= 0 && n_calls <= 4096, "n_calls must be in [0, 4096]");
  if (h->prof_ev) {
    for (cudaEvent_t e : *h->prof_ev) cudaEventDestroy(e);
    delete h->prof_ev;
    h->prof_ev = nullptr;
  }
  h->prof_cap = 0;
  h->prof_n = 0;
  if (n_calls == 0) return MTB_OK;
  h->prof_ev = new std::vector<cudaEvent_t>((size_t)n_calls * kProfMarks, nullptr);
  for (auto& e : *h->prof_ev) MTB_CUDA_TRY(cudaEventCreate(&e));
  h->prof_cap = n_calls;
  return MTB_OK;
}

extern "C" int mtb_shift_profile_read(mtb_shift* h, float* ms, int* calls) {
  MTB_ARG_CHECK(h && ms && calls, "null argument");
  for (int k = 0; k < kProfMarks - 1; ++k) ms[k] = 0.f;
  *calls = 0;
  if (h->prof_cap == 0 || h->prof_n == 0) return MTB_OK;
  const int n = h->prof_n < h->prof_cap ? h->prof_n : h->prof_cap;
  for (int c = 0; c < n; ++c) {
    cudaEvent_t* e = h->prof_ev->data() + (size_t)c * kProfMarks;
    MTB_CUDA_TRY(cudaEventSynchronize(e[kProfMarks - 1]));
    for (int k = 0; k < kProfMarks - 1; ++k) {
      float t = 0.f;
      MTB_CUDA_TRY(cudaEventElapsedTime(&t, e[k], e[k + 1]));
      ms[k] += t;
    }
  }
  *calls = n;
  return MTB_OK;
}

// ------------------------------------------------------------------ rotation tracker update
// update_rotation_estimate (src/matcha/utils/rotation_ops.py:23-34) followed by the
// rotation the shift match uses, R.from_euler('ZYZ', euler(conj(tracker))) (ShiftMatcher.py:503,
// :913), which is the rotation matrix of conj(tracker).  FP64 quaternion arithmetic.
namespace {
// Rotation matrix (row major) of conj(q) for a unit quaternion q = (w, x, y, z): the matrix
// scipy's from_euler('ZYZ', degrees) gives for the Euler angles of the conjugated tracker
// (ShiftMatcher.py:503, :913).
__device__ __forceinline__ void conj_rotation(double w, double x, double y, double z, float* R) {
  const double cw = w, cx = -x, cy = -y, cz = -z;
  R[0] = (float)(1 - 2 * (cy * cy + cz * cz)); R[1] = (float)(2 * (cx * cy - cw * cz)); R[2] = (float)(2 * (cx * cz + cw * cy));
  R[3] = (float)(2 * (cx * cy + cw * cz)); R[4] = (float)(1 - 2 * (cx * cx + cz * cz)); R[5] = (float)(2 * (cy * cz - cw * cx));
  R[6] = (float)(2 * (cx * cz - cw * cy)); R[7] = (float)(2 * (cy * cz + cw * cx)); R[8] = (float)(1 - 2 * (cx * cx + cy * cy));
}

__global__ void tracker_update_kernel(const float* __restrict__ alpha, const float* __restrict__ beta,
                                      const float* __restrict__ gamma, const double* __restrict__ tin, int B,
                                      double* __restrict__ tout, float* __restrict__ rot) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const double a = alpha[b], be = beta[b], g = gamma[b];
  double sb, cb, sp, cp, sm, cm;
  sincos(0.5 * be, &sb, &cb);
  sincos(0.5 * (a + g), &sp, &cp);
  sincos(0.5 * (a - g), &sm, &cm);
  // quaternionic.array.from_euler_angles: exp(a z/2) exp(b y/2) exp(g z/2)
  const double w = cb * cp, x = -sb * sm, y = sb * cm, z = cb * sp;
  // components 1 and 3 swapped, then conjugated
  const double qw = w, qx = -z, qy = -y, qz = -x;
  const double tw = tin[4 * b], tx = tin[4 * b + 1], ty = tin[4 * b + 2], tz = tin[4 * b + 3];
  double nw = tw * qw - tx * qx - ty * qy - tz * qz;
  double nx = tw * qx + tx * qw + ty * qz - tz * qy;
  double ny = tw * qy - tx * qz + ty * qw + tz * qx;
  double nz = tw * qz + tx * qy - ty * qx + tz * qw;
  const double inv = 1.0 / sqrt(nw * nw + nx * nx + ny * ny + nz * nz);
  nw *= inv; nx *= inv; ny *= inv; nz *= inv;
  tout[4 * b] = nw; tout[4 * b + 1] = nx; tout[4 * b + 2] = ny; tout[4 * b + 3] = nz;
  conj_rotation(nw, nx, ny, nz, rot + 9 * b);
}

__global__ void tracker_rotation_kernel(const double* __restrict__ tracker, int B, float* __restrict__ rot) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const double w = tracker[4 * b], x = tracker[4 * b + 1], y = tracker[4 * b + 2], z = tracker[4 * b + 3];
  const double inv = 1.0 / sqrt(w * w + x * x + y * y + z * z);
  conj_rotation(w * inv, x * inv, y * inv, z * inv, rot + 9 * b);
}
}  // namespace

extern "C" int mtb_update_rotation(const float* alpha, const float* beta, const float* gamma, const double* tracker_in,
                                   int B, double* tracker_out, float* rot, mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0, "negative batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(alpha && beta && gamma && tracker_in && tracker_out && rot, "null pointer");
  mtb_prof_begin((cudaStream_t)stream);
  tracker_update_kernel<<<(B + 127) / 128, 128, 0, (cudaStream_t)stream>>>(alpha, beta, gamma, tracker_in, B,
                                                                            tracker_out, rot);
  mtb_prof_end((cudaStream_t)stream, "tracker_update_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

extern "C" int mtb_tracker_rotation(const double* tracker, int B, float* rot, mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0, "negative batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(tracker && rot, "null pointer");
  mtb_prof_begin((cudaStream_t)stream);
  tracker_rotation_kernel<<<(B + 127) / 128, 128, 0, (cudaStream_t)stream>>>(tracker, B, rot);
  mtb_prof_end((cudaStream_t)stream, "tracker_rotation_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}
