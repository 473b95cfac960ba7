// Subtomogram preparation before the ball expansion, in every alternation: the patch at the
// current shift, normalised inside a spherical mask and masked, then rotated into the
// current orientation estimate.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   BatchProcessor._extract_rotated_batch   src/matcha/align_subtomograms.py:240-252
//   extract_subtomogram_patch_batch         src/matcha/utils/io_utils.py:113-178 (normalize=True)
//   normalise / mean / std                  src/matcha/utils/volume_ops.py:17-35
//   spherical mask (distance < radius)      src/matcha/utils/volume_ops.py:6-14, setup_utils.py:274-281
//   rotate_volumes_in_batches               src/matcha/utils/volume_rotation.py:49-125
//
// Both resamplings are grid_sample(mode='bilinear', align_corners=True, zero padding) in 3-D:
// corner weights (x part)(y part)(z part), corners outside the box skipped.
//
// extract_kernel: CTA = (output plane z, subtomogram b).  The sample coordinate of each axis
// depends on that axis alone (voxel + shift through the reference's normalised-grid round trip
// 2 g / (N - 1) - 1, then ((u + 1) / 2) (N - 1)): a thread keeps one column x and its axis in
// registers and walks rows, reading each row's axis from a table the CTA fills once, so the
// eight corner loads of a warp are two runs of consecutive words.  It writes the patch and
// adds the masked sum and sum of squares of its plane to the subtomogram's FP64 statistics.
//
// rotate_kernel: CTA = (output plane z, subtomogram b), a warp = an 8 x 4 patch of the plane.
// The sample point of output voxel v is R (v - c) + c (c = N / 2, the centre of the odd-padded
// linspace(-1, 1) grid), so |s - c| = |v - c|: voxels farther than radius + 2 from c read only
// masked-out corners and are written as zero without loads, voxels nearer than radius - 2
// read only corners inside the mask, and only the shell between tests the mask per corner.
// Values are normalised as they are read: (p - mean) / std inside the mask, 0 outside.
#include <math.h>
#include "common.cuh"

namespace {

constexpr int kPT = 256;

struct Axis {
  int i0;        // lower corner index
  float w0, w1;  // weights of corners i0 and i0 + 1
  bool v0, v1;   // corners inside [0, N)
};

// One axis of the patch sampling: voxel g shifted by s, through the reference's round trip.
__device__ __forceinline__ Axis patch_axis(int g, float s, int N) {
  const float size = (float)(N - 1);
  const float n = 2.f * ((float)g + s) / size - 1.f;
  float u = ((n + 1.f) / 2.f) * size;
  u = fminf(fmaxf(u, -2.f), (float)N + 1.f);  // beyond this every corner is outside the box
  const float f = floorf(u);
  Axis a;
  a.i0 = (int)f;
  a.w1 = u - f;
  a.w0 = (f + 1.f) - u;
  a.v0 = a.i0 >= 0 && a.i0 < N;
  a.v1 = a.i0 + 1 >= 0 && a.i0 + 1 < N;
  return a;
}

__device__ __forceinline__ double block_sum_d(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;
}

template <int NT>
__global__ void __launch_bounds__(kPT) extract_kernel(const float* __restrict__ vol, int n_rt,
                                                      const float* __restrict__ shift_xyz, int thresh,
                                                      float* __restrict__ patch, double* __restrict__ stats) {
  const int N = NT ? NT : n_rt;
  __shared__ double red[kPT / 32];
  extern __shared__ Axis s_y[];  // the y axis of every row (N entries)
  const int z = blockIdx.x, b = blockIdx.y;
  const int64_t NN = (int64_t)N * N;
  const float* v = vol + (int64_t)b * NN * N;
  float* out = patch + ((int64_t)b * N + z) * NN;
  const float sx = shift_xyz[3 * b], sy = shift_xyz[3 * b + 1], sz = shift_xyz[3 * b + 2];
  for (int y = threadIdx.x; y < N; y += kPT) s_y[y] = patch_axis(y, sy, N);
  __syncthreads();
  const Axis az = patch_axis(z, sz, N);
  const float* p0 = v + (int64_t)az.i0 * NN;  // planes iz0 and iz0 + 1 (dereferenced only when inside)
  const float* p1 = p0 + NN;
  const int c = N / 2;
  const int dz2 = (z - c) * (z - c);
  const int TXW = N < kPT ? N : kPT, RP = kPT / TXW;
  const int xi = threadIdx.x % TXW, yi = threadIdx.x / TXW;
  float s1 = 0.f, s2 = 0.f;
  if (yi < RP) {
    for (int x = xi; x < N; x += TXW) {
      const Axis ax = patch_axis(x, sx, N);
      const int dx2 = (x - c) * (x - c);
      for (int y = yi; y < N; y += RP) {
        const Axis ay = s_y[y];
        const int64_t r0 = (int64_t)ay.i0 * N + ax.i0, r1 = r0 + N;
        const bool q00 = az.v0 && ay.v0, q01 = az.v0 && ay.v1, q10 = az.v1 && ay.v0, q11 = az.v1 && ay.v1;
        const float c000 = (q00 && ax.v0) ? __ldg(p0 + r0) : 0.f, c001 = (q00 && ax.v1) ? __ldg(p0 + r0 + 1) : 0.f;
        const float c010 = (q01 && ax.v0) ? __ldg(p0 + r1) : 0.f, c011 = (q01 && ax.v1) ? __ldg(p0 + r1 + 1) : 0.f;
        const float c100 = (q10 && ax.v0) ? __ldg(p1 + r0) : 0.f, c101 = (q10 && ax.v1) ? __ldg(p1 + r0 + 1) : 0.f;
        const float c110 = (q11 && ax.v0) ? __ldg(p1 + r1) : 0.f, c111 = (q11 && ax.v1) ? __ldg(p1 + r1 + 1) : 0.f;
        const float w00 = ax.w0 * ay.w0, w01 = ax.w1 * ay.w0, w10 = ax.w0 * ay.w1, w11 = ax.w1 * ay.w1;
        float p = c000 * (w00 * az.w0);
        p = fmaf(c001, w01 * az.w0, p);
        p = fmaf(c010, w10 * az.w0, p);
        p = fmaf(c011, w11 * az.w0, p);
        p = fmaf(c100, w00 * az.w1, p);
        p = fmaf(c101, w01 * az.w1, p);
        p = fmaf(c110, w10 * az.w1, p);
        p = fmaf(c111, w11 * az.w1, p);
        out[(int64_t)y * N + x] = p;
        if (dz2 + (y - c) * (y - c) + dx2 < thresh) {
          s1 += p;
          s2 = fmaf(p, p, s2);
        }
      }
    }
  }
  const double t1 = block_sum_d((double)s1, red);
  const double t2 = block_sum_d((double)s2, red);
  if (threadIdx.x == 0) {
    atomicAdd(&stats[2 * b], t1);
    atomicAdd(&stats[2 * b + 1], t2);
  }
}

// BOX: the mask reaches outside the box, so a corner inside the mask may still be outside it.
template <int NT, bool BOX>
__global__ void __launch_bounds__(kPT) rotate_kernel(const float* __restrict__ patch, int n_rt,
                                                     const double* __restrict__ tracker,
                                                     const double* __restrict__ stats, double inv_count, int thresh,
                                                     int skip2, int inner2, float* __restrict__ out) {
  const int N = NT ? NT : n_rt;
  const int z = blockIdx.x, b = blockIdx.y;
  const int64_t NN = (int64_t)N * N;
  const float* p = patch + (int64_t)b * NN * N;
  float* o = out + ((int64_t)b * N + z) * NN;
  // the rotation of the tracker scaled to unit norm, as its Euler angles are
  const double qw = tracker[4 * b], qx = tracker[4 * b + 1], qy = tracker[4 * b + 2], qz = tracker[4 * b + 3];
  const double k = 2.0 / (qw * qw + qx * qx + qy * qy + qz * qz);
  const float R00 = (float)(1 - k * (qy * qy + qz * qz)), R01 = (float)(k * (qx * qy - qw * qz)),
              R02 = (float)(k * (qx * qz + qw * qy));
  const float R10 = (float)(k * (qx * qy + qw * qz)), R11 = (float)(1 - k * (qx * qx + qz * qz)),
              R12 = (float)(k * (qy * qz - qw * qx));
  const float R20 = (float)(k * (qx * qz - qw * qy)), R21 = (float)(k * (qy * qz + qw * qx)),
              R22 = (float)(1 - k * (qx * qx + qy * qy));
  // mean and standard deviation in the mask (mean(p^2) - mean^2, as the reference)
  const double m = stats[2 * b] * inv_count;
  const float mean = (float)m;
  const float inv_sd = (float)(1.0 / sqrt(fmax(stats[2 * b + 1] * inv_count - m * m, 0.0)));
  const int c = N / 2;
  const float half = (N % 2 == 0) ? 0.5f * (float)N : 0.5f * (float)(N - 1);
  const int dz = z - c;
  const float bx = fmaf(R02, (float)dz, half), by = fmaf(R12, (float)dz, half), bz = fmaf(R22, (float)dz, half);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tilesx = (N + 7) / 8, tiles = tilesx * ((N + 3) / 4);
  for (int t = warp; t < tiles; t += kPT / 32) {
    const int x = (t % tilesx) * 8 + (lane & 7), y = (t / tilesx) * 4 + (lane >> 3);
    if (x >= N || y >= N) continue;
    const int dx = x - c, dy = y - c;
    const int r2 = dx * dx + dy * dy + dz * dz;
    float val = 0.f;
    if (r2 < skip2) {
      const float sx = fmaf(R00, (float)dx, fmaf(R01, (float)dy, bx));
      const float sy = fmaf(R10, (float)dx, fmaf(R11, (float)dy, by));
      const float sz = fmaf(R20, (float)dx, fmaf(R21, (float)dy, bz));
      const float fx = floorf(sx), fy = floorf(sy), fz = floorf(sz);
      const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
      const float wx1 = sx - fx, wy1 = sy - fy, wz1 = sz - fz;
      const float wx0 = (fx + 1.f) - sx, wy0 = (fy + 1.f) - sy, wz0 = (fz + 1.f) - sz;
      const float* q = p + ((int64_t)iz * N + iy) * N + ix;
      float cv[8];
      if (!BOX && r2 < inner2) {
        // every corner lies inside the mask, hence inside the box
#pragma unroll
        for (int k = 0; k < 8; ++k)
          cv[k] = __ldg(q + (k >> 2) * NN + ((k >> 1) & 1) * N + (k & 1)) - mean;
      } else {
        const int ex0 = ix - c, ey0 = iy - c, ez0 = iz - c;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int ex = ex0 + (k & 1), ey = ey0 + ((k >> 1) & 1), ez = ez0 + (k >> 2);
          bool in = ex * ex + ey * ey + ez * ez < thresh;
          if (BOX)
            in = in && (unsigned)(ix + (k & 1)) < (unsigned)N && (unsigned)(iy + ((k >> 1) & 1)) < (unsigned)N &&
                 (unsigned)(iz + (k >> 2)) < (unsigned)N;
          cv[k] = in ? __ldg(q + (k >> 2) * NN + ((k >> 1) & 1) * N + (k & 1)) - mean : 0.f;
        }
      }
      const float w00 = wx0 * wy0, w01 = wx1 * wy0, w10 = wx0 * wy1, w11 = wx1 * wy1;
      float s = cv[0] * (w00 * wz0);
      s = fmaf(cv[1], w01 * wz0, s);
      s = fmaf(cv[2], w10 * wz0, s);
      s = fmaf(cv[3], w11 * wz0, s);
      s = fmaf(cv[4], w00 * wz1, s);
      s = fmaf(cv[5], w01 * wz1, s);
      s = fmaf(cv[6], w10 * wz1, s);
      s = fmaf(cv[7], w11 * wz1, s);
      val = s * inv_sd;
    }
    o[(int64_t)y * N + x] = val;
  }
}

template <int NT>
int launch(const float* volumes, int B, int N, const float* shift_xyz, const double* tracker, int thresh, bool box,
           int skip2, int inner2, double inv_count, float* work, double* stats, float* out, cudaStream_t st) {
  extract_kernel<NT><<<dim3(N, B), kPT, (size_t)N * sizeof(Axis), st>>>(volumes, N, shift_xyz, thresh, work, stats);
  MTB_LAUNCH_CHECK();
  if (box)
    rotate_kernel<NT, true><<<dim3(N, B), kPT, 0, st>>>(work, N, tracker, stats, inv_count, thresh, skip2, inner2,
                                                        out);
  else
    rotate_kernel<NT, false><<<dim3(N, B), kPT, 0, st>>>(work, N, tracker, stats, inv_count, thresh, skip2, inner2,
                                                         out);
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

}  // namespace

extern "C" int mtb_prepare_subtomos(const float* volumes, int B, int N, const float* shift_xyz, const double* tracker,
                                    float mask_radius, float* work, double* stats, float* out, mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0 && N >= 2 && N <= 512, "bad batch or box size");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(volumes && shift_xyz && tracker && work && stats && out, "null pointer");
  MTB_ARG_CHECK(mask_radius > 0.f && mask_radius < 1024.f, "mask radius must be in (0, 1024)");
  const cudaStream_t st = (cudaStream_t)stream;
  // integer distances squared d2 satisfy d2 < r^2 exactly when d2 < ceil(r^2)
  const double r = (double)mask_radius, r2max = r * r;
  const int thresh = (int)ceil(r2max);
  int64_t count = 0;  // voxels of the mask: per row, the dx with dx^2 < thresh - dz^2 - dy^2
  const int c = N / 2;
  for (int z = 0; z < N; ++z)
    for (int y = 0; y < N; ++y) {
      const int rem = thresh - (z - c) * (z - c) - (y - c) * (y - c);
      if (rem <= 0) continue;
      int k = (int)sqrt((double)rem);
      while (k > 0 && k * k >= rem) --k;
      while ((k + 1) * (k + 1) < rem) ++k;
      const int lo = -k > -c ? -k : -c, hi = k < N - 1 - c ? k : N - 1 - c;
      if (hi >= lo) count += hi - lo + 1;
    }
  MTB_ARG_CHECK(count > 0, "the mask is empty");
  // A rotation keeps |s - c| = |v - c|, and the corners of s lie within sqrt(3) of it: beyond
  // r + 2 all corners are outside the mask, within r - 2 all are inside.  The margins cover
  // the rounding of s.
  const int skip2 = (int)ceil((r + 2.0) * (r + 2.0));
  const int inner2 = r > 2.0 ? (int)floor((r - 2.0) * (r - 2.0)) : 0;
  // the mask stays inside the box when every offset d with d^2 < r^2 is at most min(c, N-1-c)
  const int reach = c < N - 1 - c ? c : N - 1 - c;
  const bool box = r2max > (double)(reach + 1) * (double)(reach + 1);
  MTB_CUDA_TRY(cudaMemsetAsync(stats, 0, (size_t)B * 2 * sizeof(double), st));
  const double inv_count = 1.0 / (double)count;
  if (N == 64)
    return launch<64>(volumes, B, N, shift_xyz, tracker, thresh, box, skip2, inner2, inv_count, work, stats, out, st);
  return launch<0>(volumes, B, N, shift_xyz, tracker, thresh, box, skip2, inner2, inv_count, work, stats, out, st);
}
