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
// extract_staged_kernel: CTA = (output plane z, subtomogram b).  The sample coordinate of each
// axis depends on that axis alone (voxel + shift through the reference's normalised-grid round
// trip 2 g / (N - 1) - 1, then ((u + 1) / 2) (N - 1)).  The CTA copies the rows its masked
// voxels read from planes iz0 and iz0 + 1 with 16-byte loads and stores their z interpolation
// in shared memory; a thread keeps one column x (and x + 1) and walks rows, interpolating in
// x then y.  It computes only the voxels inside the mask (nothing else reads the patch) and
// writes each as the pair (p(x), p(x + 1)), so that the rotation reads both x corners of a
// row in one 8-byte load; it adds the masked sum and sum of squares of its plane to the
// subtomogram's FP64 statistics.  extract_kernel does the same from global memory for boxes
// whose two planes do not fit in shared memory.
//
// rotate_kernel: CTA = (output plane z, subtomogram b), a warp = an 8 x 4 patch of the plane.
// The sample point of output voxel v is R (v - c) + c (c = N / 2, the centre of the odd-padded
// linspace(-1, 1) grid), so |s - c| = |v - c|: voxels farther than radius + 2 from c read only
// masked-out corners and are written as zero without loads, voxels nearer than radius - 2
// read only corners inside the mask (four pair loads), and only the shell between tests the
// mask per corner.  Values are normalised as they are read: (p - mean) / std inside the mask,
// 0 outside.  The gathers are bound by the L1 data stage (about eight lines per warp-wide
// corner read); the pair layout halves their number.
#include <math.h>
#include "common.cuh"

namespace {

constexpr int kPT = 256;

struct Axis {
  int j0, j1;    // the two corner indices, clamped into [0, N) so that every read stays in the box
  float w0, w1;  // their weights
  bool v0, v1;   // whether the unclamped corners lie in [0, N); a corner outside reads 0
};

// One axis of the patch sampling: voxel g shifted by s, through the reference's round trip.
__device__ __forceinline__ Axis patch_axis(int g, float s, int N) {
  const float size = (float)(N - 1);
  const float n = 2.f * ((float)g + s) / size - 1.f;
  float u = ((n + 1.f) / 2.f) * size;
  u = fminf(fmaxf(u, -2.f), (float)N + 1.f);  // beyond this every corner is outside the box
  const float f = floorf(u);
  const int i0 = (int)f;
  Axis a;
  a.w1 = u - f;
  a.w0 = (f + 1.f) - u;
  a.v0 = i0 >= 0 && i0 < N;
  a.v1 = i0 + 1 >= 0 && i0 + 1 < N;
  a.j0 = min(max(i0, 0), N - 1);
  a.j1 = min(max(i0 + 1, 0), N - 1);
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

// Trilinear value of the patch at one voxel from the eight corners read by at(plane, row, col)
// (plane 0 / 1 = iz0 / iz0 + 1), corners outside the box reading 0.
template <class F>
__device__ __forceinline__ float patch_value(const Axis& ax, const Axis& ay, const Axis& az, F&& at) {
  const bool q00 = az.v0 && ay.v0, q01 = az.v0 && ay.v1, q10 = az.v1 && ay.v0, q11 = az.v1 && ay.v1;
  const float c000 = (q00 && ax.v0) ? at(0, ay.j0, ax.j0) : 0.f, c001 = (q00 && ax.v1) ? at(0, ay.j0, ax.j1) : 0.f;
  const float c010 = (q01 && ax.v0) ? at(0, ay.j1, ax.j0) : 0.f, c011 = (q01 && ax.v1) ? at(0, ay.j1, ax.j1) : 0.f;
  const float c100 = (q10 && ax.v0) ? at(1, ay.j0, ax.j0) : 0.f, c101 = (q10 && ax.v1) ? at(1, ay.j0, ax.j1) : 0.f;
  const float c110 = (q11 && ax.v0) ? at(1, ay.j1, ax.j0) : 0.f, c111 = (q11 && ax.v1) ? at(1, ay.j1, ax.j1) : 0.f;
  const float w00 = ax.w0 * ay.w0, w01 = ax.w1 * ay.w0, w10 = ax.w0 * ay.w1, w11 = ax.w1 * ay.w1;
  float p = c000 * (w00 * az.w0);
  p = fmaf(c001, w01 * az.w0, p);
  p = fmaf(c010, w10 * az.w0, p);
  p = fmaf(c011, w11 * az.w0, p);
  p = fmaf(c100, w00 * az.w1, p);
  p = fmaf(c101, w01 * az.w1, p);
  p = fmaf(c110, w10 * az.w1, p);
  p = fmaf(c111, w11 * az.w1, p);
  return p;
}

template <int NT>
__global__ void __launch_bounds__(kPT) extract_kernel(const float* __restrict__ vol, int n_rt,
                                                      const float* __restrict__ shift_xyz, int thresh,
                                                      float2* __restrict__ pairs, double* __restrict__ stats) {
  const int N = NT ? NT : n_rt;
  __shared__ double red[kPT / 32];
  extern __shared__ Axis s_y[];  // the y axis of every row (N entries)
  const int z = blockIdx.x, b = blockIdx.y;
  const int64_t NN = (int64_t)N * N;
  const float* v = vol + (int64_t)b * NN * N;
  float2* out = pairs + ((int64_t)b * N + z) * NN;
  const float sx = shift_xyz[3 * b], sy = shift_xyz[3 * b + 1], sz = shift_xyz[3 * b + 2];
  for (int y = threadIdx.x; y < N; y += kPT) s_y[y] = patch_axis(y, sy, N);
  __syncthreads();
  const Axis az = patch_axis(z, sz, N);
  const float* pl[2] = {v + (int64_t)az.j0 * NN, v + (int64_t)az.j1 * NN};
  const int c = N / 2;
  const int dz2 = (z - c) * (z - c);
  const int TXW = N < kPT ? N : kPT, RP = kPT / TXW;
  const int xi = threadIdx.x % TXW, yi = threadIdx.x / TXW;
  float s1 = 0.f, s2 = 0.f;
  if (yi < RP) {
    for (int x = xi; x < N; x += TXW) {
      const Axis ax = patch_axis(x, sx, N), ax1 = patch_axis(x + 1, sx, N);
      const int dx2 = (x - c) * (x - c);
      for (int y = yi; y < N; y += RP) {
        if (dz2 + (y - c) * (y - c) + dx2 >= thresh) continue;
        const Axis ay = s_y[y];
        auto at = [&](int k, int row, int col) { return __ldg(pl[k] + (int64_t)row * N + col); };
        const float p = patch_value(ax, ay, az, at);
        const float p1 = x + 1 < N ? patch_value(ax1, ay, az, at) : 0.f;
        out[(int64_t)y * N + x] = make_float2(p, p1);
        s1 += p;
        s2 = fmaf(p, p, s2);
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

// Shared memory: one plane (N^2 floats, the z interpolation of planes iz0 and iz0 + 1) and the
// y axis table (N entries).
template <int NT>
__global__ void __launch_bounds__(kPT) extract_staged_kernel(const float* __restrict__ vol, int n_rt,
                                                             const float* __restrict__ shift_xyz, int thresh,
                                                             float2* __restrict__ pairs, double* __restrict__ stats) {
  const int N = NT ? NT : n_rt;
  __shared__ double red[kPT / 32];
  extern __shared__ float4 smem4[];
  float* s_t = reinterpret_cast<float*>(smem4);
  Axis* s_y = reinterpret_cast<Axis*>(s_t + N * N);
  const int z = blockIdx.x, b = blockIdx.y, c = N / 2;
  const int dz2 = (z - c) * (z - c);
  if (dz2 >= thresh) return;  // no voxel of this plane lies in the mask
  const int rem = thresh - dz2;  // the plane's masked voxels: (y - c)^2 + (x - c)^2 < rem
  int ky = (int)sqrtf((float)rem);
  while (ky > 0 && ky * ky >= rem) --ky;
  while ((ky + 1) * (ky + 1) < rem) ++ky;
  const int ylo = c - ky > 0 ? c - ky : 0, yhi = c + ky < N - 1 ? c + ky : N - 1;
  const int64_t NN = (int64_t)N * N;
  const float* v = vol + (int64_t)b * NN * N;
  float2* out = pairs + ((int64_t)b * N + z) * NN;
  const float sx = shift_xyz[3 * b], sy = shift_xyz[3 * b + 1], sz = shift_xyz[3 * b + 2];
  for (int y = threadIdx.x; y < N; y += kPT) s_y[y] = patch_axis(y, sy, N);
  const Axis az = patch_axis(z, sz, N);
  __syncthreads();
  // rows read: the corners of rows ylo..yhi (non-decreasing in y); rows outside are never used
  const int rlo = s_y[ylo].j0, rhi = s_y[yhi].j1;
  {
    const float* src0 = v + (int64_t)az.j0 * NN + (int64_t)rlo * N;
    const float* src1 = v + (int64_t)az.j1 * NN + (int64_t)rlo * N;
    float* dst = s_t + rlo * N;
    const int n = (rhi - rlo + 1) * N;
    if ((N & 3) == 0 && ((reinterpret_cast<uintptr_t>(src0) | reinterpret_cast<uintptr_t>(src1)) & 15) == 0) {
      const float4* a4 = reinterpret_cast<const float4*>(src0);
      const float4* b4 = reinterpret_cast<const float4*>(src1);
      float4* d4 = reinterpret_cast<float4*>(dst);
      for (int i = threadIdx.x; i < n / 4; i += kPT) {
        const float4 a = az.v0 ? __ldg(a4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 e = az.v1 ? __ldg(b4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        d4[i] = make_float4(fmaf(e.x, az.w1, a.x * az.w0), fmaf(e.y, az.w1, a.y * az.w0),
                            fmaf(e.z, az.w1, a.z * az.w0), fmaf(e.w, az.w1, a.w * az.w0));
      }
    } else {
      for (int i = threadIdx.x; i < n; i += kPT) {
        const float a = az.v0 ? __ldg(src0 + i) : 0.f, e = az.v1 ? __ldg(src1 + i) : 0.f;
        dst[i] = fmaf(e, az.w1, a * az.w0);
      }
    }
  }
  __syncthreads();
  const int TXW = N < kPT ? N : kPT, RP = kPT / TXW;
  const int xi = threadIdx.x % TXW, yi = threadIdx.x / TXW;
  float s1 = 0.f, s2 = 0.f;
  if (yi < RP) {
    for (int x = xi; x < N; x += TXW) {
      const Axis ax = patch_axis(x, sx, N), ax1 = patch_axis(x + 1, sx, N);
      const bool last = x + 1 >= N;  // p(N) lies outside the patch: the pair holds 0 there
      const int rx = rem - (x - c) * (x - c);
      for (int y = ylo + yi; y <= yhi; y += RP) {
        if ((y - c) * (y - c) >= rx) continue;
        const Axis ay = s_y[y];
        const float* t0 = s_t + ay.j0 * N;
        const float* t1 = s_t + ay.j1 * N;
        auto row = [&](const float* t, bool vy, const Axis& a) {
          const float lo = (vy && a.v0) ? t[a.j0] : 0.f, hi = (vy && a.v1) ? t[a.j1] : 0.f;
          return fmaf(hi, a.w1, lo * a.w0);
        };
        const float p = fmaf(row(t1, ay.v1, ax), ay.w1, row(t0, ay.v0, ax) * ay.w0);
        const float p1 = last ? 0.f : fmaf(row(t1, ay.v1, ax1), ay.w1, row(t0, ay.v0, ax1) * ay.w0);
        out[(int64_t)y * N + x] = make_float2(p, p1);
        s1 += p;
        s2 = fmaf(p, p, s2);
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

// Rotation.  CTA = (kZW output planes from z0, subtomogram b); a warp takes a block of
// (32 / 4 kZW) x 4 x kZW output voxels (x, y, z) at a time, so that its sample points, and
// the lines its corner reads touch, stay close together.
constexpr int kZW = 1, kXW = 32 / (4 * kZW);

// BOX: the mask reaches outside the box, so a corner inside the mask may still be outside it.
template <int NT, bool BOX>
__global__ void __launch_bounds__(kPT) rotate_kernel(const float2* __restrict__ pairs, int n_rt,
                                                     const double* __restrict__ tracker,
                                                     const double* __restrict__ stats, double inv_count, int thresh,
                                                     int skip2, int inner2, float* __restrict__ out) {
  const int N = NT ? NT : n_rt;
  const int b = blockIdx.y;
  const int64_t NN = (int64_t)N * N;
  const float2* p = pairs + (int64_t)b * NN * N;
  float* o = out + (int64_t)b * NN * N;
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
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int z = blockIdx.x * kZW + lane / (4 * kXW);
  if (z >= N) return;
  const int dz = z - c;
  const float bx = fmaf(R02, (float)dz, half), by = fmaf(R12, (float)dz, half), bz = fmaf(R22, (float)dz, half);
  const int tilesx = (N + kXW - 1) / kXW, tiles = tilesx * ((N + 3) / 4);
  for (int t = warp; t < tiles; t += kPT / 32) {
    const int x = (t % tilesx) * kXW + lane % kXW, y = (t / tilesx) * 4 + (lane / kXW) % 4;
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
      const float2* q = p + ((int64_t)iz * N + iy) * N + ix;
      float cv[8];
      if (!BOX && r2 < inner2) {
        // every corner lies inside the mask, hence inside the box: four pair loads
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const float2 e = __ldg(q + (r >> 1) * NN + (r & 1) * N);
          cv[2 * r] = e.x - mean;
          cv[2 * r + 1] = e.y - mean;
        }
      } else {
        const int ex0 = ix - c, ey0 = iy - c, ez0 = iz - c;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int ey = ey0 + (r & 1), ez = ez0 + (r >> 1), eyz = ey * ey + ez * ez;
          bool in0 = ex0 * ex0 + eyz < thresh, in1 = (ex0 + 1) * (ex0 + 1) + eyz < thresh;
          if (BOX) {
            const bool row = (unsigned)(iy + (r & 1)) < (unsigned)N && (unsigned)(iz + (r >> 1)) < (unsigned)N;
            in0 = in0 && row && (unsigned)ix < (unsigned)N;
            in1 = in1 && row && (unsigned)(ix + 1) < (unsigned)N;
          }
          const float2* qr = q + (r >> 1) * NN + (r & 1) * N;
          // a pair is written for every voxel in the mask: (p(ix), p(ix + 1)) when ix is in
          // it, else p(ix + 1) is the first value of the next pair
          float e0 = 0.f, e1 = 0.f;
          if (in0) {
            const float2 e = __ldg(qr);
            e0 = e.x - mean;
            e1 = in1 ? e.y - mean : 0.f;
          } else if (in1) {
            e1 = __ldg(reinterpret_cast<const float*>(qr + 1)) - mean;
          }
          cv[2 * r] = e0;
          cv[2 * r + 1] = e1;
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
    o[((int64_t)z * N + y) * N + x] = val;
  }
}

template <int NT>
int launch(const float* volumes, int B, int N, const float* shift_xyz, const double* tracker, int thresh, bool box,
           int skip2, int inner2, double inv_count, float2* work, double* stats, float* out, cudaStream_t st) {
  const size_t ext_smem = (size_t)N * N * sizeof(float) + (size_t)N * sizeof(Axis);
  mtb_prof_begin(st);
  if (ext_smem <= 48 * 1024)
    extract_staged_kernel<NT><<<dim3(N, B), kPT, ext_smem, st>>>(volumes, N, shift_xyz, thresh, work, stats);
  else
    extract_kernel<NT><<<dim3(N, B), kPT, (size_t)N * sizeof(Axis), st>>>(volumes, N, shift_xyz, thresh, work,
                                                                          stats);
  mtb_prof_end(st, "extract_kernel");
  MTB_LAUNCH_CHECK();
  const dim3 grid((N + kZW - 1) / kZW, B);
  mtb_prof_begin(st);
  if (box)
    rotate_kernel<NT, true><<<grid, kPT, 0, st>>>(work, N, tracker, stats, inv_count, thresh, skip2, inner2, out);
  else
    rotate_kernel<NT, false><<<grid, kPT, 0, st>>>(work, N, tracker, stats, inv_count, thresh, skip2, inner2, out);
  mtb_prof_end(st, "rotate_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

}  // namespace

extern "C" int mtb_prepare_subtomos(const float* volumes, int B, int N, const float* shift_xyz, const double* tracker,
                                    float mask_radius, float* work, double* stats, float* out, mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0 && N >= 2 && N <= 512, "bad batch or box size");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(volumes && shift_xyz && tracker && work && stats && out, "null pointer");
  MTB_ARG_CHECK((reinterpret_cast<uintptr_t>(work) & 7) == 0, "work must be 8-byte aligned");
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
  float2* pairs = reinterpret_cast<float2*>(work);
  if (N == 64)
    return launch<64>(volumes, B, N, shift_xyz, tracker, thresh, box, skip2, inner2, inv_count, pairs, stats, out,
                      st);
  return launch<0>(volumes, B, N, shift_xyz, tracker, thresh, box, skip2, inner2, inv_count, pairs, stats, out, st);
}
