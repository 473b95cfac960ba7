// Per-particle results of one alternation, packed on the device so that storing them costs
// one device-to-host copy per batch instead of a host synchronisation per value.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   store_alignment_parameters   src/matcha/utils/io_utils.py:181-225 (rotation_score,
//                                rotation = quaternionic to_euler_angles of the tracker,
//                                translation = local shift, prior_shift, shift_score per row)
//   quaternionic to_euler_angles alpha = atan2(z, w) + atan2(-x, y),
//                                beta = 2 acos(sqrt((w^2 + z^2) / |q|^2)),
//                                gamma = atan2(z, w) - atan2(-x, y)   (radians, z-y-z)
#include <math.h>
#include "common.cuh"

namespace {

constexpr int kCols = 11;

__global__ void pack_results_kernel(const float* __restrict__ rotation_score, const float* __restrict__ shift_score,
                                    const float* __restrict__ local_shift, const float* __restrict__ prior_shift,
                                    const double* __restrict__ tracker, int B, double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const double w = tracker[4 * b], x = tracker[4 * b + 1], y = tracker[4 * b + 2], z = tracker[4 * b + 3];
  const double n = w * w + x * x + y * y + z * z;
  const double t1 = atan2(z, w), t2 = atan2(-x, y);
  double* o = out + (int64_t)kCols * b;
  o[0] = (double)rotation_score[b];
  o[1] = t1 + t2;
  o[2] = 2.0 * acos(sqrt((w * w + z * z) / n));
  o[3] = t1 - t2;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    o[4 + k] = (double)local_shift[3 * b + k];
    o[7 + k] = (double)prior_shift[3 * b + k];
  }
  o[10] = (double)shift_score[b];
}

}  // namespace

extern "C" int mtb_pack_results(const float* rotation_score, const float* shift_score, const float* local_shift,
                                const float* prior_shift, const double* tracker, int B, double* out,
                                mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0, "negative batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(rotation_score && shift_score && local_shift && prior_shift && tracker && out, "null pointer");
  mtb_prof_begin((cudaStream_t)stream);
  pack_results_kernel<<<(B + 127) / 128, 128, 0, (cudaStream_t)stream>>>(rotation_score, shift_score, local_shift,
                                                                          prior_shift, tracker, B, out);
  mtb_prof_end((cudaStream_t)stream, "pack_results_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}
