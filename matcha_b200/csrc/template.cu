// The shift match's Fourier reference of a template, on the device in FP64.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   load_reference_full   src/matcha/core/ShiftMatcher.py:456-472
//   apply_soft_mask       :377-406  fftn (norm forward), fftshift, raised-cosine low-pass of
//                                   radius N voxel / 4 - 1 and edge width 2, ifftn, real part
//   gridding_correct      :409-437  divide by sinc^2(r / N), r from arange(-N//2, N//2)
//   np.roll by -N//2, fftn (norm forward), fftshift, times fftshift(get_mask_full) (:440-453:
//   frequencies with kp^2 + ip^2 + jp^2 <= (N//2 * N) // 2)
//
// Every FFT is a separable DFT here, one pass per axis, each output element a length-N dot
// product with a twiddle table computed on the host in FP64 (N^4 complex multiply-adds per
// pass: 17 M at N = 64, once per template).  The fftshifts and the roll are index maps folded
// into the elementwise passes; no volume is moved for them.
#include <math.h>

#include <vector>

#include "common.cuh"

namespace {

constexpr int kTT = 256;

struct Cd {
  double x, y;
};

__device__ __forceinline__ int wrap(int i, int N) { return i >= N ? i - N : (i < 0 ? i + N : i); }

// out = DFT of in along axis (0 = z, 1 = y, 2 = x) with twiddles tw[m] = exp(+-2 pi i m / N)
__global__ void __launch_bounds__(kTT) dft_axis_kernel(const Cd* __restrict__ in, Cd* __restrict__ out, int N,
                                                       int axis, const Cd* __restrict__ tw) {
  const int64_t total = (int64_t)N * N * N;
  const int64_t e = (int64_t)blockIdx.x * kTT + threadIdx.x;
  if (e >= total) return;
  const int x = (int)(e % N), y = (int)((e / N) % N), z = (int)(e / ((int64_t)N * N));
  const int k = axis == 0 ? z : axis == 1 ? y : x;
  const int64_t stride = axis == 0 ? (int64_t)N * N : axis == 1 ? N : 1;
  const Cd* line = in + (e - (int64_t)k * stride);
  double re = 0.0, im = 0.0;
  int m = 0;  // k * n mod N
  for (int n = 0; n < N; ++n) {
    const Cd v = line[(int64_t)n * stride], w = tw[m];
    re = fma(v.x, w.x, fma(-v.y, w.y, re));
    im = fma(v.x, w.y, fma(v.y, w.x, im));
    m += k;
    if (m >= N) m -= N;
  }
  out[e] = Cd{re, im};
}

__global__ void __launch_bounds__(kTT) load_kernel(const double* __restrict__ t, int64_t total, Cd* __restrict__ a) {
  const int64_t e = (int64_t)blockIdx.x * kTT + threadIdx.x;
  if (e < total) a[e] = Cd{t[e], 0.0};
}

// signed frequency of array index j after fftshift, measured from the centre N//2
__device__ __forceinline__ int centred(int j, int N) { return wrap(j + N / 2, N) - N / 2; }

// F <- F / N^3 * soft mask (apply_soft_mask's raised cosine at the fftshifted position)
__global__ void __launch_bounds__(kTT) soft_mask_kernel(Cd* __restrict__ a, int N, double scale, double radius,
                                                        double radius_p, double width) {
  const int64_t total = (int64_t)N * N * N;
  const int64_t e = (int64_t)blockIdx.x * kTT + threadIdx.x;
  if (e >= total) return;
  const int x = (int)(e % N), y = (int)((e / N) % N), z = (int)(e / ((int64_t)N * N));
  const double dz = centred(z, N), dy = centred(y, N), dx = centred(x, N);
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  double m = 1.0;
  if (r > radius_p)
    m = 0.0;
  else if (r >= radius)
    m = 0.5 - 0.5 * cos(M_PI * (radius_p - r) / width);
  const double s = scale * m;
  a[e] = Cd{a[e].x * s, a[e].y * s};
}

// centered[i] = real(v)[(i + N//2) mod N] / sinc^2(r / N) (gridding_correct, then the roll)
__global__ void __launch_bounds__(kTT) grid_roll_kernel(const Cd* __restrict__ v, int N, Cd* __restrict__ out) {
  const int64_t total = (int64_t)N * N * N;
  const int64_t e = (int64_t)blockIdx.x * kTT + threadIdx.x;
  if (e >= total) return;
  const int x = (int)(e % N), y = (int)((e / N) % N), z = (int)(e / ((int64_t)N * N));
  const int h = N / 2;
  const int sz = wrap(z + h, N), sy = wrap(y + h, N), sx = wrap(x + h, N);  // source voxel
  // coordinates of the source voxel on arange(-N//2, N//2) (Python floor division)
  const int lo = -((N + 1) / 2);
  const double cz = sz + lo, cy = sy + lo, cx = sx + lo;
  const double rval = sqrt(cx * cx + cy * cy + cz * cz) / (double)N;
  double corr = 1.0;
  if (rval > 0.0) {
    const double s = sin(M_PI * rval) / (M_PI * rval);
    corr = s * s;
    if (corr == 0.0) corr = 1.0;
  }
  out[e] = Cd{v[((int64_t)sz * N + sy) * N + sx].x / corr, 0.0};
}

// out[p] = faux[(p - N//2) mod N] / N^3 * mask_full at that frequency, complex64
__global__ void __launch_bounds__(kTT) final_kernel(const Cd* __restrict__ f, int N, double scale, int64_t thr,
                                                    float2* __restrict__ out) {
  const int64_t total = (int64_t)N * N * N;
  const int64_t e = (int64_t)blockIdx.x * kTT + threadIdx.x;
  if (e >= total) return;
  const int x = (int)(e % N), y = (int)((e / N) % N), z = (int)(e / ((int64_t)N * N));
  const int h = N / 2;
  const int jz = wrap(z - h, N), jy = wrap(y - h, N), jx = wrap(x - h, N);
  const int64_t kp = jz < h ? jz : jz - N, ip = jy < h ? jy : jy - N, jp = jx < h ? jx : jx - N;
  const Cd v = f[((int64_t)jz * N + jy) * N + jx];
  const bool in = kp * kp + ip * ip + jp * jp <= thr;
  out[e] = in ? make_float2((float)(v.x * scale), (float)(v.y * scale)) : make_float2(0.f, 0.f);
}

}  // namespace

extern "C" int mtb_shift_reference(const double* tmpl, int N, float voxel_size, void* workspace, float* out,
                                   mtb_stream_t stream) {
  MTB_ARG_CHECK(N >= 2 && N <= 512, "bad box size");
  MTB_ARG_CHECK(tmpl && workspace && out, "null pointer");
  MTB_ARG_CHECK((reinterpret_cast<uintptr_t>(workspace) & 15) == 0, "workspace must be 16-byte aligned");
  MTB_ARG_CHECK(voxel_size > 0.f, "voxel size must be positive");
  const cudaStream_t st = (cudaStream_t)stream;
  const int64_t total = (int64_t)N * N * N;
  Cd* a = static_cast<Cd*>(workspace);
  Cd* b = a + total;
  Cd* tw = b + total;  // forward then inverse twiddles, N each
  std::vector<Cd> h_tw(2 * (size_t)N);
  for (int m = 0; m < N; ++m) {
    const double ang = 2.0 * M_PI * (double)m / (double)N;
    h_tw[m] = Cd{cos(ang), -sin(ang)};
    h_tw[N + m] = Cd{cos(ang), sin(ang)};
  }
  MTB_CUDA_TRY(cudaMemcpyAsync(tw, h_tw.data(), h_tw.size() * sizeof(Cd), cudaMemcpyHostToDevice, st));
  const unsigned grid = (unsigned)((total + kTT - 1) / kTT);
  auto dft3 = [&](Cd* src, Cd* dst, const Cd* t) -> int {  // result in dst
    dft_axis_kernel<<<grid, kTT, 0, st>>>(src, dst, N, 2, t);
    dft_axis_kernel<<<grid, kTT, 0, st>>>(dst, src, N, 1, t);
    dft_axis_kernel<<<grid, kTT, 0, st>>>(src, dst, N, 0, t);
    MTB_LAUNCH_CHECK();
    return MTB_OK;
  };
  const double inv = 1.0 / (double)total;
  // apply_soft_mask(ori_size = N, pixel_size = voxel_size, ini_high = 4, width_fmask_edge = 2)
  const double width = 2.0;
  const double radius = (double)N * (double)voxel_size / 4.0 - width / 2.0, radius_p = radius + width;
  load_kernel<<<grid, kTT, 0, st>>>(tmpl, total, a);
  MTB_LAUNCH_CHECK();
  if (int rc = dft3(a, b, tw)) return rc;
  soft_mask_kernel<<<grid, kTT, 0, st>>>(b, N, inv, radius, radius_p, width);
  MTB_LAUNCH_CHECK();
  if (int rc = dft3(b, a, tw + N)) return rc;
  grid_roll_kernel<<<grid, kTT, 0, st>>>(a, N, b);
  MTB_LAUNCH_CHECK();
  if (int rc = dft3(b, a, tw)) return rc;
  const int64_t h = N / 2;
  final_kernel<<<grid, kTT, 0, st>>>(a, N, inv, (h * N) / 2, reinterpret_cast<float2*>(out));
  MTB_LAUNCH_CHECK();
  // the host twiddle table must outlive its copy
  MTB_CUDA_TRY(cudaStreamSynchronize(st));
  return MTB_OK;
}
