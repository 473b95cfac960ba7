// Backward kernels of the alignment score (the differentiation pattern of the alignment path).
//
// The score of subtomogram b at a rotation R is f_b(R) = Re sum_l sum_{m'm} D^l_{m'm}(R)
// sigma_b[l, m', m] (src/matcha/core/Matcha.py:184, :288), with the reference's convention
// D^l_{m'm}(alpha, beta, gamma) = exp(+i m' alpha) d^l_{m'm}(beta) exp(+i m gamma) and
// sigma_b[l, m', m] = (-1)^(m'+m) sum_k aT[l, -m, k] conj(aV_b[l, -m', k])
// (src/matcha/core/CrossCorrelationMatcher.py:183-212).
//
// score_backward_kernel regenerates D^l(R_b) for l <= L from the angles (FP64 three-term
// recurrences in l per (m', m), the forward pass stores nothing) and, in the same sweep,
//   * grad_sigma_b = w_b conj(D(R_b)): d f / d sigma in PyTorch's convention for a real
//     function of a complex tensor (d/dRe + i d/dIm);
//   * the body-frame gradient g_k = d f_b(R_b exp(t e_k)) / dt at t = 0, k = x, y, z.
//     D(R exp(t e_k)) = D(R) D(exp(t e_k)), so g_k = Re sum D(R) sigma^(k) with
//     sigma^(k)[m', n] = sum_m sigma[m', m] A_k[n, m] and A_k the generator of the
//     representation: A_z = diag(i m); A_y[m+1, m] = -sqrt((l-m)(l+m+1))/2,
//     A_y[m-1, m] = sqrt((l+m)(l-m+1))/2 (the derivative of Edmonds' d^l at beta = 0);
//     A_x[n, m] = i^(m-n) A_y[n, m] (Rx(t) = Rz(-pi/2) Ry(t) Rz(pi/2)).  Unlike the Euler
//     gradient mapped through the z-y-z kinematics, this has no singularity at beta = 0, pi.
//
// sigma_backward_template_kernel: the adjoint of the sigma contraction with respect to the
// template coefficients, grad_aT[l, -m, k] = sum_b sum_m' (-1)^(m'+m) aV_b[l, -m', k]
// grad_sigma_b[l, m', m]; one CTA per degree, the batch summed in order (deterministic).
#include <math.h>
#include "common.cuh"

namespace {

constexpr int kBT = 256;

// d^{l0}_{mp m}(beta) at l0 = max(|mp|, |m|): the single term of Edmonds' sum that survives.
__device__ double d_start(int mp, int m, double beta) {
  const int l = abs(mp) > abs(m) ? abs(mp) : abs(m);
  const int k = (m - mp) > 0 ? (m - mp) : 0;
  const double c = cos(0.5 * beta), s = sin(0.5 * beta);
  const double lognum = 0.5 * (lgamma(l + mp + 1.0) + lgamma(l - mp + 1.0) + lgamma(l + m + 1.0) + lgamma(l - m + 1.0));
  const double logden = lgamma(l + m - k + 1.0) + lgamma(k + 1.0) + lgamma(mp - m + k + 1.0) + lgamma(l - mp - k + 1.0);
  const int pc = 2 * l + m - mp - 2 * k, ps = mp - m + 2 * k;
  double v = exp(lognum - logden) * (((mp - m + k) & 1) ? -1.0 : 1.0);
  v *= (pc ? pow(c, (double)pc) : 1.0) * (ps ? pow(s, (double)ps) : 1.0);
  return v;
}

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(kBT)
score_backward_kernel(const float2* __restrict__ sigma, int64_t stride, int L, const float* __restrict__ alpha,
                      const float* __restrict__ beta, const float* __restrict__ gamma, const float* __restrict__ weight,
                      float2* __restrict__ grad_sigma, int64_t gstride, double* __restrict__ grad_body) {
  const int b = blockIdx.x;
  const double al = alpha[b], be = beta[b], ga = gamma[b];
  const double w = weight ? (double)weight[b] : 1.0;
  const double cb = cos(be);
  const float2* sg = sigma + (int64_t)b * stride;
  float2* gs = grad_sigma ? grad_sigma + (int64_t)b * gstride : nullptr;
  double gx = 0.0, gy = 0.0, gz = 0.0;
  const int P = 2 * L + 1;
  for (int e = threadIdx.x; e < P * P; e += blockDim.x) {
    const int mp = e / P - L, m = e % P - L;
    const int l0 = abs(mp) > abs(m) ? abs(mp) : abs(m);
    double sn, cs;
    sincos((double)mp * al + (double)m * ga, &sn, &cs);
    const double2 ph = make_double2(cs, sn);
    double dl = d_start(mp, m, be), dlm1 = 0.0;
    for (int l = l0; l <= L; ++l) {
      if (l > l0) {
        const int ll = l - 1;  // d^{ll+1} from d^{ll}, d^{ll-1}
        double dn;
        if (ll == 0) {
          dn = cb * dl;
        } else {
          const double a = (2.0 * ll + 1.0) * (ll * (ll + 1.0) * cb - (double)m * mp);
          const double bb = (ll + 1.0) * sqrt((double)(ll * ll - m * m) * (double)(ll * ll - mp * mp));
          const double cc = ll * sqrt((double)((ll + 1) * (ll + 1) - m * m) * (double)((ll + 1) * (ll + 1) - mp * mp));
          dn = (a * dl - bb * dlm1) / cc;
        }
        dlm1 = dl;
        dl = dn;
      }
      const int64_t idx = (int64_t)mtb_dsize(l - 1) + (int64_t)(mp + l) * (2 * l + 1) + (m + l);
      const double2 D = make_double2(dl * ph.x, dl * ph.y);
      if (gs) gs[idx] = make_float2((float)(w * D.x), (float)(-w * D.y));
      if (grad_body) {
        const float2 s0f = sg[idx];
        const double2 s0 = make_double2(s0f.x, s0f.y);
        double2 sm = make_double2(0.0, 0.0), sp = make_double2(0.0, 0.0);
        double am = 0.0, ap = 0.0;
        if (m - 1 >= -l) {
          const float2 t = sg[idx - 1];
          sm = make_double2(t.x, t.y);
          am = sqrt((double)(l - m + 1) * (double)(l + m));
        }
        if (m + 1 <= l) {
          const float2 t = sg[idx + 1];
          sp = make_double2(t.x, t.y);
          ap = sqrt((double)(l + m + 1) * (double)(l - m));
        }
        // sigma^(y) = -am/2 sigma[m-1] + ap/2 sigma[m+1]; sigma^(x) = i/2 (am sigma[m-1] + ap sigma[m+1]);
        // sigma^(z) = i m sigma[m]
        const double2 sy = make_double2(0.5 * (ap * sp.x - am * sm.x), 0.5 * (ap * sp.y - am * sm.y));
        const double2 u = make_double2(0.5 * (am * sm.x + ap * sp.x), 0.5 * (am * sm.y + ap * sp.y));
        const double2 sx = make_double2(-u.y, u.x);
        const double2 sz = make_double2(-(double)m * s0.y, (double)m * s0.x);
        gx += cmul_d(D, sx).x;
        gy += cmul_d(D, sy).x;
        gz += cmul_d(D, sz).x;
      }
    }
  }
  if (!grad_body) return;
  __shared__ double red[3][kBT];
  red[0][threadIdx.x] = gx;
  red[1][threadIdx.x] = gy;
  red[2][threadIdx.x] = gz;
  __syncthreads();
  for (int s = kBT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 3) grad_body[(int64_t)b * 3 + threadIdx.x] = w * red[threadIdx.x][0];
}

// One CTA per degree l; the rows mu = -l..l of the coefficient gather table kidx (koff[l],
// kpad[l] entries each, -1 padded) index the complex coefficients of (l, mu, k).
__global__ void __launch_bounds__(kBT)
sigma_backward_template_kernel(const float2* __restrict__ aV, int64_t v_stride, const float2* __restrict__ gsig,
                               int64_t g_stride, int B, const int* __restrict__ kpad, const int* __restrict__ koff,
                               const int* __restrict__ kidx, float2* __restrict__ grad_tmpl) {
  extern __shared__ __align__(16) float2 bsm[];
  const int l = blockIdx.x;
  const int w = 2 * l + 1;
  const int K = kpad[l];
  const int ks = K | 1;
  float2* sV = bsm;                // w rows x ks
  float2* sG = bsm + w * ks;       // w x w block of grad_sigma
  float2* acc = sG + w * w;        // w x K: the template rows' gradient
  const int* tab = kidx + koff[l];
  for (int e = threadIdx.x; e < w * K; e += blockDim.x) acc[e] = make_float2(0.f, 0.f);
  for (int b = 0; b < B; ++b) {
    __syncthreads();
    const float2* v = aV + (int64_t)b * v_stride;
    for (int e = threadIdx.x; e < w * K; e += blockDim.x) {
      const int row = e / K, k = e - (e / K) * K;
      const int idx = __ldg(&tab[e]);
      sV[row * ks + k] = idx >= 0 ? __ldg(&v[idx]) : make_float2(0.f, 0.f);
    }
    const float2* g = gsig + (int64_t)b * g_stride + mtb_dsize(l - 1);
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) sG[e] = __ldg(&g[e]);
    __syncthreads();
    // entry (rT, k) of acc: the template row rT = 2l - c (mu = -(c - l)) for the second sigma index c
    for (int e = threadIdx.x; e < w * K; e += blockDim.x) {
      const int rT = e / K, k = e - (e / K) * K;
      const int c = 2 * l - rT;
      float re = 0.f, im = 0.f;
      for (int a = 0; a < w; ++a) {
        const float2 vv = sV[(2 * l - a) * ks + k];  // aV_b[l, -(a - l), k]
        const float2 gg = sG[a * w + c];            // grad_sigma_b[l, a - l, c - l]
        const float sgn = ((a + c) & 1) ? -1.f : 1.f;
        re += sgn * (vv.x * gg.x - vv.y * gg.y);
        im += sgn * (vv.x * gg.y + vv.y * gg.x);
      }
      acc[e].x += re;
      acc[e].y += im;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < w * K; e += blockDim.x) {
    const int idx = tab[e];
    if (idx >= 0) grad_tmpl[idx] = acc[e];
  }
}

}  // namespace

extern "C" int mtb_score_backward(const float* sigma, int64_t sigma_stride, int B, int L, const float* alpha,
                                  const float* beta, const float* gamma, const float* weight, float* grad_sigma,
                                  int64_t grad_stride, double* grad_body, mtb_stream_t stream) {
  MTB_ARG_CHECK(B >= 0, "negative batch");
  MTB_ARG_CHECK(L >= 0 && L <= 128, "L must be in [0, 128]");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(alpha && beta && gamma, "null angles");
  MTB_ARG_CHECK(grad_sigma || grad_body, "nothing to compute");
  MTB_ARG_CHECK(!grad_body || (sigma && sigma_stride >= mtb_dsize(L)), "sigma row shorter than dsize(L)");
  MTB_ARG_CHECK(!grad_sigma || grad_stride >= mtb_dsize(L), "grad_sigma row shorter than dsize(L)");
  MTB_ARG_CHECK(B <= 2147483647, "batch too large");
  cudaStream_t st = (cudaStream_t)stream;
  mtb_prof_begin(st);
  score_backward_kernel<<<B, kBT, 0, st>>>(reinterpret_cast<const float2*>(sigma), sigma_stride, L, alpha, beta,
                                           gamma, weight, reinterpret_cast<float2*>(grad_sigma), grad_stride,
                                           grad_body);
  mtb_prof_end(st, "score_backward_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

// The FLE handle's gather tables (fle.cu) for the template backward.
int fle_sigma_tables(const mtb_fle* h, const int** kpad, const int** koff, const int** kidx, int* lmax, int* kmax,
                     int* ne);

extern "C" int mtb_sigma_backward_template(mtb_fle* h, const float* coeffs, int64_t coeff_stride,
                                           const float* grad_sigma, int64_t grad_stride, int B, int lmax_g,
                                           float* grad_tmpl, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  const int *kpad, *koff, *kidx;
  int lmax, kmax, ne;
  if (int rc = fle_sigma_tables(h, &kpad, &koff, &kidx, &lmax, &kmax, &ne)) return rc;
  MTB_ARG_CHECK(lmax_g >= 0 && lmax_g <= lmax, "lmax_g must be in [0, lmax of the expansion]");
  MTB_ARG_CHECK(B >= 0, "negative batch");
  MTB_ARG_CHECK(grad_tmpl, "null output");
  cudaStream_t st = (cudaStream_t)stream;
  // degrees above lmax_g (and the padding entry ne) get no gradient
  MTB_CUDA_TRY(cudaMemsetAsync(grad_tmpl, 0, (size_t)(ne + 1) * sizeof(float2), st));
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(coeffs && grad_sigma, "null pointer");
  MTB_ARG_CHECK(coeff_stride >= ne, "coefficient row shorter than ne");
  MTB_ARG_CHECK(grad_stride >= mtb_dsize(lmax_g), "grad_sigma row shorter than dsize(lmax_g)");
  const int w = 2 * lmax_g + 1, ks = kmax | 1;
  const size_t smem = ((size_t)w * ks + (size_t)w * w + (size_t)w * kmax) * sizeof(float2);
  MTB_ARG_CHECK(smem <= 227 * 1024, "degree too high for the shared-memory staging of the template backward");
  MTB_CUDA_TRY(cudaFuncSetAttribute(sigma_backward_template_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  mtb_prof_begin(st);
  sigma_backward_template_kernel<<<lmax_g + 1, kBT, smem, st>>>(
      reinterpret_cast<const float2*>(coeffs), coeff_stride, reinterpret_cast<const float2*>(grad_sigma), grad_stride,
      B, kpad, koff, kidx, reinterpret_cast<float2*>(grad_tmpl));
  mtb_prof_end(st, "sigma_backward_template_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}
