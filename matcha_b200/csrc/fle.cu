// Fourier-Bessel ball expansion (FLE) and per-degree correlation coefficients on sm_100a.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   FLE forward   src/matcha/core/FLEBasis3D.py:945-976 (evaluate_t) -- the reference
//                 approximates the discrete adjoint a = h B^H f with a type-2 NUFFT, a
//                 spherical-harmonic transform per shell and radial interpolation
//                 (tolerance 1e-4); this file evaluates the adjoint itself.
//   basis         src/matcha/core/FLEBasis3D.py:570-698 (create_denseB), :700-799
//   sigma         src/matcha/core/CrossCorrelationMatcher.py:133-212
//
// Design (B200): every real basis column -- Re or Im of conj(psi_{lkm}), m >= 0 -- has a
// definite parity under each of the reflections x->-x, y->-y, z->-z, and the voxel ball
// is closed under them.  The volume is therefore folded once into 8 parity channels over
// the positive octant (a 3-D Walsh-Hadamard transform of each orbit of 8 sign images),
// and the adjoint becomes 8 independent GEMMs of 1/8 the depth and 1/8 the width:
// 1/8 of the dense work, still exact.  Coefficients with m < 0 follow from
// a_{l,k,-m} = (-1)^m conj(a_{l,k,m}) for real volumes.
#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "fle_tc.cuh"

namespace {

constexpr int kClasses = 8;

// ------------------------------------------------------------------ basis build
// One thread per (representative, order m).  Normalised associated Legendre values
// (orthonormal, Condon-Shortley phase) by the standard recurrence in l, FP64.
__global__ void build_basis_kernel(int n_rep, int lmax, const double* __restrict__ rep_cos,
                                   const double* __restrict__ rep_phi, const int* __restrict__ rep_r2,
                                   const double* __restrict__ jtab, int n_lk,
                                   const int* __restrict__ lm_start,  // (lmax+1)^2 + 1 offsets into col list, index l*(lmax+1)+m
                                   const int* __restrict__ col_list,  // columns sorted by (l, m)
                                   const int* __restrict__ col_class, const int* __restrict__ col_pos,
                                   const int* __restrict__ col_part, const int* __restrict__ col_lk,
                                   const double* __restrict__ col_scale,
                                   float* const* __restrict__ basis,  // per class: (n_rep, n_cols_class)
                                   const int* __restrict__ class_cols) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = t % (lmax + 1);
  const int rep = t / (lmax + 1);
  if (rep >= n_rep) return;
  const double x = rep_cos[rep];
  const double s = sqrt(fmax(0.0, 1.0 - x * x));
  double pmm = 0.28209479177387814;  // 1 / sqrt(4 pi)
  for (int k = 1; k <= m; ++k) pmm *= -sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
  double sp, cp;
  sincos((double)m * rep_phi[rep], &sp, &cp);
  const double* jrow = jtab + (int64_t)rep_r2[rep] * n_lk;
  double p2 = 0.0, p1 = pmm;
  for (int l = m; l <= lmax; ++l) {
    double p;
    if (l == m) {
      p = pmm;
    } else if (l == m + 1) {
      p = sqrt(2.0 * m + 3.0) * x * pmm;
    } else {
      const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      const double b = sqrt(((double)(l - 1) * (l - 1) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
      p = a * (x * p1 - b * p2);
    }
    if (l > m) { p2 = p1; p1 = p; }
    const int key = l * (lmax + 1) + m;
    for (int q = lm_start[key]; q < lm_start[key + 1]; ++q) {
      const int col = col_list[q];
      const double ang = col_part[col] ? -sp : cp;  // conj(Y) = P e^{-i m phi}
      const double v = col_scale[col] * jrow[col_lk[col]] * p * ang;
      const int cls = col_class[col];
      basis[cls][(int64_t)rep * class_cols[cls] + col_pos[col]] = (float)v;
    }
  }
}

// ------------------------------------------------------------------ fold into channels
// A_p[b][rep] = sum over distinct sign images s of rep: f(s * rep) * chi_p(s),
// chi_p(s) = prod over flipped axes of the class parity p.  Class bits: 0 -> x odd,
// 1 -> y odd, 2 -> z odd.
__global__ void fold_kernel(const float* __restrict__ vol, int64_t vol_stride, int B, int n_rep,
                            const int* __restrict__ rep_img, float* __restrict__ A, int64_t a_stride_class) {
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (rep >= n_rep || b >= B) return;
  const float* v = vol + (int64_t)b * vol_stride;
  float f[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int idx = __ldg(&rep_img[rep * 8 + s]);
    f[s] = idx >= 0 ? __ldg(&v[idx]) : 0.f;
  }
  // Walsh-Hadamard over the three sign bits: out[p] = sum_s f[s] * (-1)^{popc(p & s)}
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      if (!(s & bit)) {
        const float u = f[s], w = f[s | bit];
        f[s] = u + w;
        f[s | bit] = u - w;
      }
    }
  }
#pragma unroll
  for (int p = 0; p < 8; ++p) A[p * a_stride_class + (int64_t)b * n_rep + rep] = f[p];
}

// ------------------------------------------------------------------ FP32 GEMM (plain path)
// C_p (B x n_p) = A_p (B x K) * Bp (K x n_p), one class per blockIdx.z.  128x128 tile,
// 256 threads, 8x8 outputs per thread, K-slices of 8 staged through shared memory.
constexpr int GM = 128, GN = 128, GK = 8;

__global__ void __launch_bounds__(256)
gemm_fp32_kernel(const float* __restrict__ A, int64_t a_stride_class, int M, int K,
                 float* const* __restrict__ Bmat, const int* __restrict__ ncols,
                 float* __restrict__ C, int64_t c_ld, const int* __restrict__ c_off) {
  const int cls = blockIdx.z;
  const int Nc = ncols[cls];
  const int n0 = blockIdx.x * GN, m0 = blockIdx.y * GM;
  if (n0 >= Nc || m0 >= M) return;
  const float* Ap = A + cls * a_stride_class;
  const float* Bp = Bmat[cls];
  __shared__ __align__(16) float As[2][GK][GM];
  __shared__ __align__(16) float Bs[2][GK][GN];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  // loaders: A tile GM x GK (row m, col k): 1024 elements, 4 per thread
  //          B tile GK x GN: 1024 elements, 4 per thread
  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      const int mm = e / GK, kk = e % GK;
      const int gm = m0 + mm, gk = k0 + kk;
      As[buf][kk][mm] = (gm < M && gk < K) ? __ldg(&Ap[(int64_t)gm * K + gk]) : 0.f;
      const int kb = e / GN, nn = e % GN;
      const int gkb = k0 + kb, gn = n0 + nn;
      Bs[buf][kb][nn] = (gkb < K && gn < Nc) ? __ldg(&Bp[(int64_t)gkb * Nc + gn]) : 0.f;
    }
  };
  int buf = 0;
  load(0, 0);
  __syncthreads();
  for (int k0 = 0; k0 < K; k0 += GK) {
    if (k0 + GK < K) load(buf ^ 1, k0 + GK);
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      float a[8], b[8];
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
      a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
      a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
      b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
      b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    buf ^= 1;
    __syncthreads();
  }
  float* Cc = C + c_off[cls];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if (gn < Nc) Cc[(int64_t)gm * c_ld + gn] = acc[i][j];
    }
  }
}

// ------------------------------------------------------------------ expand + norms
// a[b][i] = s_re * C[b][col_re[i]] + i * s_im * C[b][col_im[i]]  (col_im < 0 -> 0)
__global__ void expand_kernel(const float* __restrict__ C, int64_t c_ld, int B, int ne,
                              const int* __restrict__ col_re, const int* __restrict__ col_im,
                              const signed char* __restrict__ s_re, const signed char* __restrict__ s_im,
                              float2* __restrict__ out, int64_t out_stride, float* __restrict__ norms) {
  const int b = blockIdx.x;
  if (b >= B) return;
  const float* c = C + (int64_t)b * c_ld;
  float ss = 0.f;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const float re = s_re[i] * c[col_re[i]];
    const float im = col_im[i] >= 0 ? s_im[i] * c[col_im[i]] : 0.f;
    out[(int64_t)b * out_stride + i] = make_float2(re, im);
    ss += re * re + im * im;
  }
  if (norms) {
    __shared__ float red[32];
    ss = warp_sum(ss);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x < 32) {
      float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
      v = warp_sum(v);
      if (threadIdx.x == 0) norms[b] = sqrtf(v);
    }
  }
}

// ------------------------------------------------------------------ sigma
// sigma[b][Dindex(l, m, mp)] = (-1)^(m+mp) sum_k aT[l, -mp, k] conj(aV[b][l, -m, k])
// One CTA per (degree l, subtomogram b), largest degrees first.  The rows mu = -l..l of the
// template and of the subtomogram's coefficients (K = kpad[l] radial entries each, gathered
// through kidx) are staged in shared memory with an odd row stride; each output then reads
// two rows there: sigma[l, m, m'] = (-1)^(m+m') sum_k T[-m', k] conj(V[-m, k]).
__global__ void __launch_bounds__(256)
sigma_kernel(const float2* __restrict__ aV, int64_t v_stride, const float2* __restrict__ aT, int lout,
             const int* __restrict__ kpad, const int* __restrict__ koff, const int* __restrict__ kidx,
             float2* __restrict__ sigma, int64_t s_stride) {
  extern __shared__ __align__(16) float2 ssm[];
  const int l = lout - blockIdx.x, b = blockIdx.y;
  const int w = 2 * l + 1;
  const int K = kpad[l];
  const int ks = K | 1;  // odd row stride: neighbouring rows fall in different banks
  float2* sT = ssm;
  float2* sV = ssm + w * ks;
  const int* tab = kidx + koff[l];
  const float2* v = aV + (int64_t)b * v_stride;
  for (int e = threadIdx.x; e < w * K; e += blockDim.x) {
    const int row = e / K, k = e - (e / K) * K;
    const int idx = __ldg(&tab[e]);
    sT[row * ks + k] = idx >= 0 ? __ldg(&aT[idx]) : make_float2(0.f, 0.f);
    sV[row * ks + k] = idx >= 0 ? __ldg(&v[idx]) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* out = sigma + (int64_t)b * s_stride + mtb_dsize(l - 1);
  // a thread: one column c (m' = c - l) and four rows a = 4 aq .. 4 aq + 3 (m = a - l); the
  // lanes of a warp take consecutive c (odd row stride: no bank conflicts) and mostly share
  // aq (the four row reads are broadcasts), so one template read serves four products
  const int naq = (w + 3) >> 2;
  for (int e = threadIdx.x; e < naq * w; e += blockDim.x) {
    const int aq = e / w, c = e - (e / w) * w;
    // row of -m' is 2l - c, row of -m is 2l - a
    const float2* tr = sT + (2 * l - c) * ks;
    const float2* vr[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) vr[j] = sV + (2 * l - min(4 * aq + j, w - 1)) * ks;
    float re[4] = {0.f, 0.f, 0.f, 0.f}, im[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < K; ++k) {
      const float2 t = tr[k];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 u = vr[j][k];
        // t * conj(u)
        re[j] += t.x * u.x + t.y * u.y;
        im[j] += t.y * u.x - t.x * u.y;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = 4 * aq + j;
      if (a < w) {
        const float sgn = ((a + c) & 1) ? -1.f : 1.f;  // (-1)^(m+mp) = (-1)^(a+c-2l)
        out[a * w + c] = make_float2(sgn * re[j], sgn * im[j]);
      }
    }
  }
}

template <typename T>
int upload(T** dst, const T* src, size_t n) {
  if (n == 0) { *dst = nullptr; return MTB_OK; }
  if (cudaMalloc(dst, n * sizeof(T)) != cudaSuccess) return MTB_ERR_OOM;
  if (cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return MTB_ERR_CUDA;
  return MTB_OK;
}

}  // namespace

struct mtb_fle {
  mtb_fle_config cfg;
  int class_cols[kClasses];
  int class_off[kClasses];
  float* basis[kClasses];
  float** d_basis;
  int* d_class_cols;
  int* d_class_off;
  int* rep_img;
  int* col_re;
  int* col_im;
  signed char* s_re;
  signed char* s_im;
  float* A;      // (8, max_batch, n_rep) folded channels
  float* C;      // (max_batch, n_cols) real coefficients, class blocks side by side
  int* kpad;
  int* koff;
  int* kidx;
  int kmax;      // max over degrees of kpad
  FleTc tc;
  bool use_tc;
};

extern "C" int mtb_fle_create(const mtb_fle_config* cfg, mtb_fle** out) {
  MTB_ARG_CHECK(cfg && out, "null argument");
  *out = nullptr;
  MTB_ARG_CHECK(cfg->N >= 2 && cfg->max_batch >= 1 && cfg->ne >= 1 && cfg->n_rep >= 1 && cfg->n_cols >= 1,
                "bad FLE sizes");
  MTB_ARG_CHECK(cfg->lmax >= 0 && cfg->n_lk >= 1 && cfg->n_r2 >= 1, "bad FLE table sizes");
  MTB_ARG_CHECK(cfg->rep_img && cfg->rep_cos && cfg->rep_phi && cfg->rep_r2 && cfg->jtab && cfg->col_class &&
                    cfg->col_l && cfg->col_m && cfg->col_part && cfg->col_lk && cfg->col_scale && cfg->coef_col_re &&
                    cfg->coef_col_im && cfg->coef_sign_re && cfg->coef_sign_im && cfg->kpad && cfg->kidx,
                "null table pointer");
  mtb_fle* h = new mtb_fle();
  memset(h, 0, sizeof(*h));
  h->cfg = *cfg;
  auto fail = [&](int code) { mtb_fle_destroy(h); return code; };
  const int nc = cfg->n_cols, nr = cfg->n_rep, L = cfg->lmax;
  // columns per class and position of each column inside its class block: by degree (stable),
  // so that a 256-column tile of the tensor-core GEMM spans a narrow range of l
  std::vector<int> pos(nc);
  std::vector<std::vector<int>> by_class(kClasses);
  for (int c = 0; c < nc; ++c) {
    const int k = cfg->col_class[c];
    if (k < 0 || k >= kClasses) return fail(MTB_ERR_ARG);
    if (cfg->col_l[c] < 0 || cfg->col_l[c] > L) return fail(MTB_ERR_ARG);
    by_class[k].push_back(c);
  }
  for (int k = 0; k < kClasses; ++k) {
    std::stable_sort(by_class[k].begin(), by_class[k].end(),
                     [&](int a, int b) { return cfg->col_l[a] < cfg->col_l[b]; });
    for (size_t j = 0; j < by_class[k].size(); ++j) pos[by_class[k][j]] = (int)j;
    h->class_cols[k] = (int)by_class[k].size();
  }
  int off = 0;
  for (int k = 0; k < kClasses; ++k) { h->class_off[k] = off; off += h->class_cols[k]; }
  // columns grouped by (l, m)
  std::vector<int> lm_start((L + 1) * (L + 1) + 1, 0), col_list(nc);
  for (int c = 0; c < nc; ++c) {
    if (cfg->col_l[c] < 0 || cfg->col_l[c] > L || cfg->col_m[c] < 0 || cfg->col_m[c] > cfg->col_l[c] ||
        cfg->col_lk[c] < 0 || cfg->col_lk[c] >= cfg->n_lk)
      return fail(MTB_ERR_ARG);
    lm_start[cfg->col_l[c] * (L + 1) + cfg->col_m[c] + 1]++;
  }
  for (size_t i = 1; i < lm_start.size(); ++i) lm_start[i] += lm_start[i - 1];
  {
    std::vector<int> fillp(lm_start.begin(), lm_start.end() - 1);
    for (int c = 0; c < nc; ++c) col_list[fillp[cfg->col_l[c] * (L + 1) + cfg->col_m[c]]++] = c;
  }
  for (int i = 0; i < nr; ++i)
    if (cfg->rep_r2[i] < 0 || cfg->rep_r2[i] >= cfg->n_r2) return fail(MTB_ERR_ARG);
  for (int i = 0; i < nr * 8; ++i)
    if (cfg->rep_img[i] >= cfg->N * cfg->N * cfg->N) return fail(MTB_ERR_ARG);
  // global column index of each (class, pos): class_off + pos
  std::vector<int> gcol(nc);
  for (int c = 0; c < nc; ++c) gcol[c] = h->class_off[cfg->col_class[c]] + pos[c];
  std::vector<int> cre(cfg->ne), cim(cfg->ne);
  for (int i = 0; i < cfg->ne; ++i) {
    const int r = cfg->coef_col_re[i], m = cfg->coef_col_im[i];
    if (r < 0 || r >= nc || m >= nc) return fail(MTB_ERR_ARG);
    cre[i] = gcol[r];
    cim[i] = m >= 0 ? gcol[m] : -1;
  }
  // sigma gather table offsets
  std::vector<int> koff(L + 1);
  int kt = 0;
  for (int l = 0; l <= L; ++l) { koff[l] = kt; kt += (2 * l + 1) * cfg->kpad[l]; }
  for (int l = 0; l <= L; ++l) h->kmax = cfg->kpad[l] > h->kmax ? cfg->kpad[l] : h->kmax;
  for (int i = 0; i < kt; ++i)
    if (cfg->kidx[i] >= cfg->ne) return fail(MTB_ERR_ARG);

  int rc = MTB_OK;
  for (int k = 0; k < kClasses && !rc; ++k) {
    const size_t n = (size_t)nr * (h->class_cols[k] ? h->class_cols[k] : 1);
    if (cudaMalloc(&h->basis[k], n * sizeof(float)) != cudaSuccess) rc = MTB_ERR_OOM;
  }
  if (!rc) rc = upload(&h->d_basis, h->basis, kClasses);
  if (!rc) rc = upload(&h->d_class_cols, h->class_cols, kClasses);
  if (!rc) rc = upload(&h->d_class_off, h->class_off, kClasses);
  if (!rc) rc = upload(&h->rep_img, cfg->rep_img, (size_t)nr * 8);
  if (!rc) rc = upload(&h->col_re, cre.data(), cre.size());
  if (!rc) rc = upload(&h->col_im, cim.data(), cim.size());
  if (!rc) rc = upload(&h->s_re, cfg->coef_sign_re, (size_t)cfg->ne);
  if (!rc) rc = upload(&h->s_im, cfg->coef_sign_im, (size_t)cfg->ne);
  if (!rc) rc = upload(&h->kpad, cfg->kpad, (size_t)L + 1);
  if (!rc) rc = upload(&h->koff, koff.data(), koff.size());
  if (!rc) rc = upload(&h->kidx, cfg->kidx, (size_t)kt);
  // the FP32 fold buffer serves the CUDA-core GEMM only (the tensor-core path folds into its own bf16 operand)
  if (!rc && cfg->precision == MTB_FLE_FP32 &&
      cudaMalloc(&h->A, (size_t)kClasses * cfg->max_batch * nr * sizeof(float)) != cudaSuccess)
    rc = MTB_ERR_OOM;
  if (!rc && cudaMalloc(&h->C, (size_t)cfg->max_batch * nc * sizeof(float)) != cudaSuccess) rc = MTB_ERR_OOM;
  if (rc) return fail(rc);

  // build the basis on the device (one-time), from the compact host tables
  double *d_cos = nullptr, *d_phi = nullptr, *d_j = nullptr, *d_scale = nullptr;
  int *d_r2 = nullptr, *d_lms = nullptr, *d_cl = nullptr, *d_cls = nullptr, *d_pos = nullptr, *d_part = nullptr,
      *d_lk = nullptr;
  rc = upload(&d_cos, cfg->rep_cos, (size_t)nr);
  if (!rc) rc = upload(&d_phi, cfg->rep_phi, (size_t)nr);
  if (!rc) rc = upload(&d_r2, cfg->rep_r2, (size_t)nr);
  if (!rc) rc = upload(&d_j, cfg->jtab, (size_t)cfg->n_r2 * cfg->n_lk);
  if (!rc) rc = upload(&d_lms, lm_start.data(), lm_start.size());
  if (!rc) rc = upload(&d_cl, col_list.data(), col_list.size());
  if (!rc) rc = upload(&d_cls, cfg->col_class, (size_t)nc);
  if (!rc) rc = upload(&d_pos, pos.data(), pos.size());
  if (!rc) rc = upload(&d_part, cfg->col_part, (size_t)nc);
  if (!rc) rc = upload(&d_lk, cfg->col_lk, (size_t)nc);
  if (!rc) rc = upload(&d_scale, cfg->col_scale, (size_t)nc);
  if (!rc) {
    const int total = nr * (L + 1);
    build_basis_kernel<<<(total + 127) / 128, 128>>>(nr, L, d_cos, d_phi, d_r2, d_j, cfg->n_lk, d_lms, d_cl, d_cls,
                                                     d_pos, d_part, d_lk, d_scale, h->d_basis, h->d_class_cols);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = MTB_ERR_CUDA;
  }
  cudaFree(d_cos); cudaFree(d_phi); cudaFree(d_r2); cudaFree(d_j); cudaFree(d_lms); cudaFree(d_cl);
  cudaFree(d_cls); cudaFree(d_pos); cudaFree(d_part); cudaFree(d_lk); cudaFree(d_scale);
  if (rc) return fail(rc);
  if (cfg->precision == MTB_FLE_BF16X3 || cfg->precision == MTB_FLE_BF16_SPLIT) {
    // per class, the highest degree of each column position (columns are sorted by degree)
    std::vector<std::vector<int>> col_deg(kClasses);
    for (int k = 0; k < kClasses; ++k) {
      col_deg[k].resize(h->class_cols[k]);
      for (size_t j = 0; j < by_class[k].size(); ++j) col_deg[k][j] = cfg->col_l[by_class[k][j]];
    }
    const int split_degree = cfg->precision == MTB_FLE_BF16X3 ? -1 : cfg->split_degree;
    rc = fle_tc_prepare(&h->tc, h->basis, h->class_cols, h->class_off, nr, cfg->max_batch, nc, col_deg,
                        split_degree);
    if (rc) return fail(rc);
    h->use_tc = true;
    // the FP32 basis was only the source of the hi/lo split: release it (at 128^3, L = 64 it
    // is 33 GB, as large as the split copy)
    for (int k = 0; k < kClasses; ++k) {
      cudaFree(h->basis[k]);
      h->basis[k] = nullptr;
    }
    if (cudaGetLastError() != cudaSuccess) return fail(MTB_ERR_CUDA);
  } else if (cfg->precision != MTB_FLE_FP32) {
    return fail(MTB_ERR_ARG);
  }
  *out = h;
  return MTB_OK;
}

extern "C" void mtb_fle_destroy(mtb_fle* h) {
  if (!h) return;
  for (int k = 0; k < kClasses; ++k) if (h->basis[k]) cudaFree(h->basis[k]);
  fle_tc_release(&h->tc);
  void* ptrs[] = {h->d_basis, h->d_class_cols, h->d_class_off, h->rep_img, h->col_re, h->col_im, h->s_re, h->s_im,
                  h->A, h->C, h->kpad, h->koff, h->kidx};
  for (void* p : ptrs) if (p) cudaFree(p);
  delete h;
}

extern "C" int mtb_fle_forward(mtb_fle* h, const float* vol, int B, float* coeffs, int64_t coeff_stride,
                               float* norms, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(vol && coeffs, "null pointer");
  MTB_ARG_CHECK(coeff_stride >= h->cfg.ne, "coefficient row shorter than ne");
  cudaStream_t st = (cudaStream_t)stream;
  const int nr = h->cfg.n_rep, N = h->cfg.N;
  const int64_t vstride = (int64_t)N * N * N;
  const int64_t astride = (int64_t)h->cfg.max_batch * nr;
  if (h->use_tc) {
    const int rc = fle_tc_forward(&h->tc, vol, vstride, B, h->rep_img, h->C, st);
    if (rc) return rc;
  } else {
    dim3 fg((nr + 255) / 256, B);
    mtb_prof_begin(st);
    fold_kernel<<<fg, 256, 0, st>>>(vol, vstride, B, nr, h->rep_img, h->A, astride);
    mtb_prof_end(st, "fold_kernel");
    MTB_LAUNCH_CHECK();
    int maxc = 0;
    for (int k = 0; k < kClasses; ++k) maxc = h->class_cols[k] > maxc ? h->class_cols[k] : maxc;
    dim3 gg((maxc + GN - 1) / GN, (B + GM - 1) / GM, kClasses);
    mtb_prof_begin(st);
    gemm_fp32_kernel<<<gg, 256, 0, st>>>(h->A, astride, B, nr, h->d_basis, h->d_class_cols, h->C, h->cfg.n_cols,
                                         h->d_class_off);
    mtb_prof_end(st, "gemm_fp32_kernel");
    MTB_LAUNCH_CHECK();
  }
  mtb_prof_begin(st);
  expand_kernel<<<B, 256, 0, st>>>(h->C, h->cfg.n_cols, B, h->cfg.ne, h->col_re, h->col_im, h->s_re, h->s_im,
                                   reinterpret_cast<float2*>(coeffs), coeff_stride, norms);
  mtb_prof_end(st, "expand_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

extern "C" int mtb_sigma_upto(mtb_fle* h, const float* coeffs, int64_t coeff_stride, const float* tmpl, int B,
                              int lmax_out, float* sigma, int64_t sigma_stride, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0, "negative batch");
  MTB_ARG_CHECK(lmax_out >= 0 && lmax_out <= h->cfg.lmax, "lmax_out must be in [0, lmax of the expansion]");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(coeffs && tmpl && sigma, "null pointer");
  MTB_ARG_CHECK(coeff_stride >= h->cfg.ne, "coefficient row shorter than ne");
  MTB_ARG_CHECK(sigma_stride >= mtb_dsize(lmax_out), "sigma row shorter than dsize(lmax_out)");
  MTB_ARG_CHECK(B <= 65535, "batch too large for one launch");
  const size_t smem = (size_t)2 * (2 * lmax_out + 1) * (h->kmax | 1) * sizeof(float2);
  MTB_CUDA_TRY(cudaFuncSetAttribute(sigma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  mtb_prof_begin((cudaStream_t)stream);
  sigma_kernel<<<dim3(lmax_out + 1, B), 256, smem, (cudaStream_t)stream>>>(
      reinterpret_cast<const float2*>(coeffs), coeff_stride, reinterpret_cast<const float2*>(tmpl), lmax_out,
      h->kpad, h->koff, h->kidx, reinterpret_cast<float2*>(sigma), sigma_stride);
  mtb_prof_end((cudaStream_t)stream, "sigma_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

extern "C" int mtb_sigma(mtb_fle* h, const float* coeffs, int64_t coeff_stride, const float* tmpl, int B,
                         float* sigma, int64_t sigma_stride, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  return mtb_sigma_upto(h, coeffs, coeff_stride, tmpl, B, h->cfg.lmax, sigma, sigma_stride, stream);
}

// The sigma gather tables of a handle, for the template backward (backward.cu).
int fle_sigma_tables(const mtb_fle* h, const int** kpad, const int** koff, const int** kidx, int* lmax, int* kmax,
                     int* ne) {
  *kpad = h->kpad;
  *koff = h->koff;
  *kidx = h->kidx;
  *lmax = h->cfg.lmax;
  *kmax = h->kmax;
  *ne = h->cfg.ne;
  return MTB_OK;
}

extern "C" int mtb_fle_inject_stall(mtb_fle* h, int on) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(h->use_tc, "the stall hook acts on the tensor-core path only (precision MTB_FLE_BF16X3)");
  h->tc.stall = on ? 1 : 0;
  return MTB_OK;
}

extern "C" int mtb_fle_status(mtb_fle* h, mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  if (!h->use_tc) {
    MTB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return MTB_OK;
  }
  const int rc = fle_tc_check(&h->tc, (cudaStream_t)stream);
  if (rc) mtb_set_last_error("tensor-core FLE GEMM: a bounded wait ran out", __FILE__, __LINE__);
  return rc;
}

extern "C" int mtb_fle_split_tiles(const mtb_fle* h, int* n_split, int* n_tiles) {
  MTB_ARG_CHECK(h && n_split && n_tiles, "null argument");
  *n_split = h->use_tc ? h->tc.n_split_tiles : 0;
  *n_tiles = h->use_tc ? h->tc.n_tiles : 0;
  return MTB_OK;
}
