// Frequency-marched Wigner-D Newton refinement on sm_100a (one CTA per candidate).
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   Newton march  src/matcha/core/Matcha.py:150-205 (_take_step), 239-367 (optimize),
//                 369-398 (stage loop)
//   D             src/matcha/core/WignerDMatrices.py:281-306, 673-801, 1291-1375
//   g, H          src/matcha/core/WignerDGradients.py:155-302
//
// The score of a point (a, b, g) is f = Re sum_l sum_{m'm} e^{i m' a} d^l_{m'm}(b) e^{i m g}
// sigma_{l m' m}.  Its Euler gradient and Hessian are computed here from one sweep per
// fundamental-wedge chain instead of from the full D matrix:
//
//  * Symmetry folding.  d_{m m'} = d_{-m',-m} = (-1)^{m'-m} d_{m'm}, d_{-m,-m'} = d_{m'm}.
//    The four images (M',M), (M,M'), (-M,-M'), (-M',-M) of a wedge pair M' >= |M| carry the
//    phases z1 = e^{i(M'a + Mg)}, z2 = e^{i(Ma + M'g)} and their conjugates, so
//      sum over the images = d^l_{M'M}(b) Re(z1 S1_l + z2 S2_l)
//    with S1 = sigma(M',M) + s conj sigma(-M',-M), S2 = s sigma(M,M') + conj sigma(-M,-M'),
//    s = (-1)^{M'-M} (diagonal and anti-diagonal images coincide and are counted once).
//    S is candidate-independent: it is folded once per subtomogram into a wedge-ordered
//    array, 16 bytes per (l, wedge pair) instead of 32 bytes of sigma.
//  * Phases out of the sum.  z1 and z2 are fixed along a chain (fixed M', M, all l), so a
//    thread accumulates A = sum_l d S, B = sum_l d' S, C = sum_l d'' S per chain and applies
//    z1, z2 and the factors i M', i M of the a- and g-derivatives once at the chain's end.
//  * beta derivatives by differentiated recurrences.  d^l = (al cos b - be) d^{l-1} - ga
//    d^{l-2} (the three-term recurrence in l; al, be, ga from a candidate-independent FP64
//    table) is differentiated twice in b, so d', d'' ride along in registers: no neighbour
//    rows, no shared d blocks and no barriers inside a pass.
//
// Each thread walks whole chains (a wedge pair from l = M' to the stage degree); chains are
// dealt to threads in boustrophedon order so that long (small M') and short chains mix.
#include <math.h>
#include "common.cuh"
#include "newton.cuh"

namespace {

constexpr int kNT = kNewtonThreads;

enum { A_VAL = 0, A_GA, A_GB, A_GG, A_HAA, A_HAB, A_HAG, A_HBB, A_HBG, A_HGG, A_N };

struct Smem {
  float2* ea;   // e^{i k a}, index k + Li
  float2* eg;   // e^{i k g}, index k + Li
  double* phc;  // cos(b/2)^k, k = 0 .. 2 Li + 2
  double* pt;   // (-sin(b/2))^k
  float* red;   // (threads/32) x A_N
  float* res;   // A_N
};

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  while (n) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// Offset of degree l in the wedge-ordered arrays: sum_{j < l} (j + 1)^2.
__host__ __device__ __forceinline__ int64_t wedge_off(int l) { return (int64_t)l * (l + 1) * (2 * l + 1) / 6; }

// Wedge index p = M'^2 + M' + M, 0 <= |M| <= M'.
__device__ __forceinline__ void wedge_pair(int p, int& mp, int& m) {
  mp = (int)sqrtf((float)p);
  while (mp * mp > p) --mp;
  while ((mp + 1) * (mp + 1) <= p) ++mp;
  m = p - mp * mp - mp;
}

// Folded sigma {Re S1, Im S1, Re S2, Im S2} of wedge pair (mp, m) at degree l >= mp, read
// from the reference layout (flat [l][m'][m], w = 2l + 1).
__device__ __forceinline__ float4 fold_entry(const float2* __restrict__ sg, int l, int mp, int m) {
  const int w = 2 * l + 1;
  const float2* blk = sg + mtb_dsize(l - 1);
  auto at = [&](int r, int c) -> float2 { return __ldg(blk + (r + l) * w + (c + l)); };
  const float s = ((mp - m) & 1) ? -1.f : 1.f;
  const float2 s1 = at(mp, m);
  if (mp == 0) return make_float4(s1.x, s1.y, 0.f, 0.f);
  const float2 s4 = at(-mp, -m);
  const float r1 = s1.x + s * s4.x, i1 = s1.y - s * s4.y;
  if (m == mp || m == -mp) return make_float4(r1, i1, 0.f, 0.f);
  const float2 s2 = at(m, mp), s3 = at(-m, -mp);
  return make_float4(r1, i1, s * s2.x + s3.x, s * s2.y - s3.y);
}

// S[b][wedge_off(l) + p] for every degree l <= Lmax and wedge pair p < (l + 1)^2.
__global__ void fold_sigma_kernel(const float2* __restrict__ sigma, int64_t stride, int64_t n_fold,
                                  float4* __restrict__ S) {
  const int l = blockIdx.x, b = blockIdx.y;
  const float2* sg = sigma + (int64_t)b * stride;
  float4* out = S + (int64_t)b * n_fold + wedge_off(l);
  const int n = (l + 1) * (l + 1);
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    int mp, m;
    wedge_pair(p, mp, m);
    out[p] = fold_entry(sg, l, mp, m);
  }
}

// Recurrence factors {al, be, ga} of d^l_{M'M} = (al cos b - be) d^{l-1} - ga d^{l-2}
// for l > M', from
//   (l-1) sqrt((l^2-m^2)(l^2-m'^2)) d^l = (2l-1)(l(l-1) cos b - m m') d^{l-1}
//                                        - l sqrt(((l-1)^2-m^2)((l-1)^2-m'^2)) d^{l-2},
// in FP64; d^1_{00} = cos b d^0_{00}.  Entries with l <= M' are unused and zero.
__global__ void coef_kernel(int64_t n, float4* __restrict__ coef) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int l = 0;
    while (wedge_off(l + 1) <= t) ++l;
    const int p = (int)(t - wedge_off(l));
    int mp, m;
    wedge_pair(p, mp, m);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (l == 1 && mp == 0) {
      v.x = 1.f;
    } else if (l >= 2 && l > mp) {
      const double L = l, m2 = (double)m * m, mp2 = (double)mp * mp;
      const double inv = 1.0 / sqrt((L * L - m2) * (L * L - mp2));
      const double xl1 = ((L - 1) * (L - 1) - m2) * ((L - 1) * (L - 1) - mp2);
      v.x = (float)((2 * L - 1) * L * inv);
      v.y = (float)((2 * L - 1) * (double)m * mp * inv / (L - 1));
      v.z = (float)(L * sqrt(fmax(xl1, 0.0)) * inv / (L - 1));
    }
    coef[t] = v;
  }
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One sweep over the chains of stage degree Li at (a, be, ga): value, and with DERIVS the
// Euler gradient and Hessian, left in sm.res.  FOLDED reads the folded sigma S of this
// subtomogram; otherwise each step folds the four images from sigma itself.
template <bool DERIVS, bool FOLDED>
__device__ __forceinline__ void pass(const float4* __restrict__ S, const float2* __restrict__ sg,
                                     const float4* __restrict__ coef, const double* __restrict__ Ctab, float a,
                                     float be, float ga, int Li, const Smem sm) {
  const int tid = threadIdx.x;
  const double two_pi = 6.283185307179586;
  for (int r = tid; r < 2 * Li + 1; r += kNT) {
    double t = (double)(r - Li) * (double)a;
    t -= two_pi * rint(t / two_pi);
    float s, c;
    sincosf((float)t, &s, &c);
    sm.ea[r] = make_float2(c, s);
    t = (double)(r - Li) * (double)ga;
    t -= two_pi * rint(t / two_pi);
    sincosf((float)t, &s, &c);
    sm.eg[r] = make_float2(c, s);
  }
  double hs, hc;
  sincos(0.5 * (double)be, &hs, &hc);
  for (int k = tid; k <= 2 * Li + 2; k += kNT) {
    sm.phc[k] = ipow(hc, k);
    sm.pt[k] = ipow(-hs, k);
  }
  float sb, cb;
  sincosf(be, &sb, &cb);

  float acc[A_N];
#pragma unroll
  for (int i = 0; i < A_N; ++i) acc[i] = 0.f;
  __syncthreads();

  const int n = (Li + 1) * (Li + 1);
  int k = 0;
  for (int base = 0; base < n; base += kNT, ++k) {
    const int p = base + ((k & 1) ? kNT - 1 - tid : tid);
    if (p >= n) continue;
    int mp, m;
    wedge_pair(p, mp, m);
    // start of the chain at l = M': d = C cos^P (-sin)^Q of b/2, P = M'+M, Q = M'-M
    const int P = mp + m, Q = mp - m;
    const double C = Ctab[p];
    float d1 = (float)(C * sm.phc[P] * sm.pt[Q]), d0 = 0.f;
    float e1 = 0.f, e0 = 0.f, g1 = 0.f, g0 = 0.f;
    if (DERIVS) {
      double fp = 0.0, fpp = -(double)(2 * P * Q + P + Q) * sm.phc[P] * sm.pt[Q];
      if (P >= 1) fp += P * sm.phc[P - 1] * sm.pt[Q + 1];
      if (Q >= 1) fp -= Q * sm.phc[P + 1] * sm.pt[Q - 1];
      if (P >= 2) fpp += (double)(P * (P - 1)) * sm.phc[P - 2] * sm.pt[Q + 2];
      if (Q >= 2) fpp += (double)(Q * (Q - 1)) * sm.phc[P + 2] * sm.pt[Q - 2];
      e1 = (float)(0.5 * C * fp);
      g1 = (float)(0.25 * C * fpp);
    }
    float4 s;
    if (FOLDED) s = __ldg(S + wedge_off(mp) + p);
    else s = fold_entry(sg, mp, mp, m);
    float a1r = d1 * s.x, a1i = d1 * s.y, a2r = d1 * s.z, a2i = d1 * s.w;
    float b1r = 0.f, b1i = 0.f, b2r = 0.f, b2i = 0.f, c1r = 0.f, c1i = 0.f, c2r = 0.f, c2i = 0.f;
    if (DERIVS) {
      b1r = e1 * s.x; b1i = e1 * s.y; b2r = e1 * s.z; b2i = e1 * s.w;
      c1r = g1 * s.x; c1i = g1 * s.y; c2r = g1 * s.z; c2i = g1 * s.w;
    }
    const float4* cp = coef + wedge_off(mp + 1) + p;
    const float4* sp = FOLDED ? S + wedge_off(mp + 1) + p : nullptr;
#pragma unroll 2
    for (int l = mp + 1; l <= Li; ++l) {
      const float4 cf = __ldg(cp);
      const float t = fmaf(cf.x, cb, -cf.y);
      const float v = fmaf(t, d1, -cf.z * d0);
      if (DERIVS) {
        const float as = cf.x * sb;
        const float vp = fmaf(t, e1, -fmaf(as, d1, cf.z * e0));
        const float vpp = fmaf(t, g1, -fmaf(2.f * as, e1, fmaf(cf.x * cb, d1, cf.z * g0)));
        e0 = e1; e1 = vp;
        g0 = g1; g1 = vpp;
      }
      d0 = d1; d1 = v;
      if (FOLDED) s = __ldg(sp);
      else s = fold_entry(sg, l, mp, m);
      a1r = fmaf(v, s.x, a1r); a1i = fmaf(v, s.y, a1i);
      a2r = fmaf(v, s.z, a2r); a2i = fmaf(v, s.w, a2i);
      if (DERIVS) {
        b1r = fmaf(e1, s.x, b1r); b1i = fmaf(e1, s.y, b1i);
        b2r = fmaf(e1, s.z, b2r); b2i = fmaf(e1, s.w, b2i);
        c1r = fmaf(g1, s.x, c1r); c1i = fmaf(g1, s.y, c1i);
        c2r = fmaf(g1, s.z, c2r); c2i = fmaf(g1, s.w, c2i);
      }
      cp += (l + 1) * (l + 1);
      if (FOLDED) sp += (l + 1) * (l + 1);
    }
    // phases: z1 = e^{i(M'a + Mg)}, z2 = e^{i(Ma + M'g)}
    const float2 z1 = cmulf(sm.ea[mp + Li], sm.eg[m + Li]);
    const float2 z2 = cmulf(sm.ea[m + Li], sm.eg[mp + Li]);
    const float r1 = z1.x * a1r - z1.y * a1i, r2 = z2.x * a2r - z2.y * a2i;
    acc[A_VAL] += r1 + r2;
    if (DERIVS) {
      const float fM = (float)mp, fm = (float)m;
      const float j1 = z1.x * a1i + z1.y * a1r, j2 = z2.x * a2i + z2.y * a2r;
      const float q1 = z1.x * b1r - z1.y * b1i, q2 = z2.x * b2r - z2.y * b2i;
      const float k1 = z1.x * b1i + z1.y * b1r, k2 = z2.x * b2i + z2.y * b2r;
      const float h1 = z1.x * c1r - z1.y * c1i, h2 = z2.x * c2r - z2.y * c2i;
      acc[A_GA] -= fM * j1 + fm * j2;
      acc[A_GG] -= fm * j1 + fM * j2;
      acc[A_GB] += q1 + q2;
      acc[A_HAA] -= fM * fM * r1 + fm * fm * r2;
      acc[A_HGG] -= fm * fm * r1 + fM * fM * r2;
      acc[A_HAG] -= fM * fm * (r1 + r2);
      acc[A_HAB] -= fM * k1 + fm * k2;
      acc[A_HBG] -= fm * k1 + fM * k2;
      acc[A_HBB] += h1 + h2;
    }
  }

  // ---- block reduction
  const int lane = tid & 31, warp = tid >> 5;
  constexpr int NA = DERIVS ? A_N : 1;
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    const float v = warp_sum(acc[i]);
    if (lane == 0) sm.red[warp * A_N + i] = v;
  }
  __syncthreads();
  if (tid < NA) {
    float s = 0.f;
    for (int q = 0; q < kNT / 32; ++q) s += sm.red[q * A_N + tid];
    sm.res[tid] = s;
  }
  __syncthreads();
}

// Solve H x = g in FP64 with partial pivoting; false when a pivot is exactly zero
// (torch.linalg.solve raises "singular" there and the reference takes a zero step,
// Matcha.py:316-343).
__device__ bool solve3(const double H[3][3], const double g[3], double x[3]) {
  double A[3][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) A[i][j] = H[i][j];
    A[i][3] = g[i];
  }
  for (int c = 0; c < 3; ++c) {
    int piv = c;
    for (int r = c + 1; r < 3; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (A[piv][c] == 0.0 || !isfinite(A[piv][c])) return false;
    if (piv != c)
      for (int j = 0; j < 4; ++j) { double t = A[c][j]; A[c][j] = A[piv][j]; A[piv][j] = t; }
    for (int r = c + 1; r < 3; ++r) {
      const double f = A[r][c] / A[c][c];
      for (int j = c; j < 4; ++j) A[r][j] -= f * A[c][j];
    }
  }
  for (int r = 2; r >= 0; --r) {
    double s = A[r][3];
    for (int j = r + 1; j < 3; ++j) s -= A[r][j] * x[j];
    x[r] = s / A[r][r];
  }
  return true;
}

template <bool FOLDED>
__global__ void __launch_bounds__(kNT, 5)
newton_march_kernel(const float4* __restrict__ S, int64_t n_fold, const float2* __restrict__ sigma, int64_t stride,
                    int BC, int C, float* __restrict__ alpha, float* __restrict__ beta, float* __restrict__ gamma,
                    float* __restrict__ score, const double* __restrict__ Ctab, const float4* __restrict__ coef,
                    NewtonParams P) {
  __shared__ float2 s_ea[2 * kNewtonMaxL + 1], s_eg[2 * kNewtonMaxL + 1];
  __shared__ double s_phc[2 * kNewtonMaxL + 3], s_pt[2 * kNewtonMaxL + 3];
  __shared__ float s_red[(kNT / 32) * A_N], s_res[A_N];
  const Smem sm{s_ea, s_eg, s_phc, s_pt, s_red, s_res};

  const int cand = blockIdx.x;
  if (cand >= BC) return;
  const int b = cand / C;
  const float4* Sb = FOLDED ? S + (int64_t)b * n_fold : nullptr;
  const float2* sg = FOLDED ? nullptr : sigma + (int64_t)b * stride;
  const bool grad_step = (P.flags & MTB_SEARCH_GRADIENT_STEP) != 0;
  const float base_lr = grad_step ? 5e-7f : 1.f;

  float a = alpha[cand], be = beta[cand], ga = gamma[cand];
  float best = 0.f;
  for (int s = 0; s < P.n_stages; ++s) {
    const int Li = P.stages[s];
    if (P.num_steps > 0)
      pass<true, FOLDED>(Sb, sg, coef, Ctab, a, be, ga, Li, sm);
    else
      pass<false, FOLDED>(Sb, sg, coef, Ctab, a, be, ga, Li, sm);
    best = sm.res[A_VAL];
    double g[3] = {sm.res[A_GA], sm.res[A_GB], sm.res[A_GG]};
    double H[3][3] = {{sm.res[A_HAA], sm.res[A_HAB], sm.res[A_HAG]},
                      {sm.res[A_HAB], sm.res[A_HBB], sm.res[A_HBG]},
                      {sm.res[A_HAG], sm.res[A_HBG], sm.res[A_HGG]}};
    float lr = base_lr;
    for (int it = 0; it < P.num_steps; ++it) {
      double x[3] = {0.0, 0.0, 0.0};
      if (grad_step) {
        for (int i = 0; i < 3; ++i) x[i] = -g[i];
      } else if (!solve3(H, g, x)) {
        x[0] = x[1] = x[2] = 0.0;
      }
      const float ta = a - lr * (float)x[0];
      const float tb = be - lr * (float)x[1];
      const float tg = ga - lr * (float)x[2];
      const bool last = (it == P.num_steps - 1);
      __syncthreads();  // everyone has read the previous results
      if (last)
        pass<false, FOLDED>(Sb, sg, coef, Ctab, ta, tb, tg, Li, sm);
      else
        pass<true, FOLDED>(Sb, sg, coef, Ctab, ta, tb, tg, Li, sm);
      const float ev = sm.res[A_VAL];
      if (ev > best) {
        a = ta; be = tb; ga = tg; best = ev;
        lr *= 1.1f;
        if (!last) {
          g[0] = sm.res[A_GA]; g[1] = sm.res[A_GB]; g[2] = sm.res[A_GG];
          H[0][0] = sm.res[A_HAA]; H[0][1] = H[1][0] = sm.res[A_HAB]; H[0][2] = H[2][0] = sm.res[A_HAG];
          H[1][1] = sm.res[A_HBB]; H[1][2] = H[2][1] = sm.res[A_HBG]; H[2][2] = sm.res[A_HGG];
        }
      } else {
        lr *= 0.5f;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    alpha[cand] = a;
    beta[cand] = be;
    gamma[cand] = ga;
    score[cand] = best;
  }
}

}  // namespace

int64_t newton_fold_entries(int Lmax) { return wedge_off(Lmax + 1); }

int newton_build_coef(int Lmax, float4* coef, cudaStream_t st) {
  MTB_ARG_CHECK(Lmax >= 0 && Lmax <= kNewtonMaxL, "Lmax exceeds the Newton march limit");
  const int64_t n = newton_fold_entries(Lmax);
  const int blocks = (int)((n + 255) / 256);
  coef_kernel<<<blocks, 256, 0, st>>>(n, coef);
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

int newton_launch(const float* sigma, int64_t stride, int B, int C, float* a, float* b, float* g, float* s,
                  const double* Ctab, const float4* coef, float4* fold, const NewtonParams& P, cudaStream_t st) {
  MTB_ARG_CHECK(P.Lmax >= 0 && P.Lmax <= kNewtonMaxL, "Lmax exceeds the Newton march limit");
  if (P.flags & MTB_SEARCH_COMPAT_TOP_BLOCK) return newton_stencil_launch(sigma, stride, B, C, a, b, g, s, Ctab, P, st);
  const int BC = B * C;
  const float2* sg = reinterpret_cast<const float2*>(sigma);
  const int64_t nf = newton_fold_entries(P.Lmax);
  if (fold) {
    fold_sigma_kernel<<<dim3(P.Lmax + 1, B), 256, 0, st>>>(sg, stride, nf, fold);
    MTB_LAUNCH_CHECK();
    newton_march_kernel<true><<<BC, kNT, 0, st>>>(fold, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef, P);
  } else {
    newton_march_kernel<false><<<BC, kNT, 0, st>>>(nullptr, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef, P);
  }
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}
