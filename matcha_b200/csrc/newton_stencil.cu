// Wigner-D Newton march that reproduces the reference's final-stage top-block arithmetic
// (Matcha(..., compat_top_block=True)): the m' = -Lmax row and m = -Lmax column of the last
// degree read as zero in D, and the beta derivatives come from the reference's row-shift
// stencil applied to that zeroed block, which is not the derivative of the zeroed score.
// This kernel therefore keeps the full small-d block of every degree in shared memory.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   Newton march  src/matcha/core/Matcha.py:150-205 (_take_step), 239-367 (optimize),
//                 369-398 (stage loop)
//   D             src/matcha/core/WignerDMatrices.py:281-306, 673-801, 1291-1375
//   g, H          src/matcha/core/WignerDGradients.py:155-302
//   top block     src/matcha/core/WignerDMatrices.py:573-576 (conjugate power of index
//                 ell_max never written)
//
// Per degree l the CTA
//   1. advances the three-term recurrence in l of d^l_{m'm} for the fundamental wedge
//      m' >= |m| (state in registers) and writes the four symmetric copies into a padded
//      shared block (two zero rows above and below, so neighbours need no bounds test);
//   2. contracts the block against sigma: each thread walks down one column m with a
//      sliding window d(m'-2..m'+2), so every d value is read once, and sigma is read
//      once per element (coalesced along m).
#include <math.h>
#include "common.cuh"
#include "newton.cuh"

namespace {

constexpr int kNT = 256;

enum { A_VAL = 0, A_GA, A_GB, A_GG, A_HAA, A_HAB, A_HAG, A_HBB, A_HBG, A_HGG, A_N };

struct Smem {
  float* dbuf[2];  // (W + 4) x W, level-l block at rows 2..2l+2, cols 0..2l
  float4* rowa[2]; // per row r of level l: {Re ea, Im ea, c1, c2}
  float4* rowb[2]; // per row r of level l: {tn2, t0, tp2, m'}
  float2* ea;      // e^{i m' a}, index m' + Li
  float2* eg;      // e^{i m g},  index m + Li
  float* red;      // (threads/32) x A_N
  float* res;      // A_N
  int4* level;     // per degree l: {magic = ceil(65536 / w), G = 256 / w, chunk = ceil(w / G), w}
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

template <int KP, bool DERIVS>
__device__ void pass(const float2* __restrict__ sig, const double* __restrict__ Ctab, float a, float be, float ga,
                     int Li, bool zap_top, int W, const Smem& sm) {
  const int tid = threadIdx.x;
  for (int r = tid; r < 2 * Li + 1; r += kNT) {
    const double two_pi = 6.283185307179586;
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
  const float cb = cosf(be);
  double hs, hc;
  sincos(0.5 * (double)be, &hs, &hc);

  float d1[KP], d0[KP], sq[KP];
  int pmp[KP], pm[KP];
#pragma unroll
  for (int k = 0; k < KP; ++k) {
    const int p = tid + k * kNT;
    int mp = (int)sqrtf((float)p);
    while (mp * mp > p) --mp;
    while ((mp + 1) * (mp + 1) <= p) ++mp;
    pmp[k] = mp;
    pm[k] = p - mp * mp - mp;
    d1[k] = 0.f; d0[k] = 0.f; sq[k] = 0.f;
  }

  float acc[A_N];
#pragma unroll
  for (int i = 0; i < A_N; ++i) acc[i] = 0.f;

  for (int l = 0; l <= Li; ++l) {
    const int w = 2 * l + 1;
    float* dcur = sm.dbuf[l & 1] + 2 * W;  // logical row 0
    const bool zap = zap_top && (l == Li);
    // ---- recurrence l-1 -> l on the wedge, symmetric copies into the block
    const int npair = (l + 1) * (l + 1);
    const float fl = (float)l;
    const float inv_lm = (l > 1) ? 1.f / (float)(l - 1) : 0.f;
    const float a1 = (2.f * fl - 1.f) * (fl - 1.f) * fl;
    const float a2 = 2.f * fl - 1.f;
#pragma unroll
    for (int k = 0; k < KP; ++k) {
      const int p = tid + k * kNT;
      if (p < npair) {
        const int mp = pmp[k], m = pm[k];
        float v;
        if (mp == l) {
          // l0 = m': (-1)^(m'-m) sqrt((2m')!/((m'+m)!(m'-m)!)) c^(m'+m) s^(m'-m)
          const int pc = mp + m, ps = mp - m;
          const double dv = Ctab[p] * ipow(hc, pc) * ipow(hs, ps);
          v = (float)((ps & 1) ? -dv : dv);
          d0[k] = 0.f;
          sq[k] = 0.f;
        } else if (l == 1) {
          v = cb * d1[k];
          d0[k] = d1[k];
          sq[k] = 1.f;
        } else {
          const float x = (fl * fl - (float)(m * m)) * (fl * fl - (float)(mp * mp));
          const float inv = rsqrtf(x);
          const float aa = a1 * cb - a2 * (float)(m * mp);
          v = (aa * d1[k] - fl * sq[k] * d0[k]) * inv * inv_lm;
          d0[k] = d1[k];
          sq[k] = x * inv;
        }
        d1[k] = v;
        const float vs = ((mp - m) & 1) ? -v : v;
        const int r1 = mp + l, c1 = m + l, r2 = -m + l, c2 = -mp + l;
        // d_{m'm} at (r1, c1); d_{m m'} = (-1)^(m'-m) d at (c1, r1);
        // d_{-m,-m'} = d at (r2, c2); d_{-m',-m} = (-1)^(m'-m) d at (c2, r2)
        dcur[r1 * W + c1] = (zap && (r1 == 0 || c1 == 0)) ? 0.f : v;
        dcur[c1 * W + r1] = (zap && (c1 == 0 || r1 == 0)) ? 0.f : vs;
        dcur[r2 * W + c2] = (zap && (r2 == 0 || c2 == 0)) ? 0.f : v;
        dcur[c2 * W + r2] = (zap && (c2 == 0 || r2 == 0)) ? 0.f : vs;
      }
    }
    // rows w, w+1 below the block read as zero
    for (int e = tid; e < 2 * w; e += kNT) {
      const int hi = e >= w;
      dcur[(w + hi) * W + (e - hi * w)] = 0.f;
    }
    // per-row data of this level
    {
      float4* ra = sm.rowa[l & 1];
      float4* rb = sm.rowb[l & 1];
      for (int r = tid; r < w; r += kNT) {
        const float mp = (float)(r - l);
        const float2 e = sm.ea[r - l + Li];
        if (DERIVS) {
          const float c1 = -0.5f * sqrtf(fmaxf((fl + mp) * (fl - mp + 1.f), 0.f));
          const float c2 = 0.5f * sqrtf(fmaxf((fl - mp) * (fl + mp + 1.f), 0.f));
          const float tn2 = 0.25f * sqrtf(fmaxf((fl + mp) * (fl - mp + 1.f) * (fl + mp - 1.f) * (fl - mp + 2.f), 0.f));
          const float t0 = -0.25f * ((fl + mp) * (fl - mp + 1.f) + (fl + mp + 1.f) * (fl - mp));
          const float tp2 = 0.25f * sqrtf(fmaxf((fl + mp + 1.f) * (fl - mp) * (fl + mp + 2.f) * (fl - mp - 1.f), 0.f));
          ra[r] = make_float4(e.x, e.y, c1, c2);
          rb[r] = make_float4(tn2, t0, tp2, mp);
        } else {
          ra[r] = make_float4(e.x, e.y, 0.f, 0.f);
        }
      }
    }
    __syncthreads();
    // ---- contraction: thread (column c, row chunk g)
    // g = tid / w and c = tid % w by a multiply with ceil(2^16 / w) (exact for tid < 256,
    // w <= 129); groups of `chunk` rows, G = 256 / w groups per column
    const int4 lv = sm.level[l];  // {magic, G, chunk, w}
    const int g = (tid * lv.x) >> 16;
    const int c = tid - g * w;
    const int r0 = g * lv.z, r1 = min(w, r0 + lv.z);
    if (g < lv.y && r0 < r1) {
      const float4* ra = sm.rowa[l & 1];
      const float4* rb = sm.rowb[l & 1];
      const float2 egc = sm.eg[c - l + Li];
      const float2* sp = sig + mtb_dsize(l - 1) + r0 * w + c;
      const float* dp = dcur + r0 * W + c;
      if (DERIVS) {
        float dm2 = dp[-2 * W], dm1 = dp[-W], dc = dp[0], dp1 = dp[W];
        float T = 0.f, U = 0.f, X = 0.f, MT = 0.f;
#pragma unroll 2
        for (int r = r0; r < r1; ++r) {
          const float dp2 = dp[2 * W];
          const float2 s = __ldg(sp);
          const float4 A = ra[r], Bq = rb[r];
          const float qx = egc.x * s.x - egc.y * s.y, qy = egc.x * s.y + egc.y * s.x;
          const float er = A.x * qx - A.y * qy, ei = A.x * qy + A.y * qx;
          const float mp = Bq.w;
          const float t = dc * er, u = dc * ei;
          T += t;
          U += u;
          acc[A_GA] -= mp * u;
          const float mt = mp * t;
          MT += mt;
          acc[A_HAA] -= mp * mt;
          const float db = A.z * dm1 + A.w * dp1;
          const float dbb = Bq.y * dc + Bq.x * dm2 + Bq.z * dp2;
          acc[A_GB] += db * er;
          const float x = db * ei;
          X += x;
          acc[A_HAB] -= mp * x;
          acc[A_HBB] += dbb * er;
          dm2 = dm1; dm1 = dc; dc = dp1; dp1 = dp2;
          dp += W;
          sp += w;
        }
        const float m = (float)(c - l);
        acc[A_VAL] += T;
        acc[A_GG] -= m * U;
        acc[A_HGG] -= m * m * T;
        acc[A_HAG] -= m * MT;
        acc[A_HBG] -= m * X;
      } else {
        float T = 0.f;
#pragma unroll 4
        for (int r = r0; r < r1; ++r) {
          const float2 s = __ldg(sp);
          const float4 A = ra[r];
          const float qx = egc.x * s.x - egc.y * s.y, qy = egc.x * s.y + egc.y * s.x;
          T += dp[0] * (A.x * qx - A.y * qy);
          dp += W;
          sp += w;
        }
        acc[A_VAL] += T;
      }
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

template <int KP>
__global__ void __launch_bounds__(kNT, 2)
newton_march_kernel(const float2* __restrict__ sigma, int64_t stride, int BC, int C,
                    float* __restrict__ alpha, float* __restrict__ beta, float* __restrict__ gamma,
                    float* __restrict__ score, const double* __restrict__ Ctab, NewtonParams P) {
  extern __shared__ __align__(16) float smem[];
  const int W = 2 * P.Lmax + 1;
  Smem sm;
  float4* f4 = reinterpret_cast<float4*>(smem);
  sm.rowa[0] = f4;
  sm.rowa[1] = f4 + W;
  sm.rowb[0] = f4 + 2 * W;
  sm.rowb[1] = f4 + 3 * W;
  sm.level = reinterpret_cast<int4*>(f4 + 4 * W);
  sm.ea = reinterpret_cast<float2*>(sm.level + (P.Lmax + 1));
  sm.eg = sm.ea + W;
  sm.red = reinterpret_cast<float*>(sm.eg + W);
  sm.res = sm.red + (kNT / 32) * A_N;
  sm.dbuf[0] = sm.res + A_N + 2;
  sm.dbuf[1] = sm.dbuf[0] + (W + 4) * W;
  for (int l = threadIdx.x; l <= P.Lmax; l += kNT) {
    const int w = 2 * l + 1, G = kNT / w;
    sm.level[l] = make_int4((65536 + w - 1) / w, G, (w + G - 1) / G, w);
  }

  const int cand = blockIdx.x;
  if (cand >= BC) return;
  // the two padding rows above each block are never written: zero them once
  for (int e = threadIdx.x; e < 2 * W; e += kNT) {
    sm.dbuf[0][e] = 0.f;
    sm.dbuf[1][e] = 0.f;
  }
  const int b = cand / C;
  const float2* sig = sigma + (int64_t)b * stride;
  const bool compat = (P.flags & MTB_SEARCH_COMPAT_TOP_BLOCK) != 0;
  const bool grad_step = (P.flags & MTB_SEARCH_GRADIENT_STEP) != 0;
  const float base_lr = grad_step ? 5e-7f : 1.f;

  float a = alpha[cand], be = beta[cand], ga = gamma[cand];
  float best = 0.f;
  __syncthreads();
  for (int s = 0; s < P.n_stages; ++s) {
    const int Li = P.stages[s];
    const bool zap = compat && (Li == P.Lmax);
    if (P.num_steps > 0)
      pass<KP, true>(sig, Ctab, a, be, ga, Li, zap, W, sm);
    else
      pass<KP, false>(sig, Ctab, a, be, ga, Li, zap, W, sm);
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
        pass<KP, false>(sig, Ctab, ta, tb, tg, Li, zap, W, sm);
      else
        pass<KP, true>(sig, Ctab, ta, tb, tg, Li, zap, W, sm);
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

size_t stencil_smem_bytes(int Lmax);

template <int KP>
int launch(const float2* sigma, int64_t stride, int BC, int C, float* a, float* b, float* g, float* s,
           const double* Ctab, const NewtonParams& P, cudaStream_t st) {
  const size_t smem = stencil_smem_bytes(P.Lmax);
  MTB_CUDA_TRY(cudaFuncSetAttribute(newton_march_kernel<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  mtb_prof_begin(st);
  newton_march_kernel<KP><<<BC, kNT, smem, st>>>(sigma, stride, BC, C, a, b, g, s, Ctab, P);
  mtb_prof_end(st, "newton_march_stencil_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

size_t stencil_smem_bytes(int Lmax) {
  const int W = 2 * Lmax + 1;
  return (size_t)4 * W * sizeof(float4) + (size_t)(Lmax + 1) * sizeof(int4) + (size_t)2 * W * sizeof(float2) +
         (size_t)((kNT / 32) * A_N + A_N + 2) * sizeof(float) + (size_t)2 * (W + 4) * W * sizeof(float);
}

}  // namespace

int newton_stencil_launch(const float* sigma, int64_t stride, int B, int C, float* a, float* b, float* g, float* s,
                  const double* Ctab, const NewtonParams& P, cudaStream_t st) {
  const int BC = B * C;
  const int pairs = (P.Lmax + 1) * (P.Lmax + 1);
  const int kp = (pairs + kNT - 1) / kNT;
  const float2* sg = reinterpret_cast<const float2*>(sigma);
  if (kp <= 2) return launch<2>(sg, stride, BC, C, a, b, g, s, Ctab, P, st);
  if (kp <= 5) return launch<5>(sg, stride, BC, C, a, b, g, s, Ctab, P, st);
  if (kp <= 9) return launch<9>(sg, stride, BC, C, a, b, g, s, Ctab, P, st);
  return launch<17>(sg, stride, BC, C, a, b, g, s, Ctab, P, st);
}
