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
// Each thread walks whole chains (a wedge pair from l = M' to the stage degree), for the two
// candidates of its CTA at once; chains are dealt to threads in boustrophedon order so that
// long (small M') and short chains mix.
#include <math.h>
#include "common.cuh"
#include "newton.cuh"

namespace {

constexpr int kNT = kNewtonThreads;

enum { A_VAL = 0, A_GA, A_GB, A_GG, A_HAA, A_HAB, A_HAG, A_HBB, A_HBG, A_HGG, A_N };

// Per-candidate tables of one pass (NC candidates of one subtomogram per CTA).
template <int NC>
struct Smem {
  float2 (*ea)[2 * kNewtonMaxL + 1];   // e^{i k a}, index k + Li
  float2 (*eg)[2 * kNewtonMaxL + 1];   // e^{i k g}, index k + Li
  double (*phc)[2 * kNewtonMaxL + 3];  // cos(b/2)^k, k = 0 .. 2 Li + 2
  double (*pt)[2 * kNewtonMaxL + 3];   // (-sin(b/2))^k
  float* red;                          // (threads/32) x NC x A_N
  float* res;                          // NC x A_N
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

// One sweep over the chains of stage degree Li at the NC points (a[c], be[c], ga[c]) of one
// subtomogram's candidates: value, and with DERIVS the Euler gradient and Hessian, left in
// sm.res[c * A_N + ..].  The candidates share each chain's loads of the folded sigma and of
// the recurrence factors; their d, d', d'' run side by side.  FOLDED reads the folded sigma S
// of this subtomogram; otherwise each step folds the four images from sigma itself.
template <bool DERIVS, bool FOLDED, int NC>
__device__ __forceinline__ void pass(const float4* __restrict__ S, const float2* __restrict__ sg,
                                     const float4* __restrict__ coef, const double* __restrict__ Ctab,
                                     const float (&a)[NC], const float (&be)[NC], const float (&ga)[NC], int Li,
                                     const Smem<NC> sm) {
  const int tid = threadIdx.x;
  const double two_pi = 6.283185307179586;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    for (int r = tid; r < 2 * Li + 1; r += kNT) {
      double t = (double)(r - Li) * (double)a[c];
      t -= two_pi * rint(t / two_pi);
      float s, co;
      sincosf((float)t, &s, &co);
      sm.ea[c][r] = make_float2(co, s);
      t = (double)(r - Li) * (double)ga[c];
      t -= two_pi * rint(t / two_pi);
      sincosf((float)t, &s, &co);
      sm.eg[c][r] = make_float2(co, s);
    }
    double hs, hc;
    sincos(0.5 * (double)be[c], &hs, &hc);
    for (int k = tid; k <= 2 * Li + 2; k += kNT) {
      sm.phc[c][k] = ipow(hc, k);
      sm.pt[c][k] = ipow(-hs, k);
    }
  }
  float sb[NC], cb[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) sincosf(be[c], &sb[c], &cb[c]);

  float acc[NC][A_N];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int i = 0; i < A_N; ++i) acc[c][i] = 0.f;
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
    const double Cp = Ctab[p];
    float d1[NC], d0[NC], e1[NC], e0[NC], g1[NC], g0[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      d1[c] = (float)(Cp * sm.phc[c][P] * sm.pt[c][Q]);
      d0[c] = 0.f;
      e1[c] = e0[c] = g1[c] = g0[c] = 0.f;
      if (DERIVS) {
        double fp = 0.0, fpp = -(double)(2 * P * Q + P + Q) * sm.phc[c][P] * sm.pt[c][Q];
        if (P >= 1) fp += P * sm.phc[c][P - 1] * sm.pt[c][Q + 1];
        if (Q >= 1) fp -= Q * sm.phc[c][P + 1] * sm.pt[c][Q - 1];
        if (P >= 2) fpp += (double)(P * (P - 1)) * sm.phc[c][P - 2] * sm.pt[c][Q + 2];
        if (Q >= 2) fpp += (double)(Q * (Q - 1)) * sm.phc[c][P + 2] * sm.pt[c][Q - 2];
        e1[c] = (float)(0.5 * Cp * fp);
        g1[c] = (float)(0.25 * Cp * fpp);
      }
    }
    float4 s;
    if (FOLDED) s = __ldg(S + wedge_off(mp) + p);
    else s = fold_entry(sg, mp, mp, m);
    // per candidate: A = sum d S (a1 = S1 part, a2 = S2 part), B = sum d' S, C = sum d'' S
    float A1r[NC], A1i[NC], A2r[NC], A2i[NC];
    float B1r[NC], B1i[NC], B2r[NC], B2i[NC], C1r[NC], C1i[NC], C2r[NC], C2i[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      A1r[c] = d1[c] * s.x; A1i[c] = d1[c] * s.y; A2r[c] = d1[c] * s.z; A2i[c] = d1[c] * s.w;
      B1r[c] = B1i[c] = B2r[c] = B2i[c] = C1r[c] = C1i[c] = C2r[c] = C2i[c] = 0.f;
      if (DERIVS) {
        B1r[c] = e1[c] * s.x; B1i[c] = e1[c] * s.y; B2r[c] = e1[c] * s.z; B2i[c] = e1[c] * s.w;
        C1r[c] = g1[c] * s.x; C1i[c] = g1[c] * s.y; C2r[c] = g1[c] * s.z; C2i[c] = g1[c] * s.w;
      }
    }
    const float4* cp = coef + wedge_off(mp + 1) + p;
    const float4* sp = FOLDED ? S + wedge_off(mp + 1) + p : nullptr;
#pragma unroll 4
    for (int l = mp + 1; l <= Li; ++l) {
      const float4 cf = __ldg(cp);
      if (FOLDED) s = __ldg(sp);
      else s = fold_entry(sg, l, mp, m);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float t = fmaf(cf.x, cb[c], -cf.y);
        const float v = fmaf(t, d1[c], -cf.z * d0[c]);
        if (DERIVS) {
          const float as = cf.x * sb[c];
          const float vp = fmaf(t, e1[c], -fmaf(as, d1[c], cf.z * e0[c]));
          const float vpp = fmaf(t, g1[c], -fmaf(2.f * as, e1[c], fmaf(cf.x * cb[c], d1[c], cf.z * g0[c])));
          e0[c] = e1[c]; e1[c] = vp;
          g0[c] = g1[c]; g1[c] = vpp;
        }
        d0[c] = d1[c]; d1[c] = v;
        A1r[c] = fmaf(v, s.x, A1r[c]); A1i[c] = fmaf(v, s.y, A1i[c]);
        A2r[c] = fmaf(v, s.z, A2r[c]); A2i[c] = fmaf(v, s.w, A2i[c]);
        if (DERIVS) {
          B1r[c] = fmaf(e1[c], s.x, B1r[c]); B1i[c] = fmaf(e1[c], s.y, B1i[c]);
          B2r[c] = fmaf(e1[c], s.z, B2r[c]); B2i[c] = fmaf(e1[c], s.w, B2i[c]);
          C1r[c] = fmaf(g1[c], s.x, C1r[c]); C1i[c] = fmaf(g1[c], s.y, C1i[c]);
          C2r[c] = fmaf(g1[c], s.z, C2r[c]); C2i[c] = fmaf(g1[c], s.w, C2i[c]);
        }
      }
      cp += (l + 1) * (l + 1);
      if (FOLDED) sp += (l + 1) * (l + 1);
    }
    // phases: z1 = e^{i(M'a + Mg)}, z2 = e^{i(Ma + M'g)}
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const float2 z1 = cmulf(sm.ea[c][mp + Li], sm.eg[c][m + Li]);
      const float2 z2 = cmulf(sm.ea[c][m + Li], sm.eg[c][mp + Li]);
      const float r1 = z1.x * A1r[c] - z1.y * A1i[c], r2 = z2.x * A2r[c] - z2.y * A2i[c];
      acc[c][A_VAL] += r1 + r2;
      if (DERIVS) {
        const float fM = (float)mp, fm = (float)m;
        const float j1 = z1.x * A1i[c] + z1.y * A1r[c], j2 = z2.x * A2i[c] + z2.y * A2r[c];
        const float q1 = z1.x * B1r[c] - z1.y * B1i[c], q2 = z2.x * B2r[c] - z2.y * B2i[c];
        const float k1 = z1.x * B1i[c] + z1.y * B1r[c], k2 = z2.x * B2i[c] + z2.y * B2r[c];
        const float h1 = z1.x * C1r[c] - z1.y * C1i[c], h2 = z2.x * C2r[c] - z2.y * C2i[c];
        acc[c][A_GA] -= fM * j1 + fm * j2;
        acc[c][A_GG] -= fm * j1 + fM * j2;
        acc[c][A_GB] += q1 + q2;
        acc[c][A_HAA] -= fM * fM * r1 + fm * fm * r2;
        acc[c][A_HGG] -= fm * fm * r1 + fM * fM * r2;
        acc[c][A_HAG] -= fM * fm * (r1 + r2);
        acc[c][A_HAB] -= fM * k1 + fm * k2;
        acc[c][A_HBG] -= fm * k1 + fM * k2;
        acc[c][A_HBB] += h1 + h2;
      }
    }
  }

  // ---- block reduction
  const int lane = tid & 31, warp = tid >> 5;
  constexpr int NA = DERIVS ? A_N : 1;
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      const float v = warp_sum(acc[c][i]);
      if (lane == 0) sm.red[(warp * NC + c) * A_N + i] = v;
    }
  __syncthreads();
  if (tid < NC * A_N) {
    const int c = tid / A_N, i = tid - (tid / A_N) * A_N;
    if (i < NA) {
      float s2 = 0.f;
      for (int q = 0; q < kNT / 32; ++q) s2 += sm.red[(q * NC + c) * A_N + i];
      sm.res[c * A_N + i] = s2;
    }
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

// One CTA per NC candidates of one subtomogram (C % NC == 0).  Each candidate keeps its own
// point, learning rate, gradient and Hessian; the passes evaluate all NC together.
template <bool FOLDED, int NC>
__global__ void __launch_bounds__(kNT, 4)
newton_march_kernel(const float4* __restrict__ S, int64_t n_fold, const float2* __restrict__ sigma, int64_t stride,
                    int BC, int C, float* __restrict__ alpha, float* __restrict__ beta, float* __restrict__ gamma,
                    float* __restrict__ score, const double* __restrict__ Ctab, const float4* __restrict__ coef,
                    NewtonParams P) {
  __shared__ float2 s_ea[NC][2 * kNewtonMaxL + 1], s_eg[NC][2 * kNewtonMaxL + 1];
  __shared__ double s_phc[NC][2 * kNewtonMaxL + 3], s_pt[NC][2 * kNewtonMaxL + 3];
  __shared__ float s_red[(kNT / 32) * NC * A_N], s_res[NC * A_N];
  const Smem<NC> sm{s_ea, s_eg, s_phc, s_pt, s_red, s_res};

  const int cand0 = blockIdx.x * NC;
  if (cand0 >= BC) return;
  const int b = cand0 / C;
  const float4* Sb = FOLDED ? S + (int64_t)b * n_fold : nullptr;
  const float2* sg = FOLDED ? nullptr : sigma + (int64_t)b * stride;
  const bool grad_step = (P.flags & MTB_SEARCH_GRADIENT_STEP) != 0;
  const float base_lr = grad_step ? 5e-7f : 1.f;

  // the gradient and Hessian at each candidate's accepted point: pass results (res layout),
  // kept in shared memory so they are not live in registers across the passes
  __shared__ float s_gh[NC * A_N];
  float a[NC], be[NC], ga[NC], best[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    a[c] = alpha[cand0 + c];
    be[c] = beta[cand0 + c];
    ga[c] = gamma[cand0 + c];
    best[c] = 0.f;
  }
  for (int st = 0; st < P.n_stages; ++st) {
    const int Li = P.stages[st];
    if (P.num_steps > 0)
      pass<true, FOLDED, NC>(Sb, sg, coef, Ctab, a, be, ga, Li, sm);
    else
      pass<false, FOLDED, NC>(Sb, sg, coef, Ctab, a, be, ga, Li, sm);
    float lr[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      best[c] = sm.res[c * A_N + A_VAL];
      lr[c] = base_lr;
    }
    if (threadIdx.x < NC * A_N) s_gh[threadIdx.x] = sm.res[threadIdx.x];
    __syncthreads();
    for (int it = 0; it < P.num_steps; ++it) {
      float ta[NC], tb[NC], tg[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float* r = s_gh + c * A_N;
        const double g[3] = {r[A_GA], r[A_GB], r[A_GG]};
        const double H[3][3] = {{r[A_HAA], r[A_HAB], r[A_HAG]},
                                {r[A_HAB], r[A_HBB], r[A_HBG]},
                                {r[A_HAG], r[A_HBG], r[A_HGG]}};
        double x[3] = {0.0, 0.0, 0.0};
        if (grad_step) {
          for (int i = 0; i < 3; ++i) x[i] = -g[i];
        } else if (!solve3(H, g, x)) {
          x[0] = x[1] = x[2] = 0.0;
        }
        ta[c] = a[c] - lr[c] * (float)x[0];
        tb[c] = be[c] - lr[c] * (float)x[1];
        tg[c] = ga[c] - lr[c] * (float)x[2];
      }
      const bool last = (it == P.num_steps - 1);
      __syncthreads();  // everyone has read the previous results
      if (last)
        pass<false, FOLDED, NC>(Sb, sg, coef, Ctab, ta, tb, tg, Li, sm);
      else
        pass<true, FOLDED, NC>(Sb, sg, coef, Ctab, ta, tb, tg, Li, sm);
      bool took[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float ev = sm.res[c * A_N + A_VAL];
        took[c] = ev > best[c];
        if (took[c]) {
          a[c] = ta[c]; be[c] = tb[c]; ga[c] = tg[c]; best[c] = ev;
          lr[c] *= 1.1f;
        } else {
          lr[c] *= 0.5f;
        }
      }
      if (!last) {
        if (threadIdx.x < NC * A_N) {
          const int c = threadIdx.x / A_N;
          bool tk = false;
#pragma unroll
          for (int q = 0; q < NC; ++q) tk = (q == c) ? took[q] : tk;
          if (tk) s_gh[threadIdx.x] = sm.res[threadIdx.x];
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < NC) {
    const int c = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NC; ++q)
      if (q == c) {
        alpha[cand0 + c] = a[q];
        beta[cand0 + c] = be[q];
        gamma[cand0 + c] = ga[q];
        score[cand0 + c] = best[q];
      }
  }
}

// The score and its Euler derivatives at one given point per subtomogram, degrees <= Li:
// out[b] = (f, df/da, df/db, df/dg, d2f/da2, d2f/dadb, d2f/dadg, d2f/db2, d2f/dbdg, d2f/dg2),
// the same sweep the march makes at each Newton step, read straight from sigma.
__global__ void __launch_bounds__(kNT)
score_derivs_kernel(const float2* __restrict__ sigma, int64_t stride, const float* __restrict__ alpha,
                    const float* __restrict__ beta, const float* __restrict__ gamma, int Li,
                    const double* __restrict__ Ctab, const float4* __restrict__ coef, float* __restrict__ out) {
  __shared__ float2 s_ea[1][2 * kNewtonMaxL + 1], s_eg[1][2 * kNewtonMaxL + 1];
  __shared__ double s_phc[1][2 * kNewtonMaxL + 3], s_pt[1][2 * kNewtonMaxL + 3];
  __shared__ float s_red[(kNT / 32) * A_N], s_res[A_N];
  const Smem<1> sm{s_ea, s_eg, s_phc, s_pt, s_red, s_res};
  const int b = blockIdx.x;
  const float a[1] = {alpha[b]}, be[1] = {beta[b]}, ga[1] = {gamma[b]};
  pass<true, false, 1>(nullptr, sigma + (int64_t)b * stride, coef, Ctab, a, be, ga, Li, sm);
  if (threadIdx.x < A_N) out[(int64_t)b * A_N + threadIdx.x] = sm.res[threadIdx.x];
}

}  // namespace

int newton_eval_launch(const float* sigma, int64_t stride, int B, int Li, const float* alpha, const float* beta,
                       const float* gamma, const double* Ctab, const float4* coef, float* out, cudaStream_t st) {
  MTB_ARG_CHECK(Li >= 0 && Li <= kNewtonMaxL, "degree exceeds the Newton march limit");
  if (B == 0) return MTB_OK;
  mtb_prof_begin(st);
  score_derivs_kernel<<<B, kNT, 0, st>>>(reinterpret_cast<const float2*>(sigma), stride, alpha, beta, gamma, Li,
                                         Ctab, coef, out);
  mtb_prof_end(st, "score_derivs_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

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
  // two candidates of a subtomogram per CTA share its folded-sigma and recurrence-factor loads
  const bool pair = (C % 2) == 0;
  if (fold) {
    mtb_prof_begin(st);
    fold_sigma_kernel<<<dim3(P.Lmax + 1, B), 256, 0, st>>>(sg, stride, nf, fold);
    mtb_prof_end(st, "fold_sigma_kernel");
    MTB_LAUNCH_CHECK();
    mtb_prof_begin(st);
    if (pair)
      newton_march_kernel<true, 2><<<BC / 2, kNT, 0, st>>>(fold, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef, P);
    else
      newton_march_kernel<true, 1><<<BC, kNT, 0, st>>>(fold, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef, P);
  } else {
    mtb_prof_begin(st);
    if (pair)
      newton_march_kernel<false, 2><<<BC / 2, kNT, 0, st>>>(nullptr, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef,
                                                             P);
    else
      newton_march_kernel<false, 1><<<BC, kNT, 0, st>>>(nullptr, nf, sg, stride, BC, C, a, b, g, s, Ctab, coef, P);
  }
  mtb_prof_end(st, "newton_march_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}
