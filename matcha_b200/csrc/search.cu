// Orientation search on sm_100a: SO(3) grid search with top-k, and the
// frequency-marched Wigner-D Newton refinement.
//
// Reference behaviour restated here (paths inside swing-research/Matcha):
//   grid      src/matcha/core/SOFFT.py:30-124, src/matcha/core/Matcha.py:27-58,207-236
//   Newton    src/matcha/core/Matcha.py:150-205, 239-403
//   D, d      src/matcha/core/WignerDMatrices.py:281-306, 673-801, 1291-1375
//   g, H      src/matcha/core/WignerDGradients.py:155-302
//
// Design (B200): one CTA per (subtomogram, candidate) runs every march stage for
// its candidate.  The small-d matrix of each degree l is produced by the three-term
// recurrence in l for fixed (m', m) (state in registers, one fundamental wedge
// m' >= |m| per thread, symmetric copies written to shared memory), and contracted
// against sigma in the same sweep: value, Euler gradient and Hessian come out of one
// pass over sigma with 10 register accumulators and a warp-shuffle block reduction.
// No D matrix and no 15-column coefficient bank ever reach HBM.  The 3x3 Newton
// solve runs in FP64.
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <vector>
#include "common.cuh"
#include "newton.cuh"

namespace {

struct SearchParams {
  int Lmax;
  int n_stages;
  int stages[MTB_MAX_STAGES];
  int L0;
  int K;
  int C;
  int num_steps;
  int flags;
};

constexpr int kGridThreads = 256;
constexpr int kMaxCand = 32;

// ------------------------------------------------------------------ grid + top-k
__device__ __forceinline__ bool better(float v1, int i1, float v2, int i2) {
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

constexpr size_t kGridSmemCap = 200 * 1024;

// Dynamic shared memory of the grid kernel: sigma (l < L0), the twiddle matrix, the F, G
// buffers of JB beta values and, when staged, their d-table rows.
size_t grid_smem_bytes(int L0, int K, int JB, bool staged) {
  const int n = 2 * L0 * K, P = 2 * L0 - 1, nk = mtb_dsize(L0 - 1);
  return (size_t)(nk + n * P + JB * P * P + JB * P * n) * sizeof(float2) +
         (staged ? (size_t)JB * nk * sizeof(float) : 0);
}

// CTAs of the grid kernel an SM holds with `smem` bytes of dynamic shared memory (228 KB per
// SM, 1 KB reserved and the static arrays per CTA), at most four (the register limit of the
// 64-register instantiations at 256 threads).
int grid_ctas_per_sm(size_t smem) {
  const int c = (int)((size_t)228 * 1024 / (smem + 1024 + 256));
  return c < 4 ? c : 4;
}

struct GridPlan {
  int jb;       // beta values per pass
  bool staged;  // their d-table rows copied into shared memory (else read from the L2-resident table)
};

// The pass shape: the most CTAs per SM first (the kernel is latency-bound: a CTA runs its
// passes one after another, three barriers each), then the most beta values per pass (fewer
// passes), then staged rows.  At L0 = 16 this is two unstaged rows, two CTAs per SM (staged,
// the two rows take 150 KB and leave one).
GridPlan grid_plan(int L0, int K) {
  GridPlan best{0, true};
  int best_c = 0;
  for (int jb : {8, 4, 2, 1})
    for (bool staged : {true, false}) {
      const size_t sm = grid_smem_bytes(L0, K, jb, staged);
      if (sm > kGridSmemCap) continue;
      const int c = grid_ctas_per_sm(sm);
      if (c > best_c || (c == best_c && jb > best.jb)) {
        best = GridPlan{jb, staged};
        best_c = c;
      }
    }
  return best;
}
int grid_jb(int L0, int K) { return grid_plan(L0, K).jb; }
bool grid_staged(int L0, int K) { return grid_plan(L0, K).staged; }
size_t grid_smem_bytes(int L0, int K) {
  const GridPlan p = grid_plan(L0, K);
  return p.jb ? grid_smem_bytes(L0, K, p.jb, p.staged) : kGridSmemCap + 1;  // jb 0: nothing fits
}

// SOFFT on the (n x n x n) grid (beta_j = j pi/(n-1), alpha_a = 2 pi a/n, gamma_g = 2 pi g/n)
// for one subtomogram per CTA, kGridJB beta values per pass:
//   F_j[m'][m] = sum_{l < L0} d^l_{m'm}(beta_j) sigma_{l m' m}
//   G_j[m'][g] = sum_m F_j[m'][m] e^{2 pi i g m / n}
//   f_j[a][g]  = Re sum_{m'} G_j[m'][g] e^{2 pi i a m' / n} / n^2
// with the running top-C of every thread merged at the end.
// L0T, NT > 0 fix L0 and n at compile time (the index arithmetic then folds to constants);
// 0 takes them from the arguments.  KC >= C is the capacity of each thread's kept set, held
// in registers (statically indexed).
template <int L0T, int NT, int KC, bool STAGED>
__global__ void __launch_bounds__(kGridThreads)
so3_grid_topk_kernel(const float2* __restrict__ sigma, int64_t stride, int B,
                     const float* __restrict__ dtab, int L0_arg, int n_arg, int C, int JB,
                     float* __restrict__ alpha, float* __restrict__ beta, float* __restrict__ gamma,
                     float* __restrict__ grid_out) {
  extern __shared__ __align__(16) float gsm[];
  const int L0 = L0T > 0 ? L0T : L0_arg;
  const int n = NT > 0 ? NT : n_arg;
  const int P = 2 * L0 - 1;
  const int nk = mtb_dsize(L0 - 1);
  float2* sg = reinterpret_cast<float2*>(gsm);  // nk
  float2* TW = sg + nk;                          // n x P: e^{2 pi i g (c - L0 + 1) / n}
  float2* F = TW + n * P;                        // JB x P x P
  float2* G = F + JB * P * P;                    // JB x P x n
  float* sD = reinterpret_cast<float*>(G + JB * P * n);  // JB x nk: d^l(beta_j) of this pass
  __shared__ float mv[kGridThreads / 32];
  __shared__ int mi[kGridThreads / 32];
  __shared__ int mt[kGridThreads / 32];

  const int b = blockIdx.x;
  if (b >= B) return;
  const int tid = threadIdx.x;
  const float2* sig = sigma + (int64_t)b * stride;
  for (int k = tid; k < nk; k += blockDim.x) sg[k] = sig[k];
  for (int q = tid; q < n * P; q += blockDim.x) {
    const int g = q / P, c = q - (q / P) * P;
    int k = (g * (c - (L0 - 1))) % n;
    if (k < 0) k += n;
    double sn, cs;
    sincospi(2.0 * k / n, &sn, &cs);
    TW[q] = make_float2((float)cs, (float)sn);
  }
  float tv[KC];
  int ti[KC];
#pragma unroll
  for (int t = 0; t < KC; ++t) {
    tv[t] = -INFINITY;
    ti[t] = 0x7fffffff;
  }
  int cnt = 0, minp = 0;
  float minv = -INFINITY;
  int mini = 0x7fffffff;
  // the kept set's worst entry (for a full set of C)
  auto find_min = [&]() {
    minp = 0;
    minv = tv[0];
    mini = ti[0];
#pragma unroll
    for (int t = 1; t < KC; ++t)
      if (t < C && better(minv, mini, tv[t], ti[t])) {
        minp = t;
        minv = tv[t];
        mini = ti[t];
      }
  };
  const float inv_n2 = 1.f / (float)(n * n);
  for (int j0 = 0; j0 < n; j0 += JB) {
    const int jn = min(JB, n - j0);
    if (STAGED)
      for (int e = tid; e < jn * nk; e += blockDim.x) sD[e] = __ldg(&dtab[(int64_t)j0 * nk + e]);
    __syncthreads();
    for (int q = tid; q < jn * P * P; q += blockDim.x) {
      const int jb = q / (P * P), qq = q - jb * (P * P);
      const int mp = qq / P - (L0 - 1), m = qq % P - (L0 - 1);
      const int l0 = max(abs(mp), abs(m));
      const float* dj = STAGED ? sD + jb * nk : dtab + (int64_t)(j0 + jb) * nk;
      float re = 0.f, im = 0.f;
      if (L0T > 0) {
#pragma unroll
        for (int l = 0; l < L0T; ++l) {
          if (l >= l0) {
            const int idx = mtb_dsize(l - 1) + (mp + l) * (2 * l + 1) + (m + l);
            const float d = STAGED ? dj[idx] : __ldg(dj + idx);
            re += d * sg[idx].x;
            im += d * sg[idx].y;
          }
        }
      } else {
        for (int l = l0; l < L0; ++l) {
          const int idx = mtb_dsize(l - 1) + (mp + l) * (2 * l + 1) + (m + l);
          const float d = STAGED ? dj[idx] : __ldg(dj + idx);
          re += d * sg[idx].x;
          im += d * sg[idx].y;
        }
      }
      F[q] = make_float2(re, im);
    }
    __syncthreads();
    if constexpr (NT > 0) {
      // four outputs gg = g4 + (n/4) i per thread: one F read serves four independent chains
      constexpr int n4 = NT / 4;
      for (int q = tid; q < jn * P * n4; q += blockDim.x) {
        const int jb = q / (P * n4), qq = q - jb * (P * n4);
        const int r = qq / n4, g4 = qq - (qq / n4) * n4;
        const float2* fr = F + jb * P * P + r * P;
        float re[4] = {0.f, 0.f, 0.f, 0.f}, im[4] = {0.f, 0.f, 0.f, 0.f};
        for (int c = 0; c < P; ++c) {
          const float2 f = fr[c];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 t = TW[(g4 + n4 * i) * P + c];
            re[i] += f.x * t.x - f.y * t.y;
            im[i] += f.x * t.y + f.y * t.x;
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) G[jb * P * n + r * n + g4 + n4 * i] = make_float2(re[i], im[i]);
      }
    } else {
      for (int q = tid; q < jn * P * n; q += blockDim.x) {
        const int jb = q / (P * n), qq = q - jb * (P * n);
        const int r = qq / n, gg = qq - (qq / n) * n;
        const float2* fr = F + jb * P * P + r * P;
        const float2* tr = TW + gg * P;
        float re = 0.f, im = 0.f;
        for (int c = 0; c < P; ++c) {
          const float2 f = fr[c], t = tr[c];
          re += f.x * t.x - f.y * t.y;
          im += f.x * t.y + f.y * t.x;
        }
        G[q] = make_float2(re, im);
      }
    }
    __syncthreads();
    // offer one grid value to this thread's kept set
    auto offer = [&](float v, int flat) {
      if (grid_out) grid_out[(int64_t)b * n * n * n + flat] = v;
      // the rejection test reads the kept set's worst entry from registers
      if (cnt < C || better(v, flat, minv, mini)) {
        const int slot = cnt < C ? cnt : minp;
#pragma unroll
        for (int t = 0; t < KC; ++t)
          if (t == slot) {
            tv[t] = v;
            ti[t] = flat;
          }
        if (cnt < C) ++cnt;
        if (cnt == C) find_min();
      }
    };
    if constexpr (NT > 0) {
      // four outputs gg = g4 + (n/4) i per thread: one twiddle read serves four chains (the
      // kept set is a total order on (value, index), so the visiting order does not matter)
      constexpr int n4 = NT / 4;
      for (int q = tid; q < jn * n * n4; q += blockDim.x) {
        const int jb = q / (n * n4), qq = q - jb * (n * n4);
        const int aa = qq / n4, g4 = qq - (qq / n4) * n4;
        const float2* gc = G + jb * P * n + g4;
        const float2* ta = TW + aa * P;
        float re[4] = {0.f, 0.f, 0.f, 0.f};
        for (int r = 0; r < P; ++r) {
          const float2 t = ta[r];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 gv = gc[r * n + n4 * i];
            re[i] += gv.x * t.x - gv.y * t.y;
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) offer(re[i] * inv_n2, (j0 + jb) * n * n + aa * n + g4 + n4 * i);
      }
    } else {
      for (int q = tid; q < jn * n * n; q += blockDim.x) {
        const int jb = q / (n * n), qq = q - jb * (n * n);
        const int aa = qq / n, gg = qq - (qq / n) * n;
        const float2* gc = G + jb * P * n + gg;
        const float2* ta = TW + aa * P;
        float re = 0.f;
        for (int r = 0; r < P; ++r) {
          const float2 gv = gc[r * n], t = ta[r];
          re += gv.x * t.x - gv.y * t.y;
        }
        offer(re * inv_n2, (j0 + jb) * n * n + qq);
      }
    }
    __syncthreads();
  }
  // block merge: C rounds of block argmax over each thread's best remaining entry
  const int lane = tid & 31, warp = tid >> 5;
  const float bstep = (float)(M_PI / (double)(n - 1));
  const float astep = (float)(2.0 * M_PI / (double)n);
  uint32_t live = cnt >= 32 ? 0xffffffffu : ((1u << cnt) - 1u);
  for (int c = 0; c < C; ++c) {
    int hp = -1;
    float hv = -INFINITY;
    int hi = 0x7fffffff;
#pragma unroll
    for (int t = 0; t < KC; ++t)
      if (((live >> t) & 1u) && (hp < 0 || better(tv[t], ti[t], hv, hi))) {
        hp = t;
        hv = tv[t];
        hi = ti[t];
      }
    float v = hv;
    int i = hi, who = (hp < 0) ? -1 : tid;
    for (int o = 16; o > 0; o >>= 1) {
      const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
      const int w2 = __shfl_xor_sync(0xffffffffu, who, o);
      if (w2 >= 0 && (who < 0 || better(v2, i2, v, i))) { v = v2; i = i2; who = w2; }
    }
    if (lane == 0) { mv[warp] = v; mi[warp] = i; mt[warp] = who; }
    __syncthreads();
    if (tid == 0) {
      float bv = mv[0];
      int bi = mi[0], bw = mt[0];
      for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
        if (mt[q] >= 0 && (bw < 0 || better(mv[q], mi[q], bv, bi))) { bv = mv[q]; bi = mi[q]; bw = mt[q]; }
      mt[0] = bw;
      mi[0] = bi;
      const int jj = bi / (n * n), aa = (bi / n) % n, gg = bi % n;
      const int o = b * C + c;
      beta[o] = (float)jj * bstep;
      alpha[o] = (float)aa * astep;
      gamma[o] = (float)gg * astep;
    }
    __syncthreads();
    if (mt[0] == tid && hp >= 0) live &= ~(1u << hp);  // remove the taken entry
    __syncthreads();
  }
}

template <int L0T, int NT, int KC>
int grid_launch_t(const float2* sigma, int64_t stride, int B, const float* dtab, int L0, int K, int C, float* a,
                  float* b, float* g, float* grid, cudaStream_t st) {
  const size_t smem = grid_smem_bytes(L0, K);
  const int jb = grid_jb(L0, K);
  mtb_prof_begin(st);
  if (grid_staged(L0, K)) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(so3_grid_topk_kernel<L0T, NT, KC, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    so3_grid_topk_kernel<L0T, NT, KC, true><<<B, kGridThreads, smem, st>>>(sigma, stride, B, dtab, L0, 2 * L0 * K,
                                                                       C, jb, a, b, g, grid);
  } else {
    MTB_CUDA_TRY(cudaFuncSetAttribute(so3_grid_topk_kernel<L0T, NT, KC, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    so3_grid_topk_kernel<L0T, NT, KC, false><<<B, kGridThreads, smem, st>>>(sigma, stride, B, dtab, L0, 2 * L0 * K,
                                                                        C, jb, a, b, g, grid);
  }
  mtb_prof_end(st, "so3_grid_topk_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

// The grid search for L0 = 8, 12, 16 with K = 2 (the marches of boxes 64, 96 and 128 at
// bandlimit N/2) with its index arithmetic fixed at compile time; other grids take the general
// instantiation.
int grid_launch(const float2* sigma, int64_t stride, int B, const float* dtab, int L0, int K, int C, float* a,
                float* b, float* g, float* grid, cudaStream_t st) {
  if (L0 == 8 && K == 2 && C <= 16) return grid_launch_t<8, 32, 16>(sigma, stride, B, dtab, L0, K, C, a, b, g, grid, st);
  if (L0 == 12 && K == 2 && C <= 16)
    return grid_launch_t<12, 48, 16>(sigma, stride, B, dtab, L0, K, C, a, b, g, grid, st);
  if (L0 == 16 && K == 2 && C <= 16)
    return grid_launch_t<16, 64, 16>(sigma, stride, B, dtab, L0, K, C, a, b, g, grid, st);
  if (C <= 16) return grid_launch_t<0, 0, 16>(sigma, stride, B, dtab, L0, K, C, a, b, g, grid, st);
  return grid_launch_t<0, 0, kMaxCand>(sigma, stride, B, dtab, L0, K, C, a, b, g, grid, st);
}

__global__ void reduce_candidates_kernel(const float* __restrict__ ca, const float* __restrict__ cb,
                                         const float* __restrict__ cg, const float* __restrict__ cs,
                                         int B, int C, float* alpha, float* beta, float* gamma,
                                         float* score) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  int best = 0;
  float bv = cs[b * C];
  for (int c = 1; c < C; ++c) {
    const float v = cs[b * C + c];
    if (v > bv) { bv = v; best = c; }
  }
  alpha[b] = ca[b * C + best];
  beta[b] = cb[b * C + best];
  gamma[b] = cg[b * C + best];
  score[b] = bv;
}

// ------------------------------------------------------------------ host tables
double host_small_d_start_log(int mp, int m) {
  return 0.5 * (lgamma(2.0 * mp + 1.0) - lgamma((double)(mp + m) + 1.0) - lgamma((double)(mp - m) + 1.0));
}

// d^l_{m'm}(beta) for l < L0 in flat order, by the same recurrence in double.
void host_small_d(int Lm, double beta, double* out) {
  const double cb = cos(beta), c = cos(0.5 * beta), s = sin(0.5 * beta);
  for (int mp = -Lm; mp <= Lm; ++mp)
    for (int m = -Lm; m <= Lm; ++m) {
      const int l0 = abs(mp) > abs(m) ? abs(mp) : abs(m);
      // start value from the explicit sum at l0 (single term)
      const int kmin = (m - mp) > 0 ? (m - mp) : 0;
      const int k = kmin;
      const int l = l0;
      const double lognum = 0.5 * (lgamma(l + mp + 1.0) + lgamma(l - mp + 1.0) + lgamma(l + m + 1.0) + lgamma(l - m + 1.0));
      const double logden = lgamma(l + m - k + 1.0) + lgamma(k + 1.0) + lgamma(mp - m + k + 1.0) + lgamma(l - mp - k + 1.0);
      const int pc = 2 * l + m - mp - 2 * k, ps = mp - m + 2 * k;
      double v = exp(lognum - logden) * (((mp - m + k) & 1) ? -1.0 : 1.0);
      v *= (pc ? pow(c, pc) : 1.0) * (ps ? pow(s, ps) : 1.0);
      double dl = v, dlm1 = 0.0;
      out[mtb_dsize(l0 - 1) + (mp + l0) * (2 * l0 + 1) + (m + l0)] = dl;
      for (int ll = l0; ll < Lm; ++ll) {
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
        const int L1 = ll + 1;
        out[mtb_dsize(L1 - 1) + (mp + L1) * (2 * L1 + 1) + (m + L1)] = dl;
      }
    }
}

}  // namespace

// ------------------------------------------------------------------ C ABI
struct mtb_search {
  mtb_search_config cfg;
  SearchParams P;
  int n;            // grid size per axis
  int device;
  float* dtab;      // (n, dsize(L0-1))
  double* Ctab;     // (Lmax+1)^2 start-value coefficients of the recurrence
  float4* coef;     // recurrence factors, newton_fold_entries(Lmax)
  float4* fold;     // folded sigma, max_batch x newton_fold_entries(Lmax)
  float* cand;      // 4 x (max_batch * C): alpha, beta, gamma, score
};

extern "C" int mtb_search_create(const mtb_search_config* cfg, mtb_search** out) {
  MTB_ARG_CHECK(cfg && out, "null argument");
  *out = nullptr;
  MTB_ARG_CHECK(cfg->Lmax >= 1 && cfg->Lmax <= 64, "Lmax must be in [1, 64]");
  MTB_ARG_CHECK(cfg->n_stages >= 1 && cfg->n_stages <= MTB_MAX_STAGES, "n_stages out of range");
  MTB_ARG_CHECK(cfg->L0 >= 1 && cfg->L0 <= cfg->Lmax, "L0 must be in [1, Lmax]");
  MTB_ARG_CHECK(cfg->K >= 1 && 2 * cfg->L0 * cfg->K <= 128, "grid size 2*L0*K must be <= 128");
  MTB_ARG_CHECK(cfg->candidates >= 1 && cfg->candidates <= kMaxCand, "candidates must be in [1, 32]");
  MTB_ARG_CHECK(cfg->candidates <= 2 * cfg->L0 * cfg->K * 2 * cfg->L0 * cfg->K * 2 * cfg->L0 * cfg->K,
                "more candidates than grid points");
  MTB_ARG_CHECK(cfg->num_steps >= 0 && cfg->max_batch >= 1, "bad num_steps / max_batch");
  for (int i = 0; i < cfg->n_stages; ++i)
    MTB_ARG_CHECK(cfg->stages[i] >= 0 && cfg->stages[i] <= cfg->Lmax, "stage degree out of range");
  {
    MTB_ARG_CHECK(grid_smem_bytes(cfg->L0, cfg->K) <= kGridSmemCap,
                  "grid search too large for shared memory (reduce L0 or K)");
  }
  mtb_search* h = new mtb_search();
  memset(h, 0, sizeof(*h));
  h->cfg = *cfg;
  h->P.Lmax = cfg->Lmax;
  h->P.n_stages = cfg->n_stages;
  for (int i = 0; i < cfg->n_stages; ++i) h->P.stages[i] = cfg->stages[i];
  h->P.L0 = cfg->L0;
  h->P.K = cfg->K;
  h->P.C = cfg->candidates;
  h->P.num_steps = cfg->num_steps;
  h->P.flags = cfg->flags;
  h->n = 2 * cfg->L0 * cfg->K;
  cudaGetDevice(&h->device);

  const int n = h->n, L0 = cfg->L0, nk = mtb_dsize(L0 - 1);
  std::vector<float> dt((size_t)n * nk);
  std::vector<double> tmp(mtb_dsize(L0 - 1) > 0 ? mtb_dsize(L0 - 1) : 1);
  for (int j = 0; j < n; ++j) {
    // np.linspace(0, pi, n, endpoint=True)
    const double beta = (n > 1) ? (j == n - 1 ? M_PI : j * (M_PI / (n - 1))) : 0.0;
    host_small_d(L0 - 1, beta, tmp.data());
    for (int k = 0; k < nk; ++k) dt[(size_t)j * nk + k] = (float)tmp[k];
  }
  const int Lm = cfg->Lmax;
  std::vector<double> lc((size_t)(Lm + 1) * (Lm + 1));
  for (int mp = 0; mp <= Lm; ++mp)
    for (int m = -mp; m <= mp; ++m) lc[mp * mp + m + mp] = exp(host_small_d_start_log(mp, m));

  auto fail = [&](int code) { mtb_search_destroy(h); return code; };
  if (cudaMalloc(&h->dtab, dt.size() * sizeof(float)) != cudaSuccess) return fail(MTB_ERR_OOM);
  if (cudaMalloc(&h->Ctab, lc.size() * sizeof(double)) != cudaSuccess) return fail(MTB_ERR_OOM);
  if (cudaMalloc(&h->cand, (size_t)4 * cfg->max_batch * cfg->candidates * sizeof(float)) != cudaSuccess)
    return fail(MTB_ERR_OOM);
  const int64_t nf = newton_fold_entries(Lm);
  if (cudaMalloc(&h->coef, (size_t)nf * sizeof(float4)) != cudaSuccess) return fail(MTB_ERR_OOM);
  if (cudaMalloc(&h->fold, (size_t)cfg->max_batch * nf * sizeof(float4)) != cudaSuccess) return fail(MTB_ERR_OOM);
  if (cudaMemcpy(h->dtab, dt.data(), dt.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->Ctab, lc.data(), lc.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(MTB_ERR_CUDA);
  if (newton_build_coef(Lm, h->coef, 0) != MTB_OK) return fail(MTB_ERR_CUDA);
  if (cudaStreamSynchronize(0) != cudaSuccess) return fail(MTB_ERR_CUDA);
  *out = h;
  return MTB_OK;
}

extern "C" void mtb_search_destroy(mtb_search* h) {
  if (!h) return;
  if (h->dtab) cudaFree(h->dtab);
  if (h->Ctab) cudaFree(h->Ctab);
  if (h->cand) cudaFree(h->cand);
  if (h->coef) cudaFree(h->coef);
  if (h->fold) cudaFree(h->fold);
  delete h;
}

extern "C" int mtb_so3_grid_topk(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                                 float* alpha, float* beta, float* gamma, float* grid,
                                 mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(sigma && alpha && beta && gamma, "null pointer");
  MTB_ARG_CHECK(sigma_stride >= mtb_dsize(h->cfg.L0 - 1), "sigma row shorter than dsize(L0-1)");
  return grid_launch(reinterpret_cast<const float2*>(sigma), sigma_stride, B, h->dtab, h->cfg.L0, h->cfg.K,
                     h->cfg.candidates, alpha, beta, gamma, grid, (cudaStream_t)stream);
}

extern "C" int mtb_newton_march(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                                float* alpha, float* beta, float* gamma, float* score,
                                mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(sigma && alpha && beta && gamma && score, "null pointer");
  MTB_ARG_CHECK(sigma_stride >= mtb_dsize(h->cfg.Lmax), "sigma row shorter than dsize(Lmax)");
  NewtonParams P;
  P.Lmax = h->cfg.Lmax;
  P.n_stages = h->cfg.n_stages;
  for (int i = 0; i < MTB_MAX_STAGES; ++i) P.stages[i] = h->cfg.stages[i];
  P.num_steps = h->cfg.num_steps;
  P.flags = h->cfg.flags;
  return newton_launch(sigma, sigma_stride, B, h->cfg.candidates, alpha, beta, gamma, score, h->Ctab, h->coef,
                       h->fold, P, (cudaStream_t)stream);
}

extern "C" int mtb_score_derivatives(mtb_search* h, const float* sigma, int64_t sigma_stride, int B, int L,
                                     const float* alpha, const float* beta, const float* gamma, float* out,
                                     mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0, "negative batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(sigma && alpha && beta && gamma && out, "null pointer");
  MTB_ARG_CHECK(L >= 0 && L <= h->cfg.Lmax, "degree must be in [0, Lmax]");
  MTB_ARG_CHECK(sigma_stride >= mtb_dsize(L), "sigma row shorter than dsize(L)");
  return newton_eval_launch(sigma, sigma_stride, B, L, alpha, beta, gamma, h->Ctab, h->coef, out,
                            (cudaStream_t)stream);
}

extern "C" int mtb_search_orientations(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                                       float* alpha, float* beta, float* gamma, float* score,
                                       mtb_stream_t stream) {
  MTB_ARG_CHECK(h, "null handle");
  MTB_ARG_CHECK(B >= 0 && B <= h->cfg.max_batch, "batch exceeds max_batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(alpha && beta && gamma && score, "null pointer");
  const int C = h->cfg.candidates;
  const size_t cap = (size_t)h->cfg.max_batch * C;
  float* ca = h->cand;
  float* cb = ca + cap;
  float* cg = cb + cap;
  float* cs = cg + cap;
  int rc = mtb_so3_grid_topk(h, sigma, sigma_stride, B, ca, cb, cg, nullptr, stream);
  if (rc) return rc;
  rc = mtb_newton_march(h, sigma, sigma_stride, B, ca, cb, cg, cs, stream);
  if (rc) return rc;
  mtb_prof_begin((cudaStream_t)stream);
  reduce_candidates_kernel<<<(B + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ca, cb, cg, cs, B, C, alpha,
                                                                               beta, gamma, score);
  mtb_prof_end((cudaStream_t)stream, "reduce_candidates_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

// ------------------------------------------------------------------ allocation-free search
// mtb_search_orientations_static: the same grid search, Newton march and reduction as
// mtb_search_orientations, for callers that cannot allocate device memory.  Its tables
// (grid d-table, recurrence start coefficients) and the candidate workspace live in the
// file-scope array g_search_scratch; the tables are rebuilt on the device by every call,
// and every workspace entry is written before it is read, so nothing needs clearing.
namespace {

constexpr size_t kStaticScratchBytes = (size_t)MTB_SEARCH_STATIC_SCRATCH_BYTES;
__device__ __align__(256) unsigned char g_search_scratch[MTB_SEARCH_STATIC_SCRATCH_BYTES];

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Grid d-table d^l_{m'm}(beta_j), beta_j = j pi / (n - 1), l < L0, and the start
// coefficients sqrt((2m')!/((m'+m)!(m'-m)!)) of the Newton recurrence, FP64 on the device.
__global__ void static_tables_kernel(int L0, int n, int Lmax, float* __restrict__ dtab, double* __restrict__ Ctab) {
  const int Lm = L0 - 1;
  const int P = 2 * Lm + 1;
  const int nk = mtb_dsize(Lm);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int npairs = n * P * P;
  if (t < npairs) {
    const int j = t / (P * P), q = t % (P * P);
    const int mp = q / P - Lm, m = q % P - Lm;
    const double beta = (n > 1) ? (j == n - 1 ? M_PI : j * (M_PI / (n - 1))) : 0.0;
    const double cb = cos(beta), c = cos(0.5 * beta), s = sin(0.5 * beta);
    const int l0 = abs(mp) > abs(m) ? abs(mp) : abs(m);
    const int k = (m - mp) > 0 ? (m - mp) : 0;
    const int l = l0;
    const double lognum = 0.5 * (lgamma(l + mp + 1.0) + lgamma(l - mp + 1.0) + lgamma(l + m + 1.0) + lgamma(l - m + 1.0));
    const double logden = lgamma(l + m - k + 1.0) + lgamma(k + 1.0) + lgamma(mp - m + k + 1.0) + lgamma(l - mp - k + 1.0);
    const int pc = 2 * l + m - mp - 2 * k, ps = mp - m + 2 * k;
    double v = exp(lognum - logden) * (((mp - m + k) & 1) ? -1.0 : 1.0);
    v *= (pc ? pow(c, (double)pc) : 1.0) * (ps ? pow(s, (double)ps) : 1.0);
    double dl = v, dlm1 = 0.0;
    float* row = dtab + (int64_t)j * nk;
    row[mtb_dsize(l0 - 1) + (mp + l0) * (2 * l0 + 1) + (m + l0)] = (float)dl;
    for (int ll = l0; ll < Lm; ++ll) {
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
      const int L1 = ll + 1;
      row[mtb_dsize(L1 - 1) + (mp + L1) * (2 * L1 + 1) + (m + L1)] = (float)dl;
    }
  }
  const int u = t - npairs;
  if (u >= 0 && u < (Lmax + 1) * (Lmax + 1)) {
    int mp = (int)sqrt((double)u);
    while (mp * mp > u) --mp;
    while ((mp + 1) * (mp + 1) <= u) ++mp;
    const int m = u - mp * mp - mp;
    Ctab[u] = exp(0.5 * (lgamma(2.0 * mp + 1.0) - lgamma((double)(mp + m) + 1.0) - lgamma((double)(mp - m) + 1.0)));
  }
}

}  // namespace

extern "C" int mtb_search_orientations_static(const mtb_search_config* cfg, const float* sigma, int64_t sigma_stride,
                                              int B, float* alpha, float* beta, float* gamma, float* score,
                                              mtb_stream_t stream) {
  MTB_ARG_CHECK(cfg, "null config");
  MTB_ARG_CHECK(cfg->Lmax >= 1 && cfg->Lmax <= 64, "Lmax must be in [1, 64]");
  MTB_ARG_CHECK(cfg->n_stages >= 1 && cfg->n_stages <= MTB_MAX_STAGES, "n_stages out of range");
  MTB_ARG_CHECK(cfg->L0 >= 1 && cfg->L0 <= cfg->Lmax, "L0 must be in [1, Lmax]");
  MTB_ARG_CHECK(cfg->K >= 1 && 2 * cfg->L0 * cfg->K <= 128, "grid size 2*L0*K must be <= 128");
  MTB_ARG_CHECK(cfg->candidates >= 1 && cfg->candidates <= kMaxCand, "candidates must be in [1, 32]");
  MTB_ARG_CHECK(cfg->num_steps >= 0, "bad num_steps");
  for (int i = 0; i < cfg->n_stages; ++i)
    MTB_ARG_CHECK(cfg->stages[i] >= 0 && cfg->stages[i] <= cfg->Lmax, "stage degree out of range");
  MTB_ARG_CHECK(B >= 0, "negative batch");
  if (B == 0) return MTB_OK;
  MTB_ARG_CHECK(sigma && alpha && beta && gamma && score, "null pointer");
  MTB_ARG_CHECK(sigma_stride >= mtb_dsize(cfg->Lmax), "sigma row shorter than dsize(Lmax)");
  const int n = 2 * cfg->L0 * cfg->K, L0 = cfg->L0, P = 2 * L0 - 1, nk = mtb_dsize(L0 - 1);
  MTB_ARG_CHECK(cfg->candidates <= n * n * n, "more candidates than grid points");
  const size_t gsm = grid_smem_bytes(L0, cfg->K);
  MTB_ARG_CHECK(gsm <= kGridSmemCap, "grid search too large for shared memory (reduce L0 or K)");
  const int C = cfg->candidates;
  const size_t dtab_b = align256((size_t)n * nk * sizeof(float));
  const size_t ctab_b = align256((size_t)(cfg->Lmax + 1) * (cfg->Lmax + 1) * sizeof(double));
  const size_t coef_b = align256((size_t)newton_fold_entries(cfg->Lmax) * sizeof(float4));
  const size_t cand_b = align256((size_t)4 * B * C * sizeof(float));
  MTB_ARG_CHECK(dtab_b + ctab_b + coef_b + cand_b <= kStaticScratchBytes,
                "batch x candidates (or grid size) exceeds the static scratch of "
                "MTB_SEARCH_STATIC_SCRATCH_BYTES; use mtb_search_orientations");
  // the array's device address in the current device's context, looked up by every call (a
  // table lookup once the module is loaded), so a device reset or a context other than the
  // primary one is never served a stale address
  void* sym = nullptr;
  MTB_CUDA_TRY(cudaGetSymbolAddress(&sym, g_search_scratch));
  unsigned char* base = static_cast<unsigned char*>(sym);
  float* dtab = reinterpret_cast<float*>(base);
  double* Ctab = reinterpret_cast<double*>(base + dtab_b);
  float4* coef = reinterpret_cast<float4*>(base + dtab_b + ctab_b);
  float* ca = reinterpret_cast<float*>(base + dtab_b + ctab_b + coef_b);
  float* cb = ca + (size_t)B * C;
  float* cg = cb + (size_t)B * C;
  float* cs = cg + (size_t)B * C;
  cudaStream_t st = (cudaStream_t)stream;
  const int work = n * P * P + (cfg->Lmax + 1) * (cfg->Lmax + 1);
  static_tables_kernel<<<(work + 127) / 128, 128, 0, st>>>(L0, n, cfg->Lmax, dtab, Ctab);
  MTB_LAUNCH_CHECK();
  int rc = newton_build_coef(cfg->Lmax, coef, st);
  if (rc) return rc;
  rc = grid_launch(reinterpret_cast<const float2*>(sigma), sigma_stride, B, dtab, L0, cfg->K, C, ca, cb, cg, nullptr,
                   st);
  if (rc) return rc;
  NewtonParams NP;
  NP.Lmax = cfg->Lmax;
  NP.n_stages = cfg->n_stages;
  for (int i = 0; i < MTB_MAX_STAGES; ++i) NP.stages[i] = i < cfg->n_stages ? cfg->stages[i] : 0;
  NP.num_steps = cfg->num_steps;
  NP.flags = cfg->flags;
  rc = newton_launch(sigma, sigma_stride, B, C, ca, cb, cg, cs, Ctab, coef, nullptr, NP, st);
  if (rc) return rc;
  mtb_prof_begin(st);
  reduce_candidates_kernel<<<(B + 127) / 128, 128, 0, st>>>(ca, cb, cg, cs, B, C, alpha, beta, gamma, score);
  mtb_prof_end(st, "reduce_candidates_kernel");
  MTB_LAUNCH_CHECK();
  return MTB_OK;
}

extern "C" int mtb_so3_grid_plan(int L0, int K, int* beta_per_pass, int* staged, int64_t* smem) {
  MTB_ARG_CHECK(L0 >= 1 && K >= 1 && beta_per_pass && staged && smem, "bad argument");
  const GridPlan p = grid_plan(L0, K);
  MTB_ARG_CHECK(p.jb > 0, "grid search too large for shared memory (reduce L0 or K)");
  *beta_per_pass = p.jb;
  *staged = p.staged ? 1 : 0;
  *smem = (int64_t)grid_smem_bytes(L0, K);
  return MTB_OK;
}
