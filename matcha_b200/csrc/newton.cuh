// Interface between the orientation-search front end (search.cu) and the Newton march (newton.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include "../../include/matcha_b200.h"

constexpr int kNewtonThreads = 128;
constexpr int kNewtonMaxL = 64;

struct NewtonParams {
  int Lmax;
  int n_stages;
  int stages[MTB_MAX_STAGES];
  int num_steps;
  int flags;
};

// Entries of one subtomogram's folded sigma (and of the recurrence-factor table) for
// degrees up to Lmax: sum_{l <= Lmax} (l + 1)^2, 16 bytes each.
int64_t newton_fold_entries(int Lmax);

// Fill the candidate-independent recurrence-factor table (newton_fold_entries(Lmax) float4).
int newton_build_coef(int Lmax, float4* coef, cudaStream_t st);

// Launch the march for B subtomograms x C candidates on stream st.  Ctab holds
// sqrt((2m')!/((m'+m)!(m'-m)!)) at index m'^2 + m + m' for 0 <= |m| <= m' <= Lmax; coef is
// the table of newton_build_coef.  With fold (B x newton_fold_entries(Lmax) float4 of
// workspace) sigma is folded once per subtomogram first; with fold == nullptr every step
// reads the four sigma images itself (no workspace, more sigma traffic).
int newton_launch(const float* sigma, int64_t stride, int B, int C, float* alpha, float* beta, float* gamma,
                  float* score, const double* Ctab, const float4* coef, float4* fold, const NewtonParams& P,
                  cudaStream_t st);

// Score, Euler gradient and Hessian at one point per subtomogram (degrees <= Li <= the Lmax
// the tables were built for): out (B, 10) float = f, g (a, b, g), H (aa, ab, ag, bb, bg, gg).
int newton_eval_launch(const float* sigma, int64_t stride, int B, int Li, const float* alpha, const float* beta,
                       const float* gamma, const double* Ctab, const float4* coef, float* out, cudaStream_t st);

// The march that reproduces the reference's final-stage top block (flag
// MTB_SEARCH_COMPAT_TOP_BLOCK): full d blocks in shared memory and the reference's row-shift
// derivative stencil on the zeroed block.
int newton_stencil_launch(const float* sigma, int64_t stride, int B, int C, float* alpha, float* beta,
                          float* gamma, float* score, const double* Ctab, const NewtonParams& P, cudaStream_t st);
