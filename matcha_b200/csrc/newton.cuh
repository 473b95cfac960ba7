// Interface between the orientation-search front end (search.cu) and the Newton march (newton.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include "../../include/matcha_b200.h"

constexpr int kNewtonThreads = 256;

struct NewtonParams {
  int Lmax;
  int n_stages;
  int stages[MTB_MAX_STAGES];
  int num_steps;
  int flags;
};

// Dynamic shared memory of one Newton CTA for degrees up to Lmax.
size_t newton_smem_bytes(int Lmax);

// Launch the march for B subtomograms x C candidates on stream st.  Ctab holds
// sqrt((2m')!/((m'+m)!(m'-m)!)) at index m'^2 + m + m' for 0 <= |m| <= m' <= Lmax.
int newton_launch(const float* sigma, int64_t stride, int B, int C, float* alpha, float* beta, float* gamma,
                  float* score, const double* Ctab, const NewtonParams& P, cudaStream_t st);
