// Tensor-core (tcgen05, BF16 hi+lo split) path of the shift match's upsampled DFT; used by shift.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct ShiftTc {
  alignas(64) unsigned char mapA1[128];  // pass-1 A: rows (b, m2 < N/2, m1), K (m0, re/im)
  alignas(64) unsigned char mapA2[128];  // pass-2 A: rows (b, u0, m2 < N/2), K (m1, re/im)
  alignas(64) unsigned char mapE1[128];  // B of passes 1, 2: rows (column part, u, re/im), K (m, re/im)
  alignas(64) unsigned char mapE3[128];  // B of pass 3: rows u2, K (m2 < N/2, re/im) -> real part
  alignas(64) unsigned char mapA1n[128]; // Nyquist plane m2 = N/2, pass-1 A: rows (b, m1), K (m0, re/im)
  alignas(64) unsigned char mapA2n[128]; // and its pass-2 A: rows (b, u0), K (m1, re/im)
  alignas(64) unsigned char mapA3[128];  // unfused pass-3 A: rows (b, u0 U + u1) padded to RP3 per b,
                                         // K (m2 < N/2, re/im)
  bool fused;                            // passes 2+3 in one kernel (box 16, 32, 64 with 2U <= 256)
  int N, H, HH, U, NT12, NT3, KB12, KB3, G, TPB, CH, NB, Bmax;
  int NS, Us;                            // column parts of the passes 1, 2 N-tile; u per part
  int RP3, TPB3, R3, stages3;            // unfused pass 3: rows per subtomogram, tiles per subtomogram,
                                         // rows per hi/lo part, pipeline stages
  int R1, R2;                            // padded rows per hi/lo part of A1, A2
  int R1n, R2n;                          // and of A1n, A2n
  int stages1;                           // pipeline stages of pass 1
  int n_sm;
  size_t smem1, smem23, smem3;           // dynamic shared memory of the kernels
  void *A1, *A2, *A3, *E1, *E3;          // bf16, [part][row][K] (A3: unfused path only)
  void *A1n, *A2n;                       // bf16, [part][row][K], the Nyquist plane's operands
  float2* ENQ;                           // (NT3) (re, -im) of E2[u2, N/2], the Nyquist column's
                                         // pass-3 factor (zero past U)
  float2* nyq;                           // (Bmax, U, U) the Nyquist plane's 2-D upsampled DFT, FP32
  unsigned long long* best;              // (Bmax) argmax keys: ordered value << 32 | ~flat index
  int* err;                              // nonzero after a bounded wait ran out
};

// 0 when the tensor-core path fits this geometry, MTB_ERR_ARG otherwise: boxes 16, 32, 64 with
// 2U <= 256 run passes 2+3 fused; every other even box from 16 to 128 the front kernels take
// (48, 80, 96, 128), and U > 128 at any box, run the three passes as separate kernels, for
// U <= 256.
int shift_tc_fits(int N, int U);
int shift_tc_prepare(ShiftTc* t, int N, int H, int U, int uf, float dftshift, int max_batch);
void shift_tc_release(ShiftTc* t);
// Nyquist plane, pass 1 and passes 2+3 (fused, or pass 2 then pass 3) for B subtomograms whose
// pass-1 operands A1 and A1n have been written (fft_z split).
// marks (or null): events recorded on st after the Nyquist plane's two GEMMs, pass 1 and
// passes 2+3.
int shift_tc_passes(ShiftTc* t, int B, cudaStream_t st, const cudaEvent_t* marks = nullptr);
// Synchronises st; MTB_ERR_TIMEOUT if a device-side wait gave up, with the code of the
// wait that gave up first in *site (when site is not null).
int shift_tc_check(ShiftTc* t, cudaStream_t st, int* site = nullptr);
