// Tensor-core (tcgen05, BF16 hi+lo split) path of the shift match's upsampled DFT; used by shift.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct ShiftTc {
  alignas(64) unsigned char mapA1[128];  // pass-1 A: rows (b, m2, m1), K (m0, re/im)
  alignas(64) unsigned char mapA2[128];  // pass-2 A: rows (b, u0, m2), K (m1, re/im)
  alignas(64) unsigned char mapA3[128];  // pass-3 A: rows (b, u0, u1), K (m2, re/im)
  alignas(64) unsigned char mapE1[128];  // B of passes 1, 2: rows (u, re/im)
  alignas(64) unsigned char mapE3[128];  // B of pass 3: rows u2
  int N, H, U, NT12, NT3, KB12, KB3, Bmax;
  int R1, R2, R3;                        // padded rows per hi/lo part
  void *A1, *A2, *A3, *E1, *E3;          // bf16, [part][row][K]
  unsigned long long* best;              // (Bmax) argmax keys: ordered value << 32 | ~flat index
  int* err;                              // nonzero after a bounded wait ran out
};

int shift_tc_prepare(ShiftTc* t, int N, int H, int U, int uf, float dftshift, int max_batch);
void shift_tc_release(ShiftTc* t);
// Passes 1-3 for B subtomograms whose pass-1 operand A1 has been written (fft_z split).
int shift_tc_passes(ShiftTc* t, int B, cudaStream_t st);
// Synchronises st; MTB_ERR_TIMEOUT if a device-side wait gave up.
int shift_tc_check(ShiftTc* t, cudaStream_t st);
