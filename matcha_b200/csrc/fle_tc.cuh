// Tensor-core (tcgen05, BF16 hi+lo split) GEMM of the ball expansion; used by fle.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <vector>

struct FleTc {
  alignas(64) unsigned char mapA[128];  // CUtensorMap of the folded channels (bf16 hi/lo)
  alignas(64) unsigned char mapB[128];  // CUtensorMap of the basis (bf16 hi/lo, K-major)
  int Mpad, Npad, Kpad, n_rep, n_cols;
  int ncols[8], coff[8];
  void* A;   // (8 classes x 2 parts x Mpad, Kpad) bf16
  void* B;   // (8 classes x 2 parts x Npad, Kpad) bf16
  int* err;  // nonzero after a bounded wait ran out
  int stall; // test hook (mtb_fle_inject_stall): the producer issues no loads, waits give up early
  int ntn;   // 256-column tiles per class (Npad / 256)
  int* split;  // (8, ntn): 1 where the tile takes the hi+lo split (three MMAs per K step), 0 where
               // its columns are all of degree <= split_degree (plain BF16, one MMA)
  int n_split_tiles, n_tiles;  // how many of the valid tiles take the split, of how many
};

// Split the FP32 class bases into bf16 hi/lo K-major operands and build the tensor maps.
// col_deg[k][j]: degree of column j of class k (non-decreasing in j); split_degree < 0: every
// tile takes the split.
int fle_tc_prepare(FleTc* t, float* const* basis, const int* class_cols, const int* class_off, int n_rep,
                   int max_batch, int n_cols, const std::vector<std::vector<int>>& col_deg, int split_degree);
void fle_tc_release(FleTc* t);
// Fold + split the volumes, then C (B, n_cols) = sum over classes of the split GEMMs.
int fle_tc_forward(FleTc* t, const float* vol, int64_t vol_stride, int B, const int* rep_img, float* C,
                   cudaStream_t st);
// Synchronises st and reports MTB_ERR_TIMEOUT if a device-side wait gave up (then clears it).
int fle_tc_check(FleTc* t, cudaStream_t st);
size_t fle_tc_a_elems(int max_batch, int n_rep);
