/*
 * matcha_b200 -- C ABI of the B200-native subtomogram-alignment hot path.
 *
 * Every entry point returns an int status (MTB_OK on success) and never throws.
 * Pointers are device pointers unless the comment says "host".  Complex arrays are
 * interleaved (re, im) float32, i.e. the memory layout of torch.complex64.  Each
 * compute call takes the CUDA stream it is ordered on (cudaStream_t, passed as
 * mtb_stream_t); no call synchronises the device.  The reference path these entry
 * points replace is cited beside each one (paths inside swing-research/Matcha).
 */
#ifndef MATCHA_B200_H
#define MATCHA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MTB_OK 0
#define MTB_ERR_ARG 1     /* invalid argument (size, pointer, configuration)     */
#define MTB_ERR_OOM 2     /* device allocation failed ("out of memory")          */
#define MTB_ERR_NUMERIC 3 /* non-finite input or result                          */
#define MTB_ERR_TIMEOUT 4 /* a bounded device-side wait ran out                  */
#define MTB_ERR_CUDA 5    /* any other CUDA runtime error; see mtb_last_error()  */

typedef struct CUstream_st* mtb_stream_t; /* identical to cudaStream_t */

/* Version of this ABI (major*100 + minor). */
int mtb_version(void);

/* Host string describing the last error raised on the calling thread ("" if none). */
const char* mtb_last_error(void);

/* ------------------------------------------------------------------------------
 * Orientation search: SO(3) grid search followed by the frequency-marched
 * Wigner-D Newton refinement.
 * Replaces Matcha.__init__ / search_orientations (src/matcha/core/Matcha.py:64-118,
 * 369-403), SOFFT (src/matcha/core/SOFFT.py:11-124), WignerDMatrices.D
 * (src/matcha/core/WignerDMatrices.py:1291-1375) and WignerDGradients
 * (src/matcha/core/WignerDGradients.py:155-302).
 * ---------------------------------------------------------------------------- */
#define MTB_MAX_STAGES 16

/* flags */
#define MTB_SEARCH_COMPAT_TOP_BLOCK 1 /* zero D's m'=-Lmax row and m=-Lmax column at the
                                         final stage, as the reference's kernels return it
                                         (WignerDMatrices.py:573-576)                    */
#define MTB_SEARCH_GRADIENT_STEP 2    /* step_type "gradient" instead of "newton"
                                         (Matcha.py:14-15, 344-345)                      */

typedef struct {
  int Lmax;                  /* L_max of Matcha(...)                                 */
  int n_stages;              /* number of march stages after the skip rule           */
  int stages[MTB_MAX_STAGES];/* truncation degree of each stage (Matcha.py:381-386)  */
  int L0;                    /* grid-search degree, min(Li) (Matcha.py:77)           */
  int K;                     /* oversampling_factor_K (SOFFT.py:17-19)               */
  int candidates;            /* candidates per subtomogram                           */
  int num_steps;             /* Newton steps per stage                               */
  int max_batch;             /* largest B any call will pass                         */
  int flags;                 /* MTB_SEARCH_* bits                                    */
} mtb_search_config;

typedef struct mtb_search mtb_search;

/* Build tables (d-table of the grid, start-value table of the recursion) and the
 * per-candidate workspace on the current device.  Host pointer cfg. */
int mtb_search_create(const mtb_search_config* cfg, mtb_search** out);
void mtb_search_destroy(mtb_search* h);

/* Grid search: f(beta_j, alpha_a, gamma_g) on the (2 L0 K)^3 grid, top-`candidates`
 * peaks per subtomogram, converted to Euler angles (radians).
 * sigma: (B, sigma_stride) complex64, at least dsize(L0-1) entries per row.
 * alpha/beta/gamma: (B, candidates) float32 out.  grid: optional (B, n, n, n) float32
 * out (n = 2 L0 K), NULL to skip.  Replaces Matcha._grid_search_so3fft (Matcha.py:207-236). */
int mtb_so3_grid_topk(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                      float* alpha, float* beta, float* gamma, float* grid, mtb_stream_t stream);

/* Newton march over all stages for every candidate.  alpha/beta/gamma: (B, candidates)
 * float32 in/out; score: (B, candidates) float32 out (best Re sum D sigma).
 * sigma needs dsize(Lmax) entries per row.  Replaces the stage loop of
 * Matcha.search_orientations + Matcha.optimize (Matcha.py:239-398). */
int mtb_newton_march(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                     float* alpha, float* beta, float* gamma, float* score, mtb_stream_t stream);

/* Whole search: grid, march and the reduction over candidates (Matcha.py:19-24).
 * alpha/beta/gamma/score: (B,) float32 out.  Uses the workspace held by h. */
int mtb_search_orientations(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                            float* alpha, float* beta, float* gamma, float* score,
                            mtb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* MATCHA_B200_H */
