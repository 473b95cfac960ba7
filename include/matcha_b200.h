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

/* Host-only query of the grid kernel's pass shape for (L0, K) (no counterpart in the
 * reference): beta values per pass, whether their d-table rows are staged in shared memory,
 * and its dynamic shared memory.  MTB_ERR_ARG when the grid does not fit shared memory. */
int mtb_so3_grid_plan(int L0, int K, int* beta_per_pass, int* staged, int64_t* smem);

/* Grid search: f(beta_j, alpha_a, gamma_g) on the (2 L0 K)^3 grid, top-`candidates`
 * peaks per subtomogram, converted to Euler angles (radians).
 * sigma: (B, sigma_stride) complex64, at least dsize(L0-1) entries per row.
 * alpha/beta/gamma: (B, candidates) float32 out.  grid: optional (B, n, n, n) float32
 * out (n = 2 L0 K), NULL to skip.  Replaces Matcha._grid_search_so3fft (Matcha.py:207-236). */
int mtb_so3_grid_topk(mtb_search* h, const float* sigma, int64_t sigma_stride, int B,
                      float* alpha, float* beta, float* gamma, float* grid, mtb_stream_t stream);

/* The alignment score f = Re sum_{l <= L} D^l(alpha, beta, gamma) sigma_l at one point per
 * subtomogram, with its Euler gradient and Hessian: the quantities the Newton step reads
 * (WignerDGradients.set_so3_coeffs + get_derivatives, src/matcha/core/WignerDGradients.py:
 * 155-302), exposed for a caller's own optimiser or backward pass.  alpha, beta, gamma (B,)
 * float32; out (B, 10) float32 = f, df/d(alpha, beta, gamma), d2f/d(aa, ab, ag, bb, bg, gg).
 * L <= the handle's Lmax; sigma needs dsize(L) entries per row.  No workspace. */
int mtb_score_derivatives(mtb_search* h, const float* sigma, int64_t sigma_stride, int B, int L,
                          const float* alpha, const float* beta, const float* gamma, float* out,
                          mtb_stream_t stream);

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

/* Backward of the alignment score f_b(R) = Re sum D(R_b) sigma_b (no counterpart in the
 * reference, which differentiates only inside its Newton step, WignerDGradients.py:155-302):
 * at the rotations (alpha, beta, gamma)_b (B,) float32 it regenerates D^l(R_b), l <= L, in
 * FP64 (nothing is kept from a forward pass) and writes, each optional (NULL to skip):
 *   grad_sigma (B, >= dsize(L)) complex64 = weight_b conj(D(R_b)), d f / d sigma in PyTorch's
 *     convention for complex tensors;
 *   grad_body (B, 3) float64 = weight_b d f_b(R_b exp(t e_k)) / dt at t = 0 (k = x, y, z), the
 *     so(3) gradient in the body frame, from the generators of the representation applied to
 *     sigma (no Euler-angle singularity at beta = 0 or pi; needs sigma).
 * weight (B,) float32 or NULL (all 1). */
int mtb_score_backward(const float* sigma, int64_t sigma_stride, int B, int L, const float* alpha, const float* beta,
                       const float* gamma, const float* weight, float* grad_sigma, int64_t grad_stride,
                       double* grad_body, mtb_stream_t stream);

/* Allocation-free orientation search.  No counterpart in the reference: it is
 * mtb_search_orientations for callers that must not allocate device memory -- a host
 * program that hands all device memory to its own allocator or runs under a fixed
 * device-memory budget, or a pipeline that cannot take the device-wide synchronisation a
 * cudaMalloc/cudaFree implies.  It needs no handle and calls no allocator: its tables and
 * its candidate workspace live in one file-scope device array of
 * MTB_SEARCH_STATIC_SCRATCH_BYTES, which every GPU that loads this library holds until
 * the process exits.  Each call looks up that array's device address on the current device
 * (cudaGetSymbolAddress, which allocates nothing); the first lookup on a device loads the
 * library's device code there, so make the first call on a device before any stream
 * capture.  A device reset discards the array's contents, which every call rebuilds anyway.
 * All calls share the array: calls that can overlap on the GPU (different
 * streams, or threads without ordering between them) race with each other and must be
 * serialised by the caller.  The tables are rebuilt and every workspace entry is written
 * by each call before it is read.  Returns MTB_ERR_ARG when B x candidates (with the grid
 * tables) does not fit the array (about 250 000 candidate slots).  cfg is a host pointer
 * (its max_batch is ignored); the other arguments are those of mtb_search_orientations. */
#define MTB_SEARCH_STATIC_SCRATCH_BYTES (4 * 1024 * 1024)
int mtb_search_orientations_static(const mtb_search_config* cfg, const float* sigma, int64_t sigma_stride,
                                   int B, float* alpha, float* beta, float* gamma, float* score,
                                   mtb_stream_t stream);

/* ------------------------------------------------------------------------------
 * Ball expansion (FLE) and per-degree correlation coefficients sigma.
 * Replaces FLEBasis3D.evaluate_t (src/matcha/core/FLEBasis3D.py:945-976; its
 * cuFINUFFT + torch-harmonics + radial-interpolation pipeline, :1026-1267) and
 * CrossCorrelationMatcher.compute_sigma / get_sigma
 * (src/matcha/core/CrossCorrelationMatcher.py:183-249).
 *
 * The host supplies the basis in compact form (all pointers host, read during
 * mtb_fle_create only): octant representatives of the voxel ball and their sign
 * images, the real basis columns (Re or Im of conj(psi_{lkm}) for m >= 0) with their
 * reflection-parity class, a table of j_l(lambda_{lk} r) per squared radius, and the
 * maps from real columns back to the complex coefficients in the reference's order.
 * ---------------------------------------------------------------------------- */
typedef struct {
  int N;                    /* volume edge; volumes are (B, N, N, N) float32, C order  */
  int max_batch;            /* largest B any call will pass                            */
  int ne;                   /* complex coefficients per volume (reference order)       */
  int n_rep;                /* octant representatives (x, y, z >= 0) inside the ball   */
  int n_cols;               /* real basis columns (== ne)                              */
  int lmax;                 /* largest degree l                                        */
  int n_lk;                 /* distinct (l, k) radial functions                        */
  int n_r2;                 /* rows of jtab (squared radii)                            */
  const int* rep_img;       /* [n_rep*8] flat voxel index of the sign image with bit0=x
                               flipped, bit1=y, bit2=z; -1 if absent or a duplicate     */
  const double* rep_cos;    /* [n_rep] cos(theta) of the representative                */
  const double* rep_phi;    /* [n_rep] phi of the representative                       */
  const int* rep_r2;        /* [n_rep] row of jtab                                      */
  const double* jtab;       /* [n_r2*n_lk] j_l(lambda_lk * r / radius)                  */
  const int* col_class;     /* [n_cols] parity class, bit0 = odd in x, bit1 = y, bit2 = z */
  const int* col_l;         /* [n_cols]                                                */
  const int* col_m;         /* [n_cols] m >= 0                                         */
  const int* col_part;      /* [n_cols] 0: Re conj(Y) = P cos(m phi), 1: Im = -P sin(m phi) */
  const int* col_lk;        /* [n_cols] column of jtab                                  */
  const double* col_scale;  /* [n_cols] h * c_lk                                        */
  const int* coef_col_re;   /* [ne] column giving Re a_i (times coef_sign_re)           */
  const int* coef_col_im;   /* [ne] column giving Im a_i (times coef_sign_im), -1: zero */
  const signed char* coef_sign_re; /* [ne] +-1                                          */
  const signed char* coef_sign_im; /* [ne] +-1                                          */
  const int* kpad;          /* [lmax+1] padded k-count of degree l                      */
  const int* kidx;          /* [sum_l (2l+1) kpad[l]] coefficient index of (l, mu, k),
                               rows mu = -l..l, -1 = padding                            */
  int precision;            /* MTB_FLE_FP32: FP32 CUDA-core GEMM; MTB_FLE_BF16X3: tcgen05
                               BF16 GEMM with a hi+lo split correction; MTB_FLE_BF16_SPLIT:
                               tcgen05 BF16 GEMM, the split correction only for the columns
                               of degree l > split_degree                               */
  int split_degree;         /* MTB_FLE_BF16_SPLIT: highest degree run in plain BF16 (one MMA
                               per K step instead of three); ignored otherwise           */
} mtb_fle_config;

#define MTB_FLE_FP32 0
#define MTB_FLE_BF16X3 1
#define MTB_FLE_BF16_SPLIT 2

typedef struct mtb_fle mtb_fle;

int mtb_fle_create(const mtb_fle_config* cfg, mtb_fle** out);
void mtb_fle_destroy(mtb_fle* h);

/* Ball coefficients of B real volumes: coeffs (B, coeff_stride) complex64 out, in the
 * reference's order (FLEBasis3D.evaluate_t, without the in-place zeroing of the input);
 * norms (B,) float32 out (|a|_2, CrossCorrelationMatcher.py:244) or NULL. */
int mtb_fle_forward(mtb_fle* h, const float* vol, int B, float* coeffs, int64_t coeff_stride,
                    float* norms, mtb_stream_t stream);

/* sigma[b, Dindex(l, m, mp)] = (-1)^(m+mp) sum_k tmpl[l, -mp, k] conj(coeffs[b, l, -m, k])
 * for l <= lmax (CrossCorrelationMatcher.py:183-212).  coeffs (B, coeff_stride) and
 * tmpl (ne,) complex64; sigma (B, sigma_stride) complex64 out, dsize(lmax) entries. */
int mtb_sigma(mtb_fle* h, const float* coeffs, int64_t coeff_stride, const float* tmpl, int B,
              float* sigma, int64_t sigma_stride, mtb_stream_t stream);

/* mtb_sigma restricted to degrees l <= lmax_out (0 <= lmax_out <= lmax): the first
 * dsize(lmax_out) entries of each row, the rest of the row untouched.  No counterpart in
 * the reference, which always fills every degree of the expansion; the orientation search
 * reads degrees up to its own Lmax only. */
int mtb_sigma_upto(mtb_fle* h, const float* coeffs, int64_t coeff_stride, const float* tmpl, int B,
                   int lmax_out, float* sigma, int64_t sigma_stride, mtb_stream_t stream);

/* Synchronises stream and returns MTB_ERR_TIMEOUT if a bounded device-side wait of the
 * tensor-core path gave up since the last call (then the results of the forwards in between
 * are invalid); the flag is cleared once reported, and the handle stays usable. */
int mtb_fle_status(mtb_fle* h, mtb_stream_t stream);

/* Adjoint of the sigma contraction with respect to the template coefficients (no
 * counterpart in the reference, which has no backward; the forward is
 * CrossCorrelationMatcher.compute_sigma, src/matcha/core/CrossCorrelationMatcher.py:183-212):
 * grad_tmpl[coef(l, -m, k)] = sum_b sum_m' (-1)^(m'+m) coeffs_b[coef(l, -m', k)]
 * grad_sigma_b[l, m', m] for l <= lmax_g, zero above and in the padding entry ne.  coeffs
 * (B, ne) complex64 (the volumes' coefficients, row stride coeff_stride), grad_sigma (B,
 * >= dsize(lmax_g)) complex64, grad_tmpl (ne + 1) complex64 out; gradients in PyTorch's
 * convention for complex tensors (d/dRe + i d/dIm of a real function).  One CTA per degree,
 * the batch summed in order: deterministic. */
int mtb_sigma_backward_template(mtb_fle* h, const float* coeffs, int64_t coeff_stride, const float* grad_sigma,
                                int64_t grad_stride, int B, int lmax_g, float* grad_tmpl, mtb_stream_t stream);

/* Test hook of the failure path (no counterpart in the reference): with on != 0 the
 * tensor-core GEMM of every following forward issues no operand loads, so its MMA thread's
 * bounded wait runs out after about 20 ms; the kernel records the error, frees its tensor
 * memory and returns, and mtb_fle_status reports MTB_ERR_TIMEOUT.  Nothing faults or hangs.
 * MTB_ERR_ARG on an FP32 handle. */
int mtb_fle_inject_stall(mtb_fle* h, int on);

/* The tensor-core GEMM's 256-column tiles that take the hi+lo split (*n_split) of all its
 * valid tiles (*n_tiles): every tile under MTB_FLE_BF16X3, those holding a column of degree
 * above split_degree under MTB_FLE_BF16_SPLIT, 0 of 0 on the FP32 path. */
int mtb_fle_split_tiles(const mtb_fle* h, int* n_split, int* n_tiles);

/* ------------------------------------------------------------------------------
 * FFT shift match (RELION-style masked correlation with a local upsampled DFT).
 * Replaces estimate_shift_like_relion and what it calls
 * (src/matcha/core/ShiftMatcher.py:46-282, 491-674): rotate_complex_volume,
 * extract_shifted_patch_batch, apply_cosine_mask, rfftn and compute_shift_local.
 * ---------------------------------------------------------------------------- */
typedef struct {
  int N;                 /* box edge, power of two                                  */
  int max_batch;         /* largest B any call will pass                            */
  int upsample_factor;   /* shift_upsample_factor (ShiftMatcher.py:660)             */
  int search_radius;     /* shift_search_radius; window 2r+1 (ShiftMatcher.py:661-662) */
  float mask_radius;     /* box_size / (2 voxel_size), setup_utils.py:292-295; <0: N/2 */
  float cosine_width;    /* 5.0 in the reference (setup_utils.py:295)               */
  int precision;         /* MTB_SHIFT_FP32: upsampled DFT on CUDA cores; MTB_SHIFT_BF16X3:
                            tcgen05 BF16 GEMMs with a hi+lo split (every even box from 16 to
                            128 the shift match takes, U = ceil(uf (2r + 1)) <= 256), MTB_ERR_ARG
                            from create on a box / upsampled region they do not cover;
                            MTB_SHIFT_AUTO: the tensor cores where they cover it, else FP32 */
  int tile_rows;         /* FP32 upsampled DFT: rows u0 per CTA of its passes 2+3 (0: 2), the tile
                            shape matcha_b200.autotune chooses per box; no effect on the result */
} mtb_shift_config;

#define MTB_SHIFT_FP32 0
#define MTB_SHIFT_BF16X3 1
#define MTB_SHIFT_AUTO 2

typedef struct mtb_shift mtb_shift;

int mtb_shift_create(const mtb_shift_config* cfg, mtb_shift** out);
void mtb_shift_destroy(mtb_shift* h);

/* ref_fourier: (N, N, N) complex64, the fftshifted and masked Fourier reference of
 * load_reference_full (ShiftMatcher.py:456-472); copied into the handle. */
int mtb_shift_set_reference(mtb_shift* h, const float* ref_fourier, mtb_stream_t stream);

/* subtomos (B, N, N, N) float32; shift_zyx (B, 3) prior shifts (z, y, x); rot (B, 9)
 * row-major rotation matrices of the reference's ZYZ Euler angles
 * (R.from_euler('ZYZ', angles, degrees=True), ShiftMatcher.py:503); ctf (B, N, N, N/2+1)
 * float32 or NULL.  shift_xyz (B, 3) and score (B,) float32 out. */
int mtb_shift_search(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot,
                     const float* ctf, int B, float* shift_xyz, float* score, mtb_stream_t stream);

/* mtb_shift_search in two halves (no counterpart in the reference): mtb_shift_begin takes the
 * patch of each subtomogram at shift_zyx and its x/y transforms into the handle's workspace -
 * nothing that depends on the orientation, so a caller may issue it before the orientation is
 * known, or on another stream; mtb_shift_finish adds the rotated reference and runs the rest
 * for the same B.  The handle holds one begun batch: mtb_shift_finish must be ordered after
 * its mtb_shift_begin (the same stream, or an event between the two streams), and the next
 * mtb_shift_begin after that mtb_shift_finish. */
int mtb_shift_begin(mtb_shift* h, const float* subtomos, const float* shift_zyx, int B, mtb_stream_t stream);
int mtb_shift_finish(mtb_shift* h, const float* rot, const float* ctf, int B, float* shift_xyz, float* score,
                     mtb_stream_t stream);

/* The shift match's correlation as a function of a continuous shift, and its gradient (no
 * counterpart in the reference, which evaluates it only on the upsampled grid,
 * ShiftMatcher.py:46-91, 94-282): for the same inputs as mtb_shift_search and query shifts
 * query_xyz (B, 3) float32 in (x, y, z) voxels, score (B,) = c(s) and grad_xyz (B, 3) = dc/ds,
 *   c(s) = Re sum_m P[m] exp(2 pi i s . f(m)) / (|T| |S|),
 * P = conj(S) T the product of the rotated reference and the patch spectrum, f the
 * frequencies of the (z, y, x) data axes with the half axis taken as a full period of
 * length N/2+1 as the reference's upsampled DFT does.  On the grid s = (u - floor(U/2)) / uf
 * c(s) is the value whose maximum mtb_shift_search returns.  Uses the handle's workspace
 * (FP32 product whatever its precision); calls on one handle must be ordered. */
int mtb_shift_score_grad(mtb_shift* h, const float* subtomos, const float* shift_zyx, const float* rot,
                         const float* ctf, int B, const float* query_xyz, float* score, float* grad_xyz,
                         mtb_stream_t stream);

/* The precision a handle runs the upsampled DFT in (MTB_SHIFT_FP32 or MTB_SHIFT_BF16X3):
 * what MTB_SHIFT_AUTO resolved to.  No counterpart in the reference (a query of this build). */
int mtb_shift_precision(const mtb_shift* h, int* precision);

/* Host-only query of the tensor-core upsampled DFT's launch geometry for box N and upsampled
 * region U (no device, no allocation; no counterpart in the reference): whether passes 2 and 3
 * run fused, the column parts of the passes-1/2 N-tile and each part's width in columns, the
 * pipeline stages of the pass-1/2 kernel and of the separate pass-3 kernel (0 when fused),
 * and the largest dynamic shared memory of its kernels.  MTB_ERR_ARG where the tensor-core
 * kernels do not cover (N, U). */
int mtb_shift_tc_plan(int N, int U, int* fused, int* column_parts, int* n_tile, int* stages1, int* stages3,
                      int64_t* smem_max);

/* Synchronises stream; MTB_ERR_TIMEOUT if a bounded device-side wait of the tensor-core
 * path gave up since the handle was created (then its results are invalid). */
int mtb_shift_status(mtb_shift* h, mtb_stream_t stream);

/* Launch profile of mtb_shift_search (no counterpart in the reference; instrumentation):
 * with n_calls > 0 every search records CUDA events on its stream between its kernel
 * groups, in a ring of the last n_calls calls (0 switches it off).  mtb_shift_profile_read
 * synchronises on the recorded events and returns in ms[0..5] the summed time of
 * (patch + xy FFT, z FFT + product, Nyquist plane, upsampled-DFT pass 1, passes 2+3,
 * finalize) over those calls and their number in *calls.  For the FP32 path the Nyquist
 * entry spans no kernel and pass 1 / passes 2+3 are its two upsampled-DFT kernels. */
int mtb_shift_profile(mtb_shift* h, int n_calls);
int mtb_shift_profile_read(mtb_shift* h, float* ms, int* calls);

/* Rotation bookkeeping on the device: tracker <- normalized(tracker * conj(swap_xz(q(a, b, g))))
 * as update_rotation_estimate (src/matcha/utils/rotation_ops.py:23-34), and rot (B, 9), the
 * matrix the shift match uses for the new tracker (ShiftMatcher.py:503, :913).  alpha, beta,
 * gamma (B,) float32; tracker_in / tracker_out (B, 4) float64 (w, x, y, z), may alias. */
int mtb_update_rotation(const float* alpha, const float* beta, const float* gamma, const double* tracker_in,
                        int B, double* tracker_out, float* rot, mtb_stream_t stream);

/* The shift match's Fourier reference of a template, computed on the device in FP64 as
 * load_reference_full (src/matcha/core/ShiftMatcher.py:456-472) does in numpy: soft low-pass
 * (apply_soft_mask, ini_high 4, edge 2), sinc^2 gridding correction, roll by -N/2, fftn
 * (norm "forward"), fftshift, spherical frequency mask.  tmpl (N, N, N) float64; workspace
 * (2 N^3 + 2 N) x 16 bytes, 16-byte aligned; out (N, N, N) complex64 (interleaved floats), the
 * input of mtb_shift_set_reference.  Synchronises the stream (one-time set-up). */
int mtb_shift_reference(const double* tmpl, int N, float voxel_size, void* workspace, float* out,
                        mtb_stream_t stream);

/* Batch reader (host only): decode MRC2014 files (modes 0 int8, 1 int16, 2 float32, 6 uint16,
 * 12 float16; either byte order; any extended header) into float32 C-order (z, y, x) voxels,
 * as load_subtomogram_cpu / load_ctf_relion5_cpu do through mrcfile
 * (src/matcha/utils/io_utils.py:229-253), on a pool of n_threads threads (0: one per hardware
 * thread), the role of the reader pool of cpu_reader (src/matcha/utils/run_utils.py:430-611).
 * mtb_read_mrc decodes paths[0..n) of shape (nz, ny, nx) each, keeping the leading
 * [0, cz) x [0, cy) x [0, cx) box (the whole volume, or (nz/2, ny, nz/2+1) for a CTF weight
 * file), into dst + i cz cy cx; status[i] is MTB_READ_OK or why file i was skipped.  Returns
 * MTB_ERR_ARG for bad arguments, else MTB_OK whatever the per-file statuses. */
#define MTB_READ_OK 0
#define MTB_READ_OPEN 1   /* cannot open or stat the file */
#define MTB_READ_HEADER 2 /* not an MRC header, or a mode that is not decoded */
#define MTB_READ_SHAPE 3  /* the file's (nz, ny, nx) differs from the expected shape */
#define MTB_READ_SHORT 4  /* the file ends before its voxels do */
typedef struct mtb_reader mtb_reader;
int mtb_reader_create(int n_threads, mtb_reader** out);
int mtb_reader_destroy(mtb_reader* r);
int mtb_read_mrc(mtb_reader* r, const char* const* paths, int n, int nz, int ny, int nx, int cz, int cy, int cx,
                 float* dst, int* status);

/* The rotation the shift match uses for each tracker, on the device: rot (B, 9) float32, row
 * major, the matrix of the conjugated tracker that ShiftMatcher.search_shifts builds on the host
 * (R.from_euler('ZYZ', to_euler_angles(conj(tracker)), degrees) at src/matcha/core/
 * ShiftMatcher.py:913, :503); tracker (B, 4) float64 (w, x, y, z), any nonzero norm. */
int mtb_tracker_rotation(const double* tracker, int B, float* rot, mtb_stream_t stream);

/* One alternation's per-particle results packed for storage, the values each row of
 * store_alignment_parameters (src/matcha/utils/io_utils.py:181-225) takes from device tensors:
 * out (B, 11) float64 = rotation_score, the tracker's quaternionic to_euler_angles (alpha,
 * beta, gamma, radians), local shift (3), prior shift (3), shift_score.  rotation_score and
 * shift_score (B,) float32; local_shift and prior_shift (B, 3) float32; tracker (B, 4) float64. */
int mtb_pack_results(const float* rotation_score, const float* shift_score, const float* local_shift,
                     const float* prior_shift, const double* tracker, int B, double* out, mtb_stream_t stream);

/* The expansion's input of every alternation, BatchProcessor._extract_rotated_batch
 * (src/matcha/align_subtomograms.py:240-252): the patch of each volume at its current shift
 * (extract_subtomogram_patch_batch with normalize=True, src/matcha/utils/io_utils.py:113-178),
 * normalised by the mean and standard deviation inside the hard spherical mask of radius
 * mask_radius about voxel N/2 and multiplied by it (src/matcha/utils/volume_ops.py:6-35), then
 * rotated into the tracker's orientation (rotate_volumes, src/matcha/utils/volume_rotation.py:
 * 8-125).  volumes (B, N, N, N) float32; shift_xyz (B, 3) float32 in voxels (x, y, z);
 * tracker (B, 4) float64 (w, x, y, z); work (B, N, N, N, 2) float32 (8-byte aligned) and
 * stats (B, 2) float64 are the caller's workspace; out (B, N, N, N) float32 may not alias
 * volumes or work. */
int mtb_prepare_subtomos(const float* volumes, int B, int N, const float* shift_xyz, const double* tracker,
                         float mask_radius, float* work, double* stats, float* out, mtb_stream_t stream);

/* Library-wide launch timing (no counterpart in the reference; instrumentation).
 * mtb_profile_start(max_launches) creates 2 * max_launches CUDA events on the current device
 * and switches recording on: from then on every hot-path kernel launch of the library is
 * bracketed by two events on its stream, until max_launches launches have been recorded (the
 * rest are counted as dropped).  mtb_profile_stop switches recording off and keeps what was
 * recorded; mtb_profile_read synchronises on the recorded events and returns, per kernel name
 * in first-launch order, the summed device time (ms) and the number of launches: names is
 * max_entries * MTB_PROFILE_NAME_LEN bytes (NUL-terminated names), ms and launches have
 * max_entries entries, *n_entries the kernels found and *dropped the launches not recorded.
 * mtb_profile_start again clears the record.  Not for use during stream capture. */
#define MTB_PROFILE_NAME_LEN 64
int mtb_profile_start(int max_launches);
int mtb_profile_stop(void);
int mtb_profile_read(int max_entries, char* names, float* ms, int* launches, int* n_entries, int* dropped);

#ifdef __cplusplus
}
#endif

#endif /* MATCHA_B200_H */
