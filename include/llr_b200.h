/*
 * llr_b200.h -- C ABI of the B200-native LLR diffusion-MRI reconstruction hot path.
 *
 * Conventions (same as wyatt-A/llr-reco):
 *   - volumes are (nx, ny, nz, nq) complex64, column-major, x fastest, volume index
 *     last (src/array_utils.rs:4-17);
 *   - Casorati batches are (m, n, batch) column-major (src/block.rs:147-164);
 *   - llr_cf32 is layout-identical to Rust's Complex32 and CUDA's cuComplex.
 * Every entry point returns an int status (LLR_OK == 0, negative on error) and never
 * aborts; llr_last_error() gives the message of the calling thread's last failure.
 * "_dev" entry points take device pointers and a cudaStream_t (passed as void*, NULL =
 * legacy default stream); host-slice entry points take host pointers and block.
 */
#ifndef LLR_B200_H
#define LLR_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } llr_cf32;
typedef struct llr_ctx llr_ctx;

enum llr_status {
  LLR_OK = 0,
  LLR_ERR_INVALID = -1,     /* bad argument or configuration                     */
  LLR_ERR_CUDA = -2,        /* CUDA runtime error                                */
  LLR_ERR_CUFFT = -3,       /* cuFFT error                                        */
  LLR_ERR_NOMEM = -4,       /* device or host allocation failed                  */
  LLR_ERR_NOT_FINITE = -5,  /* non-finite objective detected                      */
  LLR_ERR_STATE = -6,       /* call out of order (e.g. iterate before upload)    */
  LLR_ERR_UNSUPPORTED = -7, /* shape outside what the kernels support            */
  LLR_ERR_NO_DEVICE = -8    /* no CUDA device                                    */
};

enum llr_prox_mode {
  LLR_PROX_HARD_RANK = 0,   /* keep the top `rank` singular triplets (low_rank.rs:10-69) */
  LLR_PROX_SOFT_THRESH = 1  /* singular values s -> max(s - lambda, 0)                   */
};

enum llr_direction { LLR_FORWARD = 0, LLR_INVERSE = 1 }; /* signal_model.rs:13-17 */

/* Recon parameters: mirrors LlrReconParams (src/lib.rs:47-81) plus the B200 build's
 * additions (prox mode, absolute threshold, wavelet choice, seed). */
typedef struct llr_config {
  int32_t vol_size[3];        /* nx, ny, nz                                          */
  int32_t nq;                 /* number of volumes                                   */
  int32_t block_size[3];      /* llr_block_size (default 32^3)                       */
  int32_t max_rand_shift[3];  /* 0 -> volume size (lib.rs:260)                       */
  int32_t prox_mode;          /* enum llr_prox_mode (default HARD_RANK)              */
  int32_t rank;               /* llr_block_rank (default 6)                          */
  float lambda;               /* absolute singular-value threshold for SOFT_THRESH   */
  float wavelet_alpha;        /* wavelet_shrink_factor; 0 disables the wavelet step  */
  int32_t wavelet_moments;    /* Daubechies order: 2 (reference) or 4                */
  int32_t wavelet_levels;     /* 0 -> maximum level (lib.rs:441)                     */
  int32_t subspace_rank;      /* 0 -> no subspace; else nq x srank matrix uploaded   */
  int32_t fft_max_batch_size; /* accepted for compatibility (lib.rs:54); unused      */
  int32_t cas_mat_max_batch_size; /* accepted for compatibility (lib.rs:56); unused  */
  int32_t n_iter;             /* default iteration count (lib.rs:62)                 */
  uint64_t seed;              /* key of the counter-based shift RNG                  */
  int32_t device;             /* CUDA device ordinal                                 */
  int32_t eig_solver;         /* 0: tridiagonal, warp per block (default); 1: Jacobi  */
  int32_t gram_mode;          /* 0: 3xTF32 tensor cores (default); 1: FP32 FMA        */
  int32_t fft_mode;           /* 0: fused FFT + DC + inverse FFT per (x, volume) plane
                                  where the plane fits (default); 1: cuFFT passes       */
  int32_t wavelet_space;      /* with a subspace: 0 = shrink the wavelet coefficients of
                                  every image volume (lib.rs:302-309, the reference);
                                  1 = of the srank subspace coefficient volumes (the
                                  blocks must tile the volume)                           */
  int32_t block_stride[3];    /* 0 -> block size (non-overlapping grid, block.rs:112-133);
                                  s < b: overlapping blocks every s voxels, each voxel
                                  the mean of its (b/s)^3 block outputs (b % s == 0 and
                                  the blocks must tile the volume)                       */
} llr_config;

/* ---- library / errors ------------------------------------------------------------ */
const char* llr_version(void);
const char* llr_last_error(void);
const char* llr_status_string(int status);
/* LlrReconParams::default() (lib.rs:67-81). */
int llr_config_default(llr_config* cfg);
/* Host-side validation of a configuration (no device access). */
int llr_config_validate(const llr_config* cfg);

/* ---- counter-based RNG, shapes and masks (host, no device access) ----------------- */
/* rand_shift (lib.rs:420-427), keyed by (seed, iteration): out[a] in [0, max_shift[a]). */
int llr_rand_shift(uint64_t seed, int64_t iteration, const int32_t max_shift[3], int32_t out[3]);
/* grid_dim (block.rs:112-118). */
int llr_grid_dim(const int32_t vol_size[3], const int32_t block_size[3], int32_t out[3]);
/* Variable-density ky-kz sampling mask, uint8 (ny, nz, nq), bit-exact with the oracle. */
int llr_vd_mask(int32_t ny, int32_t nz, int32_t nq, double accel, int32_t centre,
                uint64_t seed, uint8_t* out);
/* Orthogonal Daubechies filters (order 1..10): lo_d, hi_d, lo_r, hi_r of 2*order taps
 * (the bank the dwt crate supplies at cudwt3.rs:27-31). */
int llr_daubechies_filters(int32_t order, float* lo_d, float* hi_d, float* lo_r, float* hi_r);

/* ---- context: device-resident reconstruction -------------------------------------- */
int llr_ctx_create(const llr_config* cfg, llr_ctx** out);
int llr_ctx_destroy(llr_ctx* ctx);
int llr_ctx_set_stream(llr_ctx* ctx, void* stream);
int llr_ctx_get_config(const llr_ctx* ctx, llr_config* out);
/* Measurements y (host, (nx,ny,nz,nq)); the data-consistency set is {y != 0}
 * (lib.rs:392-406).  Line-structured sets (whole x-lines, data_import.rs:416-438) take
 * the hybrid-space fast path; any other pattern takes the element-wise path. */
int llr_upload_kspace(llr_ctx* ctx, const llr_cf32* y);
/* Same, from a device buffer in reference layout (left unmodified). */
int llr_upload_kspace_dev(llr_ctx* ctx, const llr_cf32* d_y);
/* Linear phase corrections, nq x 3 floats each (signal_model.rs:28-33); NULL = zeros.
 * Must precede llr_upload_kspace. */
int llr_set_linear_corrections(llr_ctx* ctx, const float* lin_ksp, const float* lin_img);
/* estimate_linear_correction (signal_model.rs:100-106) for every volume of y (host). */
int llr_estimate_linear_corrections(const llr_cf32* y, const int32_t vol_size[3], int32_t nq,
                                    float* lin_ksp_out);
/* Subspace matrix S, nq x srank column-major (lib.rs:210-219). */
int llr_upload_subspace(llr_ctx* ctx, const llr_cf32* S);
/* Set the iterate to the zero-filled image A^H y (lib.rs:233-242). */
int llr_init_zero_filled(llr_ctx* ctx);
int llr_upload_image(llr_ctx* ctx, const llr_cf32* x);
int llr_upload_image_dev(llr_ctx* ctx, const llr_cf32* d_x);
int llr_download_image(llr_ctx* ctx, llr_cf32* x);
int llr_download_image_dev(llr_ctx* ctx, llr_cf32* d_x);
/* Run n iterations of lib.rs:262-341 (LLR -> wavelet -> A -> hard DC -> A^H) as one
 * CUDA graph per iteration.  resid_hist (host, may be NULL) receives the per-iteration
 * sum of squared data-consistency errors (f64). */
int llr_iterate(llr_ctx* ctx, int32_t n_iter, double* resid_hist);
/* Enqueue n iterations on the context stream without synchronising (no history copy). */
int llr_iterate_async(llr_ctx* ctx, int32_t n_iter);
/* Same iterations, each stage captured as its own graph with CUDA events recorded on the
 * context stream between stages.  stage_ms[5] (may be NULL) receives the summed device
 * time of: LLR prox, wavelet, forward FFT, data consistency, inverse FFT; total_ms the
 * device time from the first to the last event.  Synchronises. */
int llr_iterate_profiled(llr_ctx* ctx, int32_t n_iter, double* stage_ms, double* total_ms);
/* Device time of n single-graph iterations (events on the context stream). */
int llr_iterate_timed(llr_ctx* ctx, int32_t n_iter, double* total_ms);
/* Copy of the iterate in the context's internal layout (V * nq complex), and the relative
 * RMS distance ||x - ref|| / ||ref|| of the current iterate to such a copy taken from a
 * context with the same configuration and k-space (the internal layout differs from the
 * image by a per-element phase and one scale, so the ratio is that of the images).
 * No reference counterpart: convergence measurement without host copies. */
int llr_ctx_snapshot(llr_ctx* ctx, llr_cf32* d_dst);
int llr_ctx_nrmse(llr_ctx* ctx, const llr_cf32* d_ref, double* nrmse);
/* Number of this library's kernels that one captured iteration launches (cuFFT's kernels
 * are not counted).  Valid after the first llr_iterate* call; no reference counterpart. */
int llr_ctx_kernel_launches(const llr_ctx* ctx, int32_t* per_iteration);
/* Blocks the last prox step handed to the Jacobi kernel (more kept components than the
 * tridiagonal path holds, or eigenvectors failing its residual check); 0 for the Jacobi and
 * subspace solvers.  Synchronises.  No reference counterpart: a solver diagnostic. */
int llr_ctx_fallback_blocks(llr_ctx* ctx, int64_t* count);
int llr_get_iteration(const llr_ctx* ctx, int64_t* it);
int llr_set_iteration(llr_ctx* ctx, int64_t it);
/* Residual history of the last `count` iterations ending at the current one. */
int llr_get_residual_history(llr_ctx* ctx, double* out, int32_t count);
/* Objective history, same window: F(x) = 0.5 ||M A x - y||^2 + lambda sum_b ||X_b||_* of each
 * iteration's prox output x (FP64 sums; the nuclear norms from the prox's own singular values).
 * Defined for the soft threshold on one non-overlapping tiling with no wavelet or subspace term
 * (hard rank: the data term alone); NaN otherwise.  With a fixed block partition it is the
 * function the proximal-gradient iteration (step 1, unitary A) decreases monotonically.  No
 * reference counterpart (lib.rs:321-325 records only the residual). */
int llr_get_objective_history(llr_ctx* ctx, double* out, int32_t count);
/* sum |y|^2 and numel/nnz of the measurements (lib.rs:409-417). */
int llr_measurement_stats(llr_ctx* ctx, double* total_energy, double* undersampling);
/* Largest block singular value of the current iterate at `shift` (FP32 Gram + Jacobi). */
int llr_sigma_max(llr_ctx* ctx, const int32_t shift[3], double* sigma_max);
int llr_set_lambda(llr_ctx* ctx, float lambda);
/* Single operator steps on the context iterate (for tests and custom loops). */
int llr_ctx_prox_llr(llr_ctx* ctx, const int32_t shift[3]);
int llr_ctx_wavelet(llr_ctx* ctx);
int llr_ctx_data_consistency(llr_ctx* ctx, double* resid);
/* Bytes of device memory held by the context. */
int llr_ctx_device_bytes(const llr_ctx* ctx, size_t* bytes);

/* ---- device-pointer operators (reference layout) ---------------------------------- */
/* signal_model (signal_model.rs:34-79): in place on d_x (nx,ny,nz,batch). lin_* are
 * host arrays of batch x 3 floats (NULL = zeros). */
int llr_signal_model_dev(llr_cf32* d_x, const int32_t image_size[3], int32_t batch,
                         const float* lin_ksp, const float* lin_img, int32_t direction,
                         void* stream);
/* lift_data_set / un_lift_data_set (block.rs:147-184) on device buffers. */
int llr_lift_data_set_dev(const llr_cf32* d_vol, int32_t nq, llr_cf32* d_mat,
                          const int32_t vol_size[3], const int32_t block_size[3],
                          const int32_t shift[3], int64_t start, int64_t n, void* stream);
int llr_un_lift_data_set_dev(llr_cf32* d_vol, int32_t nq, const llr_cf32* d_mat,
                             const int32_t vol_size[3], const int32_t block_size[3],
                             const int32_t shift[3], int64_t start, int64_t n, void* stream);
/* cu_low_rank_approx_batch (low_rank.rs:10-69) in place on (m, n, batch), n <= 128 (n > 64 runs
 * the wide Jacobi kernel). */
int llr_low_rank_batch_dev(int32_t m, int32_t n, int32_t rank, int32_t batch,
                           llr_cf32* d_mats, void* stream);
/* Same operation as llr_low_rank_batch_dev, for callers that cannot let the library
 * allocate device memory (a caller replaying its own CUDA graph under a fixed memory plan,
 * a device whose memory belongs to another framework's pool, a loop that must not pay an
 * allocator call per invocation).  No counterpart in the reference.  It allocates nothing:
 * it runs the fused tridiagonal prox kernel (no per-matrix Gram scratch; the allocating call
 * runs the split Gram / eigen / apply kernels, so the two agree to the prox tolerance,
 * relative 5e-5, not bitwise), and the list of matrices keeping more than 16 components,
 * which the Jacobi kernel finishes, lives in a static 256 KiB device array per GPU (held
 * until exit), so batch must be <= 65536 (LLR_ERR_INVALID otherwise).  The first call on a
 * device looks up that array's device address and caches it; make that first call before
 * any stream capture, and do not use this entry point on a device after cudaDeviceReset().
 * All calls on a GPU share the array and it keeps the last call's contents (the count word
 * is cleared by every call), so calls that can run at the same time on one GPU, e.g. on two
 * streams, race: serialise them. */
int llr_low_rank_batch_dev_noalloc(int32_t m, int32_t n, int32_t rank, int32_t batch,
                                   llr_cf32* d_mats, void* stream);
/* Singular-value soft threshold of every (m, n) matrix, n <= 128. */
int llr_soft_threshold_batch_dev(int32_t m, int32_t n, float lambda, int32_t batch,
                                 llr_cf32* d_mats, void* stream);
/* LR(X S) S^H per Casorati matrix (lib.rs:281-289, dti_subspace.rs:141-221). */
int llr_subspace_low_rank_batch_dev(int32_t m, int32_t nq, int32_t srank, int32_t prox_mode,
                                    int32_t rank, float lambda, const llr_cf32* d_S,
                                    int32_t batch, llr_cf32* d_mats, void* stream);
/* rhsCdgmmBatched (kernels.cu:49-67): A[:, j, b] *= d[j, b]. Returns a cudaError_t. */
int rhsCdgmmBatched(int m, int n, int batch_size, llr_cf32* d_matrix, float* d_diag);
/* cublas_cgemm_strided_batched_device (cublas.rs:12-105) semantics, own kernel. */
int llr_cgemm_strided_batched_dev(int32_t m, int32_t k, int32_t n, int32_t batch,
                                  int32_t broadcast_a, llr_cf32 alpha, llr_cf32 beta,
                                  int32_t transpose_a, int32_t transpose_b,
                                  const llr_cf32* d_a, const llr_cf32* d_b, llr_cf32* d_c,
                                  void* stream);
/* dwt3_axis / idwt3_axis (kernels.cu:273-348): one-level analysis / synthesis along
 * `axis`; sizes and shift are HOST arrays; filters are device arrays.  The circular
 * shift wraps each axis by its own extent (kernels.cu:80-95 wraps all by vol_size[0]). */
int llr_dwt3_axis_dev(const llr_cf32* d_vol, llr_cf32* d_decomp, const uint32_t vol_size[3],
                      const uint32_t decomp_size[3], uint32_t axis, uint32_t filter_len,
                      const float* d_lo_d, const float* d_hi_d, const int32_t shift[3],
                      void* stream);
int llr_idwt3_axis_dev(llr_cf32* d_vol, const llr_cf32* d_decomp, const uint32_t vol_size[3],
                       const uint32_t decomp_size[3], uint32_t axis, uint32_t filter_len,
                       const float* d_lo_r, const float* d_hi_r, const int32_t shift[3],
                       void* stream);
/* The reference's native DWT launchers with their exact C signatures, as cudwt3.rs:97-100
 * binds them (kernels.cu:273-310 dwt3_axis, kernels.cu:312-348 idwt3_axis): vol_size and
 * decomp_size are HOST arrays of 3 (x fastest); vol_data, decomp, the filters and rand_shift
 * (3 ints) are DEVICE pointers.  Default stream; the call synchronises and returns a
 * cudaError_t (0 = success; cudaErrorInvalidValue for a bad argument).  dwt3_axis writes the
 * approximation (first sub_band_size(n, filter_len) coefficients) then the detail along
 * `axis`; idwt3_axis keeps the centre vol_size[axis] samples.  The circular shift wraps each
 * axis by its own extent (kernels.cu:80-95 wraps all three by vol_size[0]; equal when the
 * shift is zero). */
int dwt3_axis(llr_cf32* vol_data, llr_cf32* decomp, unsigned int* vol_size, unsigned int* decomp_size,
              unsigned int axis, unsigned int filter_len, float* lo_d, float* hi_d, int* rand_shift);
int idwt3_axis(llr_cf32* vol_data, llr_cf32* decomp, unsigned int* vol_size, unsigned int* decomp_size,
               unsigned int axis, unsigned int filter_len, float* lo_r, float* hi_r, int* rand_shift);
/* wavelet_denoise (lib.rs:430-458) on nvol volumes in place; levels 0 -> max. */
int llr_wavelet_denoise_dev(llr_cf32* d_vols, const int32_t vol_size[3], int32_t nvol,
                            int32_t moments, int32_t levels, float alpha, void* stream);
/* hard_project (lib.rs:392-406): where y != 0, accumulate |x - y|^2 (f64) and x := y. */
int llr_hard_project_dev(llr_cf32* d_x, const llr_cf32* d_y, int64_t n, double* sum_sq_error,
                         void* stream);

/* ---- host-slice entry points with the reference's argument order ------------------ */
/* cu_low_rank_approx_batch(m, n, rank, batch_size, &mut [Complex32]) (low_rank.rs:10). */
int llr_cu_low_rank_approx_batch(size_t m, size_t n, size_t rank, size_t batch_size,
                                 llr_cf32* matrix_data);
/* signal_model(x, image_size, batch_size, lin_ksp_corr, lin_img_corr, direction)
 * (signal_model.rs:34). */
int llr_signal_model(llr_cf32* x, const size_t image_size[3], size_t batch_size,
                     const float* lin_ksp_corr, const float* lin_img_corr, int32_t direction);
/* lift_data_set(volumes, matrix_data, vol_size, block_size, shift, start, n)
 * (block.rs:147); volumes is nvols contiguous volumes. */
int llr_lift_data_set(const llr_cf32* volumes, size_t nvols, llr_cf32* matrix_data,
                      const size_t vol_size[3], const size_t block_size[3],
                      const size_t shift[3], size_t matrix_idx_start, size_t n_matrices);
int llr_un_lift_data_set(llr_cf32* volumes, size_t nvols, const llr_cf32* matrix_data,
                         const size_t vol_size[3], const size_t block_size[3],
                         const size_t shift[3], size_t matrix_idx_start, size_t n_matrices);
/* dti_project / dti_back_project (dti_subspace.rs:141,172). */
int llr_dti_project(const llr_cf32* subspace_matrix, const llr_cf32* image_matrices,
                    llr_cf32* compressed_matrices, size_t batch_size, size_t nq, size_t nvox,
                    size_t srank);
int llr_dti_back_project(const llr_cf32* subspace_matrix, llr_cf32* image_matrices,
                         const llr_cf32* compressed_matrices, size_t batch_size, size_t nq,
                         size_t nvox, size_t srank);
/* cu_dwt_denoise(vol, vol_size, lo_d, hi_d, lo_r, hi_r, rand_shift) (cudwt3.rs:102):
 * one-level 3-axis analysis followed by synthesis (no shrinkage). */
int llr_cu_dwt_denoise(llr_cf32* vol_data, const size_t vol_size[3], const float* lo_d,
                       const float* hi_d, const float* lo_r, const float* hi_r,
                       size_t filter_len, const int32_t rand_shift[3]);

/* ---- pinned host memory helpers (for end-to-end callers) -------------------------- */
int llr_host_alloc(size_t bytes, void** out);
int llr_host_free(void* p);
int llr_device_alloc(size_t bytes, void** out);
int llr_device_free(void* p);
int llr_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream);
int llr_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream);
int llr_stream_sync(void* stream);
int llr_device_count(int32_t* n);

/* ---- data-set files (host only, no GPU) --------------------------------------------
 * CFL volumes as the reference's dataset builder and writer use them (data_import.rs:67-108,
 * lib.rs:353-362, the cfl crate's format): <name>.hdr ("# Dimensions" and the sizes, first
 * fastest) and <name>.cfl (raw complex64, column-major).  A ".cfl"/".hdr" suffix on the path is
 * ignored.  The b-table reader takes four numbers per volume, b-value and gradient vector
 * (data_import.rs:110-145; ".txt" is appended when the path has no extension); the b0 mask
 * marks gradient vectors of norm <= tol (data_import.rs:322-328). */
int llr_cfl_dims(const char* path, int64_t* dims, int32_t max_dims, int32_t* ndims);
int llr_cfl_read(const char* path, llr_cf32* dst, int64_t count);
int llr_cfl_write(const char* path, const int64_t* dims, int32_t ndims, const llr_cf32* src);
int llr_read_b_table(const char* path, int32_t n_vols, float* b_vals, float* b_vecs);
int llr_b0_mask(const float* b_vecs, int32_t n_vols, float tol, uint8_t* is_b0);
/* read_affine_translation (signal_model.rs:119-176): the first line holding "Parameters:" must
 * carry 12 numbers (a 3 x 4 affine, translation last); translation = entries 9..11 * multiplier.
 * Translations feed the image-space linear corrections (llr_set_linear_corrections). */
int llr_read_affine_translation(const char* path, float multiplier, float* translation);

/* ---- DTI scalar maps (diffusion_models.rs:21-129, calc_scalars) --------------------
 * Per voxel: s0 = mean |b0|, ln-signal ratios clamped as build_rhs, the least-squares tensor
 * of build_design_matrix's columns, its eigenvalues e1 >= e2 >= e3, MD, RD, FA.  Volumes are
 * (n_vox) complex64 each, volume-major; out receives 7 planes of n_vox floats: b0av, e1, e2,
 * e3, md, rd, fa.  nq >= 6 diffusion-weighted volumes with b_vals (nq), b_vecs (nq x 3). */
int llr_dti_fit_dev(const llr_cf32* d_dwi, int32_t nq, const llr_cf32* d_b0, int32_t nb0, int64_t n_vox,
                    const float* b_vals, const float* b_vecs, float* d_out, void* stream);
int llr_dti_fit(const llr_cf32* dwi, int32_t nq, const llr_cf32* b0, int32_t nb0, int64_t n_vox,
                const float* b_vals, const float* b_vecs, float* out);

/* ---- temporal subspace built on the GPU (no reference counterpart: the reference only
 * loads one, lib.rs:212-222) -------------------------------------------------------------
 * n_signals simulated tensor signals exp(-b g^T D g) (eigenvalues uniform in [lam_lo, lam_hi],
 * principal direction uniform on the sphere, frame as eigenvector_matrix, dti_subspace.rs:13-76)
 * from counter-based draws keyed by seed; FP64 Gram matrix on the GPU, FP64 Jacobi eigenvectors.
 * S_out: nq x rank column-major (largest-magnitude entry of each column positive), sv_out: the
 * rank singular values of the nq x n_signals signal matrix.  nq <= 64. */
int llr_dti_subspace(const float* b_vals, const float* b_vecs, int32_t nq, int32_t rank, int64_t n_signals,
                     uint64_t seed, float lam_lo, float lam_hi, llr_cf32* S_out, double* sv_out);

/* ---- learned warm start: 3-D residual CNN ----------------------------------------
 * No reference counterpart: the reference has no learned component.  A network of
 * n_layers conv3d 3x3x3 layers (zero padding, ReLU between layers, out = in + net(in));
 * channels[0..n_layers], channels[0] == channels[n_layers]; built layer shapes are
 * 14->32, 32->32 and 32->14.  Activations are channels-last FP32 over a volume
 * dims[3] (x fastest); weights are used in BF16 with FP32 accumulation, the optimizer
 * (Adam) keeps FP32 master parameters.  Parameter order per layer: W[27][cin][cout]
 * (tap = dx + 3 (dy + 3 dz)), then b[cout]. */
typedef struct llr_cnn llr_cnn;
int llr_cnn_create(int32_t n_layers, const int32_t* channels, int32_t device, uint64_t seed, llr_cnn** out);
int llr_cnn_destroy(llr_cnn* net);
int llr_cnn_param_count(const llr_cnn* net, int64_t* count);
int llr_cnn_get_params(llr_cnn* net, float* host);
int llr_cnn_set_params(llr_cnn* net, const float* host);
int llr_cnn_get_grads(llr_cnn* net, float* host);
int llr_cnn_forward_dev(llr_cnn* net, const float* d_in, float* d_out, const int32_t* dims, void* stream);
/* forward, mean-squared-error loss against d_target, backward: gradients kept in the net */
int llr_cnn_loss_grad_dev(llr_cnn* net, const float* d_in, const float* d_target, const int32_t* dims,
                          double* loss, void* stream);
int llr_cnn_adam_step(llr_cnn* net, float lr, float beta1, float beta2, float eps, void* stream);
int llr_cnn_train_step_dev(llr_cnn* net, const float* d_in, const float* d_target, const int32_t* dims,
                           float lr, double* loss, void* stream);
/* CNN channels of subspace coefficients: chan[v][2k + {0,1}] = scale (re, im)(sum_q u*[v + V q]
 * x[v + V q] S[q + nq k]) (dti_subspace.rs:141-166), and the image back: x = u (1/scale) c S^H, or
 * x += u (1/scale) c S^H with accumulate != 0 (dti_subspace.rs:172-207).  u is the unit phase of
 * d_phase_ref (a reference image of the same shape, e.g. a low-resolution reconstruction; 0 maps
 * to 1), or 1 when d_phase_ref is NULL: the demodulation that lets a real temporal subspace hold
 * volumes that each carry their own smooth phase.  Images in the reference layout; 1 <= srank <= 16. */
int llr_subspace_channels_dev(const llr_cf32* d_x, const int32_t* vol, int32_t nq, const llr_cf32* d_S,
                              int32_t srank, float scale, const llr_cf32* d_phase_ref, float* d_chan,
                              void* stream);
int llr_subspace_image_dev(const float* d_chan, const int32_t* vol, int32_t nq, const llr_cf32* d_S,
                           int32_t srank, float scale, const llr_cf32* d_phase_ref, int32_t accumulate,
                           llr_cf32* d_x, void* stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* LLR_B200_H */
