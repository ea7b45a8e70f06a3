//! Raw declarations of the C ABI in include/llr_b200.h (same names, argument order and types).
//! Every function returns an `llr_status` (0 = success) unless noted; `llr_last_error` holds
//! the message of the last failure on the calling thread.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_float, c_int, c_uint, c_void};

/// Complex f32 with the layout of cuComplex and num_complex::Complex32.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct llr_cf32 {
    pub re: f32,
    pub im: f32,
}

/// Opaque reconstruction context.
#[repr(C)]
pub struct llr_ctx {
    _private: [u8; 0],
}

/// Opaque warm-start network.
#[repr(C)]
pub struct llr_cnn {
    _private: [u8; 0],
}

pub const LLR_OK: c_int = 0;
pub const LLR_ERR_INVALID: c_int = -1;
pub const LLR_ERR_CUDA: c_int = -2;
pub const LLR_ERR_CUFFT: c_int = -3;
pub const LLR_ERR_NOMEM: c_int = -4;
pub const LLR_ERR_NOT_FINITE: c_int = -5;
pub const LLR_ERR_STATE: c_int = -6;
pub const LLR_ERR_UNSUPPORTED: c_int = -7;
pub const LLR_ERR_NO_DEVICE: c_int = -8;

pub const LLR_PROX_HARD_RANK: i32 = 0;
pub const LLR_PROX_SOFT_THRESH: i32 = 1;
pub const LLR_FORWARD: i32 = 0;
pub const LLR_INVERSE: i32 = 1;

/// Recon parameters (LlrReconParams, lib.rs:47-81, plus the B200 build's options).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct llr_config {
    pub vol_size: [i32; 3],
    pub nq: i32,
    pub block_size: [i32; 3],
    pub max_rand_shift: [i32; 3],
    pub prox_mode: i32,
    pub rank: i32,
    pub lambda: f32,
    pub wavelet_alpha: f32,
    pub wavelet_moments: i32,
    pub wavelet_levels: i32,
    pub subspace_rank: i32,
    pub fft_max_batch_size: i32,
    pub cas_mat_max_batch_size: i32,
    pub n_iter: i32,
    pub seed: u64,
    pub device: i32,
    pub eig_solver: i32,
    pub gram_mode: i32,
    pub fft_mode: i32,
    pub wavelet_space: i32,
    pub block_stride: [i32; 3],
}

extern "C" {
    pub fn llr_version() -> *const c_char;
    pub fn llr_last_error() -> *const c_char;
    pub fn llr_status_string(status: c_int) -> *const c_char;
    pub fn llr_config_default(cfg: *mut llr_config) -> c_int;
    pub fn llr_config_validate(cfg: *const llr_config) -> c_int;
    pub fn llr_rand_shift(seed: u64, iteration: i64, max_shift: *const i32, out: *mut i32) -> c_int;
    pub fn llr_grid_dim(vol_size: *const i32, block_size: *const i32, out: *mut i32) -> c_int;
    pub fn llr_vd_mask(ny: i32, nz: i32, nq: i32, accel: f64, centre: i32, seed: u64, out: *mut u8) -> c_int;
    pub fn llr_daubechies_filters(order: i32, lo_d: *mut f32, hi_d: *mut f32, lo_r: *mut f32, hi_r: *mut f32)
        -> c_int;

    // reconstruction context (lib.rs:113-363 as one device-resident object)
    pub fn llr_ctx_create(cfg: *const llr_config, out: *mut *mut llr_ctx) -> c_int;
    pub fn llr_ctx_destroy(ctx: *mut llr_ctx) -> c_int;
    pub fn llr_ctx_set_stream(ctx: *mut llr_ctx, stream: *mut c_void) -> c_int;
    pub fn llr_ctx_get_config(ctx: *const llr_ctx, out: *mut llr_config) -> c_int;
    pub fn llr_upload_kspace(ctx: *mut llr_ctx, y: *const llr_cf32) -> c_int;
    pub fn llr_upload_kspace_dev(ctx: *mut llr_ctx, d_y: *const llr_cf32) -> c_int;
    pub fn llr_set_linear_corrections(ctx: *mut llr_ctx, lin_ksp: *const f32, lin_img: *const f32) -> c_int;
    pub fn llr_estimate_linear_corrections(y: *const llr_cf32, vol_size: *const i32, nq: i32, lin_ksp: *mut f32)
        -> c_int;
    pub fn llr_upload_subspace(ctx: *mut llr_ctx, s: *const llr_cf32) -> c_int;
    pub fn llr_init_zero_filled(ctx: *mut llr_ctx) -> c_int;
    pub fn llr_upload_image(ctx: *mut llr_ctx, x: *const llr_cf32) -> c_int;
    pub fn llr_upload_image_dev(ctx: *mut llr_ctx, d_x: *const llr_cf32) -> c_int;
    pub fn llr_download_image(ctx: *mut llr_ctx, x: *mut llr_cf32) -> c_int;
    pub fn llr_download_image_dev(ctx: *mut llr_ctx, d_x: *mut llr_cf32) -> c_int;
    pub fn llr_iterate(ctx: *mut llr_ctx, n_iter: i32, resid_hist: *mut f64) -> c_int;
    pub fn llr_iterate_async(ctx: *mut llr_ctx, n_iter: i32) -> c_int;
    pub fn llr_iterate_profiled(ctx: *mut llr_ctx, n_iter: i32, stage_ms: *mut f64, total_ms: *mut f64) -> c_int;
    pub fn llr_iterate_timed(ctx: *mut llr_ctx, n_iter: i32, total_ms: *mut f64) -> c_int;
    pub fn llr_ctx_snapshot(ctx: *mut llr_ctx, d_dst: *mut llr_cf32) -> c_int;
    pub fn llr_ctx_nrmse(ctx: *mut llr_ctx, d_ref: *const llr_cf32, nrmse: *mut f64) -> c_int;
    pub fn llr_ctx_kernel_launches(ctx: *const llr_ctx, per_iteration: *mut i32) -> c_int;
    pub fn llr_ctx_fallback_blocks(ctx: *mut llr_ctx, count: *mut i64) -> c_int;
    pub fn llr_get_iteration(ctx: *const llr_ctx, it: *mut i64) -> c_int;
    pub fn llr_set_iteration(ctx: *mut llr_ctx, it: i64) -> c_int;
    pub fn llr_get_residual_history(ctx: *mut llr_ctx, out: *mut f64, count: i32) -> c_int;
    pub fn llr_get_objective_history(ctx: *mut llr_ctx, out: *mut f64, count: i32) -> c_int;
    pub fn llr_measurement_stats(ctx: *mut llr_ctx, total_energy: *mut f64, undersampling: *mut f64) -> c_int;
    pub fn llr_sigma_max(ctx: *mut llr_ctx, shift: *const i32, sigma_max: *mut f64) -> c_int;
    pub fn llr_set_lambda(ctx: *mut llr_ctx, lambda: f32) -> c_int;
    pub fn llr_ctx_prox_llr(ctx: *mut llr_ctx, shift: *const i32) -> c_int;
    pub fn llr_ctx_wavelet(ctx: *mut llr_ctx) -> c_int;
    pub fn llr_ctx_data_consistency(ctx: *mut llr_ctx, resid: *mut f64) -> c_int;
    pub fn llr_ctx_device_bytes(ctx: *const llr_ctx, bytes: *mut usize) -> c_int;

    // host-slice entry points with the reference's argument order
    pub fn llr_cu_low_rank_approx_batch(m: usize, n: usize, rank: usize, batch_size: usize,
                                        matrix_data: *mut llr_cf32) -> c_int;
    pub fn llr_signal_model(x: *mut llr_cf32, image_size: *const usize, batch_size: usize, lin_ksp_corr: *const f32,
                            lin_img_corr: *const f32, direction: i32) -> c_int;
    pub fn llr_lift_data_set(volumes: *const llr_cf32, nvols: usize, matrix_data: *mut llr_cf32,
                             vol_size: *const usize, block_size: *const usize, shift: *const usize,
                             matrix_idx_start: usize, n_matrices: usize) -> c_int;
    pub fn llr_un_lift_data_set(volumes: *mut llr_cf32, nvols: usize, matrix_data: *const llr_cf32,
                                vol_size: *const usize, block_size: *const usize, shift: *const usize,
                                matrix_idx_start: usize, n_matrices: usize) -> c_int;
    pub fn llr_dti_project(subspace_matrix: *const llr_cf32, image_matrices: *const llr_cf32,
                           compressed_matrices: *mut llr_cf32, batch_size: usize, nq: usize, nvox: usize,
                           srank: usize) -> c_int;
    pub fn llr_dti_back_project(subspace_matrix: *const llr_cf32, image_matrices: *mut llr_cf32,
                                compressed_matrices: *const llr_cf32, batch_size: usize, nq: usize, nvox: usize,
                                srank: usize) -> c_int;
    pub fn llr_cu_dwt_denoise(vol_data: *mut llr_cf32, vol_size: *const usize, lo_d: *const f32, hi_d: *const f32,
                              lo_r: *const f32, hi_r: *const f32, filter_len: usize, rand_shift: *const i32)
        -> c_int;

    // device-pointer entry points (d_* arguments are device memory; stream may be null)
    pub fn llr_signal_model_dev(d_x: *mut llr_cf32, image_size: *const i32, batch: i32, lin_ksp: *const f32,
                                lin_img: *const f32, direction: i32, stream: *mut c_void) -> c_int;
    pub fn llr_low_rank_batch_dev(m: i32, n: i32, rank: i32, batch: i32, d_mats: *mut llr_cf32,
                                  stream: *mut c_void) -> c_int;
    pub fn llr_soft_threshold_batch_dev(m: i32, n: i32, lambda: f32, batch: i32, d_mats: *mut llr_cf32,
                                        stream: *mut c_void) -> c_int;
    pub fn llr_wavelet_denoise_dev(d_vols: *mut llr_cf32, vol_size: *const i32, nvol: i32, moments: i32, levels: i32,
                                   alpha: f32, stream: *mut c_void) -> c_int;
    pub fn rhsCdgmmBatched(m: c_int, n: c_int, batch_size: c_int, d_matrix: *mut llr_cf32, d_diag: *mut f32)
        -> c_int;

    // the native DWT launchers cudwt3.rs:97-100 binds (cudaError_t return, 0 = success)
    pub fn dwt3_axis(vol_data: *mut llr_cf32, decomp: *mut llr_cf32, vol_size: *mut c_uint,
                     decomp_size: *mut c_uint, axis: c_uint, filter_len: c_uint, lo_d: *mut c_float,
                     hi_d: *mut c_float, rand_shift: *mut c_int) -> c_int;
    pub fn idwt3_axis(vol_data: *mut llr_cf32, decomp: *mut llr_cf32, vol_size: *mut c_uint,
                      decomp_size: *mut c_uint, axis: c_uint, filter_len: c_uint, lo_r: *mut c_float,
                      hi_r: *mut c_float, rand_shift: *mut c_int) -> c_int;

    // memory helpers
    pub fn llr_host_alloc(bytes: usize, out: *mut *mut c_void) -> c_int;
    pub fn llr_host_free(p: *mut c_void) -> c_int;
    pub fn llr_device_alloc(bytes: usize, out: *mut *mut c_void) -> c_int;
    pub fn llr_device_free(p: *mut c_void) -> c_int;
    pub fn llr_stream_sync(stream: *mut c_void) -> c_int;
    pub fn llr_device_count(n: *mut i32) -> c_int;
}
