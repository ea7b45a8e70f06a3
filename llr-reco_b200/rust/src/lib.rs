//! Safe Rust API of libllr_b200: the llr-reco LLR reconstruction hot path on B200 (sm_100a).
//!
//! The free functions keep the names, argument order and in-place semantics of the llr-reco
//! operators they replace (`cu_low_rank_approx_batch` low_rank.rs:10, `signal_model`
//! signal_model.rs:34, `lift_data_set` / `un_lift_data_set` block.rs:147,166, `dti_project` /
//! `dti_back_project` dti_subspace.rs:141,172, `cu_dwt_denoise` cudwt3.rs:102); they return a
//! `Result` where the reference panics, so a drop-in call site adds `.expect(..)`.  `Recon`
//! holds the whole iteration of lib.rs:262-341 on the device (one CUDA graph per iteration).
//!
//! Element slices may be of `Cf32` or, with the `num-complex` feature, of
//! `num_complex::Complex32` (the element type of the llr-reco crate): both are two f32 (re, im).
pub mod ffi;

use std::ffi::CStr;
use std::fmt;

pub use ffi::llr_cf32 as Cf32;

/// Element types laid out as two consecutive f32 (re, im).
///
/// # Safety
/// Implementors must be `repr(C)` pairs of f32 with no padding.
pub unsafe trait ComplexF32: Copy {}
unsafe impl ComplexF32 for ffi::llr_cf32 {}
#[cfg(feature = "num-complex")]
unsafe impl ComplexF32 for num_complex::Complex32 {}

/// A failed library call: its status and the library's message.
#[derive(Debug, Clone)]
pub struct Error {
    pub status: i32,
    pub message: String,
}

impl fmt::Display for Error {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "llr_b200 error {}: {}", self.status, self.message)
    }
}

impl std::error::Error for Error {}

pub type Result<T> = std::result::Result<T, Error>;

fn check(status: i32) -> Result<()> {
    if status == ffi::LLR_OK {
        return Ok(());
    }
    let message = unsafe {
        let p = ffi::llr_last_error();
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(Error { status, message })
}

fn ptr<T: ComplexF32>(s: &[T]) -> *const Cf32 {
    s.as_ptr() as *const Cf32
}

fn ptr_mut<T: ComplexF32>(s: &mut [T]) -> *mut Cf32 {
    s.as_mut_ptr() as *mut Cf32
}

/// signal_model.rs:13-17.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum ModelDirection {
    Forward,
    Inverse,
}

impl ModelDirection {
    fn code(self) -> i32 {
        match self {
            ModelDirection::Forward => ffi::LLR_FORWARD,
            ModelDirection::Inverse => ffi::LLR_INVERSE,
        }
    }
}

/// The block low-rank operator: the reference's truncated SVD (keep `rank` components) or the
/// singular-value soft threshold.
#[derive(Clone, Copy, Debug, PartialEq)]
pub enum Prox {
    HardRank(i32),
    SoftThreshold(f32),
}

/// Reconstruction parameters (LlrReconParams, lib.rs:47-81, plus the B200 build's options).
#[derive(Clone, Copy, Debug)]
pub struct Config(pub ffi::llr_config);

impl Default for Config {
    fn default() -> Self {
        let mut c = ffi::llr_config::default();
        unsafe { ffi::llr_config_default(&mut c) };
        Config(c)
    }
}

impl Config {
    /// Volume (nx, ny, nz), volume count and block size; everything else at its default.
    pub fn new(vol_size: [usize; 3], nq: usize, block_size: [usize; 3], prox: Prox) -> Self {
        let mut c = Config::default();
        c.0.vol_size = vol_size.map(|v| v as i32);
        c.0.nq = nq as i32;
        c.0.block_size = block_size.map(|v| v as i32);
        c.set_prox(prox);
        c
    }

    pub fn set_prox(&mut self, prox: Prox) {
        match prox {
            Prox::HardRank(r) => {
                self.0.prox_mode = ffi::LLR_PROX_HARD_RANK;
                self.0.rank = r;
            }
            Prox::SoftThreshold(l) => {
                self.0.prox_mode = ffi::LLR_PROX_SOFT_THRESH;
                self.0.lambda = l;
            }
        }
    }

    pub fn validate(&self) -> Result<()> {
        check(unsafe { ffi::llr_config_validate(&self.0) })
    }

    fn elements(&self) -> usize {
        self.0.vol_size.iter().map(|&v| v as usize).product::<usize>() * self.0.nq as usize
    }
}

/// cu_low_rank_approx_batch (low_rank.rs:10): each of `batch_size` column-major m x n matrices
/// is replaced in place by its best rank-`rank` approximation.
pub fn cu_low_rank_approx_batch<T: ComplexF32>(m: usize, n: usize, rank: usize, batch_size: usize,
                                               matrix_data: &mut [T]) -> Result<()> {
    assert!(matrix_data.len() >= m * n * batch_size, "matrix data buffer is too small");
    check(unsafe { ffi::llr_cu_low_rank_approx_batch(m, n, rank, batch_size, ptr_mut(matrix_data)) })
}

/// signal_model (signal_model.rs:34): the forward (image -> k-space) or inverse operator on
/// `batch_size` volumes of `image_size`, with per-volume linear phase corrections.
pub fn signal_model<T: ComplexF32>(x: &mut [T], image_size: &[usize; 3], batch_size: usize,
                                   lin_ksp_corr: &[[f32; 3]], lin_img_corr: &[[f32; 3]],
                                   direction: ModelDirection) -> Result<()> {
    assert!(x.len() >= image_size.iter().product::<usize>() * batch_size, "volume buffer is too small");
    assert!(lin_ksp_corr.len() >= batch_size && lin_img_corr.len() >= batch_size, "one correction per volume");
    check(unsafe {
        ffi::llr_signal_model(ptr_mut(x), image_size.as_ptr(), batch_size, lin_ksp_corr.as_ptr() as *const f32,
                              lin_img_corr.as_ptr() as *const f32, direction.code())
    })
}

/// lift_data_set (block.rs:147): gather blocks start..start+n of `nvols` contiguous volumes at
/// `shift` into Casorati matrices (block voxels x volumes, column-major, one after another).
pub fn lift_data_set<T: ComplexF32>(volumes: &[T], nvols: usize, matrix_data: &mut [T], vol_size: &[usize; 3],
                                    block_size: &[usize; 3], shift: &[usize; 3], matrix_idx_start: usize,
                                    n_matrices: usize) -> Result<()> {
    let m = block_size.iter().product::<usize>();
    assert!(volumes.len() >= vol_size.iter().product::<usize>() * nvols, "volume buffer is too small");
    assert!(matrix_data.len() >= m * nvols * n_matrices, "matrix buffer is too small");
    check(unsafe {
        ffi::llr_lift_data_set(ptr(volumes), nvols, ptr_mut(matrix_data), vol_size.as_ptr(), block_size.as_ptr(),
                               shift.as_ptr(), matrix_idx_start, n_matrices)
    })
}

/// un_lift_data_set (block.rs:166): scatter the matrices back into the volumes.
pub fn un_lift_data_set<T: ComplexF32>(volumes: &mut [T], nvols: usize, matrix_data: &[T], vol_size: &[usize; 3],
                                       block_size: &[usize; 3], shift: &[usize; 3], matrix_idx_start: usize,
                                       n_matrices: usize) -> Result<()> {
    let m = block_size.iter().product::<usize>();
    assert!(volumes.len() >= vol_size.iter().product::<usize>() * nvols, "volume buffer is too small");
    assert!(matrix_data.len() >= m * nvols * n_matrices, "matrix buffer is too small");
    check(unsafe {
        ffi::llr_un_lift_data_set(ptr_mut(volumes), nvols, ptr(matrix_data), vol_size.as_ptr(), block_size.as_ptr(),
                                  shift.as_ptr(), matrix_idx_start, n_matrices)
    })
}

/// dti_project (dti_subspace.rs:141): compressed = images * S for `batch_size` nvox x nq
/// matrices (S nq x srank, column-major).
pub fn dti_project<T: ComplexF32>(subspace_matrix: &[T], image_matrices: &[T], compressed_matrices: &mut [T],
                                  batch_size: usize, nq: usize, nvox: usize, srank: usize) -> Result<()> {
    assert!(subspace_matrix.len() >= nq * srank, "subspace matrix is too small");
    assert!(image_matrices.len() >= nvox * nq * batch_size, "image buffer is too small");
    assert!(compressed_matrices.len() >= nvox * srank * batch_size, "coefficient buffer is too small");
    check(unsafe {
        ffi::llr_dti_project(ptr(subspace_matrix), ptr(image_matrices), ptr_mut(compressed_matrices), batch_size,
                             nq, nvox, srank)
    })
}

/// dti_back_project (dti_subspace.rs:172): images = compressed * S^H.
pub fn dti_back_project<T: ComplexF32>(subspace_matrix: &[T], image_matrices: &mut [T], compressed_matrices: &[T],
                                       batch_size: usize, nq: usize, nvox: usize, srank: usize) -> Result<()> {
    assert!(subspace_matrix.len() >= nq * srank, "subspace matrix is too small");
    assert!(image_matrices.len() >= nvox * nq * batch_size, "image buffer is too small");
    assert!(compressed_matrices.len() >= nvox * srank * batch_size, "coefficient buffer is too small");
    check(unsafe {
        ffi::llr_dti_back_project(ptr(subspace_matrix), ptr_mut(image_matrices), ptr(compressed_matrices),
                                  batch_size, nq, nvox, srank)
    })
}

/// cu_dwt_denoise (cudwt3.rs:102): one-level analysis along every axis then synthesis, with
/// the periodic `rand_shift` applied on the way in and removed on the way out.
pub fn cu_dwt_denoise<T: ComplexF32>(vol_data: &mut [T], vol_size: &[usize; 3], lo_d: &[f32], hi_d: &[f32],
                                     lo_r: &[f32], hi_r: &[f32], rand_shift: &[i32; 3]) -> Result<()> {
    let f = lo_d.len();
    assert!(hi_d.len() == f && lo_r.len() == f && hi_r.len() == f, "four filters of one length");
    assert!(vol_data.len() >= vol_size.iter().product::<usize>(), "volume buffer is too small");
    check(unsafe {
        ffi::llr_cu_dwt_denoise(ptr_mut(vol_data), vol_size.as_ptr(), lo_d.as_ptr(), hi_d.as_ptr(), lo_r.as_ptr(),
                                hi_r.as_ptr(), f, rand_shift.as_ptr())
    })
}

/// rand_shift (lib.rs:420-427) with the counter-based draw the library uses on the device.
pub fn rand_shift(seed: u64, iteration: i64, max_shift: [i32; 3]) -> Result<[i32; 3]> {
    let mut out = [0i32; 3];
    check(unsafe { ffi::llr_rand_shift(seed, iteration, max_shift.as_ptr(), out.as_mut_ptr()) })?;
    Ok(out)
}

/// Orthogonal Daubechies filters of `order` (2 * order taps): (lo_d, hi_d, lo_r, hi_r).
pub fn daubechies_filters(order: usize) -> Result<[Vec<f32>; 4]> {
    let t = 2 * order;
    let (mut a, mut b, mut c, mut d) = (vec![0f32; t], vec![0f32; t], vec![0f32; t], vec![0f32; t]);
    check(unsafe {
        ffi::llr_daubechies_filters(order as i32, a.as_mut_ptr(), b.as_mut_ptr(), c.as_mut_ptr(), d.as_mut_ptr())
    })?;
    Ok([a, b, c, d])
}

/// The device-resident reconstruction (lib.rs:113-363): k-space, iterate and every workspace
/// stay on the GPU; each iteration (LLR prox -> wavelet -> A -> hard DC -> A^H) is one graph.
pub struct Recon {
    ctx: *mut ffi::llr_ctx,
    elements: usize,
    nq: usize,
    srank: usize,
}

impl Recon {
    pub fn new(cfg: &Config) -> Result<Self> {
        let mut ctx = std::ptr::null_mut();
        check(unsafe { ffi::llr_ctx_create(&cfg.0, &mut ctx) })?;
        Ok(Recon { ctx, elements: cfg.elements(), nq: cfg.0.nq as usize, srank: cfg.0.subspace_rank.max(0) as usize })
    }

    /// Measured k-space (nx, ny, nz, nq), column-major, zero where not sampled.
    pub fn upload_kspace<T: ComplexF32>(&mut self, y: &[T]) -> Result<()> {
        assert!(y.len() >= self.elements, "k-space buffer is too small");
        check(unsafe { ffi::llr_upload_kspace(self.ctx, ptr(y)) })
    }

    /// Temporal subspace S (nq x srank, column-major) of a context created with a subspace rank.
    pub fn upload_subspace<T: ComplexF32>(&mut self, s: &[T]) -> Result<()> {
        assert!(s.len() >= self.nq * self.srank, "subspace buffer is too small");
        check(unsafe { ffi::llr_upload_subspace(self.ctx, ptr(s)) })
    }

    /// Per-volume linear phase corrections (k-space and image), one [f32; 3] per volume.
    pub fn set_linear_corrections(&mut self, lin_ksp: &[[f32; 3]], lin_img: &[[f32; 3]]) -> Result<()> {
        assert!(lin_ksp.len() >= self.nq && lin_img.len() >= self.nq, "one correction per volume");
        check(unsafe {
            ffi::llr_set_linear_corrections(self.ctx, lin_ksp.as_ptr() as *const f32, lin_img.as_ptr() as *const f32)
        })
    }

    /// x0 = A^H y (lib.rs:233-242).
    pub fn init_zero_filled(&mut self) -> Result<()> {
        check(unsafe { ffi::llr_init_zero_filled(self.ctx) })
    }

    /// Start from a given image (for example a learned warm start).
    pub fn upload_image<T: ComplexF32>(&mut self, x: &[T]) -> Result<()> {
        assert!(x.len() >= self.elements, "image buffer is too small");
        check(unsafe { ffi::llr_upload_image(self.ctx, ptr(x)) })
    }

    /// `n` iterations; returns the per-iteration data-consistency residual (FP64).
    pub fn iterate(&mut self, n: usize) -> Result<Vec<f64>> {
        let mut h = vec![0f64; n];
        check(unsafe { ffi::llr_iterate(self.ctx, n as i32, h.as_mut_ptr()) })?;
        Ok(h)
    }

    /// Device milliseconds of `n` iterations (no history copy).
    pub fn iterate_timed(&mut self, n: usize) -> Result<f64> {
        let mut ms = 0f64;
        check(unsafe { ffi::llr_iterate_timed(self.ctx, n as i32, &mut ms) })?;
        Ok(ms)
    }

    /// Objective 0.5 ||M A x - y||^2 + lambda sum_b ||X_b||_* of the last `count` iterations
    /// (NaN where the configuration defines none).
    pub fn objective_history(&mut self, count: usize) -> Result<Vec<f64>> {
        let mut h = vec![0f64; count];
        check(unsafe { ffi::llr_get_objective_history(self.ctx, h.as_mut_ptr(), count as i32) })?;
        Ok(h)
    }

    pub fn residual_history(&mut self, count: usize) -> Result<Vec<f64>> {
        let mut h = vec![0f64; count];
        check(unsafe { ffi::llr_get_residual_history(self.ctx, h.as_mut_ptr(), count as i32) })?;
        Ok(h)
    }

    pub fn download_image<T: ComplexF32>(&mut self, x: &mut [T]) -> Result<()> {
        assert!(x.len() >= self.elements, "image buffer is too small");
        check(unsafe { ffi::llr_download_image(self.ctx, ptr_mut(x)) })
    }

    /// Largest block singular value of the current iterate at `shift` (the lambda scale).
    pub fn sigma_max(&mut self, shift: [i32; 3]) -> Result<f64> {
        let mut s = 0f64;
        check(unsafe { ffi::llr_sigma_max(self.ctx, shift.as_ptr(), &mut s) })?;
        Ok(s)
    }

    pub fn set_lambda(&mut self, lambda: f32) -> Result<()> {
        check(unsafe { ffi::llr_set_lambda(self.ctx, lambda) })
    }

    /// (sum |y|^2, numel / nnz) of the measurements (lib.rs:409-417).
    pub fn measurement_stats(&mut self) -> Result<(f64, f64)> {
        let (mut e, mut u) = (0f64, 0f64);
        check(unsafe { ffi::llr_measurement_stats(self.ctx, &mut e, &mut u) })?;
        Ok((e, u))
    }

    pub fn iteration(&self) -> Result<i64> {
        let mut it = 0i64;
        check(unsafe { ffi::llr_get_iteration(self.ctx, &mut it) })?;
        Ok(it)
    }
}

impl Drop for Recon {
    fn drop(&mut self) {
        unsafe {
            ffi::llr_ctx_destroy(self.ctx);
        }
    }
}

/// The recon loop of lib.rs:113-363 without file IO: zero-filled start, `n_iter` iterations,
/// the image into `image`; returns the residual history.  With a soft threshold whose lambda
/// is 0, lambda becomes `lam_rel` times the largest block singular value of the start image.
pub fn llr_recon<T: ComplexF32>(cfg: &Config, kspace: &[T], subspace: Option<&[T]>, n_iter: usize, lam_rel: f32,
                                image: &mut [T]) -> Result<Vec<f64>> {
    let mut r = Recon::new(cfg)?;
    r.upload_kspace(kspace)?;
    if let Some(s) = subspace {
        r.upload_subspace(s)?;
    }
    r.init_zero_filled()?;
    if cfg.0.prox_mode == ffi::LLR_PROX_SOFT_THRESH && cfg.0.lambda == 0.0 {
        let s = r.sigma_max([0, 0, 0])?;
        r.set_lambda(lam_rel * s as f32)?;
    }
    let h = r.iterate(n_iter)?;
    r.download_image(image)?;
    Ok(h)
}

#[cfg(test)]
mod tests {
    use super::*;

    #[test]
    fn config_layout_matches_the_c_struct() {
        assert_eq!(std::mem::size_of::<ffi::llr_config>(), 120);
        assert_eq!(std::mem::align_of::<ffi::llr_config>(), 8);
        assert_eq!(std::mem::size_of::<Cf32>(), 8);
    }

    #[test]
    fn host_functions_need_no_device() {
        let s = rand_shift(7, 3, [8, 8, 8]).unwrap();
        assert!(s.iter().all(|&v| (0..8).contains(&v)));
        let [lo_d, hi_d, lo_r, hi_r] = daubechies_filters(2).unwrap();
        assert_eq!(lo_d.len(), 4);
        let e: f32 = lo_d.iter().map(|v| v * v).sum();
        assert!((e - 1.0).abs() < 1e-6);
        assert_eq!((hi_d.len(), lo_r.len(), hi_r.len()), (4, 4, 4));
        let mut c = Config::new([64, 64, 64], 17, [8, 8, 8], Prox::SoftThreshold(0.1));
        c.validate().unwrap();
        c.0.eig_solver = 2;
        assert!(c.validate().is_err());
    }
}
