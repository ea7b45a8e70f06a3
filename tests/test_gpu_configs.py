"""GPU parity at the benchmark configurations' own sizes (or their shape class where the FP64
oracle would take minutes), through the C-ABI context against ``oracle.recon``.

Tolerance as in test_gpu_recon.py: relative L2 error of the image <= 2e-4 (complex FP32 vs
FP64) and of every per-iteration data-consistency residual <= 2e-4.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import llr_oracle as O

from llr_b200 import ReconContext, ReconParams, _lib as L
from llr_b200.phantom import dti_subspace, make_dataset

pytestmark = pytest.mark.gpu

TOL = 2e-4


def test_c1_full_configuration(gpu):
    """Config 1 exactly: 64^3 x 17 (1 b0 + 16 directions at b=1000), 4x VD ky-kz line sampling with
    a fully sampled 16 x 16 centre, SNR 30, 8^3 blocks (Casorati 512 x 17) with a random shift per
    iteration, soft threshold 0.02 sigma_max, 50 proximal-gradient iterations (lib.rs:262-341).
    The blocks the prox hands to the Jacobi kernel are counted every iteration: at most 5 % of
    the 512 blocks may take that path."""
    vol, bs, n_iter = (64, 64, 64), (8, 8, 8), 50
    d = make_dataset(vol, [(0, 1), (1000, 16)], 4.0, 0, centre=16, mask_fn=O.vd_mask)
    y = d.y
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=11)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=17, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=11)
    hist, fallback = [], []
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        ctx.init_zero_filled()
        assert rel_err(ctx.download_image(), x0) < 2e-6
        for _ in range(n_iter):
            hist.extend(ctx.iterate(1))
            fallback.append(ctx.fallback_blocks)
        gx = ctx.download_image()
    ox, oh = O.recon(y.astype(np.complex128), ocfg, n_iter, x0=x0)
    print(f"C1: image rel err {rel_err(gx, ox):.2e}; Jacobi-fallback blocks per iteration: max {max(fallback)}, "
          f"mean {np.mean(fallback):.2f} of 512")
    assert np.all(np.isfinite(hist))
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL)
    assert max(fallback) <= 0.05 * 512, fallback


def test_c3_shape_class(gpu):
    """Config-3 shape class: 61 volumes (b = 0 / 1000 / 2000, 1 / 30 / 30), 10x sampling, rank-7
    temporal subspace, LLR on the subspace coefficients with 8^3 blocks (X <- LR(X S) S^H,
    dti_subspace.rs:141-221), soft threshold 0.02 sigma_max, then the 3-level db4 wavelet shrink with
    alpha 0.005 on every volume (lib.rs:430-465); a 64 x 56 x 56 volume, the smallest on which a
    3-level db4 decomposition runs along every axis."""
    vol, bs, n_iter = (64, 56, 56), (8, 8, 8), 2
    d = make_dataset(vol, [(0, 1), (1000, 30), (2000, 30)], 10.0, 0, centre=16, mask_fn=O.vd_mask)
    S = dti_subspace(d.b, d.g, 7, 20000, 1)
    y = d.y
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=13, wavelet_alpha=0.005, wavelet_moments=4,
                         wavelet_levels=3)
    ocfg.subspace = S.astype(np.complex128)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=61, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=13,
                    subspace_rank=7)
    p.wavelet_alpha, p.wavelet_moments, p.wavelet_levels = 0.005, 4, 3
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        ctx.upload_subspace(S)
        ctx.init_zero_filled()
        hist = ctx.iterate(n_iter)
        gx = ctx.download_image()
    ox, oh = O.recon(y.astype(np.complex128), ocfg, n_iter, x0=x0)
    assert np.all(np.isfinite(hist))
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL)


def test_c3_coefficient_wavelet(gpu):
    """Config 3 as run by the benchmark: the 3-level db4 shrink (alpha 0.005) acts on the 7 subspace
    coefficient volumes LR(X S) and the image is C S^H (wavelet_space 1); 64^3 x 61, 10x sampling,
    8^3 blocks, soft threshold 0.02 sigma_max, 3 iterations against the oracle's coefficient form."""
    vol, bs, n_iter = (64, 64, 64), (8, 8, 8), 3
    d = make_dataset(vol, [(0, 1), (1000, 30), (2000, 30)], 10.0, 1, centre=16, mask_fn=O.vd_mask)
    S = dti_subspace(d.b, d.g, 7, 20000, 2)
    y = d.y
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=17, wavelet_alpha=0.005, wavelet_moments=4,
                         wavelet_levels=3, wavelet_space="coeffs")
    ocfg.subspace = S.astype(np.complex128)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=61, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=17,
                    subspace_rank=7, wavelet_space=1)
    p.wavelet_alpha, p.wavelet_moments, p.wavelet_levels = 0.005, 4, 3
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        ctx.upload_subspace(S)
        ctx.init_zero_filled()
        hist = ctx.iterate(n_iter)
        gx = ctx.download_image()
    ox, oh = O.recon(y.astype(np.complex128), ocfg, n_iter, x0=x0)
    assert np.all(np.isfinite(hist))
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL)


def test_c5_shape_class_overlapping_blocks(gpu):
    """Config-5 shape class: 106 volumes (6 b0 + 100 over b = 1000 / 2000 / 3000), 12x sampling,
    8^3 blocks at stride 4 (Casorati 512 x 106, each voxel the mean of its 8 block outputs),
    random shift per iteration, soft threshold 0.02 sigma_max; a 32^3 volume, 2 iterations."""
    vol, bs, st, n_iter = (32, 32, 32), (8, 8, 8), (4, 4, 4), 2
    d = make_dataset(vol, [(0, 6), (1000, 34), (2000, 33), (3000, 33)], 12.0, 2, centre=8, mask_fn=O.vd_mask)
    y = d.y
    assert y.shape[3] == 106
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=19, block_stride=st)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=106, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=19,
                    block_stride=st)
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        ctx.init_zero_filled()
        hist = ctx.iterate(n_iter)
        gx = ctx.download_image()
    ox, oh = O.recon(y.astype(np.complex128), ocfg, n_iter, x0=x0)
    assert np.all(np.isfinite(hist))
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL)


@pytest.mark.parametrize("lam_rel", [0.02, 0.002])
def test_plain_512x61_blocks(gpu, lam_rel):
    """8^3 blocks of 61 volumes without a subspace (Casorati 512 x 61): a whole block does not fit the
    Jacobi kernel's shared memory, so the blocks the tridiagonal path hands back (more than 8 kept
    components) go to the wide kernel, which streams row chunks.  At lambda = 0.002 sigma_max most
    blocks keep more than 8 components and take that path; 2 iterations against the oracle.  Image
    within TOL in both cases.  At 0.002 sigma_max nearly every component is kept, and FP32 Jacobi on
    the FP32 Gram (squared conditioning) leaves relative errors ~1e-4 on such dense spectra; the
    residual, a small difference of images (||M A x - y|| << ||x||), magnifies them, so its bound
    there is 1e-3 (measured 7e-4)."""
    vol, bs = (16, 16, 24), (8, 8, 8)
    d = make_dataset(vol, [(0, 1), (1000, 60)], 4.0, 5, centre=6, mask_fn=O.vd_mask)
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=31)
    x0 = O.zero_filled(d.y.astype(np.complex128), ocfg)
    ocfg.lam = lam_rel * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=61, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=31)
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        hist = ctx.iterate(2)
        fallback = ctx.fallback_blocks
        gx = ctx.download_image()
    ox, oh = O.recon(d.y.astype(np.complex128), ocfg, 2, x0=x0)
    if lam_rel < 0.01:
        assert fallback > 0, fallback
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL if lam_rel >= 0.01 else 1e-3)


@pytest.mark.parametrize("nq,stride", [(17, (4, 4, 4)), (80, None), (20, (2, 4, 8))])
def test_overlap_and_wide_paths(gpu, nq, stride):
    """Overlapping blocks with the split prox path (17 volumes; anisotropic strides 2 / 4 / 8, i.e.
    8 phases of 4 x 2 x 1) and the wide Jacobi kernel on a non-overlapping grid (80 volumes)."""
    vol, bs = (24, 24, 16), (8, 8, 8)
    d = make_dataset(vol, [(0, 1), (1000, nq - 1)], 4.0, 3, centre=6, mask_fn=O.vd_mask)
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=23, block_stride=stride)
    x0 = O.zero_filled(d.y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=nq, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=23,
                    block_stride=stride)
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        hist = ctx.iterate(3)
        gx = ctx.download_image()
    ox, oh = O.recon(d.y.astype(np.complex128), ocfg, 3, x0=x0)
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(hist, oh, rtol=TOL)


def test_fp32_converged_matches_fp64_converged(gpu):
    """The headline's reference: the FP32 GPU recon run to convergence (fixed partition) against the
    FP64 oracle run the same 300 iterations on a 24 x 24 x 16 x 17 set; the two converged images
    differ by far less than the 1e-3 NRMSE target (bound 1e-4)."""
    vol, bs, n_iter = (24, 24, 16), (4, 4, 4), 300
    d = make_dataset(vol, [(0, 1), (1000, 16)], 4.0, 4, centre=6, mask_fn=O.vd_mask)
    ocfg = O.ReconConfig(block_size=bs, mode="soft", seed=29, max_rand_shift=(1, 1, 1))
    x0 = O.zero_filled(d.y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=vol, nq=17, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam, seed=29,
                    max_rand_shift=(1, 1, 1))
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        hist = ctx.iterate(n_iter)
        gx = ctx.download_image()
    ox, oh = O.recon(d.y.astype(np.complex128), ocfg, n_iter, x0=x0)
    step = O.nrmse(O.recon(d.y.astype(np.complex128), ocfg, 1, x0=ox, it0=n_iter)[0], ox)
    assert step < 1e-4, step                      # the FP64 run has converged
    assert rel_err(gx, ox) < 1e-4, rel_err(gx, ox)
    assert abs(hist[-1] - oh[-1]) <= 1e-4 * oh[-1]
