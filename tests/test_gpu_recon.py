"""GPU parity of the device-resident reconstruction (C-ABI context) against the FP64 oracle.

Every case runs the same seeded phantom through ``llr_iterate`` (CUDA graph replay, shifts
drawn on the device) and through ``oracle.recon`` with the same counter-based shift
sequence.  Tolerance: relative L2 error of the image <= 2e-4 (complex FP32 vs FP64) and of
each per-iteration data-consistency residual <= 2e-4.
"""
import numpy as np
import pytest

from conftest import crandn, rel_err
from oracle import llr_oracle as O

import llr_b200
from llr_b200 import ReconContext, ReconParams, _lib as L
from llr_b200.phantom import dti_subspace, make_dataset

pytestmark = pytest.mark.gpu

TOL = 2e-4


def dataset(vol, nq, accel=3.0, seed=0, centre=6):
    shells = [(0, 1), (1000, nq - 1)]
    return make_dataset(vol, shells, accel, seed, centre=centre, mask_fn=O.vd_mask)


def oracle_cfg(bs, mode, rank=0, lam=0.0, seed=0, **kw):
    return O.ReconConfig(block_size=tuple(bs), mode=mode, rank=rank, lam=lam, seed=seed, **kw)


def run_both(y, bs, mode, n_iter, rank=2, lam_rel=0.02, seed=5, lin=None, wavelet=None, subspace=None,
             max_shift=None, eig_solver=0, gram_mode=0, fft_mode=0):
    nx, ny, nz, nq = y.shape
    ocfg = oracle_cfg(bs, "hard" if mode == L.LLR_PROX_HARD_RANK else "soft", rank=rank, seed=seed,
                      max_rand_shift=max_shift)
    if lin is not None:
        ocfg.lin_ksp, ocfg.lin_img = lin
    if subspace is not None:
        ocfg.subspace = subspace.astype(np.complex128)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    lam = 0.0
    if mode == L.LLR_PROX_SOFT_THRESH:
        lam = lam_rel * O.sigma_max(x0, bs)
        ocfg.lam = lam
    if wavelet is not None:
        ocfg.wavelet_alpha, ocfg.wavelet_moments, ocfg.wavelet_levels = wavelet
    p = ReconParams(vol_size=(nx, ny, nz), nq=nq, block_size=bs, prox_mode=mode, rank=rank, lam=lam, seed=seed,
                    max_rand_shift=max_shift, eig_solver=eig_solver, gram_mode=gram_mode, fft_mode=fft_mode,
                    subspace_rank=0 if subspace is None else subspace.shape[1])
    if wavelet is not None:
        p.wavelet_alpha, p.wavelet_moments, p.wavelet_levels = wavelet
    with ReconContext(p) as ctx:
        if lin is not None:
            ctx.set_linear_corrections(lin[0], lin[1])
        ctx.upload_kspace(y)
        if subspace is not None:
            ctx.upload_subspace(subspace)
        ctx.init_zero_filled()
        g0 = ctx.download_image()
        assert rel_err(g0, x0) < 2e-6, "zero-filled image"
        hist = ctx.iterate(n_iter)
        gx = ctx.download_image()
        it = ctx.iteration
    ox, ohist = O.recon(y.astype(np.complex128), ocfg, n_iter, x0=x0)
    return gx, ox, np.asarray(hist), np.asarray(ohist), it


def check(gx, ox, gh, oh):
    assert np.all(np.isfinite(gh))
    assert rel_err(gx, ox) < TOL, rel_err(gx, ox)
    np.testing.assert_allclose(gh, oh, rtol=TOL)


def test_soft_threshold_hybrid_path(gpu):
    d = dataset((24, 20, 16), 6)
    gx, ox, gh, oh, it = run_both(d.y, (4, 4, 4), L.LLR_PROX_SOFT_THRESH, 5)
    assert it == 5
    check(gx, ox, gh, oh)
    assert gh[-1] < gh[0]


@pytest.mark.parametrize("eig_solver", [0, 1])
def test_hard_rank_c1_like(gpu, eig_solver):
    """Config-1 shape class: 8^3 blocks, 17 volumes (Casorati 512 x 17), reduced volume."""
    d = dataset((32, 32, 32), 17, accel=4.0, centre=8)
    gx, ox, gh, oh, _ = run_both(d.y, (8, 8, 8), L.LLR_PROX_HARD_RANK, 4, rank=4, eig_solver=eig_solver)
    check(gx, ox, gh, oh)


@pytest.mark.parametrize("eig_solver,gram_mode", [(0, 0), (1, 0), (0, 1)])
def test_soft_c2_like(gpu, eig_solver, gram_mode):
    """Config-2 shape class: 6^3 blocks, 61 volumes (Casorati 216 x 61), reduced volume; both
    eigen-solvers (tridiagonal + bisection, Jacobi) and both Gram paths (3xTF32 tensor cores,
    FP32 FMA)."""
    d = dataset((24, 24, 12), 61, accel=8.0, centre=6)
    gx, ox, gh, oh, _ = run_both(d.y, (6, 6, 6), L.LLR_PROX_SOFT_THRESH, 4, eig_solver=eig_solver,
                                 gram_mode=gram_mode)
    check(gx, ox, gh, oh)


@pytest.mark.parametrize("nq,bs,max_shift,gram_mode", [(61, (6, 6, 6), None, 0), (17, (8, 8, 8), (1, 1, 1), 0),
                                                       (9, (4, 4, 4), None, 1)])
def test_objective_history_matches_oracle(gpu, nq, bs, max_shift, gram_mode):
    """FP64 objective 0.5 ||M A x - y||^2 + lam sum_b ||X_b||_* of every iteration's prox output
    against the oracle's (relative 2e-4, the complex-FP32 tolerance of the residual): random and
    fixed partitions, both Gram paths (the nuclear norms come from the apply kernel's FP64
    singular values and, for blocks the Jacobi kernel takes, its own)."""
    d = dataset((24, 24, 16), nq, accel=4.0, centre=6)
    ocfg = oracle_cfg(bs, "soft", seed=9, max_rand_shift=max_shift)
    x0 = O.zero_filled(d.y.astype(np.complex128), ocfg)
    ocfg.lam = 0.02 * O.sigma_max(x0, bs)
    p = ReconParams(vol_size=(24, 24, 16), nq=nq, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=ocfg.lam,
                    seed=9, max_rand_shift=max_shift, gram_mode=gram_mode)
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        hist = ctx.iterate(4)
        obj = ctx.objective_history(4)
    _, oh, oo = O.recon_objective(d.y.astype(np.complex128), ocfg, 4, x0=x0)
    np.testing.assert_allclose(hist, oh, rtol=2e-4)
    np.testing.assert_allclose(obj, oo, rtol=2e-4)


@pytest.mark.parametrize("bs,srank", [((6, 6, 6), 0), ((8, 8, 8), 7)])
def test_sigma_max_large_blocks(gpu, bs, srank):
    """sigma_max (the lambda scale) of 61-volume blocks, 216 x 61 without a subspace and 512 x 61 with
    one (the config-3 block, too large to stage whole in shared memory), against the oracle's FP64
    SVD of every block."""
    from llr_b200.phantom import dti_subspace
    d = dataset((24, 24, 24), 61, accel=4.0, centre=6)
    x0 = O.zero_filled(d.y.astype(np.complex128), oracle_cfg(bs, "soft"))
    p = ReconParams(vol_size=(24, 24, 24), nq=61, block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH, lam=1.0,
                    subspace_rank=srank)
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        if srank:
            ctx.upload_subspace(dti_subspace(d.b, d.g, srank, 5000, 1))
        ctx.init_zero_filled()
        for sh in ((0, 0, 0), (3, 5, 1)):
            s = ctx.sigma_max(sh)
            e = O.sigma_max(x0, bs, sh)
            assert abs(s - e) <= 1e-5 * e, (sh, s, e)


def test_objective_monotone_with_fixed_partition(gpu):
    """With the tiling fixed the objective never rises (proximal gradient, step 1, unitary A):
    60 iterations on the GPU, each step checked, allowing an FP32-level relative 1e-6 wobble;
    the hard-rank objective is half the residual; a wavelet run has none (NaN)."""
    d = dataset((24, 24, 16), 17, accel=4.0, centre=6)
    ocfg = oracle_cfg((6, 6, 4), "soft", seed=4, max_rand_shift=(1, 1, 1))
    lam = 0.02 * O.sigma_max(O.zero_filled(d.y.astype(np.complex128), ocfg), (6, 6, 4))
    p = ReconParams(vol_size=(24, 24, 16), nq=17, block_size=(6, 6, 4), prox_mode=L.LLR_PROX_SOFT_THRESH, lam=lam,
                    seed=4, max_rand_shift=(1, 1, 1))
    with ReconContext(p) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        ctx.iterate(60)
        obj = ctx.objective_history(60)
    assert np.all(np.isfinite(obj))
    assert np.all(obj[1:] <= obj[:-1] * (1 + 1e-6)), np.diff(obj).max()
    assert obj[-1] < 0.99 * obj[0]
    ph = ReconParams(vol_size=(24, 24, 16), nq=17, block_size=(6, 6, 4), prox_mode=L.LLR_PROX_HARD_RANK, rank=2,
                     seed=4)
    with ReconContext(ph) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        h = ctx.iterate(3)
        np.testing.assert_array_equal(ctx.objective_history(3), 0.5 * np.asarray(h))
    pw = ReconParams(vol_size=(24, 24, 16), nq=17, block_size=(6, 6, 4), prox_mode=L.LLR_PROX_SOFT_THRESH, lam=lam,
                     seed=4)
    pw.wavelet_alpha, pw.wavelet_moments, pw.wavelet_levels = 0.005, 2, 1
    with ReconContext(pw) as ctx:
        ctx.upload_kspace(d.y)
        ctx.init_zero_filled()
        ctx.iterate(2)
        assert np.all(np.isnan(ctx.objective_history(2)))


@pytest.mark.parametrize("vol,fft_mode", [((16, 24, 12), 0), ((16, 24, 12), 1), ((6, 48, 32), 0)])
def test_fused_fft_dc(gpu, vol, fft_mode):
    """Hybrid path with the fused per-plane FFT + DC + inverse FFT kernel (fft_mode 0; plane
    sizes 24 = 6 x 4, 12 = 4 x 3, 48 = 8 x 6, 32 = 8 x 4) and with cuFFT passes (fft_mode 1)."""
    d = dataset(vol, 7, accel=4.0, centre=4)
    gx, ox, gh, oh, _ = run_both(d.y, (4, 4, 4), L.LLR_PROX_SOFT_THRESH, 4, fft_mode=fft_mode)
    check(gx, ox, gh, oh)


@pytest.mark.parametrize("nx,nq", [(6, 5), (48, 7)])
def test_fused_fft_dc_c2_plane(gpu, nx, nq):
    """The 192 x 96 (y, z) plane of the production configuration (16 x 12 and 12 x 8 register
    DFTs), fused against cuFFT on the same data.  6 x 5 planes: one plane per CTA; 48 x 7 = 336
    planes: every CTA transforms several, so the next plane's rows are staged while the current
    one is transformed."""
    d = dataset((nx, 192, 96), nq, accel=8.0, centre=8)
    out = {}
    for mode in (0, 1):
        p = ReconParams(vol_size=(nx, 192, 96), nq=nq, block_size=(6, 6, 6), prox_mode=L.LLR_PROX_SOFT_THRESH,
                        lam=0.5, seed=3, fft_mode=mode)
        with ReconContext(p) as ctx:
            ctx.upload_kspace(d.y)
            ctx.init_zero_filled()
            h = ctx.iterate(3)
            out[mode] = (ctx.download_image(), np.asarray(h))
    assert rel_err(out[0][0], out[1][0]) < 2e-6
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=2e-6)


def test_element_wise_sampling_path(gpu):
    """A sampling set that is not whole x-lines takes the element-wise (3-D FFT) path."""
    d = dataset((16, 12, 8), 5)
    rng = np.random.default_rng(3)
    y = d.y.copy()
    y[rng.random(y.shape) < 0.3] = 0
    gx, ox, gh, oh, _ = run_both(y, (4, 4, 4), L.LLR_PROX_SOFT_THRESH, 4)
    check(gx, ox, gh, oh)


@pytest.mark.parametrize("element_wise", [False, True])
def test_linear_corrections(gpu, element_wise):
    d = dataset((16, 12, 10), 4)
    rng = np.random.default_rng(4)
    lk = rng.uniform(-2, 2, (4, 3)).astype(np.float32)
    li = rng.uniform(-2, 2, (4, 3)).astype(np.float32)
    y = d.y.copy()
    if element_wise:
        y[rng.random(y.shape) < 0.2] = 0
    gx, ox, gh, oh, _ = run_both(y, (4, 4, 2), L.LLR_PROX_SOFT_THRESH, 3,
                                 lin=(lk.astype(np.float64), li.astype(np.float64)))
    check(gx, ox, gh, oh)


def test_volume_not_divisible_by_block(gpu):
    """Voxels outside floor(vol/block) blocks pass through the prox unchanged (block.rs:112-118)."""
    d = dataset((20, 18, 14), 5)
    gx, ox, gh, oh, _ = run_both(d.y, (8, 8, 8), L.LLR_PROX_SOFT_THRESH, 3)
    check(gx, ox, gh, oh)


def test_bounded_random_shift(gpu):
    d = dataset((16, 16, 8), 5)
    gx, ox, gh, oh, _ = run_both(d.y, (4, 4, 4), L.LLR_PROX_HARD_RANK, 3, rank=2, max_shift=(4, 4, 4))
    check(gx, ox, gh, oh)


def test_wavelet_term(gpu):
    d = dataset((32, 24, 20), 4)
    gx, ox, gh, oh, _ = run_both(d.y, (4, 4, 4), L.LLR_PROX_SOFT_THRESH, 3, wavelet=(0.002, 2, 2))
    check(gx, ox, gh, oh)


def test_subspace_llr(gpu):
    vol, nq = (24, 16, 16), 13
    d = make_dataset(vol, [(0, 1), (1000, 6), (2000, 6)], 3.0, 2, centre=6, mask_fn=O.vd_mask)
    S = dti_subspace(d.b, d.g, 4, 2000, 1)
    gx, ox, gh, oh, _ = run_both(d.y, (8, 8, 8), L.LLR_PROX_HARD_RANK, 3, rank=2, subspace=S)
    check(gx, ox, gh, oh)


def test_single_steps_and_sigma_max(gpu):
    d = dataset((24, 20, 16), 6)
    y = d.y
    bs = (4, 4, 4)
    ocfg = oracle_cfg(bs, "soft", seed=1)
    x0 = O.zero_filled(y.astype(np.complex128), ocfg)
    smax = O.sigma_max(x0, bs, (3, 5, 7))
    p = ReconParams(vol_size=y.shape[:3], nq=y.shape[3], block_size=bs, prox_mode=L.LLR_PROX_SOFT_THRESH,
                    lam=0.05 * smax, seed=1)
    ocfg.lam = 0.05 * smax
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        e, us = ctx.measurement_stats()
        oe = O.calc_undersampling_factor(y)
        assert abs(us - oe[0]) < 1e-9 * oe[0] and abs(e - oe[1]) < 1e-5 * oe[1]
        ctx.init_zero_filled()
        assert abs(ctx.sigma_max((3, 5, 7)) - smax) < 1e-4 * smax
        ctx.prox((3, 5, 7))
        px = O.llr_prox(x0, ocfg, (3, 5, 7))
        assert rel_err(ctx.download_image(), px) < 5e-5
        r = ctx.data_consistency()
        k = O.signal_model(px, np.zeros((6, 3)), np.zeros((6, 3)), O.FORWARD)
        k, err = O.hard_project(k, y.astype(np.complex128))
        assert abs(r - err) < 1e-4 * err
        xd = O.signal_model(k, np.zeros((6, 3)), np.zeros((6, 3)), O.INVERSE)
        assert rel_err(ctx.download_image(), xd) < 5e-5


def test_upload_download_round_trip_and_resume(gpu):
    d = dataset((16, 16, 8), 5)
    bs = (4, 4, 4)
    p = ReconParams(vol_size=(16, 16, 8), nq=5, block_size=bs, prox_mode=L.LLR_PROX_HARD_RANK, rank=2, seed=9)
    with ReconContext(p) as a:
        a.upload_kspace(d.y)
        a.init_zero_filled()
        a.iterate(3)
        assert a.kernel_launches_per_iteration >= 3   # prox, DC, residual finalise at least
        mid = a.download_image()
        a.iterate(2)
        straight = a.download_image()
        h_all = a.residual_history(5)
    with ReconContext(p) as b:
        b.upload_kspace(d.y)
        b.upload_image(mid)
        assert rel_err(b.download_image(), mid) < 1e-6
        b.iteration = 3                     # checkpoint/resume: same shift sequence from it 3
        b.iterate(2)
        assert rel_err(b.download_image(), straight) < 1e-5
        np.testing.assert_allclose(b.residual_history(2), h_all[3:], rtol=1e-5)


def test_state_errors(gpu):
    p = ReconParams(vol_size=(16, 16, 8), nq=3, block_size=(4, 4, 4), rank=1)
    with ReconContext(p) as ctx:
        with pytest.raises(llr_b200.LlrError) as e:
            ctx.iterate(1)
        assert e.value.status == L.LLR_ERR_STATE
        with pytest.raises(llr_b200.LlrError) as e:
            ctx.kernel_launches_per_iteration
        assert e.value.status == L.LLR_ERR_STATE
        with pytest.raises(llr_b200.LlrError):
            ctx.download_image()


def test_unsupported_casorati_is_reported(gpu):
    """More than 128 Casorati columns is outside every prox kernel."""
    p = ReconParams(vol_size=(64, 64, 64), nq=130, block_size=(8, 8, 8), rank=2)
    with pytest.raises(llr_b200.LlrError) as e:
        ReconContext(p)
    assert e.value.status == L.LLR_ERR_UNSUPPORTED
