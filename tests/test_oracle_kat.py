"""Pins the CPU oracle to every known-answer test the reference holds for this path.

Each test restates the reference test's inputs and expected values (cited file:line);
sizes are reduced where the reference used hundreds of MB.
"""
import math

import numpy as np
import pytest

from conftest import crandn, rel_err
from oracle import llr_oracle as O


def test_cgemm_4x4_known_answer():
    """low_rank.rs:107-180: A(i,j) = i + j i, B(i,j) = j + i i, C = A*B, batch 2."""
    m, k, n, batch = 4, 3, 4, 2
    A = np.zeros((m, k, batch), dtype=np.complex64)
    B = np.zeros((k, n, batch), dtype=np.complex64)
    for b in range(batch):
        for i in range(m):
            for j in range(k):
                A[i, j, b] = complex(i, j)
        for i in range(k):
            for j in range(n):
                B[i, j, b] = complex(j, i)
    C = np.zeros(m * n * batch, dtype=np.complex64)
    out = O.cgemm_strided_batched(m, k, n, batch, False, 1.0, 0.0, False, False,
                                  A.reshape(-1, order="F"), B.reshape(-1, order="F"), C)
    expected = np.array([-5 + 0j, -5 + 3j, -5 + 6j, -5 + 9j, -5 + 3j, -2 + 6j, 1 + 9j, 4 + 12j,
                         -5 + 6j, 1 + 9j, 7 + 12j, 13 + 15j, -5 + 9j, 4 + 12j, 13 + 15j, 22 + 18j])
    np.testing.assert_array_equal(out[:16], expected)
    np.testing.assert_array_equal(out[16:], expected)


def test_rhs_cdgmm_known_answer():
    """cublas.rs:137-183: A = 1+1i, d = j+1  ->  (j+1)(1+1i) exactly (smaller m, batch)."""
    m, n, batch = 270, 67, 5
    A = np.full((m, n, batch), 1 + 1j, dtype=np.complex64)
    d = np.tile((np.arange(n) + 1.0)[:, None], (1, batch)).astype(np.float32)
    out = O.rhs_cdgmm_batched(A, d)
    exp = ((np.arange(n) + 1.0) * (1 + 1j))[None, :, None] * np.ones((m, 1, batch))
    np.testing.assert_array_equal(out, exp.astype(np.complex64))


def test_fft_round_trip_of_ones_is_exact():
    """cufft.rs:413-422: forward then inverse FFT of ones(128^3) equals ones."""
    x = np.ones((32, 32, 32, 1), dtype=np.complex128)
    k = O.fftn_unitary(x, O.FORWARD)
    y = O.fftn_unitary(k, O.INVERSE)
    np.testing.assert_allclose(y, x, atol=1e-12)


def test_dwt_single_level_reconstructs_ijk():
    """cudwt3.rs:18-93: DWT -> IDWT of i+j+k (Daubechies2) rounds back exactly."""
    n = 40
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    v = (i + j + k).astype(np.complex64)
    bank = O.daubechies_bank(2)
    for axis in range(3):
        d = O.dwt_axis(v, axis, bank.lo_d, bank.hi_d)
        assert d.shape[axis] == 2 * O.sub_band_size(n, 4)
        r = O.idwt_axis(d, axis, bank.lo_r, bank.hi_r, n)
        np.testing.assert_array_equal(np.round(r.real), v.real)
    r = O.idwt3(O.dwt3(v, bank), bank, v.shape)
    np.testing.assert_array_equal(np.round(r.real), v.real)


def test_lift_un_lift_identity():
    """block.rs:284-343: lift then un-lift every block restores the data (reduced sizes)."""
    vol, nvol, bs, shift = (40, 30, 20), 5, (8, 6, 4), (28, 14, 6)
    x = np.zeros(vol + (nvol,), dtype=np.complex64, order="F")
    I, J, K, L = np.meshgrid(*[np.arange(s) for s in vol + (nvol,)], indexing="ij")
    x[...] = I + J + K + L
    orig = x.copy()
    nb = int(np.prod(O.grid_dim(vol, bs)))
    mats = O.lift_data_set(x, bs, shift, 0, nb)
    assert mats.shape == (int(np.prod(bs)), nvol, nb)
    x[...] = 0
    O.un_lift_data_set(x, mats, bs, shift, 0, nb)
    np.testing.assert_array_equal(x, orig)


def test_identity_subspace_round_trip():
    """dti_subspace.rs:238-261: identity subspace maps X back to itself."""
    nq, rank, nvox, batch = 3, 3, 100, 10
    S = np.eye(nq, rank, dtype=np.complex64)
    X = np.zeros((nvox, nq, batch), dtype=np.complex64)
    for i in range(nvox):
        for j in range(nq):
            X[i, j, :] = i + j
    flat = X.reshape(-1, order="F")
    out = O.subspace_constraint(S, flat, batch, nq, nvox, rank)
    np.testing.assert_array_equal(out, flat)


def test_periodic_coordinate_wrap():
    """fftshift.rs:127-134: coord [0, 0, -1] in [256, 128, 256] -> [0, 0, 255]."""
    idx = O.coord_to_col_maj_index([0, 0, -1], [256, 128, 256])
    assert O.col_maj_index_to_coord(idx, [256, 128, 256]) == [0, 0, 255]


def test_conj_transpose():
    """dti_subspace.rs:263-281 (printed there; asserted here)."""
    m, n = 3, 2
    a = np.arange(m * n).astype(np.complex64) * (1 + 0.5j)
    out = O.conj_transpose_matrix(a, m, n, 1)
    np.testing.assert_array_equal(out.reshape(n, m, order="F"), a.reshape(m, n, order="F").conj().T)


# ---- properties the oracle must satisfy ---------------------------------------------------
def test_signal_model_is_unitary_and_invertible():
    rng = np.random.default_rng(1)
    x = crandn(rng, (12, 10, 8, 3)).astype(np.complex128)
    lk = rng.standard_normal((3, 3))
    li = rng.standard_normal((3, 3))
    k = O.signal_model(x, lk, li, O.FORWARD)
    assert abs(np.linalg.norm(k) / np.linalg.norm(x) - 1) < 1e-12
    xb = O.signal_model(k, lk, li, O.INVERSE)
    assert rel_err(xb, x) < 1e-12


def test_zero_correction_forward_is_centred_fft():
    """phase_shift_example.m:9-18: pi ramps around a plain FFT == fftshift-centred FFT.

    Equal exactly when every n/2 is even (otherwise up to the global sign (-1)^(sum n/2)).
    """
    rng = np.random.default_rng(2)
    x = crandn(rng, (8, 4, 12, 1)).astype(np.complex128)
    k = O.signal_model(x, np.zeros((1, 3)), np.zeros((1, 3)), O.FORWARD)[..., 0]
    ref = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x[..., 0]), norm="ortho"))
    assert rel_err(k, ref) < 1e-12


def test_hard_rank_equals_projector_form():
    """U_r S_r V_r^H == C V_r V_r^H (the identity the fused prox kernel relies on)."""
    rng = np.random.default_rng(3)
    C = crandn(rng, (40, 9, 4)).astype(np.complex128)
    out = O.low_rank_hard(C, 3)
    for b in range(4):
        _, _, Vh = np.linalg.svd(C[:, :, b], full_matrices=False)
        Vr = Vh[:3].conj().T
        assert rel_err(out[:, :, b], C[:, :, b] @ Vr @ Vr.conj().T) < 1e-12


def test_soft_threshold_via_gram_eigen():
    """C max(s - l, 0)/s V V^H equals the SVD soft threshold."""
    rng = np.random.default_rng(4)
    C = crandn(rng, (30, 7, 3)).astype(np.complex128)
    lam = 3.0
    out = O.low_rank_soft(C, lam)
    for b in range(3):
        G = C[:, :, b].conj().T @ C[:, :, b]
        w, V = np.linalg.eigh(G)
        s = np.sqrt(np.maximum(w, 0))
        gfun = np.where(s > lam, 1 - lam / np.where(s > 0, s, 1), 0)
        W = (V * gfun) @ V.conj().T
        assert rel_err(out[:, :, b], C[:, :, b] @ W) < 1e-10


def test_hybrid_space_identity():
    """A^H (1-M) A == I_x (x) A_yz^H (1-M) A_yz for a line mask (x fully sampled)."""
    rng = np.random.default_rng(5)
    nx, ny, nz, nq = 8, 6, 4, 2
    x = crandn(rng, (nx, ny, nz, nq)).astype(np.complex128)
    lk = rng.standard_normal((nq, 3))
    li = rng.standard_normal((nq, 3))
    mask = (rng.random((ny, nz, nq)) < 0.4)
    k = O.signal_model(x, lk, li, O.FORWARD)
    k[:, mask] = 0
    full = O.signal_model(k, lk, li, O.INVERSE)
    # yz-only operator: apply A along y,z with the reference ramps, mask, invert
    out = np.empty_like(x)
    for q in range(nq):
        sy = O.calc_shift(lk[q], (nx, ny, nz))
        si = O.calc_shift(li[q], (nx, ny, nz))
        pk = np.exp(1j * (O.phase_axis(ny, sy[1])[:, None] + O.phase_axis(nz, sy[2])[None, :]))
        pi_ = np.exp(1j * (O.phase_axis(ny, si[1])[:, None] + O.phase_axis(nz, si[2])[None, :]))
        u = np.fft.fftn(x[..., q] * pk[None], axes=(1, 2), norm="ortho") * np.conj(pi_)[None]
        u[:, mask[..., q]] = 0
        out[..., q] = np.fft.ifftn(u * pi_[None], axes=(1, 2), norm="ortho") * np.conj(pk)[None]
    assert rel_err(out, full) < 1e-12


@pytest.mark.parametrize("moments", [2, 4])
def test_daubechies_filters_match_published_values(moments):
    h = O.daubechies_lowpass(moments)
    published = {
        2: [0.48296291314469025, 0.836516303737469, 0.22414386804185735, -0.12940952255092145],
        4: [0.23037781330885523, 0.7148465705525415, 0.6308807679295904, -0.02798376941698385,
            -0.18703481171888114, 0.030841381835986965, 0.032883011666982945, -0.010597401784997278],
    }[moments]
    np.testing.assert_allclose(h, published, atol=1e-12)
    assert abs(h.sum() - math.sqrt(2)) < 1e-12 and abs((h * h).sum() - 1) < 1e-12


@pytest.mark.parametrize("moments,levels", [(2, 0), (4, 3)])
def test_multilevel_wavelet_perfect_reconstruction(moments, levels):
    rng = np.random.default_rng(6)
    x = crandn(rng, (36, 28, 20)).astype(np.complex128)
    bank = O.daubechies_bank(moments)
    L = levels or O.w_max_level(min(x.shape), bank.flen)
    r = O.waverec3(O.wavedec3(x, bank, L), bank, x.shape)
    assert rel_err(r, x) < 1e-12
    # alpha = 0 shrink is the identity
    assert rel_err(O.wavelet_denoise(x, 0.0, bank, levels), x) < 1e-12


def test_shrink_complex_zero_maps_to_zero():
    out = O.shrink_complex(np.array([0j, 3 + 4j], dtype=np.complex64), 1.0)
    np.testing.assert_allclose(out, [0, (3 + 4j) * 0.8], atol=1e-7)


def test_rand_shift_is_deterministic_and_in_range():
    a = [O.rand_shift(11, it, (64, 48, 32)) for it in range(50)]
    b = [O.rand_shift(11, it, (64, 48, 32)) for it in range(50)]
    assert a == b
    arr = np.array(a)
    assert (arr >= 0).all() and (arr < np.array([64, 48, 32])).all()
    assert len({tuple(v) for v in a}) > 40


def test_vd_mask_rate_and_centre():
    m = O.vd_mask(48, 40, 3, 4.0, 16, 9)
    assert m.shape == (48, 40, 3)
    assert (m[24 - 8:24 + 8, 20 - 8:20 + 8, :] == 1).all()
    r = m.size / m.sum()
    assert 3.6 < r < 4.4
    assert not np.array_equal(m[..., 0], m[..., 1])


def test_recon_residual_decreases_small():
    """The oracle's plain method lowers the DC residual on a tiny phantom."""
    rng = np.random.default_rng(7)
    nx, ny, nz, nq = 16, 16, 8, 5
    x = crandn(rng, (nx, ny, nz, 1)) * np.ones((1, 1, 1, nq), dtype=np.complex64)
    x = x * np.linspace(1, 0.5, nq)[None, None, None, :]
    mask = O.vd_mask(ny, nz, nq, 2.0, 4, 1)
    k = O.signal_model(x.astype(np.complex128), np.zeros((nq, 3)), np.zeros((nq, 3)), O.FORWARD)
    y = O.under_sample_kspace(k, mask)
    cfg = O.ReconConfig(block_size=(4, 4, 4), mode="hard", rank=1, seed=3)
    _, hist = O.recon(y, cfg, 6)
    assert hist[-1] < hist[0]


def test_objective_decreases_with_fixed_partition():
    """Proximal gradient with step 1 on 0.5 ||M A x - y||^2 + lam sum_b ||X_b||_* (A unitary,
    lib.rs:262-341) never raises the objective when the tiling stays fixed; the objective of an
    iterate is 0.5 err + lam * (sum of the thresholded singular values)."""
    rng = np.random.default_rng(8)
    nx, ny, nz, nq = 12, 12, 8, 5
    x = crandn(rng, (nx, ny, nz, 1)) * np.ones((1, 1, 1, nq), dtype=np.complex64)
    x = x * np.linspace(1, 0.5, nq)[None, None, None, :] + 0.1 * crandn(rng, (nx, ny, nz, nq))
    mask = O.vd_mask(ny, nz, nq, 2.0, 4, 2)
    k = O.signal_model(x.astype(np.complex128), np.zeros((nq, 3)), np.zeros((nq, 3)), O.FORWARD)
    y = O.under_sample_kspace(k, mask)
    cfg = O.ReconConfig(block_size=(4, 4, 4), mode="soft", seed=3, max_rand_shift=(1, 1, 1))
    cfg.lam = 0.05 * O.sigma_max(O.zero_filled(y, cfg), (4, 4, 4))
    _, hist, obj = O.recon_objective(y, cfg, 12)
    assert all(b <= a * (1 + 1e-12) for a, b in zip(obj, obj[1:])), obj
    assert obj[-1] < obj[0]
    # the objective's terms: data term from the DC residual, nuclear term non-negative
    assert all(o >= 0.5 * h for o, h in zip(obj, hist))
    hcfg = O.ReconConfig(block_size=(4, 4, 4), mode="hard", rank=1, seed=3)
    _, hh, ho = O.recon_objective(y, hcfg, 2)
    assert ho == [0.5 * v for v in hh]


def test_dti_eigenvalue_known_answer():
    """diffusion_models.rs:148-157: tensor (2, 1.5, 1, 0, 0, 0) has eigenvalues 1, 1.5, 2."""
    np.testing.assert_allclose(O.tensor_eigenvalues(np.array([2.0, 1.5, 1.0, 0, 0, 0])), [2.0, 1.5, 1.0])


def test_dti_fit_recovers_noise_free_tensor():
    """A noise-free tensor signal S0 exp(-b g^T D g) is fitted exactly (diffusion_models.rs:61-112)."""
    from llr_b200.phantom import b_table, eigenvector_matrix, sample_unit_sphere, tensor_signal
    rng = np.random.default_rng(2)
    b, g = b_table([(0, 2), (1000, 15), (2000, 15)], rng)
    R = eigenvector_matrix(sample_unit_sphere(0.3, 0.7))
    D = R @ np.diag([1.7e-3, 0.5e-3, 0.3e-3]) @ R.T
    s = tensor_signal(np.array([0.8]), D[None], b, g)[0]
    dwi = s[b > 0][None].astype(np.complex128)
    b0 = s[b == 0][None].astype(np.complex128)
    r = O.dti_fit(dwi, b0, b[b > 0], g[b > 0])
    np.testing.assert_allclose([r["e1"][0], r["e2"][0], r["e3"][0]], [1.7e-3, 0.5e-3, 0.3e-3], rtol=1e-9)
    np.testing.assert_allclose(r["md"][0], 2.5e-3 / 3, rtol=1e-9)


def test_overlapping_prox_is_the_mean_over_covering_blocks():
    """The oracle's overlapping prox (phases of non-overlapping tilings) equals the direct
    definition: every block of the stride-s grid (lift_data_set with a stride) low-ranked, its
    output added to every voxel it covers, divided by the number of covering blocks."""
    rng = np.random.default_rng(5)
    vol, bs, st, nq = (16, 8, 16), (8, 4, 8), (4, 2, 8), 5
    x = np.asfortranarray((rng.standard_normal(vol + (nq,)) + 1j * rng.standard_normal(vol + (nq,))))
    shift = (3, 5, 1)
    cfg = O.ReconConfig(block_size=bs, mode="soft", lam=1.5, block_stride=st)
    got = O.llr_prox(x, cfg, shift)
    g = O.grid_dim_strided(vol, bs, st)
    nb = int(np.prod(g))
    mats = O.low_rank_soft(O.lift_data_set(x, bs, shift, 0, nb, stride=st), 1.5)
    acc = np.zeros((int(np.prod(vol)), nq), dtype=complex)
    cnt = np.zeros(int(np.prod(vol)))
    for b in range(nb):
        idx = O._block_voxel_index(vol, bs, O.block_coord(b, vol, bs, shift, st))
        acc[idx] += mats[:, :, b]
        cnt[idx] += 1
    assert np.all(cnt == 2 * 2 * 1)
    exp = (acc / cnt[:, None]).reshape(vol + (nq,), order="F")
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)
