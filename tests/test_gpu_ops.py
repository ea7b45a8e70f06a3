"""GPU parity of the stand-alone operators against the CPU oracle (through the C ABI).

Tolerances (complex FP32 against FP64): relative L2 error <= 2e-6 for the FFT-based signal
model, exact for gathers/scatters and the reference's exact known answers, <= 5e-5 for the
low-rank prox and the wavelet.
"""
import numpy as np
import pytest

from conftest import crandn, rel_err
from oracle import llr_oracle as O

import llr_b200
from llr_b200 import DeviceBuffer, _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,nq", [((16, 12, 8), 3), ((9, 10, 7), 2)])
@pytest.mark.parametrize("direction", [L.LLR_FORWARD, L.LLR_INVERSE])
def test_signal_model_matches_oracle(gpu, dims, nq, direction):
    rng = np.random.default_rng(10)
    x = crandn(rng, dims + (nq,))
    lk = rng.standard_normal((nq, 3)).astype(np.float32)
    li = rng.standard_normal((nq, 3)).astype(np.float32)
    buf = np.asfortranarray(x).reshape(-1, order="F").copy()
    llr_b200.signal_model(buf, dims, nq, lk, li, direction)
    got = buf.reshape(dims + (nq,), order="F")
    exp = O.signal_model(x.astype(np.complex128), lk.astype(np.float64), li.astype(np.float64), direction)
    assert rel_err(got, exp) < 2e-6


def test_fft_round_trip_of_ones(gpu):
    """cufft.rs:413-422 on the device: forward then inverse of ones returns ones."""
    dims = (64, 64, 64)
    buf = np.ones(int(np.prod(dims)), dtype=np.complex64)
    llr_b200.signal_model(buf, dims, 1, None, None, L.LLR_FORWARD)
    llr_b200.signal_model(buf, dims, 1, None, None, L.LLR_INVERSE)
    np.testing.assert_allclose(buf, 1.0, atol=2e-6)


@pytest.mark.parametrize("vol,bs,shift", [((40, 30, 20), (8, 6, 4), (28, 14, 6)), ((17, 13, 9), (4, 5, 3), (3, 12, 8))])
def test_lift_unlift_match_oracle_exactly(gpu, vol, bs, shift):
    rng = np.random.default_rng(11)
    nq = 4
    x = np.asfortranarray(crandn(rng, vol + (nq,)))
    nb = int(np.prod(O.grid_dim(vol, bs)))
    m = int(np.prod(bs))
    mats = np.zeros(m * nq * nb, dtype=np.complex64)
    flat = x.reshape(-1, order="F").copy()
    llr_b200.lift_data_set(flat, nq, mats, vol, bs, shift, 0, nb)
    exp = O.lift_data_set(x, bs, shift, 0, nb)
    np.testing.assert_array_equal(mats, exp.reshape(-1, order="F"))
    # partial batch from an offset (block.rs:153-163 numbers matrices from 0 within the batch)
    part = np.zeros(m * nq * 3, dtype=np.complex64)
    llr_b200.lift_data_set(flat, nq, part, vol, bs, shift, 2, 3)
    np.testing.assert_array_equal(part, O.lift_data_set(x, bs, shift, 2, 3).reshape(-1, order="F"))
    # un-lift restores (block.rs:284-343)
    zero = np.zeros_like(flat)
    llr_b200.un_lift_data_set(zero, nq, mats, vol, bs, shift, 0, nb)
    ref = np.zeros_like(x)
    O.un_lift_data_set(ref, exp, bs, shift, 0, nb)
    np.testing.assert_array_equal(zero, ref.reshape(-1, order="F"))


@pytest.mark.parametrize("m,n,rank", [(64, 9, 3), (216, 61, 6), (512, 17, 5), (100, 33, 1), (20, 10, 10),
                                    (512, 106, 6), (150, 128, 20), (200, 65, 65)])
def test_hard_rank_batch_matches_oracle(gpu, m, n, rank):
    rng = np.random.default_rng(12)
    batch = 7
    # a low-rank signal plus noise so that the rank-r subspace is well separated
    U = crandn(rng, (batch, m, rank))
    V = crandn(rng, (batch, rank, n))
    A = np.moveaxis(U @ V, 0, 2) * 3 + 0.3 * crandn(rng, (m, n, batch))
    A = A.astype(np.complex64)
    buf = A.reshape(-1, order="F").copy()
    llr_b200.cu_low_rank_approx_batch(m, n, rank, batch, buf)
    exp = O.low_rank_hard(A.astype(np.complex128), rank)
    assert rel_err(buf.reshape(m, n, batch, order="F"), exp) < 5e-5


@pytest.mark.parametrize("m,n", [(64, 9), (216, 61), (512, 17), (40, 40), (512, 7), (512, 106), (128, 100)])
def test_soft_threshold_batch_matches_oracle(gpu, m, n):
    rng = np.random.default_rng(13)
    batch = 9
    A = crandn(rng, (m, n, batch))
    s = O.block_singular_values(A)
    lam = float(np.median(s))
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, lam, batch, d.ptr, None))
    got = d.download(np.empty_like(A, order="F"))
    exp = O.low_rank_soft(A.astype(np.complex128), lam)
    # n > 64 runs the wide Jacobi kernel: FP32 rotations of the n x n Gram matrix without the FP64
    # gain refinement; with lambda at the median of a dense random spectrum (the worst case) its
    # error is ~1e-4 (a float32 emulation of the same sweeps gives 4e-5)
    assert rel_err(got, exp) < (5e-5 if n <= 64 else 2e-4)


@pytest.mark.parametrize("m,n,batch", [(216, 61, 1200), (27, 10, 3000)])
def test_soft_threshold_many_blocks_per_cta(gpu, m, n, batch):
    """More blocks than resident CTAs, so every kernel of the split path runs several blocks
    per CTA: the tensor-core Gram with its loads prefetched across block boundaries, the eigen
    kernel's block queue and the apply kernel.  m = 27 is one 32-row chunk per block (the Gram
    kernel then keeps three row tables).  Half the blocks are rank-3 signal plus noise (three
    kept components), half noise only (zero output)."""
    rng = np.random.default_rng(31)
    r = 3
    U = crandn(rng, (batch, m, r))
    V = crandn(rng, (batch, r, n))
    on = (rng.random(batch) < 0.5).astype(np.float64)
    A = np.moveaxis(U @ V, 0, 2) * on[None, None, :] + 0.3 * crandn(rng, (m, n, batch))
    A = A.astype(np.complex64)
    s = O.block_singular_values(A)
    lam = 1.1 * float(max(s[on == 0, 0].max(), s[on == 1, r].max()))   # noise below, signal's 3 above
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, lam, batch, d.ptr, None))
    got = d.download(np.empty_like(A, order="F"))
    exp = O.low_rank_soft(A.astype(np.complex128), lam)
    err = np.linalg.norm((got - exp).reshape(m * n, batch), axis=0)
    scale = np.maximum(np.linalg.norm(A.reshape(m * n, batch), axis=0), 1e-30)
    assert float((err / scale).max()) < 5e-5
    assert np.count_nonzero(np.abs(got[:, :, on == 0]).max(axis=(0, 1))) == 0   # noise-only blocks: zero


def _spectrum_blocks(rng, m, n, sigmas):
    """Blocks C = U diag(sigma) V^H with Haar-like random U (m x n) and V (n x n)."""
    out = np.empty((m, n, len(sigmas)), dtype=np.complex128)
    for b, sg in enumerate(sigmas):
        U, _ = np.linalg.qr(crandn(rng, (m, n)))
        V, _ = np.linalg.qr(crandn(rng, (n, n)))
        out[:, :, b] = (U * np.asarray(sg)[None, :]) @ V.conj().T
    return out


@pytest.mark.parametrize("n", [61, 17])
def test_soft_threshold_eigen_branches(gpu, n):
    """Every branch of the eigen stage: all singular values below the threshold with
    ||G||_F <= lambda^2 (zero at once) and with ||G||_F above it (zero certified by a
    Cholesky factorisation of lambda^2 I - G), 1..8 kept components, more than 8 kept
    (Jacobi fallback), a singular value just above the threshold, and an all-zero block."""
    rng = np.random.default_rng(21)
    m, lam = 216, 1.0
    low = lambda k: list(rng.uniform(0.05, 0.95, k))
    sig = []
    sig.append([0.01] * n)                                   # ||G||_F tiny
    sig.append(low(n))                                       # below, Frobenius above lambda^2
    sig.append([0.97] * 3 + low(n - 3))                      # close below
    for r in range(1, 9):
        sig.append(list(np.linspace(4.0, 1.2, r)) + low(n - r))
    sig.append(list(np.linspace(5.0, 1.5, 12)) + low(n - 12))  # 12 kept: fallback
    sig.append([1.0 + 1e-4] + low(n - 1))                    # just above the threshold
    sig.append([0.0] * n)                                    # all zero
    A = _spectrum_blocks(rng, m, n, sig).astype(np.complex64)
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, lam, A.shape[2], d.ptr, None))
    got = d.download(np.empty_like(A, order="F"))
    exp = O.low_rank_soft(A.astype(np.complex128), lam)
    for b in range(A.shape[2]):
        scale = max(np.linalg.norm(A[:, :, b]), 1e-30)
        assert np.linalg.norm(got[:, :, b] - exp[:, :, b]) / scale < 5e-5, b
    assert rel_err(got, exp) < 5e-5


def test_zero_and_rank_deficient_blocks(gpu):
    m, n, batch = 64, 8, 3
    A = np.zeros((m, n, batch), dtype=np.complex64)
    A[:, 0, 1] = 1 + 1j          # rank 1
    A[:, :, 2] = 2.0             # rank 1, all columns equal
    buf = A.reshape(-1, order="F").copy()
    llr_b200.cu_low_rank_approx_batch(m, n, 2, batch, buf)
    assert rel_err(buf.reshape(m, n, batch, order="F"), A) < 1e-6
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, 0.0, batch, d.ptr, None))
    assert rel_err(d.download(np.empty_like(A, order="F")), A) < 1e-6


def test_rhs_cdgmm_known_answer(gpu):
    """cublas.rs:137-183 on the device (smaller m): exact."""
    m, n, batch = 2700, 67, 50
    A = np.full((m, n, batch), 1 + 1j, dtype=np.complex64)
    d = np.tile((np.arange(n) + 1.0)[:, None], (1, batch)).astype(np.float32)
    dA, dd = DeviceBuffer.from_array(A), DeviceBuffer.from_array(np.asfortranarray(d))
    assert L.lib.rhsCdgmmBatched(m, n, batch, dA.ptr, dd.ptr) == 0
    got = dA.download(np.empty_like(A, order="F"))
    exp = ((np.arange(n) + 1.0) * (1 + 1j))[None, :, None] * np.ones((m, 1, batch))
    np.testing.assert_array_equal(got, exp.astype(np.complex64))


def test_cgemm_known_answer(gpu):
    """low_rank.rs:107-180: the 4x4 expected matrix, exact, batch 2."""
    m, k, n, batch = 4, 3, 4, 2
    A = np.zeros((m, k, batch), dtype=np.complex64, order="F")
    B = np.zeros((k, n, batch), dtype=np.complex64, order="F")
    for i in range(m):
        for j in range(k):
            A[i, j, :] = complex(i, j)
    for i in range(k):
        for j in range(n):
            B[i, j, :] = complex(j, i)
    dA, dB = DeviceBuffer.from_array(A), DeviceBuffer.from_array(B)
    dC = DeviceBuffer.from_array(np.zeros((m, n, batch), dtype=np.complex64))
    one, zero = L.llr_cf32(1, 0), L.llr_cf32(0, 0)
    L.check(L.lib.llr_cgemm_strided_batched_dev(m, k, n, batch, 0, one, zero, 0, 0, dA.ptr, dB.ptr, dC.ptr, None))
    L.check(L.lib.llr_stream_sync(None))
    got = dC.download(np.empty((m, n, batch), dtype=np.complex64, order="F"))
    expected = np.array([-5 + 0j, -5 + 3j, -5 + 6j, -5 + 9j, -5 + 3j, -2 + 6j, 1 + 9j, 4 + 12j,
                         -5 + 6j, 1 + 9j, 7 + 12j, 13 + 15j, -5 + 9j, 4 + 12j, 13 + 15j, 22 + 18j])
    np.testing.assert_array_equal(got[:, :, 0].reshape(-1, order="F"), expected)
    np.testing.assert_array_equal(got[:, :, 1], got[:, :, 0])


@pytest.mark.parametrize("ta,tb,bcast", [(0, 0, 0), (1, 1, 1), (0, 1, 0), (1, 0, 1)])
def test_cgemm_ops_match_oracle(gpu, ta, tb, bcast):
    rng = np.random.default_rng(14)
    m, k, n, batch = 13, 21, 17, 3
    a = crandn(rng, (m * k * (1 if bcast else batch),))
    b = crandn(rng, (k * n * batch,))
    c = crandn(rng, (m * n * batch,))
    dA, dB, dC = DeviceBuffer.from_array(a), DeviceBuffer.from_array(b), DeviceBuffer.from_array(c)
    alpha, beta = L.llr_cf32(0.5, -1.0), L.llr_cf32(2.0, 0.25)
    L.check(L.lib.llr_cgemm_strided_batched_dev(m, k, n, batch, bcast, alpha, beta, ta, tb, dA.ptr, dB.ptr, dC.ptr,
                                                None))
    got = dC.download(np.empty_like(c))
    exp = O.cgemm_strided_batched(m, k, n, batch, bool(bcast), 0.5 - 1j, 2 + 0.25j, bool(ta), bool(tb),
                                  a.astype(np.complex128), b.astype(np.complex128), c.astype(np.complex128))
    assert rel_err(got, exp) < 1e-6


def test_dti_project_and_back_project_match_oracle(gpu):
    rng = np.random.default_rng(15)
    nq, srank, nvox, batch = 17, 5, 64, 6
    S = np.asfortranarray(crandn(rng, (nq, srank)))
    X = crandn(rng, (nvox * nq * batch,))
    out = np.zeros(srank * nvox * batch, dtype=np.complex64)
    llr_b200.dti_project(S, X, out, batch, nq, nvox, srank)
    exp = O.dti_project(S.astype(np.complex128), X.astype(np.complex128), batch, nq, nvox, srank)
    assert rel_err(out, exp) < 1e-6
    Xb = np.zeros_like(X)
    comp = crandn(rng, (srank * nvox * batch,))
    llr_b200.dti_back_project(S, Xb, comp, batch, nq, nvox, srank)
    expb = O.dti_back_project(S.astype(np.complex128), comp.astype(np.complex128), batch, nq, nvox, srank)
    assert rel_err(Xb, expb) < 1e-6


def test_identity_subspace_round_trip(gpu):
    """dti_subspace.rs:238-261 through the fused subspace prox with rank = srank (identity)."""
    nq, srank, m, batch = 3, 3, 100, 10
    S = np.eye(nq, srank, dtype=np.complex64)
    X = np.zeros((m, nq, batch), dtype=np.complex64)
    for i in range(m):
        for j in range(nq):
            X[i, j, :] = i + j
    dS, dX = DeviceBuffer.from_array(np.asfortranarray(S)), DeviceBuffer.from_array(np.asfortranarray(X))
    L.check(L.lib.llr_subspace_low_rank_batch_dev(m, nq, srank, L.LLR_PROX_HARD_RANK, srank, 0.0, dS.ptr, batch,
                                                  dX.ptr, None))
    got = dX.download(np.empty_like(X, order="F"))
    assert rel_err(got, X) < 1e-6


@pytest.mark.parametrize("mode", ["hard", "soft"])
def test_subspace_low_rank_matches_oracle(gpu, mode):
    rng = np.random.default_rng(16)
    m, nq, srank, batch, rank = 512, 61, 7, 5, 3
    Q, _ = np.linalg.qr(crandn(rng, (nq, srank)).astype(np.complex128))
    S = np.asfortranarray(Q.astype(np.complex64))
    X = np.asfortranarray(crandn(rng, (m, nq, batch)))
    lam = 20.0
    dS, dX = DeviceBuffer.from_array(S), DeviceBuffer.from_array(X)
    L.check(L.lib.llr_subspace_low_rank_batch_dev(m, nq, srank, L.LLR_PROX_HARD_RANK if mode == "hard" else
                                                  L.LLR_PROX_SOFT_THRESH, rank, lam, dS.ptr, batch, dX.ptr, None))
    got = dX.download(np.empty_like(X, order="F"))
    exp = O.subspace_low_rank(X.astype(np.complex128), S.astype(np.complex128), mode, rank, lam)
    assert rel_err(got, exp) < 5e-5


def test_dwt_axis_reconstructs_ijk(gpu):
    """cudwt3.rs:18-93 on the device: single-level DWT -> IDWT of i+j+k, every axis."""
    n = 48
    vol = (n, n, n)
    i, j, k = np.meshgrid(*[np.arange(n)] * 3, indexing="ij")
    v = np.asfortranarray((i + j + k).astype(np.complex64))
    lo_d, hi_d, lo_r, hi_r = llr_b200.daubechies_filters(2)
    F = 4
    nc = O.sub_band_size(n, F)
    filt = [DeviceBuffer.from_array(f) for f in (lo_d, hi_d, lo_r, hi_r)]
    for axis in range(3):
        ds = list(vol)
        ds[axis] = 2 * nc
        dv = DeviceBuffer.from_array(v)
        dd = DeviceBuffer(int(np.prod(ds)) * 8)
        L.check(L.lib.llr_dwt3_axis_dev(dv.ptr, dd.ptr, L.u32x3(vol), L.u32x3(ds), axis, F, filt[0].ptr, filt[1].ptr,
                                        L.i32x3((0, 0, 0)), None))
        dec = dd.download(np.empty(ds, dtype=np.complex64, order="F"))
        exp = O.dwt_axis(v.astype(np.complex128), axis, O.daubechies_bank(2).lo_d, O.daubechies_bank(2).hi_d)
        assert rel_err(dec, exp) < 1e-6
        L.check(L.lib.llr_idwt3_axis_dev(dv.ptr, dd.ptr, L.u32x3(vol), L.u32x3(ds), axis, F, filt[2].ptr,
                                         filt[3].ptr, L.i32x3((0, 0, 0)), None))
        L.check(L.lib.llr_stream_sync(None))
        r = dv.download(np.empty(vol, dtype=np.complex64, order="F"))
        np.testing.assert_array_equal(np.round(r.real), v.real)


def test_reference_dwt_symbols_round_trip_and_shift(gpu):
    """dwt3_axis / idwt3_axis with the reference's own C signatures (kernels.cu:273,312 as
    cudwt3.rs:97-100 binds them: host sizes, device filters and device shift pointer):
    the i+j+k round trip of cudwt3.rs:18-93 on every axis, and a shifted analysis against the
    oracle with the shift applied per axis."""
    n = (40, 36, 32)
    i, j, k = np.meshgrid(*[np.arange(a) for a in n], indexing="ij")
    v = np.asfortranarray((i + j + k).astype(np.complex64))
    bank = O.daubechies_bank(2)
    F = 4
    filt = [DeviceBuffer.from_array(np.asarray(f, dtype=np.float32)) for f in llr_b200.daubechies_filters(2)]
    for shift in ((0, 0, 0), (5, -3, 7)):
        dsh = DeviceBuffer.from_array(np.asarray(shift, dtype=np.int32))
        vs = np.asarray(n, dtype=np.uint32)
        for axis in range(3):
            ds = np.asarray(n, dtype=np.uint32)
            ds[axis] = 2 * O.sub_band_size(n[axis], F)
            dv = DeviceBuffer.from_array(v)
            dd = DeviceBuffer(int(np.prod(ds)) * 8)
            e = L.lib.dwt3_axis(dv.ptr, dd.ptr, vs.ctypes.data_as(L.PU32), ds.ctypes.data_as(L.PU32), axis, F,
                                filt[0].ptr, filt[1].ptr, dsh.ptr)
            assert e == 0
            dec = dd.download(np.empty(tuple(ds), dtype=np.complex64, order="F"))
            src = np.roll(v.astype(np.complex128), [-s for s in shift], axis=(0, 1, 2))
            exp = O.dwt_axis(src, axis, bank.lo_d, bank.hi_d)
            assert rel_err(dec, exp) < 1e-6, (shift, axis)
            dv2 = DeviceBuffer(v.nbytes)
            e = L.lib.idwt3_axis(dv2.ptr, dd.ptr, vs.ctypes.data_as(L.PU32), ds.ctypes.data_as(L.PU32), axis, F,
                                 filt[2].ptr, filt[3].ptr, dsh.ptr)
            assert e == 0
            r = dv2.download(np.empty(n, dtype=np.complex64, order="F"))
            np.testing.assert_array_equal(np.round(r.real), v.real)
    bad = np.asarray(n, dtype=np.uint32)
    assert L.lib.dwt3_axis(dv.ptr, dd.ptr, bad.ctypes.data_as(L.PU32), bad.ctypes.data_as(L.PU32), 0, F,
                           filt[0].ptr, filt[1].ptr, dsh.ptr) != 0   # decomposition extent too small


def test_cu_dwt_denoise_round_trip(gpu):
    """cu_dwt_denoise (cudwt3.rs:102-247): analysis + synthesis without shrink is the identity."""
    rng = np.random.default_rng(17)
    vol = (40, 36, 28)
    x = np.asfortranarray(crandn(rng, vol))
    lo_d, hi_d, lo_r, hi_r = llr_b200.daubechies_filters(2)
    buf = x.reshape(-1, order="F").copy()
    llr_b200.cu_dwt_denoise(buf, vol, lo_d, hi_d, lo_r, hi_r, (0, 0, 0))
    assert rel_err(buf, x.reshape(-1, order="F")) < 2e-6


@pytest.mark.parametrize("vol,moments,levels", [((32, 32, 32), 2, 0), ((40, 36, 28), 4, 2), ((33, 30, 26), 2, 2),
                                                 ((70, 50, 45), 4, 3), ((24, 20, 18), 1, 2), ((40, 40, 40), 8, 1)])
def test_wavelet_denoise_matches_oracle(gpu, vol, moments, levels):
    rng = np.random.default_rng(18)
    nvol = 2
    x = np.asfortranarray(crandn(rng, vol + (nvol,)))
    alpha = 0.8
    d = DeviceBuffer.from_array(x)
    L.check(L.lib.llr_wavelet_denoise_dev(d.ptr, L.i32x3(vol), nvol, moments, levels, alpha, None))
    got = d.download(np.empty_like(x, order="F"))
    bank = O.daubechies_bank(moments)
    exp = np.stack([O.wavelet_denoise(x[..., v].astype(np.complex128), alpha, bank, levels) for v in range(nvol)], -1)
    assert rel_err(got, exp) < 5e-5


def test_hard_project_matches_reference(gpu):
    """lib.rs:392-406: replace where y != 0 and return sum |x - y|^2."""
    rng = np.random.default_rng(19)
    n = 100_000
    x = crandn(rng, (n,))
    y = crandn(rng, (n,))
    y[rng.random(n) < 0.6] = 0
    dx, dy = DeviceBuffer.from_array(x), DeviceBuffer.from_array(y)
    import ctypes as C
    err = C.c_double()
    L.check(L.lib.llr_hard_project_dev(dx.ptr, dy.ptr, n, C.byref(err), None))
    got = dx.download(np.empty_like(x, order="F"))
    exp, e = O.hard_project(x, y)
    np.testing.assert_array_equal(got, exp)
    assert abs(err.value - e) <= 1e-6 * e


def test_near_threshold_gains_refined(gpu):
    """Singular values within 0.2 % of the threshold next to a dominant one (sigma_1 = 40 lambda):
    the Gram eigenvalues carry an absolute error ~ eps sigma_1^2, the refinement sweep takes the
    gains from ||C v||^2 with FP64 accumulation.  The output restricted to the near-threshold
    singular vectors must match the FP64 oracle to 1e-4 lambda."""
    rng = np.random.default_rng(31)
    m, n, lam = 216, 61, 1.0
    sig = []
    for k in range(12):
        s = [40.0, 1.0 + 2e-3, 1.0 - 2e-3, 1.0 + 5e-4] + list(rng.uniform(0.05, 0.6, n - 4))
        sig.append(s)
    A = _spectrum_blocks(rng, m, n, sig).astype(np.complex64)
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, lam, A.shape[2], d.ptr, None))
    got = d.download(np.empty_like(A, order="F")).astype(np.complex128)
    A64 = A.astype(np.complex128)
    exp = O.low_rank_soft(A64, lam)
    for b in range(A.shape[2]):
        _, s, Vh = np.linalg.svd(A64[:, :, b], full_matrices=False)
        near = Vh[1:4].conj().T                      # right singular vectors at 1 +- 2e-3, 1 + 5e-4
        err = np.linalg.norm((got[:, :, b] - exp[:, :, b]) @ near)
        assert err < 1e-4 * lam, (b, err, s[:4])


def test_near_threshold_vector_error_bounded(gpu):
    """The refinement sweep fixes gains, not vectors: the eigenvectors still come from the FP32-level
    Gram, whose eigenvalues carry an absolute error ~ eps sigma_1^2.  Bound what that leaves, on the
    construction above (sigma_1 = 40 lambda beside singular values within 0.2 % of lambda):
    * the whole output, not only its projection on the near-threshold vectors: ||C' - C'_64||_F
      <= 2e-4 lambda per block;
    * the dominant right singular vector (gap sigma_1^2 - 1 ~ 1600 lambda^2, so its perturbation is
      ~ eps): sin of its angle to the FP64 one <= 1e-5;
    * the near-threshold vectors may turn inside their cluster by ~ eps sigma_1^2 / gap (gap ~ 3e-3
      lambda^2 here, a few per cent), but not out of it: the output's component outside the span of
      the FP64 kept vectors (sigma > lambda) is <= 2e-4 lambda."""
    rng = np.random.default_rng(37)
    m, n, lam = 216, 61, 1.0
    sig = [[40.0, 1.0 + 2e-3, 1.0 - 2e-3, 1.0 + 5e-4] + list(rng.uniform(0.05, 0.6, n - 4)) for _ in range(12)]
    A = _spectrum_blocks(rng, m, n, sig).astype(np.complex64)
    d = DeviceBuffer.from_array(A)
    L.check(L.lib.llr_soft_threshold_batch_dev(m, n, lam, A.shape[2], d.ptr, None))
    got = d.download(np.empty_like(A, order="F")).astype(np.complex128)
    A64 = A.astype(np.complex128)
    exp = O.low_rank_soft(A64, lam)
    worst = [0.0, 0.0, 0.0]
    for b in range(A.shape[2]):
        _, s, Vh = np.linalg.svd(A64[:, :, b], full_matrices=False)
        full = np.linalg.norm(got[:, :, b] - exp[:, :, b])
        _, _, Vg = np.linalg.svd(got[:, :, b], full_matrices=False)
        sin1 = np.sqrt(max(0.0, 1.0 - abs(np.vdot(Vh[0], Vg[0])) ** 2))
        kept = Vh[s > lam].conj().T                  # FP64 kept right singular vectors
        outside = np.linalg.norm(got[:, :, b] - got[:, :, b] @ kept @ kept.conj().T)
        worst = [max(worst[0], full), max(worst[1], sin1), max(worst[2], outside)]
    print(f"near-threshold blocks: max ||C' - C'_64||_F {worst[0]:.2e} lambda, max sin(v1) {worst[1]:.2e}, "
          f"max component outside the kept span {worst[2]:.2e} lambda")
    assert worst[0] <= 2e-4 * lam, worst
    assert worst[1] <= 1e-5, worst
    assert worst[2] <= 2e-4 * lam, worst


def test_subspace_construction_matches_oracle(gpu):
    """GPU temporal subspace (simulated signals, FP64 Gram, FP64 Jacobi) against the oracle's
    restatement with the same counter-based draws: the same subspace and singular values."""
    from llr_b200.phantom import b_table, dti_subspace_gpu
    b, g = b_table([(0, 1), (1000, 30), (2000, 30)], np.random.default_rng(3))
    S, sv = dti_subspace_gpu(b, g, 7, 20000, 5)
    f32 = lambda v: np.float64(np.float32(v))              # the ABI takes the b-table and ranges in FP32
    Se, sve = O.dti_subspace_counter(b.astype(np.float32), g.astype(np.float32), 7, 20000, 5, f32(0.1e-3), f32(3.0e-3))
    np.testing.assert_allclose(sv, sve, rtol=1e-9)
    assert np.abs(S.imag).max() == 0
    P, Pe = S.astype(np.complex128) @ S.conj().T.astype(np.complex128), Se @ Se.conj().T
    assert np.linalg.norm(P - Pe) < 1e-6
    np.testing.assert_allclose(S.real, Se.real, atol=1e-6)   # same sign convention
