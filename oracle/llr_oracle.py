"""CPU oracle for the llr-reco LLR reconstruction hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  Nothing in the product library routes through it.

It restates, in numpy (complex128 by default, complex64 on request), the algorithm of
wyatt-A/llr-reco.  Every function cites the reference file:line it follows.  Array
conventions follow the reference: volumes are ``(nx, ny, nz, nq)`` arrays addressed
column-major with x fastest (``array_utils.rs:4-17``); Casorati batches are
``(m, n, batch)`` column-major (``block.rs:147-164``).

Parity status: the reference cannot be built here (Rust toolchain and its unvendored
``dwt``/``cfl`` git crates are absent).  The oracle is pinned against every known-answer
test the reference holds for this path (see ``tests/test_oracle_kat.py``): the CGEMM
4x4 matrix (``low_rank.rs:149-179``), the diagonal scale (``cublas.rs:158-181``), the FFT
round trip of ones (``cufft.rs:415-421``), the single-level DWT perfect reconstruction
(``cudwt3.rs:18-93``), the lift/un-lift identity (``block.rs:285-343``), the identity
subspace round trip (``dti_subspace.rs:238-261``) and the periodic wrap
(``fftshift.rs:127-134``).  The multi-level wavelet shrink lives in the unpinned ``dwt``
crate and is restated from the filter-bank definition in ``kernels.cu:155-268``; its
parity is unpinned beyond perfect reconstruction.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

MASK64 = (1 << 64) - 1
GOLDEN64 = 0x9E3779B97F4A7C15


# ----------------------------------------------------------------------------------------
# counter-based RNG (replaces the unseeded rand::rng() of lib.rs:420-427)
# ----------------------------------------------------------------------------------------
def splitmix64(x: int) -> int:
    """SplitMix64 finaliser (Steele, Lea & Flood 2014) on a 64-bit counter."""
    z = (x + GOLDEN64) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def rng_u64(seed: int, stream: int, index: int) -> int:
    """Keyed draw: one SplitMix64 step of ``seed`` advanced by (stream, index)."""
    return splitmix64((seed + GOLDEN64 * ((stream << 32) + index + 1)) & MASK64)


SHIFT_STREAM = 0x5348  # "SH"


def rand_shift(seed: int, iteration: int, max_shift: Sequence[int]) -> list[int]:
    """Uniform shift in [0, max_a) per axis for one iteration.

    Follows ``rand_shift`` (lib.rs:420-427) with the unseeded thread RNG replaced by a
    counter-based draw keyed by (seed, iteration, axis), so that the GPU path and this
    oracle produce bit-identical shift sequences.
    """
    return [int(rng_u64(seed, SHIFT_STREAM, 3 * iteration + a) % int(max_shift[a])) for a in range(3)]


# ----------------------------------------------------------------------------------------
# index helpers (array_utils.rs:4-17, block.rs:112-133, fftshift.rs:257-276)
# ----------------------------------------------------------------------------------------
def index_to_subscript_col_maj3(index: int, size: Sequence[int]) -> list[int]:
    """array_utils.rs:4-10."""
    iz = index // (size[0] * size[1])
    rem = index % (size[0] * size[1])
    return [rem % size[0], rem // size[0], iz]


def coord_to_col_maj_index(coords: Sequence[int], dims: Sequence[int]) -> int:
    """fftshift.rs:257-267 (Euclidean wrap per axis)."""
    idx, stride = 0, 1
    for c, d in zip(coords, dims):
        idx += (c % d) * stride
        stride *= d
    return idx


def col_maj_index_to_coord(idx: int, dims: Sequence[int]) -> list[int]:
    """fftshift.rs:269-276."""
    out = []
    for d in dims:
        out.append(idx % d)
        idx //= d
    return out


def grid_dim(vol_size: Sequence[int], block_size: Sequence[int]) -> list[int]:
    """block.rs:112-118: floor(vol/block) blocks per axis."""
    return [int(v) // int(b) for v, b in zip(vol_size, block_size)]


def block_coord(block_idx: int, vol_size, block_size, shift, stride=None) -> list[int]:
    """block.rs:122-133: lower corner of block ``block_idx`` (col-major grid) plus shift.

    ``stride`` generalises the non-overlapping grid (stride == block size, the reference)
    to overlapping blocks.
    """
    stride = list(block_size) if stride is None else list(stride)
    g = grid_dim_strided(vol_size, block_size, stride)
    ix, iy, iz = index_to_subscript_col_maj3(block_idx, g)
    return [ix * stride[0] + shift[0], iy * stride[1] + shift[1], iz * stride[2] + shift[2]]


def grid_dim_strided(vol_size, block_size, stride) -> list[int]:
    """Blocks per axis for a stride-s grid; equals grid_dim when stride == block size."""
    if list(stride) == list(block_size):
        return grid_dim(vol_size, block_size)
    return [int(v) // int(s) for v, s in zip(vol_size, stride)]


def _block_voxel_index(vol_size, block_size, corner) -> np.ndarray:
    """Linear voxel addresses of one block, in block col-major order (block.rs:8-28)."""
    bx, by, bz = block_size
    ix = (np.arange(bx) + corner[0]) % vol_size[0]
    iy = (np.arange(by) + corner[1]) % vol_size[1]
    iz = (np.arange(bz) + corner[2]) % vol_size[2]
    # r = ix + bx*(iy + by*iz)  -> x fastest
    lin = ix[:, None, None] + vol_size[0] * (iy[None, :, None] + vol_size[1] * iz[None, None, :])
    return lin.reshape(-1, order="F")


def lift_data_set(x: np.ndarray, block_size, shift, start: int, n: int, stride=None) -> np.ndarray:
    """block.rs:147-164 (+ read_matrix :64-84, _read_block_unchecked :8-28).

    Gather ``n`` blocks starting at block index ``start`` into a column-major Casorati
    batch ``(m, nq, n)``: ``C[r, q, j] = x_q[wrap(corner_j + sub(r))]``.
    """
    nx, ny, nz, nq = x.shape
    vol = (nx, ny, nz)
    flat = x.reshape(nx * ny * nz, nq, order="F")
    m = int(np.prod(block_size))
    out = np.empty((m, nq, n), dtype=x.dtype)
    for c, i in enumerate(range(start, start + n)):
        corner = block_coord(i, vol, block_size, shift, stride)
        out[:, :, c] = flat[_block_voxel_index(vol, block_size, corner), :]
    return out


def un_lift_data_set(x: np.ndarray, mats: np.ndarray, block_size, shift, start: int, n: int) -> None:
    """block.rs:166-184 (+ write_matrix :86-109, _write_block_unchecked :33-62); in place."""
    nx, ny, nz, nq = x.shape
    vol = (nx, ny, nz)
    flat = x.reshape(nx * ny * nz, nq, order="F")  # view when x is F-contiguous
    assert np.shares_memory(flat, x), "un_lift_data_set needs an F-contiguous volume array"
    for c, i in enumerate(range(start, start + n)):
        corner = block_coord(i, vol, block_size, shift)
        flat[_block_voxel_index(vol, block_size, corner), :] = mats[:, :, c]


# ----------------------------------------------------------------------------------------
# signal model (signal_model.rs:34-117, cufft.rs:124-180, 269-337)
# ----------------------------------------------------------------------------------------
def calc_shift(linear_correction, image_size) -> list[float]:
    """signal_model.rs:110-117: s_a = corr_a + n_a/2."""
    return [float(c) + 0.5 * float(n) for c, n in zip(linear_correction, image_size)]


def phase_axis(n: int, shift_samples: float) -> np.ndarray:
    """cufft.rs:320-326: 2*pi*s*(i - n/2)/n for i in [0, n) (radians, float64)."""
    i = np.arange(n, dtype=np.float64)
    return (i - n / 2.0) * (2.0 * np.pi * shift_samples / n)


def phase_ramp3(dims, shift, sign: float) -> np.ndarray:
    """cufft.rs:290-304: exp(i*sign*sum_a phi_a) on a (nx, ny, nz) grid.

    ``sign`` is +1 for the reference's ``FftDirection::Inverse`` and -1 for ``Forward``.
    """
    px = phase_axis(dims[0], shift[0])
    py = phase_axis(dims[1], shift[1])
    pz = phase_axis(dims[2], shift[2])
    total = px[:, None, None] + py[None, :, None] + pz[None, None, :]
    return np.exp(1j * sign * total)


FORWARD, INVERSE = 0, 1


def fftn_unitary(x: np.ndarray, direction: int) -> np.ndarray:
    """cufft.rs:124-180 with NormalizationType::Unitary: 3-D C2C over axes 0..2, 1/sqrt(N)."""
    if direction == FORWARD:
        return np.fft.fftn(x, axes=(0, 1, 2), norm="ortho")
    return np.fft.ifftn(x, axes=(0, 1, 2), norm="ortho")


def signal_model(x: np.ndarray, lin_ksp, lin_img, direction: int) -> np.ndarray:
    """signal_model.rs:34-79 for a (nx, ny, nz, nq) batch; returns a new array.

    Forward:  x * e^{+i phi_ksp} -> unitary FFT -> * e^{-i phi_img}
    Inverse:  x * e^{+i phi_img} -> unitary IFFT -> * e^{-i phi_ksp}
    """
    nx, ny, nz, nq = x.shape
    dims = (nx, ny, nz)
    out = np.empty_like(x)
    for q in range(nq):
        if direction == FORWARD:
            pre = phase_ramp3(dims, calc_shift(lin_ksp[q], dims), +1.0)
            post = phase_ramp3(dims, calc_shift(lin_img[q], dims), -1.0)
        else:
            pre = phase_ramp3(dims, calc_shift(lin_img[q], dims), +1.0)
            post = phase_ramp3(dims, calc_shift(lin_ksp[q], dims), -1.0)
        v = x[..., q] * pre
        v = fftn_unitary(v, direction)
        out[..., q] = (v * post).astype(x.dtype)
    return out


def max_coord(vol: np.ndarray) -> list[int]:
    """cufft.rs:329-337: col-major coordinate of max |k|^2 (last index on ties)."""
    e = (np.abs(vol) ** 2).reshape(-1, order="F")
    mx = e.max()
    idx = int(np.flatnonzero(e == mx)[-1])
    return index_to_subscript_col_maj3(idx, vol.shape)


def estimate_linear_correction(ksp: np.ndarray) -> list[float]:
    """signal_model.rs:100-106: argmax |k|^2 minus (n+1)//2 per axis."""
    c = max_coord(ksp)
    return [float(c[a] - (ksp.shape[a] + 1) // 2) for a in range(3)]


def hard_project(x: np.ndarray, y: np.ndarray) -> tuple[np.ndarray, float]:
    """lib.rs:392-406: where y != 0 accumulate |x-y|^2 (f64) and set x := y."""
    nz_mask = y != 0
    d = (x - y)[nz_mask]
    err = float(np.sum(np.abs(d.astype(np.complex128)) ** 2))
    out = x.copy()
    out[nz_mask] = y[nz_mask]
    return out, err


def calc_undersampling_factor(y: np.ndarray) -> tuple[float, float]:
    """lib.rs:409-417: (numel / nnz, sum |y|^2)."""
    nnz = np.count_nonzero(y)
    return y.size / nnz, float(np.sum(np.abs(y.astype(np.complex128)) ** 2))


def under_sample_kspace(k: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """data_import.rs:416-438: zero the x-line k[:, ky, kz, q] where mask(ky, kz, q) == 0."""
    assert mask.shape == k.shape[1:]
    return k * (mask != 0)[None, :, :, :]


# ----------------------------------------------------------------------------------------
# low-rank prox (low_rank.rs:10-69, cusolver.rs:20-151, kernels.cu:11-67, cublas.rs:12-105)
# ----------------------------------------------------------------------------------------
def rhs_cdgmm_batched(mats: np.ndarray, diag: np.ndarray) -> np.ndarray:
    """kernels.cu:11-44: A[:, j, b] *= d[j, b] (complex times real)."""
    return mats * diag[None, :, :]


def cgemm_strided_batched(m, k, n, batch, broadcast_a, alpha, beta, transpose_a, transpose_b,
                          a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """cublas.rs:12-105: C = alpha*op(A)*op(B) + beta*C on flat column-major buffers.

    ``op`` is the conjugate transpose when the transpose flag is set; ``broadcast_a``
    sets A's batch stride to zero.  Returns the new flat C buffer.
    """
    lda_rows, lda_cols = (k, m) if transpose_a else (m, k)
    ldb_rows, ldb_cols = (n, k) if transpose_b else (k, n)
    sa = 0 if broadcast_a else m * k
    out = c.copy()
    for i in range(batch):
        A = a[i * sa:i * sa + lda_rows * lda_cols].reshape(lda_rows, lda_cols, order="F")
        B = b[i * k * n:(i + 1) * k * n].reshape(ldb_rows, ldb_cols, order="F")
        A = A.conj().T if transpose_a else A
        B = B.conj().T if transpose_b else B
        C = c[i * m * n:(i + 1) * m * n].reshape(m, n, order="F")
        out[i * m * n:(i + 1) * m * n] = (alpha * (A @ B) + beta * C).reshape(-1, order="F")
    return out


def low_rank_hard(mats: np.ndarray, rank: int) -> np.ndarray:
    """low_rank.rs:10-69: keep the top ``rank`` singular triplets, C <- U_r S_r V_r^H."""
    m, n, b = mats.shape
    A = np.moveaxis(mats, 2, 0).astype(np.complex128)
    U, s, Vh = np.linalg.svd(A, full_matrices=False)
    r = int(rank)
    out = (U[:, :, :r] * s[:, None, :r]) @ Vh[:, :r, :]
    return np.moveaxis(out, 0, 2).astype(mats.dtype)


def low_rank_soft(mats: np.ndarray, lam: float) -> np.ndarray:
    """Singular-value soft threshold C <- U max(S - lam, 0) V^H (the build's SOFT_THRESH mode).

    Same operator shape as low_rank.rs:10-69; only the singular-value map differs.
    """
    A = np.moveaxis(mats, 2, 0).astype(np.complex128)
    U, s, Vh = np.linalg.svd(A, full_matrices=False)
    s2 = np.maximum(s - lam, 0.0)
    out = (U * s2[:, None, :]) @ Vh
    return np.moveaxis(out, 0, 2).astype(mats.dtype)


def block_singular_values(mats: np.ndarray) -> np.ndarray:
    """Singular values of every Casorati matrix, shape (batch, min(m, n)) descending."""
    A = np.moveaxis(mats, 2, 0).astype(np.complex128)
    return np.linalg.svd(A, compute_uv=False)


# ----------------------------------------------------------------------------------------
# DTI subspace (dti_subspace.rs:141-221, lib.rs:281-289)
# ----------------------------------------------------------------------------------------
def conj_transpose_matrix(data: np.ndarray, m: int, n: int, batch: int) -> np.ndarray:
    """dti_subspace.rs:211-221 on a flat column-major buffer: (m x n) -> (n x m), conj."""
    out = np.empty_like(data)
    for i in range(batch):
        A = data[i * m * n:(i + 1) * m * n].reshape(m, n, order="F")
        out[i * m * n:(i + 1) * m * n] = A.conj().T.reshape(-1, order="F")
    return out


def dti_project(S: np.ndarray, X: np.ndarray, batch: int, nq: int, nvox: int, srank: int) -> np.ndarray:
    """dti_subspace.rs:141-166: flat (srank x nvox) per batch = S^H * X^H."""
    a = S.reshape(-1, order="F")
    c = np.zeros(nvox * srank * batch, dtype=X.dtype)
    return cgemm_strided_batched(srank, nq, nvox, batch, True, 1.0, 0.0, True, True, a, X, c)


def dti_back_project(S: np.ndarray, compressed: np.ndarray, batch: int, nq: int, nvox: int, srank: int) -> np.ndarray:
    """dti_subspace.rs:172-207: S * L^H then conj transpose -> flat (nvox x nq) per batch."""
    a = S.reshape(-1, order="F")
    c = np.zeros(nq * nvox * batch, dtype=compressed.dtype)
    out = cgemm_strided_batched(nq, srank, nvox, batch, True, 1.0, 0.0, False, False, a, compressed, c)
    return conj_transpose_matrix(out, nq, nvox, batch)


def subspace_low_rank(mats: np.ndarray, S: np.ndarray, mode: str, rank: int = 0, lam: float = 0.0) -> np.ndarray:
    """lib.rs:281-289: X <- LR(X S) S^H for each Casorati matrix X (m x nq)."""
    m, nq, b = mats.shape
    srank = S.shape[1]
    flat = mats.reshape(-1, order="F")
    comp = dti_project(S, flat, b, nq, m, srank)
    comp = conj_transpose_matrix(comp, srank, m, b)                # (m x srank) = X S
    z = comp.reshape(m, srank, b, order="F")
    z = low_rank_hard(z, rank) if mode == "hard" else low_rank_soft(z, lam)
    comp = conj_transpose_matrix(z.reshape(-1, order="F"), m, srank, b)
    out = dti_back_project(S, comp, b, nq, m, srank)
    return out.reshape(m, nq, b, order="F")


def subspace_constraint(S: np.ndarray, X: np.ndarray, batch: int, nq: int, nvox: int, srank: int) -> np.ndarray:
    """dti_subspace.rs:89-134 restated on matrices: X <- X S S^H per batch.

    (The reference stores its result through an explicit transpose loop; with an
    orthonormal or identity subspace the observable effect is the projection X S S^H.)
    """
    out = np.empty_like(X)
    for i in range(batch):
        A = X[i * nq * nvox:(i + 1) * nq * nvox].reshape(nvox, nq, order="F")
        out[i * nq * nvox:(i + 1) * nq * nvox] = (A @ S @ S.conj().T).reshape(-1, order="F")
    return out


# ----------------------------------------------------------------------------------------
# wavelets (kernels.cu:97-105, 150-268; lib.rs:430-465; dwt crate wavedec3/waverec3)
# ----------------------------------------------------------------------------------------
def daubechies_lowpass(n_moments: int) -> np.ndarray:
    """Daubechies minimum-phase scaling filter with ``n_moments`` vanishing moments.

    Spectral factorisation (Daubechies, Ten Lectures on Wavelets, 1992, sec. 6.1):
    P(y) = sum_k C(N-1+k, k) y^k, y = (2 - z - 1/z)/4; keep roots inside the unit circle.
    Returned in reconstruction order h[0..2N) with sum(h) = sqrt(2).
    """
    N = int(n_moments)
    if N == 1:
        return np.array([1.0, 1.0]) / math.sqrt(2.0)
    p = [math.comb(N - 1 + k, k) for k in range(N)]
    yroots = np.roots(p[::-1])
    zr = []
    for y in yroots:
        # z + 1/z = 2 - 4y  ->  z^2 - (2-4y) z + 1 = 0
        r = np.roots([1.0, -(2.0 - 4.0 * y), 1.0])
        zr.append(r[np.argmin(np.abs(r))])
    poly = np.array([1.0 + 0j])
    for _ in range(N):
        poly = np.convolve(poly, [1.0, 1.0])
    for z in zr:
        poly = np.convolve(poly, [1.0, -z])
    h = np.real(poly)
    h = h * (math.sqrt(2.0) / h.sum())
    return h


@dataclass
class FilterBank:
    lo_d: np.ndarray
    hi_d: np.ndarray
    lo_r: np.ndarray
    hi_r: np.ndarray

    @property
    def flen(self) -> int:
        return len(self.lo_d)


def daubechies_bank(n_moments: int) -> FilterBank:
    """Orthogonal analysis/synthesis bank in the pywt ordering that kernels.cu expects."""
    h = daubechies_lowpass(n_moments)
    F = len(h)
    lo_r = h.copy()
    hi_r = np.array([(-1.0) ** k * h[F - 1 - k] for k in range(F)])
    return FilterBank(lo_d=lo_r[::-1].copy(), hi_d=hi_r[::-1].copy(), lo_r=lo_r, hi_r=hi_r)


def sub_band_size(n: int, flen: int) -> int:
    """kernels.cu:150-152."""
    return (int(n) + int(flen) - 1) // 2


def w_max_level(n: int, flen: int) -> int:
    """Maximum useful decomposition level floor(log2(n / (F - 1))) (dwt crate, lib.rs:441)."""
    if flen <= 1 or n < flen - 1:
        return 0
    return int(math.floor(math.log2(n / (flen - 1))))


def _sym_index(idx: np.ndarray, n: int) -> np.ndarray:
    """kernels.cu:97-105 half-sample symmetric extension."""
    idx = np.where(idx < 0, -idx - 1, idx)
    idx = np.where(idx >= n, 2 * n - idx - 1, idx)
    return idx


def dwt_axis(x: np.ndarray, axis: int, lo_d: np.ndarray, hi_d: np.ndarray) -> np.ndarray:
    """kernels.cu:155-212: one-level analysis along ``axis``; output [a | d] of 2*nc."""
    F = len(lo_d)
    n = x.shape[axis]
    nc = sub_band_size(n, F)
    xm = np.moveaxis(x, axis, 0)
    c = np.arange(nc)
    a = np.zeros((nc,) + xm.shape[1:], dtype=np.result_type(x.dtype, np.float64))
    d = np.zeros_like(a)
    for j in range(F):
        src = _sym_index(2 * c - F + 2 + j, n)
        a += lo_d[F - 1 - j] * xm[src]
        d += hi_d[F - 1 - j] * xm[src]
    out = np.concatenate([a, d], axis=0).astype(x.dtype)
    return np.moveaxis(out, 0, axis)


def idwt_axis(dec: np.ndarray, axis: int, lo_r: np.ndarray, hi_r: np.ndarray, n_out: int) -> np.ndarray:
    """kernels.cu:215-268: one-level synthesis along ``axis`` keeping ``n_out`` samples."""
    F = len(lo_r)
    dm = np.moveaxis(dec, axis, 0)
    nc = dm.shape[0] // 2
    a, d = dm[:nc], dm[nc:]
    full_len = 2 * nc + F - 1
    keep_len = 2 * nc - F + 2
    start = (full_len - keep_len) // 2
    out = np.zeros((n_out,) + dm.shape[1:], dtype=np.result_type(dec.dtype, np.float64))
    s = np.arange(n_out)
    for j in range(F):
        idx = start + s - j
        ok = (idx >= 0) & (idx < 2 * nc) & (idx % 2 == 0)
        h = np.where(ok, idx // 2, 0)
        term = lo_r[j] * a[h] + hi_r[j] * d[h]
        term[~ok] = 0
        out += term
    return np.moveaxis(out.astype(dec.dtype), 0, axis)


def dwt3(x: np.ndarray, bank: FilterBank) -> np.ndarray:
    """cudwt3.rs:146-183: analysis along axis 0, 1, 2 -> (2ncx, 2ncy, 2ncz)."""
    for ax in range(3):
        x = dwt_axis(x, ax, bank.lo_d, bank.hi_d)
    return x


def idwt3(dec: np.ndarray, bank: FilterBank, out_shape) -> np.ndarray:
    """cudwt3.rs:185-219: synthesis along axis 2, 1, 0 down to ``out_shape``."""
    for ax in (2, 1, 0):
        dec = idwt_axis(dec, ax, bank.lo_r, bank.hi_r, out_shape[ax])
    return dec


def wavedec3(x: np.ndarray, bank: FilterBank, levels: int) -> list[np.ndarray]:
    """Multi-level 3-D decomposition (dwt crate ``wavedec3``, call site lib.rs:444).

    Returns one decomposition array per level (finest first).  Level l+1 decomposes the
    approximation corner of level l.
    """
    decs = []
    cur = x
    for _ in range(levels):
        dec = dwt3(cur, bank)
        decs.append(dec)
        nc = [s // 2 for s in dec.shape]
        cur = dec[:nc[0], :nc[1], :nc[2]]
    return decs


def waverec3(decs: list[np.ndarray], bank: FilterBank, out_shape) -> np.ndarray:
    """Inverse of :func:`wavedec3` (dwt crate ``waverec3``, call site lib.rs:454)."""
    shapes = [tuple(out_shape)] + [tuple(s // 2 for s in d.shape) for d in decs[:-1]]
    rec = None
    for lvl in range(len(decs) - 1, -1, -1):
        dec = decs[lvl].copy()
        if rec is not None:
            nc = [s // 2 for s in dec.shape]
            dec[:nc[0], :nc[1], :nc[2]] = rec
        rec = idwt3(dec, bank, shapes[lvl])
    return rec


def shrink_complex(x: np.ndarray, alpha: float) -> np.ndarray:
    """lib.rs:460-465: c * max(|c| - alpha, 0) / |c|, with 0 -> 0 (the reference yields NaN)."""
    m = np.abs(x)
    with np.errstate(divide="ignore", invalid="ignore"):
        f = np.where(m > 0, np.maximum(m - alpha, 0.0) / np.where(m > 0, m, 1.0), 0.0)
    return (x * f).astype(x.dtype)


def wavelet_denoise(vol: np.ndarray, alpha: float, bank: FilterBank, levels: Optional[int] = None) -> np.ndarray:
    """lib.rs:430-458: wavedec3 -> shrink every sub-band -> waverec3 for one volume."""
    if levels is None or levels <= 0:
        levels = w_max_level(min(vol.shape), bank.flen)
    if levels == 0:
        return shrink_complex(vol, alpha)
    decs = wavedec3(vol, bank, levels)
    # Shrink: every level's detail sub-bands once, and the final approximation once.
    shrunk = []
    for lvl, d in enumerate(decs):
        s = shrink_complex(d, alpha)
        if lvl < len(decs) - 1:
            nc = [t // 2 for t in d.shape]
            s[:nc[0], :nc[1], :nc[2]] = d[:nc[0], :nc[1], :nc[2]]
        shrunk.append(s)
    return waverec3(shrunk, bank, vol.shape)


# ----------------------------------------------------------------------------------------
# synthetic variable-density mask (bit-exact twin of llr_vd_mask in the C ABI)
# ----------------------------------------------------------------------------------------
MASK_STREAM = 0x4D41  # "MA"


def vd_mask(ny: int, nz: int, nq: int, accel: float, centre: int, seed: int) -> np.ndarray:
    """Variable-density random ky-kz mask, one per volume, uint8 (ny, nz, nq).

    The ``centre`` x ``centre`` block around (ny/2, nz/2) is always sampled.  Other points
    are kept with probability min(1, a*w(r)), w = (1 - min(r, 1))^2 + 0.02 where r is the
    normalised radius; ``a`` is found by bisection so the expected count equals
    ny*nz/accel.  Probabilities are quantised to 32-bit fixed point and the sampling test
    is integer, so the C implementation reproduces this bit for bit.
    """
    cy, cz = ny // 2, nz // 2
    ky = np.arange(ny, dtype=np.float64)
    kz = np.arange(nz, dtype=np.float64)
    dy = (ky - cy) / (ny / 2.0)
    dz = (kz - cz) / (nz / 2.0)
    w = np.empty((ny, nz))
    for j in range(ny):
        for k in range(nz):
            r = math.sqrt(dy[j] * dy[j] + dz[k] * dz[k])
            t = 1.0 - (r if r < 1.0 else 1.0)
            w[j, k] = t * t + 0.02
    h0 = centre // 2
    inc = np.zeros((ny, nz), dtype=bool)
    inc[max(cy - h0, 0):min(cy - h0 + centre, ny), max(cz - h0, 0):min(cz - h0 + centre, nz)] = True
    target = int(round(ny * nz / float(accel)))
    rest = max(target - int(inc.sum()), 0)
    TWO32 = 4294967296.0

    def quant(a: float) -> np.ndarray:
        qv = np.zeros((ny, nz), dtype=np.uint64)
        for j in range(ny):
            for k in range(nz):
                if inc[j, k]:
                    continue
                p = a * w[j, k]
                p = 1.0 if p > 1.0 else p
                qv[j, k] = int(math.floor(p * TWO32))
        return qv

    lo, hi = 0.0, 1.0
    while int(quant(hi).sum()) < rest * (1 << 32) and hi < 1e12:
        hi *= 2.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if int(quant(mid).sum()) < rest * (1 << 32):
            lo = mid
        else:
            hi = mid
    qv = quant(hi)
    out = np.zeros((ny, nz, nq), dtype=np.uint8)
    for q in range(nq):
        for k in range(nz):
            for j in range(ny):
                if inc[j, k]:
                    out[j, k, q] = 1
                    continue
                u = rng_u64(seed, MASK_STREAM + (q << 8), j + ny * k) >> 32
                out[j, k, q] = 1 if u < int(qv[j, k]) else 0
    return out


# ----------------------------------------------------------------------------------------
# prox, iteration and recon (lib.rs:113-363)
# ----------------------------------------------------------------------------------------
@dataclass
class ReconConfig:
    block_size: tuple = (8, 8, 8)
    mode: str = "soft"           # "soft" (north-star objective) | "hard" (reference gesvda)
    rank: int = 6
    lam: float = 0.0             # absolute singular-value threshold for "soft"
    wavelet_alpha: float = 0.0
    wavelet_moments: int = 2     # db2 (reference) / db4
    wavelet_levels: int = 0      # 0 -> w_max_level (reference)
    max_rand_shift: Optional[tuple] = None  # None -> vol size (lib.rs:260)
    seed: int = 0
    subspace: Optional[np.ndarray] = None
    lin_ksp: Optional[np.ndarray] = None
    lin_img: Optional[np.ndarray] = None
    wavelet_space: str = "image"  # with a subspace: "image" (lib.rs:302-309) | "coeffs" (srank volumes)
    block_stride: Optional[tuple] = None   # None / == block size: non-overlapping grid (block.rs:112-133)


def llr_prox_coeffs(x: np.ndarray, cfg: ReconConfig, shift) -> np.ndarray:
    """The subspace prox of lib.rs:281-289 stopped before the back-projection: the coefficient
    volumes LR(X S) (nx, ny, nz, srank), blocks un-lifted into them (the blocks tile the volume)."""
    nx, ny, nz, nq = x.shape
    S = np.asarray(cfg.subspace)
    nb = int(np.prod(grid_dim((nx, ny, nz), cfg.block_size)))
    mats = lift_data_set(np.asfortranarray(x), cfg.block_size, shift, 0, nb)
    Z = np.einsum("mqb,qk->mkb", mats, S)
    Z = low_rank_hard(Z, cfg.rank) if cfg.mode == "hard" else low_rank_soft(Z, cfg.lam)
    out = np.zeros((nx, ny, nz, S.shape[1]), dtype=np.result_type(x.dtype, S.dtype), order="F")
    un_lift_data_set(out, Z, cfg.block_size, shift, 0, nb)
    return out


def llr_prox(x: np.ndarray, cfg: ReconConfig, shift) -> np.ndarray:
    """lib.rs:270-296: lift every block, low-rank it, un-lift.

    With ``cfg.block_stride`` s < b (overlapping blocks every s voxels, b % s == 0, the blocks
    tiling the volume) every voxel becomes the mean of the outputs of the (b/s)^3 blocks that
    cover it: the strided grid splits into (b/s)^3 non-overlapping tilings, at the shift plus an
    offset in {0, s, ..., b - s} per axis, and the result is the mean of their prox outputs."""
    bs = tuple(cfg.block_size)
    st = tuple(cfg.block_stride) if cfg.block_stride is not None else bs
    if st != bs:
        per = [b // s if 0 < s < b else 1 for b, s in zip(bs, st)]
        offs = [[k * s for k in range(p)] if p > 1 else [0] for p, s in zip(per, st)]
        acc = np.zeros_like(x)
        for oz in offs[2]:
            for oy in offs[1]:
                for ox in offs[0]:
                    acc += _llr_prox_tiling(x, cfg, (shift[0] + ox, shift[1] + oy, shift[2] + oz))
        return np.asfortranarray(acc / float(np.prod(per)))
    return _llr_prox_tiling(x, cfg, shift)


def _llr_prox_tiling(x: np.ndarray, cfg: ReconConfig, shift) -> np.ndarray:
    """One non-overlapping tiling at ``shift`` (the reference's grid)."""
    nx, ny, nz, nq = x.shape
    g = grid_dim((nx, ny, nz), cfg.block_size)
    nb = int(np.prod(g))
    out = np.asfortranarray(x.copy())
    if nb == 0:
        return out
    mats = lift_data_set(out, cfg.block_size, shift, 0, nb)
    if cfg.subspace is not None:
        mats = subspace_low_rank(mats, cfg.subspace, cfg.mode, cfg.rank, cfg.lam)
    elif cfg.mode == "hard":
        mats = low_rank_hard(mats, cfg.rank)
    else:
        mats = low_rank_soft(mats, cfg.lam)
    un_lift_data_set(out, mats, cfg.block_size, shift, 0, nb)
    return out


def _corrections(cfg: ReconConfig, nq: int):
    z = np.zeros((nq, 3))
    ksp = z if cfg.lin_ksp is None else np.asarray(cfg.lin_ksp, dtype=np.float64)
    img = z if cfg.lin_img is None else np.asarray(cfg.lin_img, dtype=np.float64)
    return ksp, img


def iterate(x: np.ndarray, y: np.ndarray, cfg: ReconConfig, it: int):
    """One pass of lib.rs:262-341: LLR -> wavelet -> A -> hard DC -> A^H.

    Returns (x_next, sum_sq_error).
    """
    nx, ny, nz, nq = x.shape
    maxs = cfg.max_rand_shift or (nx, ny, nz)
    shift = rand_shift(cfg.seed, it, maxs)
    coeffs = cfg.subspace is not None and cfg.wavelet_alpha > 0 and cfg.wavelet_space == "coeffs"
    if coeffs:
        # shrink in the subspace coefficient domain, then X = C S^H
        c = llr_prox_coeffs(x, cfg, shift)
        bank = daubechies_bank(cfg.wavelet_moments)
        for k in range(c.shape[3]):
            c[..., k] = wavelet_denoise(c[..., k], cfg.wavelet_alpha, bank, cfg.wavelet_levels)
        z = np.asfortranarray(np.einsum("xyzk,qk->xyzq", c, np.conj(cfg.subspace)))
    else:
        z = llr_prox(x, cfg, shift)
    if cfg.wavelet_alpha > 0 and not coeffs:
        bank = daubechies_bank(cfg.wavelet_moments)
        for q in range(nq):
            z[..., q] = wavelet_denoise(z[..., q], cfg.wavelet_alpha, bank, cfg.wavelet_levels)
    ksp, img = _corrections(cfg, nq)
    k = signal_model(z, ksp, img, FORWARD)
    k, err = hard_project(k, y)
    xn = signal_model(k, ksp, img, INVERSE)
    return np.asfortranarray(xn), err


def objective(z: np.ndarray, err: float, cfg: ReconConfig, shift) -> float:
    """Objective of the prox output ``z`` of an iteration whose hard DC measured ``err`` =
    ||M A z - y||^2: 0.5 err + lam sum_b ||Z_b||_* over the tiling at ``shift`` (soft threshold;
    hard rank: 0.5 err).  Proximal gradient with step 1 (A unitary, lib.rs:262-341) minimises
    this function; with a fixed tiling it decreases every iteration."""
    if cfg.mode == "hard":
        return 0.5 * err
    nx, ny, nz, nq = z.shape
    nb = int(np.prod(grid_dim((nx, ny, nz), cfg.block_size)))
    if nb == 0:
        return 0.5 * err
    mats = lift_data_set(np.asfortranarray(z), cfg.block_size, shift, 0, nb)
    return 0.5 * err + cfg.lam * float(block_singular_values(mats).sum())


def recon_objective(y: np.ndarray, cfg: ReconConfig, n_iter: int, x0: Optional[np.ndarray] = None, it0: int = 0):
    """``recon`` that also returns the objective of every iteration's prox output (plain soft or
    hard LLR on one tiling: no wavelet, subspace or overlapping blocks)."""
    assert cfg.wavelet_alpha <= 0 and cfg.subspace is None
    assert cfg.block_stride is None or tuple(cfg.block_stride) == tuple(cfg.block_size)
    x = zero_filled(y, cfg) if x0 is None else np.asfortranarray(x0.copy())
    nx, ny, nz, nq = x.shape
    hist, obj = [], []
    for it in range(it0, it0 + n_iter):
        shift = rand_shift(cfg.seed, it, cfg.max_rand_shift or (nx, ny, nz))
        z = llr_prox(x, cfg, shift)
        ksp, img = _corrections(cfg, nq)
        k, err = hard_project(signal_model(z, ksp, img, FORWARD), y)
        obj.append(objective(z, err, cfg, shift))
        hist.append(err)
        x = np.asfortranarray(signal_model(k, ksp, img, INVERSE))
    return x, hist, obj


def zero_filled(y: np.ndarray, cfg: ReconConfig) -> np.ndarray:
    """lib.rs:233-242: x0 = A^H y."""
    ksp, img = _corrections(cfg, y.shape[3])
    return np.asfortranarray(signal_model(y, ksp, img, INVERSE))


def recon(y: np.ndarray, cfg: ReconConfig, n_iter: int, x0: Optional[np.ndarray] = None, it0: int = 0):
    """lib.rs:113-363 without file IO: returns (x, residual history)."""
    x = zero_filled(y, cfg) if x0 is None else np.asfortranarray(x0.copy())
    hist = []
    for it in range(it0, it0 + n_iter):
        x, err = iterate(x, y, cfg, it)
        hist.append(err)
    return x, hist


def sigma_max(x: np.ndarray, block_size, shift=(0, 0, 0)) -> float:
    """Largest singular value over every block of ``x`` at ``shift`` (FP64)."""
    nx, ny, nz, nq = x.shape
    nb = int(np.prod(grid_dim((nx, ny, nz), block_size)))
    mats = lift_data_set(np.asfortranarray(x), block_size, shift, 0, nb)
    return float(block_singular_values(mats)[:, 0].max())


def nrmse(x: np.ndarray, ref: np.ndarray) -> float:
    """||x - ref||_2 / ||ref||_2 over all volumes."""
    return float(np.linalg.norm((x - ref).ravel()) / np.linalg.norm(ref.ravel()))


# ---------------------------------------------------------------------------------------
# DTI scalar maps (diffusion_models.rs:21-129)
# ---------------------------------------------------------------------------------------
def dti_design_matrix(b: np.ndarray, g: np.ndarray) -> np.ndarray:
    """build_design_matrix (diffusion_models.rs:219-253): (nq, 6), columns -b gx^2, -b gy^2,
    -b gz^2, -2 b gx gy, -2 b gx gz, -2 b gy gz."""
    b = np.asarray(b, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    return np.stack([-b * g[:, 0] ** 2, -b * g[:, 1] ** 2, -b * g[:, 2] ** 2, -2 * b * g[:, 0] * g[:, 1],
                     -2 * b * g[:, 0] * g[:, 2], -2 * b * g[:, 1] * g[:, 2]], axis=1)


def tensor_eigenvalues(t: np.ndarray) -> np.ndarray:
    """solve_eigenvalues (diffusion_models.rs:160-185): t (..., 6) = Dxx Dyy Dzz Dxy Dxz Dyz;
    returns (..., 3) descending (e1 >= e2 >= e3)."""
    t = np.asarray(t, dtype=np.float64)
    M = np.zeros(t.shape[:-1] + (3, 3))
    M[..., 0, 0], M[..., 1, 1], M[..., 2, 2] = t[..., 0], t[..., 1], t[..., 2]
    M[..., 1, 0] = M[..., 0, 1] = t[..., 3]
    M[..., 2, 0] = M[..., 0, 2] = t[..., 4]
    M[..., 2, 1] = M[..., 1, 2] = t[..., 5]
    return np.linalg.eigvalsh(M)[..., ::-1]


def dti_fit(dwi: np.ndarray, b0: np.ndarray, b: np.ndarray, g: np.ndarray) -> dict:
    """calc_scalars (diffusion_models.rs:21-112) on (V, nq) and (V, nb0) complex arrays: b0 average
    of magnitudes, rhs = ln(clamp(|s| / max(s0, FLT_MIN), FLT_MIN, 1)), least-squares tensor,
    eigenvalues, MD, RD, FA."""
    tiny = np.finfo(np.float32).tiny
    s0 = np.abs(b0).mean(axis=1) if b0.shape[1] else np.zeros(dwi.shape[0])
    rhs = np.log(np.clip(np.abs(dwi) / np.maximum(s0, tiny)[:, None], tiny, 1.0))
    A = dti_design_matrix(b, g)
    t = np.linalg.lstsq(A, rhs.T, rcond=None)[0].T
    e = tensor_eigenvalues(t)
    md = e.mean(axis=1)
    rd = 0.5 * (e[:, 1] + e[:, 2])
    with np.errstate(invalid="ignore", divide="ignore"):
        fa = np.sqrt(1.5) * np.sqrt(((e - md[:, None]) ** 2).sum(axis=1)) / np.sqrt((e ** 2).sum(axis=1))
    return dict(b0av=s0, e1=e[:, 0], e2=e[:, 1], e3=e[:, 2], md=md, rd=rd, fa=fa, tensor=t)


# ---------------------------------------------------------------------------------------
# Temporal subspace from simulated tensor signals (the library's GPU construction)
# ---------------------------------------------------------------------------------------
SUBSPACE_STREAM = 0x5342  # "SB"


def _rng_u64_vec(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """rng_u64 over an array of indices (uint64 arithmetic wraps modulo 2^64)."""
    with np.errstate(over="ignore"):
        g = np.uint64(GOLDEN64)
        x = np.uint64(seed) + g * ((np.uint64(stream) << np.uint64(32)) + index.astype(np.uint64) + np.uint64(1))
        z = x + g
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def dti_subspace_counter(b, g, rank: int, n_signals: int, seed: int, lam_lo=0.1e-3, lam_hi=3.0e-3):
    """Leading left singular vectors of n_signals simulated tensor signals (S0 = 1), drawn with the
    counter RNG: direction (sample_unit_sphere, dti_subspace.rs:65-76) from draws 5i, 5i+1,
    eigenvalues uniform in [lam_lo, lam_hi] from draws 5i+2..5i+4, frame as eigenvector_matrix
    (dti_subspace.rs:13-44).  Returns (S (nq, rank) with the largest-magnitude entry of each column
    positive, singular values (rank,))."""
    b = np.asarray(b, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    i = np.arange(n_signals, dtype=np.uint64)
    u = [((_rng_u64_vec(seed, SUBSPACE_STREAM, 5 * i + k) >> np.uint64(11)).astype(np.float64) + 0.5) / 2.0 ** 53
         for k in range(5)]
    th, ph = 2 * np.pi * u[0], np.arccos(2 * u[1] - 1)
    e1 = np.stack([np.sin(ph) * np.cos(th), np.sin(ph) * np.sin(th), np.cos(ph)], axis=1)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    near_x = np.abs(e1[:, 0] - 1.0) < np.finfo(np.float32).eps
    tmp = np.where(near_x[:, None], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0])
    e2 = np.cross(e1, tmp)
    e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
    e3 = np.cross(e1, e2)
    lam = np.stack([lam_lo + (lam_hi - lam_lo) * u[k] for k in (2, 3, 4)], axis=1)
    proj = np.stack([e1 @ g.T, e2 @ g.T, e3 @ g.T], axis=2)          # (n, nq, 3)
    sig = np.exp(-b[None, :] * np.einsum("nqa,na->nq", proj ** 2, lam))
    G = sig.T @ sig
    w, V = np.linalg.eigh(G)
    order = np.argsort(w)[::-1][:rank]
    S = V[:, order]
    idx = np.argmax(np.abs(S), axis=0)
    S = S * np.sign(S[idx, np.arange(rank)])
    return S.astype(np.complex128), np.sqrt(np.maximum(w[order], 0.0))
