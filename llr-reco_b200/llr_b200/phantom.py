"""Seeded synthetic diffusion-MRI datasets (the reference reads private CFL files instead).

Signal model S_q = S0 exp(-b_q g_q^T D g_q) with the design-matrix convention of
``diffusion_models.rs:221-253``; gradient directions from ``sample_unit_sphere``
(``dti_subspace.rs:65-76``) and tensor frames from ``eigenvector_matrix``
(``dti_subspace.rs:13-44``).  Everything is drawn from ``numpy.random.Generator(PCG64(seed))``
so a seed fixes the dataset.  Sampling masks come from the library's counter-based
``llr_vd_mask`` (bit-exact twin in the oracle).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np


def sample_unit_sphere(u1: float, u2: float) -> np.ndarray:
    """dti_subspace.rs:65-76."""
    theta = 2.0 * math.pi * u1
    phi = math.acos(2.0 * u2 - 1.0)
    return np.array([math.sin(phi) * math.cos(theta), math.sin(phi) * math.sin(theta), math.cos(phi)])


def eigenvector_matrix(principal_dir) -> np.ndarray:
    """dti_subspace.rs:13-44: orthonormal frame whose first column is the principal direction."""
    e1 = np.asarray(principal_dir, dtype=np.float64)
    e1 = e1 / np.linalg.norm(e1)
    temp = np.array([1.0, 0.0, 0.0])
    if abs(e1[0] - 1.0) < np.finfo(np.float32).eps:
        temp = np.array([0.0, 1.0, 0.0])
    e2 = np.cross(e1, temp)
    e2 = e2 / np.linalg.norm(e2)
    e3 = np.cross(e1, e2)
    return np.stack([e1, e2, e3], axis=1)


def b_table(shells, rng) -> tuple[np.ndarray, np.ndarray]:
    """shells: list of (b_value, count).  Returns (b (nq,), g (nq, 3))."""
    b, g = [], []
    for bv, cnt in shells:
        for _ in range(cnt):
            b.append(float(bv))
            g.append(np.zeros(3) if bv == 0 else sample_unit_sphere(rng.random(), rng.random()))
    return np.array(b), np.array(g)


def tensor_signal(S0: np.ndarray, D: np.ndarray, b: np.ndarray, g: np.ndarray) -> np.ndarray:
    """S0 * exp(-b g^T D g); D (..., 3, 3), returns (..., nq)."""
    quad = np.einsum("qi,...ij,qj->...q", g, D, g)
    return S0[..., None] * np.exp(-b * quad)


@dataclass
class Dataset:
    x_true: np.ndarray        # (nx, ny, nz, nq) complex64, F-order
    mask: np.ndarray          # (ny, nz, nq) uint8
    b: np.ndarray
    g: np.ndarray
    noise_sigma: float
    y: Optional[np.ndarray] = None   # measured k-space (nx, ny, nz, nq) complex64, F-order


def phantom_image(vol, b, g, rng, n_ellipsoids=6, lam=(1.7e-3, 0.3e-3, 0.3e-3), d_bg=3.0e-3,
                  phase_range=math.pi) -> np.ndarray:
    """Ellipsoid phantom: an isotropic background object and ``n_ellipsoids`` anisotropic ones."""
    nx, ny, nz = vol
    nq = len(b)
    xs = (np.arange(nx) - nx / 2 + 0.5) / (nx / 2)
    ys = (np.arange(ny) - ny / 2 + 0.5) / (ny / 2)
    zs = (np.arange(nz) - nz / 2 + 0.5) / (nz / 2)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    img = np.zeros((nx, ny, nz, nq), dtype=np.float32)
    # background object: isotropic D, S0 ~ U[0.5, 1]
    outer = (X / 0.9) ** 2 + (Y / 0.85) ** 2 + (Z / 0.8) ** 2 <= 1.0
    s0 = rng.uniform(0.5, 1.0)
    sig_bg = s0 * np.exp(-b * d_bg)
    img[outer] = sig_bg.astype(np.float32)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.45, 0.45, size=3)
        r = rng.uniform(0.12, 0.35, size=3)
        R = eigenvector_matrix(sample_unit_sphere(rng.random(), rng.random()))
        P = np.stack([X - c[0], Y - c[1], Z - c[2]], axis=-1) @ R
        inside = ((P / r) ** 2).sum(-1) <= 1.0
        inside &= outer
        Rt = eigenvector_matrix(sample_unit_sphere(rng.random(), rng.random()))
        D = Rt @ np.diag(lam) @ Rt.T
        s0e = rng.uniform(0.5, 1.0)
        sig = tensor_signal(np.array(s0e), D, b, g)
        img[inside] = sig.astype(np.float32)
    # smooth 2nd-order polynomial phase per volume, scaled to +-phase_range
    mon = [X, Y, Z, X * X, Y * Y, Z * Z, X * Y, X * Z, Y * Z]
    out = np.empty((nx, ny, nz, nq), dtype=np.complex64, order="F")
    for q in range(nq):
        coef = rng.standard_normal(len(mon))
        ph = sum(cf * m for cf, m in zip(coef, mon))
        mx = np.abs(ph).max()
        ph = ph * (phase_range / mx) if mx > 0 else ph
        out[..., q] = img[..., q] * np.exp(1j * ph).astype(np.complex64)
    return out


def centred_fft_unitary(x: np.ndarray) -> np.ndarray:
    """Forward operator with zero linear corrections (signal_model.rs:34-79) via numpy.

    With s = n/2 the reference's ramps are exp(+-i pi (i - n/2)); this is the centred,
    unitary 3-D FFT of every volume.
    """
    try:
        import scipy.fft as sf
        fftn = lambda a: sf.fftn(a, axes=(0, 1, 2), norm="ortho", workers=-1)
    except Exception:  # pragma: no cover
        fftn = lambda a: np.fft.fftn(a, axes=(0, 1, 2), norm="ortho")
    nx, ny, nz, nq = x.shape
    ramps = []
    for n in (nx, ny, nz):
        i = np.arange(n)
        ramps.append(np.exp(1j * math.pi * (i - n / 2.0)))
    pre = (ramps[0][:, None, None] * ramps[1][None, :, None] * ramps[2][None, None, :])
    out = np.empty_like(x, order="F")
    for q in range(nq):
        out[..., q] = (fftn(x[..., q] * pre) * np.conj(pre)).astype(x.dtype)
    return out


def make_dataset(vol, shells, accel, seed, centre=16, snr=30.0, n_ellipsoids=6,
                 mask_fn: Optional[Callable] = None, forward: Optional[Callable] = None,
                 protocol_seed: Optional[int] = None) -> Dataset:
    """Phantom, per-volume VD ky-kz mask, complex Gaussian noise at ``snr``.

    Noise: sigma = mean |x_true| over the object / snr, added with standard deviation sigma
    to the real and to the imaginary part of every sampled k-space sample.  With
    ``protocol_seed`` the b-table (the acquisition protocol) comes from that seed and only the
    phantom, mask and noise from ``seed``, so that many subjects share one protocol.
    """
    rng = np.random.default_rng(seed)
    b, g = b_table(shells, np.random.default_rng(protocol_seed) if protocol_seed is not None else rng)
    x = phantom_image(vol, b, g, rng, n_ellipsoids=n_ellipsoids)
    nx, ny, nz = vol
    nq = len(b)
    if mask_fn is None:
        from .api import vd_mask
        mask_fn = vd_mask
    mask = mask_fn(ny, nz, nq, float(accel), int(centre), int(seed))
    obj = np.abs(x[..., 0]) > 0
    sigma = float(np.abs(x[..., 0])[obj].mean() / snr) if obj.any() else 0.0
    k = (forward or centred_fft_unitary)(x)
    noise = (rng.standard_normal(k.shape, dtype=np.float32) + 1j * rng.standard_normal(k.shape, dtype=np.float32))
    k = k + (sigma * noise).astype(np.complex64)
    k *= (mask != 0)[None, :, :, :]
    return Dataset(x_true=x, mask=mask, b=b, g=g, noise_sigma=sigma, y=np.asfortranarray(k.astype(np.complex64)))


# Seed of the b-table every benchmark subject shares (the acquisition protocol the learned warm
# start was trained in); phantom, mask and noise come from the subject's own seed.
PROTOCOL_SEED = 1234

# Configurations of the benchmark suite (shapes and acquisition parameters).
CONFIGS = {
    "c1": dict(vol=(64, 64, 64), shells=[(0, 1), (1000, 16)], accel=4.0, block=(8, 8, 8), n_iter=50),
    "c2": dict(vol=(192, 192, 96), shells=[(0, 7), (3000, 54)], accel=8.0, block=(6, 6, 6), n_iter=100),
    # config-2 geometry class at 1/8 of the volume (216 MB per copy, still > L2): profiling case
    "c2_small": dict(vol=(96, 96, 48), shells=[(0, 7), (3000, 54)], accel=8.0, block=(6, 6, 6), n_iter=100),
    "c3": dict(vol=(256, 256, 256), shells=[(0, 1), (1000, 30), (2000, 30)], accel=10.0, block=(8, 8, 8),
               n_iter=80, srank=7, wavelet_alpha=0.005, wavelet_moments=4, wavelet_levels=3, wavelet_space=1),
    "c5": dict(vol=(256, 256, 256), shells=[(0, 6), (1000, 34), (2000, 33), (3000, 33)], accel=12.0,
               block=(8, 8, 8), stride=(4, 4, 4), n_iter=80),
    # config-5 geometry class at 1/8 of the volume (1.78 GB per copy): measurement case
    "c5_small": dict(vol=(128, 128, 128), shells=[(0, 6), (1000, 34), (2000, 33), (3000, 33)], accel=12.0,
                     block=(8, 8, 8), stride=(4, 4, 4), n_iter=80),
}


def dti_subspace(b: np.ndarray, g: np.ndarray, rank: int, n_signals: int, seed: int) -> np.ndarray:
    """Temporal subspace: top-``rank`` left singular vectors of ``n_signals`` simulated tensor
    signals (eigenvalues U[0.1, 3.0]e-3, random orientation, S0 = 1).  Returns (nq, rank)."""
    rng = np.random.default_rng(seed)
    lam = rng.uniform(0.1e-3, 3.0e-3, size=(n_signals, 3))
    D = np.empty((n_signals, 3, 3))
    for i in range(n_signals):
        R = eigenvector_matrix(sample_unit_sphere(rng.random(), rng.random()))
        D[i] = R @ np.diag(lam[i]) @ R.T
    sig = tensor_signal(np.ones(n_signals), D, b, g)     # (n, nq)
    U, s, _ = np.linalg.svd(sig.T, full_matrices=False)
    return np.asfortranarray(U[:, :rank].astype(np.complex64))


def dti_subspace_gpu(b: np.ndarray, g: np.ndarray, rank: int, n_signals: int, seed: int,
                     lam_lo: float = 0.1e-3, lam_hi: float = 3.0e-3):
    """The same subspace construction on the GPU (llr_dti_subspace, counter-based draws):
    returns (S (nq, rank) complex64, singular values)."""
    import ctypes as C
    from . import _lib as L
    nq = len(b)
    bb = np.ascontiguousarray(b, dtype=np.float32)
    gg = np.ascontiguousarray(g, dtype=np.float32)
    S = np.empty((nq, rank), dtype=np.complex64, order="F")
    sv = np.empty(rank, dtype=np.float64)
    L.check(L.lib.llr_dti_subspace(L.fptr(bb), L.fptr(gg), nq, rank, int(n_signals), C.c_uint64(seed),
                                   float(lam_lo), float(lam_hi), L.ptr(S), sv.ctypes.data_as(L.PF64)))
    return S, sv
