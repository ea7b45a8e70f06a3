"""Timed CPU baseline: FP32 numpy/scipy restatement of the reference's iteration.

TEST/BENCH INFRASTRUCTURE ONLY (the ``cpu_baseline`` and ``--impl reference`` legs of
bench.py).  The reference cannot be built here (no Rust toolchain, unvendored git crates),
so its CPU path is restated as written in ``lib.rs:262-341``: per batch of Casorati
matrices lift (block.rs:147-164) -> low-rank (batched LAPACK SVD in place of cuSOLVER
gesvda, low_rank.rs:10-69) -> un-lift (block.rs:166-184); then the signal model
(signal_model.rs:34-79, scipy.fft with all host threads) -> hard_project (lib.rs:392-406) ->
inverse signal model.  FP32 arithmetic throughout, with the f64 residual of the reference.

A full iteration of the production-size configuration takes tens of seconds on a host, so
``time_iteration_sample`` times a bounded, stated sample (a number of blocks and a number
of volumes) and scales it to one iteration.
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import llr_oracle as O


def _threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:  # pragma: no cover
        return os.cpu_count() or 1


def prox_blocks(x: np.ndarray, block_size, shift, blocks: np.ndarray, mode: str, rank: int, lam: float,
                batch: int = 200, threads: int = 1) -> None:
    """lift -> low rank -> un-lift for the listed block indices, in place, FP32."""
    nx, ny, nz, nq = x.shape
    flat = x.reshape(nx * ny * nz, nq, order="F")
    vol = (nx, ny, nz)
    idx = [O._block_voxel_index(vol, block_size, O.block_coord(int(b), vol, block_size, shift)) for b in blocks]

    def work(chunk):
        ids = [idx[i] for i in chunk]
        mats = np.stack([flat[v, :] for v in ids], axis=0)            # (b, m, nq) complex64
        U, s, Vh = np.linalg.svd(mats, full_matrices=False)
        if mode == "hard":
            out = (U[:, :, :rank] * s[:, None, :rank]) @ Vh[:, :rank, :]
        else:
            out = (U * np.maximum(s - lam, 0)[:, None, :].astype(np.float32)) @ Vh
        for v, o in zip(ids, out):
            flat[v, :] = o

    chunks = [list(range(i, min(i + batch, len(blocks)))) for i in range(0, len(blocks), batch)]
    if threads > 1:
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(work, chunks))
    else:
        for c in chunks:
            work(c)


def signal_dc(x: np.ndarray, y: np.ndarray, threads: int) -> float:
    """A -> hard_project -> A^H on every volume of x (zero corrections), FP32, in place."""
    import scipy.fft as sf
    nx, ny, nz, nq = x.shape
    ramps = [np.exp(1j * np.pi * (np.arange(n) - n / 2.0)).astype(np.complex64) for n in (nx, ny, nz)]
    pre = ramps[0][:, None, None] * ramps[1][None, :, None] * ramps[2][None, None, :]
    err = 0.0
    for q in range(nq):
        k = sf.fftn(x[..., q] * pre, norm="ortho", workers=threads) * np.conj(pre)
        yq = y[..., q]
        m = yq != 0
        d = (k - yq)[m]
        err += float(np.sum((d.real.astype(np.float64) ** 2 + d.imag.astype(np.float64) ** 2)))
        k[m] = yq[m]
        x[..., q] = sf.ifftn(k * pre, norm="ortho", workers=threads) * np.conj(pre)
    return err


def sigma_max_all_blocks(x: np.ndarray, block_size, shift=(0, 0, 0), batch: int = 512,
                         threads: int | None = None) -> float:
    """Largest singular value over every block of ``x`` at ``shift`` (lift_data_set order,
    block.rs:147-164), from the FP64 Gram matrix of each Casorati block (eigvalsh), in batches
    over host threads.  The threshold rule lambda = 0.02 sigma_max uses it."""
    threads = threads or _threads()
    nx, ny, nz, nq = x.shape
    vol = (nx, ny, nz)
    total = int(np.prod(O.grid_dim(vol, block_size)))
    flat = x.reshape(nx * ny * nz, nq, order="F")

    def work(b0):
        ids = [O._block_voxel_index(vol, block_size, O.block_coord(b, vol, block_size, shift))
               for b in range(b0, min(b0 + batch, total))]
        mats = np.stack([flat[v, :] for v in ids], axis=0).astype(np.complex128)
        G = np.conj(np.swapaxes(mats, 1, 2)) @ mats
        return float(np.sqrt(max(np.linalg.eigvalsh(G)[:, -1].max(), 0.0)))

    with ThreadPoolExecutor(threads) as ex:
        return max(ex.map(work, range(0, total, batch)))


def time_iteration_sample(x: np.ndarray, y: np.ndarray, block_size, mode: str, rank: int, lam: float,
                          n_blocks: int, n_vols: int, seed: int = 0, threads: int | None = None) -> dict:
    """Time ``n_blocks`` blocks of the prox and ``n_vols`` volumes of A/DC/A^H; scale to one
    full iteration.  Returns seconds per iteration and the sample description."""
    threads = threads or _threads()
    nx, ny, nz, nq = x.shape
    total_blocks = int(np.prod(O.grid_dim((nx, ny, nz), block_size)))
    n_blocks = max(1, min(n_blocks, total_blocks))
    n_vols = max(1, min(n_vols, nq))
    rng = np.random.default_rng(seed)
    blocks = np.sort(rng.choice(total_blocks, size=n_blocks, replace=False))
    shift = O.rand_shift(seed, 0, (nx, ny, nz))
    xs = np.asfortranarray(x.copy())
    t0 = time.perf_counter()
    prox_blocks(xs, block_size, shift, blocks, mode, rank, lam, threads=threads)
    t_prox = time.perf_counter() - t0
    xv = np.asfortranarray(xs[..., :n_vols].copy())
    t0 = time.perf_counter()
    signal_dc(xv, y[..., :n_vols], threads)
    t_sig = time.perf_counter() - t0
    per_iter = t_prox * total_blocks / n_blocks + t_sig * nq / n_vols
    return {
        "seconds_per_iteration": per_iter,
        "prox_seconds_sampled": t_prox,
        "signal_seconds_sampled": t_sig,
        "threads": threads,
        "sample": (f"{n_blocks} of {total_blocks} Casorati blocks (prox) + {n_vols} of {nq} volumes "
                   f"(A, hard DC, A^H), scaled to one iteration"),
    }
