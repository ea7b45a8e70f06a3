"""Python host side of the C ABI: device buffers and the reconstruction context.

Names and argument meanings follow the reference operators (``llr_recon_exec``,
``signal_model``, ``cu_low_rank_approx_batch``, ``lift_data_set`` ...); every call goes
through ``libllr_b200.so``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import check, lib

CF32 = np.complex64


def to_ref_layout(x: np.ndarray) -> np.ndarray:
    """(nx, ny, nz, nq) array -> contiguous column-major complex64 buffer (x fastest)."""
    return np.asfortranarray(x, dtype=CF32)


def device_count() -> int:
    n = C.c_int32(0)
    st = lib.llr_device_count(C.byref(n))
    return int(n.value) if st == L.LLR_OK else 0


class DeviceBuffer:
    """Raw device allocation owned by Python (freed on close/GC)."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        check(lib.llr_device_alloc(self.nbytes, C.byref(p)))
        self.ptr = p

    @classmethod
    def from_array(cls, a: np.ndarray) -> "DeviceBuffer":
        """Copy ``a`` to the device in column-major order (the library's convention)."""
        a = np.asfortranarray(a)
        b = cls(a.nbytes)
        check(lib.llr_memcpy_h2d(b.ptr, L.ptr(a), a.nbytes, None))
        check(lib.llr_stream_sync(None))
        return b

    def upload(self, a: np.ndarray) -> None:
        assert a.nbytes <= self.nbytes
        check(lib.llr_memcpy_h2d(self.ptr, L.ptr(a), a.nbytes, None))
        check(lib.llr_stream_sync(None))

    def download(self, a: np.ndarray) -> np.ndarray:
        """Copy device bytes into ``a``, which must be column-major (or 1-D)."""
        assert a.nbytes <= self.nbytes
        assert a.flags["F_CONTIGUOUS"], "download target must be column-major"
        check(lib.llr_stream_sync(None))
        check(lib.llr_memcpy_d2h(L.ptr(a), self.ptr, a.nbytes, None))
        check(lib.llr_stream_sync(None))
        return a

    def close(self) -> None:
        if self.ptr is not None and self.ptr.value:
            lib.llr_device_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host buffer exposed as a numpy array."""

    def __init__(self, shape, dtype=CF32, order="F"):
        dtype = np.dtype(dtype)
        n = int(np.prod(shape)) * dtype.itemsize
        p = C.c_void_p()
        check(lib.llr_host_alloc(n, C.byref(p)))
        self.ptr = p
        buf = (C.c_char * n).from_address(p.value)
        self.array = np.ndarray(shape, dtype=dtype, buffer=buf, order=order)

    def close(self):
        if self.ptr is not None and self.ptr.value:
            lib.llr_host_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ReconParams:
    """Mirror of ``LlrReconParams`` (lib.rs:47-81) plus the B200 build's additions."""
    vol_size: Sequence[int]
    nq: int
    block_size: Sequence[int] = (32, 32, 32)
    max_rand_shift: Optional[Sequence[int]] = None
    prox_mode: int = L.LLR_PROX_HARD_RANK
    rank: int = 6
    lam: float = 0.0
    wavelet_alpha: float = 0.0
    wavelet_moments: int = 2
    wavelet_levels: int = 0
    subspace_rank: int = 0
    n_iter: int = 60
    seed: int = 0
    device: int = 0
    eig_solver: int = 0
    gram_mode: int = 0
    fft_mode: int = 0
    wavelet_space: int = 0
    block_stride: Optional[Sequence[int]] = None

    def to_c(self) -> L.llr_config:
        c = L.llr_config()
        check(lib.llr_config_default(C.byref(c)))
        c.vol_size = L.i32x3(self.vol_size)
        c.nq = int(self.nq)
        c.block_size = L.i32x3(self.block_size)
        c.max_rand_shift = L.i32x3(self.max_rand_shift or (0, 0, 0))
        c.prox_mode = int(self.prox_mode)
        c.rank = int(self.rank)
        c.lambda_ = float(self.lam)
        c.wavelet_alpha = float(self.wavelet_alpha)
        c.wavelet_moments = int(self.wavelet_moments)
        c.wavelet_levels = int(self.wavelet_levels)
        c.subspace_rank = int(self.subspace_rank)
        c.n_iter = int(self.n_iter)
        c.seed = int(self.seed)
        c.device = int(self.device)
        c.eig_solver = int(self.eig_solver)
        c.gram_mode = int(self.gram_mode)
        c.fft_mode = int(self.fft_mode)
        c.wavelet_space = int(self.wavelet_space)
        c.block_stride = L.i32x3(self.block_stride or (0, 0, 0))
        return c


class ReconContext:
    """Device-resident reconstruction (replacement of ``llr_recon_exec``, lib.rs:113-363)."""

    def __init__(self, params: ReconParams):
        self.params = params
        self._cfg = params.to_c()
        h = C.c_void_p()
        check(lib.llr_ctx_create(C.byref(self._cfg), C.byref(h)))
        self.h = h
        nx, ny, nz = (int(v) for v in params.vol_size)
        self.shape = (nx, ny, nz, int(params.nq))

    # -- data ---------------------------------------------------------------------------
    def set_linear_corrections(self, lin_ksp=None, lin_img=None) -> None:
        k = None if lin_ksp is None else np.ascontiguousarray(lin_ksp, dtype=np.float32)
        i = None if lin_img is None else np.ascontiguousarray(lin_img, dtype=np.float32)
        check(lib.llr_set_linear_corrections(self.h, None if k is None else L.fptr(k),
                                             None if i is None else L.fptr(i)))

    def upload_kspace(self, y: np.ndarray) -> None:
        y = to_ref_layout(y)
        assert y.shape == self.shape, (y.shape, self.shape)
        check(lib.llr_upload_kspace(self.h, L.ptr(y)))

    def upload_subspace(self, S: np.ndarray) -> None:
        S = np.asfortranarray(S, dtype=CF32)
        check(lib.llr_upload_subspace(self.h, L.ptr(S)))

    def init_zero_filled(self) -> None:
        check(lib.llr_init_zero_filled(self.h))

    def upload_image(self, x: np.ndarray) -> None:
        x = to_ref_layout(x)
        check(lib.llr_upload_image(self.h, L.ptr(x)))

    def download_image(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=CF32, order="F")
        check(lib.llr_download_image(self.h, L.ptr(out)))
        return out

    # -- iteration ----------------------------------------------------------------------
    def iterate(self, n: int, history: bool = True) -> Optional[np.ndarray]:
        if history:
            h = np.empty(max(n, 1), dtype=np.float64)
            check(lib.llr_iterate(self.h, int(n), h.ctypes.data_as(L.PF64)))
            return h[:n]
        check(lib.llr_iterate(self.h, int(n), None))
        return None

    def iterate_async(self, n: int) -> None:
        check(lib.llr_iterate_async(self.h, int(n)))

    def iterate_timed(self, n: int) -> float:
        """Device milliseconds of ``n`` single-graph iterations (CUDA events on the context stream)."""
        ms = C.c_double()
        check(lib.llr_iterate_timed(self.h, int(n), C.byref(ms)))
        return ms.value

    def iterate_profiled(self, n: int) -> tuple[np.ndarray, float]:
        """Per-stage device milliseconds (prox, wavelet, FFT, DC, IFFT) summed over ``n`` iterations."""
        st = np.zeros(5, dtype=np.float64)
        tot = C.c_double()
        check(lib.llr_iterate_profiled(self.h, int(n), st.ctypes.data_as(L.PF64), C.byref(tot)))
        return st, tot.value

    def snapshot(self) -> DeviceBuffer:
        """Device copy of the iterate in the internal layout (for nrmse())."""
        b = DeviceBuffer(8 * int(np.prod(self.shape)))
        check(lib.llr_ctx_snapshot(self.h, b.ptr))
        return b

    def nrmse(self, snap: DeviceBuffer) -> float:
        """||x - ref|| / ||ref|| against a snapshot of a context with the same configuration."""
        v = C.c_double()
        check(lib.llr_ctx_nrmse(self.h, snap.ptr, C.byref(v)))
        return float(v.value)

    @property
    def fallback_blocks(self) -> int:
        """Blocks the last prox step handed to the Jacobi kernel."""
        v = C.c_int64()
        check(lib.llr_ctx_fallback_blocks(self.h, C.byref(v)))
        return int(v.value)

    @property
    def kernel_launches_per_iteration(self) -> int:
        """Library kernels (not cuFFT's) one captured iteration launches."""
        v = C.c_int32()
        check(lib.llr_ctx_kernel_launches(self.h, C.byref(v)))
        return int(v.value)

    @property
    def iteration(self) -> int:
        v = C.c_int64()
        check(lib.llr_get_iteration(self.h, C.byref(v)))
        return int(v.value)

    @iteration.setter
    def iteration(self, it: int) -> None:
        check(lib.llr_set_iteration(self.h, int(it)))

    def residual_history(self, count: int) -> np.ndarray:
        h = np.empty(count, dtype=np.float64)
        check(lib.llr_get_residual_history(self.h, h.ctypes.data_as(L.PF64), int(count)))
        return h

    def objective_history(self, count: int) -> np.ndarray:
        """0.5 ||M A x - y||^2 + lambda sum_b ||X_b||_* of the last ``count`` prox outputs (FP64;
        NaN where the configuration defines no single objective)."""
        h = np.empty(count, dtype=np.float64)
        check(lib.llr_get_objective_history(self.h, h.ctypes.data_as(L.PF64), int(count)))
        return h

    def measurement_stats(self) -> tuple[float, float]:
        e, u = C.c_double(), C.c_double()
        check(lib.llr_measurement_stats(self.h, C.byref(e), C.byref(u)))
        return e.value, u.value

    def sigma_max(self, shift=(0, 0, 0)) -> float:
        v = C.c_double()
        check(lib.llr_sigma_max(self.h, L.i32x3(shift), C.byref(v)))
        return v.value

    def set_lambda(self, lam: float) -> None:
        check(lib.llr_set_lambda(self.h, float(lam)))
        self.params.lam = float(lam)

    def prox(self, shift) -> None:
        check(lib.llr_ctx_prox_llr(self.h, L.i32x3(shift)))

    def wavelet(self) -> None:
        check(lib.llr_ctx_wavelet(self.h))

    def data_consistency(self) -> float:
        v = C.c_double()
        check(lib.llr_ctx_data_consistency(self.h, C.byref(v)))
        return v.value

    def device_bytes(self) -> int:
        v = C.c_size_t()
        check(lib.llr_ctx_device_bytes(self.h, C.byref(v)))
        return int(v.value)

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            lib.llr_ctx_destroy(self.h)
        self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- host-slice operators with the reference's argument order ---------------------------
def cu_low_rank_approx_batch(m: int, n: int, rank: int, batch: int, matrix_data: np.ndarray) -> None:
    """low_rank.rs:10 — in place on a flat complex64 buffer of (m, n, batch) column-major."""
    assert matrix_data.dtype == CF32 and matrix_data.size >= m * n * batch
    check(lib.llr_cu_low_rank_approx_batch(m, n, rank, batch, L.ptr(matrix_data)))


def signal_model(x: np.ndarray, image_size, batch: int, lin_ksp=None, lin_img=None, direction=L.LLR_FORWARD):
    """signal_model.rs:34 — in place on a flat complex64 buffer of ``batch`` volumes."""
    assert x.dtype == CF32
    k = None if lin_ksp is None else np.ascontiguousarray(lin_ksp, dtype=np.float32)
    i = None if lin_img is None else np.ascontiguousarray(lin_img, dtype=np.float32)
    check(lib.llr_signal_model(L.ptr(x), L.szx3(image_size), batch, None if k is None else L.fptr(k),
                               None if i is None else L.fptr(i), int(direction)))


def lift_data_set(volumes: np.ndarray, nvols: int, matrix_data: np.ndarray, vol_size, block_size, shift,
                  start: int, n: int) -> None:
    """block.rs:147 — volumes: flat (V*nvols) complex64; matrix_data: flat (m*nvols*n)."""
    check(lib.llr_lift_data_set(L.ptr(volumes), nvols, L.ptr(matrix_data), L.szx3(vol_size),
                                L.szx3(block_size), L.szx3(shift), start, n))


def un_lift_data_set(volumes: np.ndarray, nvols: int, matrix_data: np.ndarray, vol_size, block_size, shift,
                     start: int, n: int) -> None:
    """block.rs:166."""
    check(lib.llr_un_lift_data_set(L.ptr(volumes), nvols, L.ptr(matrix_data), L.szx3(vol_size),
                                   L.szx3(block_size), L.szx3(shift), start, n))


def dti_project(S, X, out, batch, nq, nvox, srank) -> None:
    """dti_subspace.rs:141."""
    check(lib.llr_dti_project(L.ptr(S), L.ptr(X), L.ptr(out), batch, nq, nvox, srank))


def dti_back_project(S, X, comp, batch, nq, nvox, srank) -> None:
    """dti_subspace.rs:172."""
    check(lib.llr_dti_back_project(L.ptr(S), L.ptr(X), L.ptr(comp), batch, nq, nvox, srank))


def cu_dwt_denoise(vol: np.ndarray, vol_size, lo_d, hi_d, lo_r, hi_r, rand_shift=(0, 0, 0)) -> None:
    """cudwt3.rs:102 — one-level three-axis analysis + synthesis, in place."""
    f = [np.ascontiguousarray(v, dtype=np.float32) for v in (lo_d, hi_d, lo_r, hi_r)]
    check(lib.llr_cu_dwt_denoise(L.ptr(vol), L.szx3(vol_size), L.fptr(f[0]), L.fptr(f[1]), L.fptr(f[2]),
                                 L.fptr(f[3]), len(f[0]), L.i32x3(rand_shift)))


def rand_shift(seed: int, iteration: int, max_shift) -> list[int]:
    out = L.i32x3((0, 0, 0))
    check(lib.llr_rand_shift(int(seed), int(iteration), L.i32x3(max_shift), out))
    return [int(v) for v in out]


def vd_mask(ny: int, nz: int, nq: int, accel: float, centre: int, seed: int) -> np.ndarray:
    out = np.zeros((ny, nz, nq), dtype=np.uint8, order="F")
    check(lib.llr_vd_mask(ny, nz, nq, float(accel), int(centre), int(seed),
                          out.ctypes.data_as(L.PU8)))
    return out


def daubechies_filters(order: int):
    F = 2 * order
    bufs = [np.zeros(F, dtype=np.float32) for _ in range(4)]
    check(lib.llr_daubechies_filters(order, *[L.fptr(b) for b in bufs]))
    return tuple(bufs)
