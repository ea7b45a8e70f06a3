"""CFL files and b-tables through the library (llr_cfl_*, llr_read_b_table, llr_b0_mask)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check, lib


def cfl_dims(path: str) -> tuple:
    d = (C.c_int64 * 16)()
    nd = C.c_int32()
    check(lib.llr_cfl_dims(str(path).encode(), d, 16, C.byref(nd)))
    return tuple(int(d[i]) for i in range(nd.value))


def read_cfl(path: str) -> np.ndarray:
    """Complex64 array with the file's dimensions, column-major."""
    dims = cfl_dims(path)
    out = np.empty(dims, dtype=np.complex64, order="F")
    check(lib.llr_cfl_read(str(path).encode(), L.ptr(out), int(out.size)))
    return out


def write_cfl(path: str, a: np.ndarray) -> None:
    a = np.asfortranarray(a, dtype=np.complex64)
    dims = (C.c_int64 * a.ndim)(*a.shape)
    check(lib.llr_cfl_write(str(path).encode(), dims, a.ndim, L.ptr(a)))


def read_b_table(path: str, n_vols: int):
    """(b-values (n,), gradient vectors (n, 3))."""
    b = np.empty(n_vols, dtype=np.float32)
    g = np.empty((n_vols, 3), dtype=np.float32)
    check(lib.llr_read_b_table(str(path).encode(), int(n_vols), L.fptr(b), L.fptr(g)))
    return b, g


def b0_mask(g: np.ndarray, tol: float = 0.0) -> np.ndarray:
    g = np.ascontiguousarray(g, dtype=np.float32)
    out = np.empty(g.shape[0], dtype=np.uint8)
    check(lib.llr_b0_mask(L.fptr(g), int(g.shape[0]), float(tol), L.ptr(out)))
    return out.astype(bool)


def read_affine_translation(path: str, multiplier: float = 1.0) -> np.ndarray:
    """Translation (3,) of an affine transform file, times ``multiplier``."""
    out = np.empty(3, dtype=np.float32)
    check(lib.llr_read_affine_translation(str(path).encode(), float(multiplier), L.fptr(out)))
    return out


def read_affine_translations(paths, multiplier: float = 1.0) -> np.ndarray:
    """(n, 3) translations, e.g. per-volume image-space corrections for set_linear_corrections."""
    return np.stack([read_affine_translation(p, multiplier) for p in paths])
