"""Learned warm start: host side of the 3-D residual CNN (llr_cnn_* in the C ABI).

The network maps the subspace coefficients of an adjoint (zero-filled) image to those of the
converged plain reconstruction; its output, taken back through S^H, is the starting image of
the same proximal-gradient LLR iteration, which still decides the answer (its fixed point).
Training runs on the GPU with the library's own conv3d forward / backward kernels and Adam.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L
from ._lib import check, lib
from .api import DeviceBuffer

DEFAULT_CHANNELS = (14, 32, 32, 32, 32, 32, 32, 32, 14)


def _i32(v) -> C.Array:
    return (C.c_int32 * len(v))(*[int(a) for a in v])


class DeviceArray:
    """Row-major float32 device array (raw bytes, no reordering)."""

    def __init__(self, shape):
        self.shape = tuple(int(s) for s in shape)
        self.buf = DeviceBuffer(4 * int(np.prod(self.shape)))

    @classmethod
    def from_numpy(cls, a: np.ndarray) -> "DeviceArray":
        a = np.ascontiguousarray(a, dtype=np.float32)
        d = cls(a.shape)
        d.buf.upload(a.reshape(-1))
        return d

    @property
    def ptr(self):
        return self.buf.ptr

    def numpy(self) -> np.ndarray:
        out = np.empty(int(np.prod(self.shape)), dtype=np.float32)
        self.buf.download(out)
        return out.reshape(self.shape)

    def close(self):
        self.buf.close()


class Cnn:
    """conv3d 3x3x3 residual network, channels-last activations of shape (nz, ny, nx, C)."""

    def __init__(self, channels: Sequence[int] = DEFAULT_CHANNELS, device: int = 0, seed: int = 0):
        self.channels = tuple(int(c) for c in channels)
        h = C.c_void_p()
        check(lib.llr_cnn_create(len(self.channels) - 1, _i32(self.channels), int(device), C.c_uint64(seed),
                                 C.byref(h)))
        self.h = h
        n = C.c_int64()
        check(lib.llr_cnn_param_count(self.h, C.byref(n)))
        self.n_params = int(n.value)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.llr_cnn_destroy(self.h)
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

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        check(lib.llr_cnn_get_params(self.h, L.ptr(out)))
        return out

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        check(lib.llr_cnn_set_params(self.h, L.ptr(p)))

    @property
    def grads(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        check(lib.llr_cnn_get_grads(self.h, L.ptr(out)))
        return out

    @staticmethod
    def _dims(shape) -> C.Array:
        nz, ny, nx = shape[:3]
        return _i32((nx, ny, nz))

    def forward_dev(self, x: DeviceArray, out: DeviceArray) -> None:
        check(lib.llr_cnn_forward_dev(self.h, x.ptr, out.ptr, self._dims(x.shape), None))

    def forward(self, x: np.ndarray) -> np.ndarray:
        dx = DeviceArray.from_numpy(x)
        do = DeviceArray(dx.shape[:3] + (self.channels[-1],))
        self.forward_dev(dx, do)
        check(lib.llr_stream_sync(None))
        out = do.numpy()
        dx.close()
        do.close()
        return out

    def loss_grad_dev(self, x: DeviceArray, target: DeviceArray) -> float:
        loss = C.c_double()
        check(lib.llr_cnn_loss_grad_dev(self.h, x.ptr, target.ptr, self._dims(x.shape), C.byref(loss), None))
        return float(loss.value)

    def adam_step(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
        check(lib.llr_cnn_adam_step(self.h, float(lr), float(beta1), float(beta2), float(eps), None))

    def train_step_dev(self, x: DeviceArray, target: DeviceArray, lr: float) -> float:
        loss = C.c_double()
        check(lib.llr_cnn_train_step_dev(self.h, x.ptr, target.ptr, self._dims(x.shape), float(lr), C.byref(loss),
                                         None))
        return float(loss.value)

    def save(self, path: str) -> None:
        np.savez(path, channels=np.asarray(self.channels, dtype=np.int32), params=self.params)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Cnn":
        z = np.load(path)
        net = cls(tuple(int(c) for c in z["channels"]), device=device)
        net.params = z["params"]
        return net


def subspace_channels_dev(d_x, vol, nq: int, d_S, srank: int, scale: float, out: DeviceArray,
                          d_phase_ref=None) -> None:
    """CNN channels scale * ((u* x) S) of a device image in the reference layout; u is the unit
    phase of the device image ``d_phase_ref`` (1 when None)."""
    check(lib.llr_subspace_channels_dev(d_x, _i32(vol), int(nq), d_S, int(srank), float(scale), d_phase_ref,
                                        out.ptr, None))


def subspace_image_dev(chan: DeviceArray, vol, nq: int, d_S, srank: int, scale: float, d_x,
                       accumulate: bool = False, d_phase_ref=None) -> None:
    """Image u (1 / scale) c S^H from CNN channels into a device image (reference layout); added
    to what the image holds when ``accumulate``."""
    check(lib.llr_subspace_image_dev(chan.ptr, _i32(vol), int(nq), d_S, int(srank), float(scale), d_phase_ref,
                                     1 if accumulate else 0, d_x, None))
