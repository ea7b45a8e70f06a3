"""ctypes binding of ``libllr_b200.so`` (declarations mirror ``include/llr_b200.h``).

The shared library is loaded from the package directory (``llr-reco_b200/``).  There is
no fallback: if the library is missing the import raises, so no CPU path can stand in
for the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libllr_b200.so")

LLR_OK = 0
LLR_ERR_INVALID = -1
LLR_ERR_CUDA = -2
LLR_ERR_CUFFT = -3
LLR_ERR_NOMEM = -4
LLR_ERR_NOT_FINITE = -5
LLR_ERR_STATE = -6
LLR_ERR_UNSUPPORTED = -7
LLR_ERR_NO_DEVICE = -8

LLR_PROX_HARD_RANK = 0
LLR_PROX_SOFT_THRESH = 1
LLR_FORWARD = 0
LLR_INVERSE = 1


class llr_cf32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class llr_config(C.Structure):
    _fields_ = [
        ("vol_size", C.c_int32 * 3),
        ("nq", C.c_int32),
        ("block_size", C.c_int32 * 3),
        ("max_rand_shift", C.c_int32 * 3),
        ("prox_mode", C.c_int32),
        ("rank", C.c_int32),
        ("lambda_", C.c_float),
        ("wavelet_alpha", C.c_float),
        ("wavelet_moments", C.c_int32),
        ("wavelet_levels", C.c_int32),
        ("subspace_rank", C.c_int32),
        ("fft_max_batch_size", C.c_int32),
        ("cas_mat_max_batch_size", C.c_int32),
        ("n_iter", C.c_int32),
        ("seed", C.c_uint64),
        ("device", C.c_int32),
        ("eig_solver", C.c_int32),
        ("gram_mode", C.c_int32),
        ("fft_mode", C.c_int32),
        ("wavelet_space", C.c_int32),
        ("block_stride", C.c_int32 * 3),
    ]


P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
U32 = C.c_uint32
U64 = C.c_uint64
SZ = C.c_size_t
F32 = C.c_float
F64 = C.c_double
PI32 = C.POINTER(C.c_int32)
PU32 = C.POINTER(C.c_uint32)
PSZ = C.POINTER(C.c_size_t)
PF32 = C.POINTER(C.c_float)
PF64 = C.POINTER(C.c_double)
PU8 = C.POINTER(C.c_uint8)
PCFG = C.POINTER(llr_config)

# name -> (restype, argtypes); every function declared in include/llr_b200.h.
SIGNATURES = {
    "llr_version": (C.c_char_p, []),
    "llr_last_error": (C.c_char_p, []),
    "llr_status_string": (C.c_char_p, [C.c_int]),
    "llr_config_default": (C.c_int, [PCFG]),
    "llr_config_validate": (C.c_int, [PCFG]),
    "llr_rand_shift": (C.c_int, [U64, I64, PI32, PI32]),
    "llr_grid_dim": (C.c_int, [PI32, PI32, PI32]),
    "llr_vd_mask": (C.c_int, [I32, I32, I32, F64, I32, U64, PU8]),
    "llr_daubechies_filters": (C.c_int, [I32, PF32, PF32, PF32, PF32]),
    "llr_ctx_create": (C.c_int, [PCFG, C.POINTER(P)]),
    "llr_ctx_destroy": (C.c_int, [P]),
    "llr_ctx_set_stream": (C.c_int, [P, P]),
    "llr_ctx_get_config": (C.c_int, [P, PCFG]),
    "llr_upload_kspace": (C.c_int, [P, P]),
    "llr_upload_kspace_dev": (C.c_int, [P, P]),
    "llr_set_linear_corrections": (C.c_int, [P, PF32, PF32]),
    "llr_estimate_linear_corrections": (C.c_int, [P, PI32, I32, PF32]),
    "llr_upload_subspace": (C.c_int, [P, P]),
    "llr_init_zero_filled": (C.c_int, [P]),
    "llr_upload_image": (C.c_int, [P, P]),
    "llr_upload_image_dev": (C.c_int, [P, P]),
    "llr_download_image": (C.c_int, [P, P]),
    "llr_download_image_dev": (C.c_int, [P, P]),
    "llr_iterate": (C.c_int, [P, I32, PF64]),
    "llr_iterate_async": (C.c_int, [P, I32]),
    "llr_iterate_profiled": (C.c_int, [P, I32, PF64, PF64]),
    "llr_iterate_timed": (C.c_int, [P, I32, PF64]),
    "llr_ctx_kernel_launches": (C.c_int, [P, C.POINTER(I32)]),
    "llr_ctx_fallback_blocks": (C.c_int, [P, C.POINTER(I64)]),
    "llr_ctx_snapshot": (C.c_int, [P, P]),
    "llr_ctx_nrmse": (C.c_int, [P, P, PF64]),
    "llr_get_iteration": (C.c_int, [P, C.POINTER(I64)]),
    "llr_set_iteration": (C.c_int, [P, I64]),
    "llr_get_residual_history": (C.c_int, [P, PF64, I32]),
    "llr_get_objective_history": (C.c_int, [P, PF64, I32]),
    "llr_measurement_stats": (C.c_int, [P, PF64, PF64]),
    "llr_sigma_max": (C.c_int, [P, PI32, PF64]),
    "llr_set_lambda": (C.c_int, [P, F32]),
    "llr_ctx_prox_llr": (C.c_int, [P, PI32]),
    "llr_ctx_wavelet": (C.c_int, [P]),
    "llr_ctx_data_consistency": (C.c_int, [P, PF64]),
    "llr_ctx_device_bytes": (C.c_int, [P, PSZ]),
    "llr_signal_model_dev": (C.c_int, [P, PI32, I32, PF32, PF32, I32, P]),
    "llr_lift_data_set_dev": (C.c_int, [P, I32, P, PI32, PI32, PI32, I64, I64, P]),
    "llr_un_lift_data_set_dev": (C.c_int, [P, I32, P, PI32, PI32, PI32, I64, I64, P]),
    "llr_low_rank_batch_dev": (C.c_int, [I32, I32, I32, I32, P, P]),
    "llr_low_rank_batch_dev_noalloc": (C.c_int, [I32, I32, I32, I32, P, P]),
    "llr_soft_threshold_batch_dev": (C.c_int, [I32, I32, F32, I32, P, P]),
    "llr_subspace_low_rank_batch_dev": (C.c_int, [I32, I32, I32, I32, I32, F32, P, I32, P, P]),
    "rhsCdgmmBatched": (C.c_int, [C.c_int, C.c_int, C.c_int, P, P]),
    "llr_cgemm_strided_batched_dev": (C.c_int, [I32, I32, I32, I32, I32, llr_cf32, llr_cf32, I32, I32, P, P, P, P]),
    "llr_dwt3_axis_dev": (C.c_int, [P, P, PU32, PU32, U32, U32, P, P, PI32, P]),
    "llr_idwt3_axis_dev": (C.c_int, [P, P, PU32, PU32, U32, U32, P, P, PI32, P]),
    "dwt3_axis": (C.c_int, [P, P, PU32, PU32, C.c_uint, C.c_uint, P, P, P]),
    "idwt3_axis": (C.c_int, [P, P, PU32, PU32, C.c_uint, C.c_uint, P, P, P]),
    "llr_wavelet_denoise_dev": (C.c_int, [P, PI32, I32, I32, I32, F32, P]),
    "llr_hard_project_dev": (C.c_int, [P, P, I64, PF64, P]),
    "llr_cu_low_rank_approx_batch": (C.c_int, [SZ, SZ, SZ, SZ, P]),
    "llr_signal_model": (C.c_int, [P, PSZ, SZ, PF32, PF32, I32]),
    "llr_lift_data_set": (C.c_int, [P, SZ, P, PSZ, PSZ, PSZ, SZ, SZ]),
    "llr_un_lift_data_set": (C.c_int, [P, SZ, P, PSZ, PSZ, PSZ, SZ, SZ]),
    "llr_dti_project": (C.c_int, [P, P, P, SZ, SZ, SZ, SZ]),
    "llr_dti_back_project": (C.c_int, [P, P, P, SZ, SZ, SZ, SZ]),
    "llr_cu_dwt_denoise": (C.c_int, [P, PSZ, PF32, PF32, PF32, PF32, SZ, PI32]),
    "llr_host_alloc": (C.c_int, [SZ, C.POINTER(P)]),
    "llr_host_free": (C.c_int, [P]),
    "llr_device_alloc": (C.c_int, [SZ, C.POINTER(P)]),
    "llr_device_free": (C.c_int, [P]),
    "llr_memcpy_h2d": (C.c_int, [P, P, SZ, P]),
    "llr_memcpy_d2h": (C.c_int, [P, P, SZ, P]),
    "llr_stream_sync": (C.c_int, [P]),
    "llr_device_count": (C.c_int, [PI32]),
    "llr_cfl_dims": (C.c_int, [C.c_char_p, C.POINTER(I64), I32, PI32]),
    "llr_cfl_read": (C.c_int, [C.c_char_p, P, I64]),
    "llr_cfl_write": (C.c_int, [C.c_char_p, C.POINTER(I64), I32, P]),
    "llr_read_b_table": (C.c_int, [C.c_char_p, I32, PF32, PF32]),
    "llr_b0_mask": (C.c_int, [PF32, I32, C.c_float, P]),
    "llr_read_affine_translation": (C.c_int, [C.c_char_p, C.c_float, PF32]),
    "llr_dti_fit_dev": (C.c_int, [P, I32, P, I32, I64, PF32, PF32, P, P]),
    "llr_dti_subspace": (C.c_int, [PF32, PF32, I32, I32, I64, U64, C.c_float, C.c_float, P, PF64]),
    "llr_dti_fit": (C.c_int, [P, I32, P, I32, I64, PF32, PF32, PF32]),
    "llr_cnn_create": (C.c_int, [I32, PI32, I32, U64, C.POINTER(P)]),
    "llr_cnn_destroy": (C.c_int, [P]),
    "llr_cnn_param_count": (C.c_int, [P, C.POINTER(I64)]),
    "llr_cnn_get_params": (C.c_int, [P, P]),
    "llr_cnn_set_params": (C.c_int, [P, P]),
    "llr_cnn_get_grads": (C.c_int, [P, P]),
    "llr_cnn_forward_dev": (C.c_int, [P, P, P, PI32, P]),
    "llr_cnn_loss_grad_dev": (C.c_int, [P, P, P, PI32, PF64, P]),
    "llr_cnn_adam_step": (C.c_int, [P, C.c_float, C.c_float, C.c_float, C.c_float, P]),
    "llr_cnn_train_step_dev": (C.c_int, [P, P, P, PI32, C.c_float, PF64, P]),
    "llr_subspace_channels_dev": (C.c_int, [P, PI32, I32, P, I32, C.c_float, P, P, P]),
    "llr_subspace_image_dev": (C.c_int, [P, PI32, I32, P, I32, C.c_float, P, I32, P, P]),
}


class LlrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"llr status {status}: {message}")
        self.status = status


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `make -C llr-reco_b200` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != LLR_OK:
        raise LlrError(status, lib.llr_last_error().decode(errors="replace"))


def i32x3(v) -> C.Array:
    return (C.c_int32 * 3)(*[int(a) for a in v])


def u32x3(v) -> C.Array:
    return (C.c_uint32 * 3)(*[int(a) for a in v])


def szx3(v) -> C.Array:
    return (C.c_size_t * 3)(*[int(a) for a in v])


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def fptr(a: np.ndarray):
    return a.ctypes.data_as(PF32)
