"""C-ABI checks that need no GPU: the library loads, exports every declared symbol, and its
host-only functions (config, RNG, masks, filters) agree with the oracle bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import llr_oracle as O

import llr_b200
from llr_b200 import _lib as L


def header_functions():
    text = open(os.path.join(ROOT, "include", "llr_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


def test_library_exports_every_header_symbol():
    names = header_functions()
    assert len(names) > 50
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)


def test_library_is_built_for_sm100a():
    assert b"sm_100a" in L.lib.llr_version()


def test_config_default_mirrors_reference():
    """LlrReconParams::default (lib.rs:67-81)."""
    c = L.llr_config()
    L.check(L.lib.llr_config_default(C.byref(c)))
    assert list(c.block_size) == [32, 32, 32]
    assert c.rank == 6 and c.n_iter == 60
    assert abs(c.wavelet_alpha - 0.005) < 1e-9
    assert c.fft_max_batch_size == 200 and c.cas_mat_max_batch_size == 200
    assert c.prox_mode == L.LLR_PROX_HARD_RANK and c.wavelet_moments == 2


def _cfg(**kw):
    p = llr_b200.ReconParams(vol_size=(32, 32, 32), nq=10, block_size=(8, 8, 8), rank=3)
    for k, v in kw.items():
        setattr(p, k, v)
    return p.to_c()


@pytest.mark.parametrize("kw,msg", [
    (dict(rank=0), "rank should not be less than 1"),
    (dict(rank=11), "rank must not exceed n"),
    (dict(block_size=(40, 8, 8)), "block dimension"),
    (dict(nq=0), "nq"),
    (dict(max_rand_shift=(33, 1, 1)), "max_rand_shift"),
    (dict(subspace_rank=11), "subspace rank"),
    (dict(eig_solver=2), "eig_solver"),
    (dict(gram_mode=2), "gram_mode"),
    (dict(fft_mode=2), "fft_mode"),
])
def test_config_validation_errors(kw, msg):
    c = _cfg(**kw)
    st = L.lib.llr_config_validate(C.byref(c))
    assert st == L.LLR_ERR_INVALID
    assert msg in L.lib.llr_last_error().decode()


def test_config_validation_ok():
    c = _cfg()
    assert L.lib.llr_config_validate(C.byref(c)) == L.LLR_OK


def test_status_strings():
    assert L.lib.llr_status_string(0) == b"ok"
    assert L.lib.llr_status_string(-7) == b"unsupported shape"


def test_rand_shift_bit_exact_with_oracle():
    for seed in (0, 1, 12345, 2 ** 63 + 17):
        for it in range(0, 400, 7):
            mx = (192, 192, 96)
            assert llr_b200.rand_shift(seed, it, mx) == O.rand_shift(seed, it, mx)


@pytest.mark.parametrize("ny,nz,nq,R,centre,seed", [(64, 64, 3, 4.0, 16, 0), (48, 30, 2, 8.0, 8, 77),
                                                   (20, 16, 2, 2.0, 0, 5)])
def test_vd_mask_bit_exact_with_oracle(ny, nz, nq, R, centre, seed):
    a = llr_b200.vd_mask(ny, nz, nq, R, centre, seed)
    b = O.vd_mask(ny, nz, nq, R, centre, seed)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 6, 8])
def test_daubechies_filters_match_oracle(order):
    lo_d, hi_d, lo_r, hi_r = llr_b200.daubechies_filters(order)
    bank = O.daubechies_bank(order)
    for a, b in ((lo_d, bank.lo_d), (hi_d, bank.hi_d), (lo_r, bank.lo_r), (hi_r, bank.hi_r)):
        np.testing.assert_allclose(a, b, atol=2e-7)


def test_grid_dim():
    out = L.i32x3((0, 0, 0))
    L.check(L.lib.llr_grid_dim(L.i32x3((788, 480, 480)), L.i32x3((32, 32, 32)), out))
    assert list(out) == [24, 15, 15]


def test_estimate_linear_corrections_matches_oracle():
    rng = np.random.default_rng(0)
    vol = (9, 8, 6)
    y = np.asfortranarray((rng.standard_normal(vol + (3,)) + 1j * rng.standard_normal(vol + (3,))).astype(np.complex64))
    y[4, 2, 5, 1] = 50  # clear peak
    out = np.zeros(9, dtype=np.float32)
    L.check(L.lib.llr_estimate_linear_corrections(L.ptr(y), L.i32x3(vol), 3, L.fptr(out)))
    for q in range(3):
        np.testing.assert_array_equal(out[3 * q:3 * q + 3], O.estimate_linear_correction(y[..., q]))


def test_context_without_device_reports_no_device():
    if llr_b200.device_count() > 0:
        pytest.skip("a CUDA device is present")
    c = _cfg()
    h = C.c_void_p()
    st = L.lib.llr_ctx_create(C.byref(c), C.byref(h))
    assert st == L.LLR_ERR_NO_DEVICE


def test_product_package_does_not_import_oracle():
    pkg = os.path.join(ROOT, "llr-reco_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert not re.search(r"^\s*(import|from)\s+oracle", txt, flags=re.M), os.path.join(dirpath, f)
                assert "llr_oracle" not in txt, os.path.join(dirpath, f)
