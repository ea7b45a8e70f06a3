"""The allocation-free batched low-rank entry point.

``llr_low_rank_batch_dev_noalloc`` exists for callers that cannot let the library allocate
device memory (their own CUDA-graph replay under a fixed memory plan, a device pool owned by
another framework, a loop that must not pay an allocator call per invocation).  It must give
the same result as ``llr_low_rank_batch_dev``, call after call, since it reuses one static
scratch list.  This file sorts last so that a stop-at-first-failure run has already run every
other test.
"""
import numpy as np
import pytest

from conftest import crandn, rel_err

from llr_b200 import DeviceBuffer, _lib as L
from oracle import llr_oracle as O

pytestmark = pytest.mark.gpu

TOL = 5e-5   # the low-rank prox tolerance used by the other GPU tests


def _batch(rng, m, n, rank, batch):
    U = crandn(rng, (batch, m, rank))
    V = crandn(rng, (batch, rank, n))
    A = np.moveaxis(U @ V, 0, 2) * 3 + 0.3 * crandn(rng, (m, n, batch))
    return np.asfortranarray(A.astype(np.complex64))


@pytest.mark.parametrize("m,n,rank", [(216, 61, 6), (512, 17, 4)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(gpu, m, n, rank):
    rng = np.random.default_rng(31)
    for call in range(2):
        A = _batch(rng, m, n, rank, 40 + 13 * call)
        batch = A.shape[2]
        d_ref, d_new = DeviceBuffer.from_array(A), DeviceBuffer.from_array(A)
        L.check(L.lib.llr_low_rank_batch_dev(m, n, rank, batch, d_ref.ptr, None))
        L.check(L.lib.llr_low_rank_batch_dev_noalloc(m, n, rank, batch, d_new.ptr, None))
        L.check(L.lib.llr_stream_sync(None))
        ref = d_ref.download(np.empty_like(A, order="F"))
        got = d_new.download(np.empty_like(A, order="F"))
        assert np.all(np.isfinite(got))
        assert rel_err(got, ref) <= TOL, (call, rel_err(got, ref))


@pytest.mark.parametrize("m,n,rank", [(216, 61, 20), (64, 40, 24)])
def test_noalloc_static_list_path_on_two_calls(gpu, m, n, rank):
    """Ranks above 16 send every matrix through the static list to the Jacobi kernel: the list
    is filled, read and its count cleared again on the second call (different batch size)."""
    rng = np.random.default_rng(47)
    for call, batch in enumerate((37, 23)):
        A = _batch(rng, m, n, rank, batch)
        d_ref, d_new = DeviceBuffer.from_array(A), DeviceBuffer.from_array(A)
        L.check(L.lib.llr_low_rank_batch_dev(m, n, rank, batch, d_ref.ptr, None))
        L.check(L.lib.llr_low_rank_batch_dev_noalloc(m, n, rank, batch, d_new.ptr, None))
        L.check(L.lib.llr_stream_sync(None))
        ref = d_ref.download(np.empty_like(A, order="F"))
        got = d_new.download(np.empty_like(A, order="F"))
        exact = O.low_rank_hard(A.astype(np.complex128), rank)
        assert np.all(np.isfinite(got))
        assert rel_err(got, ref) <= TOL, (call, rel_err(got, ref))
        assert rel_err(got, exact) <= TOL, (call, rel_err(got, exact))


def test_noalloc_rejects_batches_beyond_its_static_list(gpu):
    d = DeviceBuffer(8 * 4 * 2 * 16)
    st = L.lib.llr_low_rank_batch_dev_noalloc(4, 2, 1, 65537, d.ptr, None)
    assert st == L.LLR_ERR_INVALID
    assert "65536" in L.lib.llr_last_error().decode()
