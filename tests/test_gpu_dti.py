"""DTI scalar maps on the GPU (llr_dti_fit, llr-dti-scalars) against the FP64 oracle
(diffusion_models.rs:21-129)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, rel_err
from oracle import llr_oracle as O

pytestmark = pytest.mark.gpu


def _fit(dwi, b0, b, g):
    from llr_b200 import _lib as L
    V, nq = dwi.shape
    nb0 = b0.shape[1]
    out = np.empty((7, V), dtype=np.float32)
    dwi = np.asfortranarray(dwi.astype(np.complex64))
    b0 = np.asfortranarray(b0.astype(np.complex64))
    bb = np.ascontiguousarray(b, dtype=np.float32)
    gg = np.ascontiguousarray(g, dtype=np.float32)
    L.check(L.lib.llr_dti_fit(L.ptr(dwi), nq, L.ptr(b0) if nb0 else None, nb0, V, L.fptr(bb), L.fptr(gg), L.fptr(out)))
    return dict(zip(["b0av", "e1", "e2", "e3", "md", "rd", "fa"], out))


def test_dti_fit_matches_oracle_on_phantom(gpu):
    from llr_b200.phantom import make_dataset
    d = make_dataset((20, 20, 10), [(0, 3), (1000, 30), (2000, 30)], 2.0, 4, centre=4)
    x = d.x_true.reshape(-1, d.x_true.shape[3], order="F")
    rng = np.random.default_rng(1)
    x = x + 0.01 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    dwi, b0 = x[:, d.b > 0], x[:, d.b == 0]
    got = _fit(dwi, b0, d.b[d.b > 0], d.g[d.b > 0])
    exp = O.dti_fit(dwi.astype(np.complex64).astype(np.complex128), b0.astype(np.complex64).astype(np.complex128),
                    d.b[d.b > 0], d.g[d.b > 0])
    for k in ("b0av", "e1", "e2", "e3", "md", "rd"):
        assert rel_err(got[k], exp[k]) < 1e-4, k
    ok = np.isfinite(exp["fa"])
    assert np.array_equal(np.isfinite(got["fa"]), ok)
    assert np.max(np.abs(got["fa"][ok] - exp["fa"][ok])) < 1e-3


def test_dti_fit_noise_free_tensor(gpu):
    from llr_b200.phantom import b_table, eigenvector_matrix, sample_unit_sphere, tensor_signal
    rng = np.random.default_rng(2)
    b, g = b_table([(0, 2), (1000, 15), (2000, 15)], rng)
    R = eigenvector_matrix(sample_unit_sphere(0.3, 0.7))
    D = R @ np.diag([1.7e-3, 0.5e-3, 0.3e-3]) @ R.T
    s = tensor_signal(np.array([0.8, 0.0]), np.stack([D, D]), b, g)     # second voxel: zero signal
    got = _fit(s[:, b > 0], s[:, b == 0], b[b > 0], g[b > 0])
    np.testing.assert_allclose([got["e1"][0], got["e2"][0], got["e3"][0]], [1.7e-3, 0.5e-3, 0.3e-3], rtol=2e-4)
    assert got["b0av"][1] == 0.0


def test_dti_scalars_cli(gpu, tmp_path):
    from llr_b200.cfl import read_cfl, write_cfl
    from llr_b200.phantom import make_dataset
    exe = os.path.join(PKG, "llr-dti-scalars")
    d = make_dataset((12, 10, 8), [(0, 2), (1000, 12)], 2.0, 5, centre=4)
    n = d.x_true.shape[3]
    for q in range(n):
        write_cfl(str(tmp_path / f"v{q:02d}"), d.x_true[..., q])
    with open(tmp_path / "bt.txt", "w") as f:
        for bv, gv in zip(d.b, d.g):
            f.write(f"{bv:g} {gv[0]:.9f} {gv[1]:.9f} {gv[2]:.9f}\n")
    out = tmp_path / "maps"
    out.mkdir()
    r = subprocess.run([exe, str(tmp_path), "v*", str(tmp_path / "bt"), str(out), str(n)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    x = d.x_true.reshape(-1, n, order="F")
    exp = _fit(x[:, d.b > 0], x[:, d.b == 0], d.b[d.b > 0], d.g[d.b > 0])
    for k in ("b0av", "e1", "md", "fa"):
        m = read_cfl(str(out / k)).reshape(-1, order="F")
        assert np.all(m.imag == 0)
        np.testing.assert_allclose(m.real, exp[k], rtol=1e-6)   # the b-table went through text
