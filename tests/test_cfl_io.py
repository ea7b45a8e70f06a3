"""Data-set files without a GPU: CFL volumes (the cfl crate's format used by the reference's
dataset builder and writer, data_import.rs:67-108, lib.rs:353-362), the b-table reader
(data_import.rs:110-145), the b0 mask (data_import.rs:322-328), and the llr-recon driver's
input handling up to the point where it needs a GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG


def _write_cfl_py(base, a):
    """Reference writer restated from the format: text header, raw complex64 column-major."""
    with open(base + ".hdr", "w") as f:
        f.write("# Dimensions\n" + " ".join(str(d) for d in a.shape) + "\n")
    np.asfortranarray(a, dtype=np.complex64).ravel(order="F").tofile(base + ".cfl")


def test_cfl_round_trip_both_ways(tmp_path):
    from llr_b200.cfl import cfl_dims, read_cfl, write_cfl
    rng = np.random.default_rng(0)
    a = (rng.standard_normal((5, 4, 3, 2)) + 1j * rng.standard_normal((5, 4, 3, 2))).astype(np.complex64)
    p = str(tmp_path / "vol")
    write_cfl(p, a)
    assert open(p + ".hdr").read().split("\n")[:2] == ["# Dimensions", "5 4 3 2"]
    raw = np.fromfile(p + ".cfl", dtype=np.complex64)
    np.testing.assert_array_equal(raw, a.ravel(order="F"))
    q = str(tmp_path / "ref")
    _write_cfl_py(q, a[:, :, :, 1:])
    assert cfl_dims(q + ".cfl") == (5, 4, 3, 1)
    np.testing.assert_array_equal(read_cfl(q), a[:, :, :, 1:])


def test_cfl_errors(tmp_path):
    from llr_b200 import LlrError
    from llr_b200.cfl import read_cfl
    p = str(tmp_path / "short")
    with open(p + ".hdr", "w") as f:
        f.write("# Dimensions\n4 4\n")
    np.zeros(10, dtype=np.complex64).tofile(p + ".cfl")
    with pytest.raises(LlrError):
        read_cfl(p)
    with pytest.raises(LlrError):
        read_cfl(str(tmp_path / "missing"))


def test_b_table_and_b0_mask(tmp_path):
    from llr_b200 import LlrError
    from llr_b200.cfl import b0_mask, read_b_table
    p = tmp_path / "btab.txt"
    p.write_text("0 0 0 0\n1000 1 0 0\n1000 0 0.6 0.8\n5 0.001 0 0\n")
    b, g = read_b_table(str(tmp_path / "btab"), 4)                 # ".txt" appended
    np.testing.assert_array_equal(b, [0, 1000, 1000, 5])
    np.testing.assert_allclose(g[2], [0, 0.6, 0.8])
    np.testing.assert_array_equal(b0_mask(g, 0.0), [True, False, False, False])
    np.testing.assert_array_equal(b0_mask(g, 0.01), [True, False, False, True])
    with pytest.raises(LlrError):
        read_b_table(str(p), 5)
    (tmp_path / "bad.txt").write_text("0 0 0 x\n")
    with pytest.raises(LlrError):
        read_b_table(str(tmp_path / "bad.txt"), 1)


def _cli():
    exe = os.path.join(PKG, "llr-recon")
    if not os.path.exists(exe):
        pytest.skip("llr-recon not built")
    return exe


def test_cli_reports_bad_inputs(tmp_path):
    exe = _cli()
    r = subprocess.run([exe, str(tmp_path / "none"), str(tmp_path), "vol*", str(tmp_path), "out", "bt"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "failed to open config file" in r.stderr
    (tmp_path / "p.toml").write_text("llr_block_size = [4, 4, 4]\nbogus = 1\n")
    r = subprocess.run([exe, str(tmp_path / "p"), str(tmp_path), "vol*", str(tmp_path), "out", "bt"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "unknown recon parameter: bogus" in r.stderr
    (tmp_path / "p.toml").write_text("llr_block_size = [4, 4, 4]\nn_iter = 2\n")
    r = subprocess.run([exe, str(tmp_path / "p"), str(tmp_path), "vol*", str(tmp_path), "out", "bt"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "no files found" in r.stderr


def test_affine_translation_reader(tmp_path):
    """read_affine_translation (signal_model.rs:119-176): translation = entries 9..11 of the first
    "Parameters:" line, times the multiplier."""
    from llr_b200 import LlrError
    from llr_b200.cfl import read_affine_translations
    p = tmp_path / "a0.txt"
    p.write_text("#Insight Transform File V1.0\n#Transform 0\nTransform: AffineTransform_double_3_3\n"
                 "Parameters: 1 0 0 0 1 0 0 0 1 1.5 -2 0.25\nFixedParameters: 0 0 0\n")
    q = tmp_path / "a1.txt"
    q.write_text("Parameters: 0.9 0.1 0 -0.1 0.9 0 0 0 1 3 4 5\nParameters: 9 9 9 9 9 9 9 9 9 9 9 9\n")
    t = read_affine_translations([p, q], 2.0)
    np.testing.assert_allclose(t, [[3.0, -4.0, 0.5], [6.0, 8.0, 10.0]])
    (tmp_path / "bad.txt").write_text("Parameters: 1 2 3\n")
    with pytest.raises(LlrError):
        read_affine_translations([tmp_path / "bad.txt"])
    (tmp_path / "none.txt").write_text("FixedParameters: 0 0 0\n")
    with pytest.raises(LlrError):
        read_affine_translations([tmp_path / "none.txt"])
