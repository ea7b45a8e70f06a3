"""llr-recon end to end on the GPU: CFL volumes, b-table, sampling mask and a TOML parameter
file in; reconstructed volumes and error_history.json out -- against the same reconstruction
through the Python host API."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, rel_err

pytestmark = pytest.mark.gpu


def test_cli_matches_api(gpu, tmp_path):
    import llr_b200
    from llr_b200 import ReconContext, ReconParams, _lib as L
    from llr_b200.cfl import read_cfl, write_cfl
    from llr_b200.phantom import make_dataset
    from oracle import llr_oracle as O
    exe = os.path.join(PKG, "llr-recon")
    vol, shells = (24, 24, 12), [(0, 1), (1000, 8)]
    d = make_dataset(vol, shells, 4.0, 7, centre=6, mask_fn=O.vd_mask)
    n_all = d.y.shape[3]
    inp = tmp_path / "in"
    out = tmp_path / "out"
    inp.mkdir()
    out.mkdir()
    for q in range(n_all):
        write_cfl(str(inp / f"vol{q:02d}"), d.y[..., q])
    write_cfl(str(tmp_path / "mask"), d.mask.astype(np.complex64))
    with open(tmp_path / "btab.txt", "w") as f:
        for b, g in zip(d.b, d.g):
            f.write(f"{b:g} {g[0]:.8f} {g[1]:.8f} {g[2]:.8f}\n")
    (tmp_path / "params.toml").write_text(
        "llr_block_size = [6, 6, 6]\nllr_block_rank = 3\nwavelet_shrink_factor = 0.0\nn_iter = 5\n"
        'prox_mode = "soft"\nlambda_rel = 0.02\nseed = 3\n')
    r = subprocess.run([exe, str(tmp_path / "params"), str(inp), "vol*", str(out), "img", str(tmp_path / "btab"),
                        "--sample-mask-cfl", str(tmp_path / "mask")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    dti = [q for q in range(n_all) if d.b[q] > 0]
    got = np.stack([read_cfl(str(out / f"img{q}")) for q in dti], axis=-1)
    hist = json.loads((out / "error_history.json").read_text())
    assert len(hist) == 5

    # the same through the host API
    y = np.asfortranarray(d.y[..., dti] * (d.mask[None, :, :, dti] != 0))
    nq = len(dti)
    lin = np.zeros((nq, 3), dtype=np.float32)
    L.check(L.lib.llr_estimate_linear_corrections(L.ptr(y), L.i32x3(vol), nq, L.fptr(lin)))
    p = ReconParams(vol_size=vol, nq=nq, block_size=(6, 6, 6), prox_mode=llr_b200.LLR_PROX_SOFT_THRESH, rank=3,
                    lam=0.0, seed=3)
    p.wavelet_alpha = 0.0
    with ReconContext(p) as ctx:
        ctx.set_linear_corrections(lin, np.zeros_like(lin))
        ctx.upload_kspace(y)
        ctx.init_zero_filled()
        ctx.set_lambda(0.02 * ctx.sigma_max((0, 0, 0)))
        h = ctx.iterate(5)
        energy = ctx.measurement_stats()[0]
        exp = ctx.download_image()
    assert rel_err(got, exp) < 1e-6
    np.testing.assert_allclose(hist, np.asarray(h) / energy, rtol=1e-9)
