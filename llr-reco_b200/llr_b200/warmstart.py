"""Learned warm start of the plain LLR reconstruction.

The network (llr_b200.cnn, trained with the library's own conv3d kernels) maps the temporal-
subspace coefficients of the adjoint (zero-filled) image to those of the converged plain
reconstruction.  Its output, taken back through S^H, starts the same proximal-gradient LLR
iteration, so the final answer is still the method's own fixed point.  The comparison this
module measures is the one the learned start is for: iterations and device time until the
iterate is within a relative RMS error of the converged image, from the zero-filled start and
from the network's start (network time included).

The comparison runs with a fixed block partition (no random shift): with a new random shift
every iteration the iterate keeps moving by a few per cent per iteration and there is no
single converged image to measure against.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import check, lib
from ._lib import LLR_PROX_SOFT_THRESH
from .api import DeviceBuffer, ReconContext, ReconParams
from .cnn import Cnn, DeviceArray, subspace_channels_dev, subspace_image_dev
from .phantom import PROTOCOL_SEED, b_table, dti_subspace, make_dataset


@dataclass
class Protocol:
    """Acquisition and reconstruction settings shared by every subject."""
    vol: tuple = (48, 48, 48)
    shells: list = field(default_factory=lambda: [(0, 7), (3000, 54)])
    accel: float = 8.0
    block: tuple = (6, 6, 6)
    centre: int = 12
    lam_rel: float = 0.02
    srank: int = 7
    protocol_seed: int = PROTOCOL_SEED
    recon_seed: int = 3
    fixed_partition: bool = True
    gram_mode: int = 0
    demodulate: bool = True     # channels of the phase-demodulated image (phase of the calibration image)

    @property
    def nq(self) -> int:
        return int(sum(c for _, c in self.shells))

    def subspace(self) -> np.ndarray:
        b, g = b_table(self.shells, np.random.default_rng(self.protocol_seed))
        return dti_subspace(b, g, self.srank, 100000, self.protocol_seed + 1)

    def params(self, lam: float = 0.0) -> ReconParams:
        return ReconParams(vol_size=tuple(self.vol), nq=self.nq, block_size=tuple(self.block),
                           prox_mode=LLR_PROX_SOFT_THRESH, lam=lam, seed=self.recon_seed,
                           max_rand_shift=(1, 1, 1) if self.fixed_partition else None,
                           gram_mode=self.gram_mode)

    def subject(self, seed: int):
        return make_dataset(self.vol, self.shells, self.accel, seed, centre=self.centre,
                            protocol_seed=self.protocol_seed)


def nrmse(x: np.ndarray, ref: np.ndarray) -> float:
    return float(np.linalg.norm((x - ref).ravel()) / np.linalg.norm(ref.ravel()))


def reference(proto: Protocol, y: np.ndarray, n_iter: int, snapshot: bool = False):
    """Zero-filled image, lambda = lam_rel * sigma_max of it, the plain recon after n_iter and the
    measured k-space energy; with ``snapshot`` also a device copy of the final iterate."""
    with ReconContext(proto.params()) as ctx:
        ctx.upload_kspace(y)
        ctx.init_zero_filled()
        x_zf = ctx.download_image()
        lam = proto.lam_rel * ctx.sigma_max((0, 0, 0))
        ctx.set_lambda(lam)
        ctx.iterate(n_iter)
        energy = ctx.measurement_stats()[0]
        if snapshot:
            return x_zf, ctx.download_image(), lam, energy, ctx.snapshot()
        return x_zf, ctx.download_image(), lam, energy


def calibration_kspace(proto: Protocol, y: np.ndarray) -> np.ndarray:
    """The fully sampled k-space centre of y (|ky - ny/2|, |kz - nz/2| < centre/2, every x), zero
    elsewhere."""
    nx, ny, nz, nq = y.shape
    h = proto.centre // 2
    yc = np.zeros(y.shape, dtype=np.complex64, order="F")
    sl = (slice(None), slice(ny // 2 - h, ny // 2 + h), slice(nz // 2 - h, nz // 2 + h), slice(None))
    yc[sl] = y[sl]
    return yc


def calibration_image(proto: Protocol, y: np.ndarray) -> Optional[DeviceBuffer]:
    """Device image A^H of the calibration k-space: a low-resolution reconstruction whose phase is
    the smooth phase of each volume.  The network works on the temporal-subspace coefficients of
    the image demodulated by this phase, since every volume carries its own phase and a real
    subspace cannot hold it (None: no demodulation)."""
    if not proto.demodulate:
        return None
    d = DeviceBuffer.from_array(calibration_kspace(proto, y))
    check(lib.llr_signal_model_dev(d.ptr, L.i32x3(proto.vol), proto.nq, None, None, L.LLR_INVERSE, None))
    check(lib.llr_stream_sync(None))
    return d


def channel_scale(proto: Protocol, energy: float) -> float:
    """Unit-RMS channels: the coefficients carry about the image energy (A is unitary)."""
    V = int(np.prod(proto.vol))
    return float(np.sqrt(V * 2 * proto.srank / max(energy, 1e-30)))


class SubspaceCodec:
    """Device-side c = scale * x S (channels) and x = c S^H / scale for one protocol."""

    def __init__(self, proto: Protocol, S: Optional[np.ndarray] = None):
        self.proto = proto
        self.S = proto.subspace() if S is None else S
        self.dS = DeviceBuffer.from_array(np.asfortranarray(self.S.astype(np.complex64)))

    def channels(self, x: np.ndarray, scale: float, ph: Optional[DeviceBuffer] = None) -> DeviceArray:
        p = self.proto
        dx = DeviceBuffer.from_array(x.astype(np.complex64))
        out = DeviceArray((p.vol[2], p.vol[1], p.vol[0], 2 * p.srank))
        subspace_channels_dev(dx.ptr, p.vol, p.nq, self.dS.ptr, p.srank, scale, out, ph.ptr if ph else None)
        check(lib.llr_stream_sync(None))
        dx.close()
        return out

    def image(self, chan: DeviceArray, scale: float, ph: Optional[DeviceBuffer] = None) -> np.ndarray:
        p = self.proto
        dx = DeviceBuffer(8 * int(np.prod(p.vol)) * p.nq)
        subspace_image_dev(chan, p.vol, p.nq, self.dS.ptr, p.srank, scale, dx.ptr, d_phase_ref=ph.ptr if ph else None)
        out = dx.download(np.empty(tuple(p.vol) + (p.nq,), dtype=np.complex64, order="F"))
        dx.close()
        return out


def training_pairs(proto: Protocol, codec: SubspaceCodec, seeds: Sequence[int], n_ref: int):
    """(input channels, target channels) on the device for each training subject."""
    pairs = []
    for s in seeds:
        d = proto.subject(s)
        x_zf, x_ref, _, energy = reference(proto, d.y, n_ref)
        sc = channel_scale(proto, energy)
        ph = calibration_image(proto, d.y)
        pairs.append((codec.channels(x_zf, sc, ph), codec.channels(x_ref, sc, ph)))
        if ph is not None:
            ph.close()
    return pairs


def train(net: Cnn, pairs, epochs: int, lr: float, lr_final: Optional[float] = None) -> list:
    """Adam over the training pairs (one subject per step), cosine-decayed learning rate."""
    losses = []
    steps = max(1, epochs * len(pairs))
    lr_final = lr * 0.05 if lr_final is None else lr_final
    k = 0
    for _ in range(epochs):
        ep = []
        for xin, tgt in pairs:
            a = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * k / steps))
            ep.append(net.train_step_dev(xin, tgt, a))
            k += 1
        losses.append(float(np.mean(ep)))
    return losses


def warm_start_image(net: Cnn, codec: SubspaceCodec, x_zf: np.ndarray, energy: float, y: np.ndarray):
    """Network start image x0 = x_zf + u (c_out - c_in) S^H / scale -- the network corrects the
    demodulated subspace part of the zero-filled image and keeps the rest; u is the unit phase of
    the calibration image -- and the milliseconds of device work producing it (calibration image,
    channels, network, image), measured between stream synchronisations; host copies are outside."""
    import time
    p = codec.proto
    sc = channel_scale(p, energy)
    dx = DeviceBuffer.from_array(x_zf.astype(np.complex64))
    chan = DeviceArray((p.vol[2], p.vol[1], p.vol[0], 2 * p.srank))
    out = DeviceArray(chan.shape)
    # host masking and upload of the calibration lines are data preparation (outside the timing)
    dc = DeviceBuffer.from_array(calibration_kspace(p, y)) if p.demodulate else None
    check(lib.llr_stream_sync(None))
    t0 = time.perf_counter()
    if dc is not None:
        check(lib.llr_signal_model_dev(dc.ptr, L.i32x3(p.vol), p.nq, None, None, L.LLR_INVERSE, None))
    ph = dc.ptr if dc is not None else None
    subspace_channels_dev(dx.ptr, p.vol, p.nq, codec.dS.ptr, p.srank, sc, chan, ph)
    net.forward_dev(chan, out)
    subspace_image_dev(out, p.vol, p.nq, codec.dS.ptr, p.srank, sc, dx.ptr, accumulate=True, d_phase_ref=ph)
    subspace_image_dev(chan, p.vol, p.nq, codec.dS.ptr, p.srank, -sc, dx.ptr, accumulate=True, d_phase_ref=ph)
    check(lib.llr_stream_sync(None))
    ms = 1e3 * (time.perf_counter() - t0)
    x0 = dx.download(np.empty_like(x_zf, dtype=np.complex64, order="F"))
    for b in (dx, chan, out, dc):
        if b is not None:
            b.close()
    return x0, ms


def time_to_targets(proto: Protocol, y: np.ndarray, lam: float, x_start: np.ndarray, snap,
                    targets: Sequence[float], max_iter: int, chunk: int = 10):
    """For each target t: (iterations, device ms) until the relative RMS distance of the iterate
    to the reference snapshot (ReconContext.snapshot of the converged run) is <= t, or None.
    The distance is taken on the device between chunks of ``chunk`` timed iterations."""
    res = {t: None for t in targets}
    curve = []
    with ReconContext(proto.params(lam)) as ctx:
        ctx.upload_kspace(y)
        ctx.upload_image(x_start)
        ctx.iteration = 0
        it, ms = 0, 0.0
        e = ctx.nrmse(snap)
        curve.append((0, e))
        for t in targets:
            if e <= t:
                res[t] = (0, 0.0)
        while it < max_iter and any(v is None for v in res.values()):
            ms += ctx.iterate_timed(chunk)
            it += chunk
            e = ctx.nrmse(snap)
            curve.append((it, e))
            for t in targets:
                if res[t] is None and e <= t:
                    res[t] = (it, ms)
    return res, curve


def default_weights_path() -> str:
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warm_start_net.npz")


def main(argv=None) -> None:
    """python -m llr_b200.warmstart train: builds adjoint -> converged pairs with the plain
    recon and trains the network on the GPU; writes the parameters and the protocol."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("cmd", choices=["train"])
    ap.add_argument("--out", default=default_weights_path())
    ap.add_argument("--vol", type=int, nargs=3, default=[96, 96, 48])
    ap.add_argument("--centre", type=int, default=8)
    ap.add_argument("--subjects", type=int, default=32)
    ap.add_argument("--n-ref", type=int, default=600)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=5)
    a = ap.parse_args(argv)
    proto = Protocol(vol=tuple(a.vol), centre=a.centre)
    codec = SubspaceCodec(proto)
    t0 = time.time()
    pairs = training_pairs(proto, codec, list(range(1000, 1000 + a.subjects)), a.n_ref)
    t1 = time.time()
    net = Cnn(seed=a.seed)
    losses = train(net, pairs, a.epochs, a.lr)
    t2 = time.time()
    import os
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    info = dict(vol=list(proto.vol), centre=proto.centre, subjects=a.subjects, n_ref=a.n_ref, epochs=a.epochs,
                lr=a.lr, seed=a.seed, protocol_seed=proto.protocol_seed, srank=proto.srank,
                loss_first=losses[0], loss_last=losses[-1], pairs_s=round(t1 - t0, 1), train_s=round(t2 - t1, 1))
    np.savez(a.out, channels=np.asarray(net.channels, dtype=np.int32), params=net.params,
             info=np.asarray(json.dumps(info)))
    print(json.dumps(info))


if __name__ == "__main__":
    main()
