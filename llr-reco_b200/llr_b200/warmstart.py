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
import json
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


def start_state(proto: Protocol, y: np.ndarray):
    """Zero-filled image, lambda = lam_rel * sigma_max of it and the measured k-space energy."""
    with ReconContext(proto.params()) as ctx:
        ctx.upload_kspace(y)
        ctx.init_zero_filled()
        return ctx.download_image(), proto.lam_rel * ctx.sigma_max((0, 0, 0)), ctx.measurement_stats()[0]


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


def _synth_kspace(args):
    """Worker of the synthesis pool: the measured k-space of one subject (host only)."""
    vol, shells, accel, seed, centre, protocol_seed = args
    return make_dataset(vol, shells, accel, seed, centre=centre, protocol_seed=protocol_seed).y


def subject_stream(proto: Protocol, seeds: Sequence[int], workers: int):
    """Yields (seed, y) in order; the phantoms are synthesised on ``workers`` host processes
    (started with spawn, so they hold no CUDA state) while the caller uses the GPU.  At most
    ``workers`` finished or running subjects are outstanding, which bounds host memory."""
    args = [(tuple(proto.vol), proto.shells, proto.accel, int(s), proto.centre, proto.protocol_seed) for s in seeds]
    if workers <= 1:
        for a in args:
            yield a[3], _synth_kspace(a)
        return
    import collections
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(workers) as pool:
        pending = collections.deque()
        nxt = 0
        while nxt < len(args) or pending:
            while nxt < len(args) and len(pending) < workers:
                pending.append((args[nxt][3], pool.apply_async(_synth_kspace, (args[nxt],))))
                nxt += 1
            seed, res = pending.popleft()
            yield seed, res.get()


def objective_run(proto: Protocol, y: np.ndarray, lam: float, x_start: Optional[np.ndarray], n_iter: int,
                  gram_mode: Optional[int] = None):
    """n_iter fixed-partition iterations from x_start (None: the zero-filled image); returns the
    objective of every iteration (FP64, ReconContext.objective_history) and the device ms."""
    p = proto.params(lam)
    if gram_mode is not None:
        p.gram_mode = gram_mode
    with ReconContext(p) as ctx:
        ctx.upload_kspace(y)
        if x_start is None:
            ctx.init_zero_filled()
        else:
            ctx.upload_image(x_start)
        ctx.iteration = 0
        ms = ctx.iterate_timed(n_iter)
        obj = ctx.objective_history(n_iter)
    return obj, ms


def iterations_to(obj: np.ndarray, f_star: float, tol: float) -> Optional[int]:
    """First iteration count k with F_k <= F* + tol |F*| (None: never within the run)."""
    hit = np.flatnonzero(obj <= f_star + tol * abs(f_star))
    return int(hit[0]) + 1 if hit.size else None


def protocol_eval(net: Cnn, proto: Protocol, codec: SubspaceCodec, seeds: Sequence[int], n_conv: int, tol: float,
                  workers: int, log=print) -> dict:
    """The learned start judged on held-out subjects: for each, the plain FP32 method (FMA Gram)
    and the mixed-precision method (3xTF32 tensor-core Gram) from the zero-filled image, and the
    mixed method from the network's image, each run n_conv fixed-partition iterations; F* is the
    lowest objective any of the three reached; reported are the iterations and device seconds
    until F_k <= F* + tol |F*| (the network's time included in the learned run)."""
    per = []
    for seed, y in subject_stream(proto, seeds, workers):
        x_zf, lam, energy = start_state(proto, y)
        x0, net_ms = warm_start_image(net, codec, x_zf, energy, y)
        runs = {"plain_fp32": objective_run(proto, y, lam, None, n_conv, gram_mode=1),
                "plain_mixed": objective_run(proto, y, lam, None, n_conv, gram_mode=0),
                "learned_mixed": objective_run(proto, y, lam, x0, n_conv, gram_mode=0)}
        f_star = min(float(np.nanmin(o)) for o, _ in runs.values())
        rec = {"seed": int(seed), "f_star": f_star, "network_ms": round(net_ms, 3),
               "tail_change": float(abs(runs["plain_mixed"][0][-101] - runs["plain_mixed"][0][-1]) / abs(f_star))}
        for name, (o, ms) in runs.items():
            k = iterations_to(o, f_star, tol)
            t_it = ms / n_conv
            extra = net_ms if name == "learned_mixed" else 0.0
            rec[name] = {"iterations": k, "ms_per_iteration": round(t_it, 4),
                         "seconds": None if k is None else round(1e-3 * (k * t_it + extra), 5),
                         "start_gap": float((o[0] - f_star) / abs(f_star))}
        log(json.dumps(rec))
        per.append(rec)

    def stat(key, field):
        v = [r[key][field] for r in per if r[key][field] is not None]
        return {"median": float(np.median(v)), "mean": float(np.mean(v)), "n": len(v)} if v else None

    summary = {k: {"iterations": stat(k, "iterations"), "seconds": stat(k, "seconds")}
               for k in ("plain_fp32", "plain_mixed", "learned_mixed")}
    ratios = [r["plain_fp32"]["seconds"] / r["learned_mixed"]["seconds"] for r in per
              if r["plain_fp32"]["seconds"] and r["learned_mixed"]["seconds"]]
    it_ratio = [r["plain_mixed"]["iterations"] / r["learned_mixed"]["iterations"] for r in per
                if r["plain_mixed"]["iterations"] and r["learned_mixed"]["iterations"]]
    summary["speedup_learned_mixed_vs_plain_fp32"] = {"median": float(np.median(ratios)),
                                                      "min": float(np.min(ratios)), "max": float(np.max(ratios))} \
        if ratios else None
    summary["iteration_ratio_zero_filled_vs_learned"] = {"median": float(np.median(it_ratio)),
                                                         "min": float(np.min(it_ratio)),
                                                         "max": float(np.max(it_ratio))} if it_ratio else None
    summary["learned_fewer_iterations"] = sum(
        1 for r in per if r["plain_mixed"]["iterations"] and r["learned_mixed"]["iterations"]
        and r["learned_mixed"]["iterations"] < r["plain_mixed"]["iterations"])
    return {"subjects": per, "summary": summary}


def run_protocol(a) -> dict:
    """Training on ``a.train`` seeded phantoms reconstructed by the plain method (``a.n_ref``
    fixed-partition iterations), then the held-out evaluation (protocol_eval)."""
    import time
    proto = Protocol(vol=tuple(a.vol), centre=a.centre)
    codec = SubspaceCodec(proto)
    t0 = time.time()
    pairs = []
    for seed, y in subject_stream(proto, range(a.train_seed0, a.train_seed0 + a.train), a.workers):
        x_zf, x_ref, _, energy = reference(proto, y, a.n_ref)
        sc = channel_scale(proto, energy)
        ph = calibration_image(proto, y)
        pairs.append((codec.channels(x_zf, sc, ph), codec.channels(x_ref, sc, ph)))
        if ph is not None:
            ph.close()
    t1 = time.time()
    net = Cnn(seed=a.seed)
    losses = train(net, pairs, a.epochs, a.lr)
    t2 = time.time()
    for xin, tgt in pairs:
        xin.close()
        tgt.close()
    ev = protocol_eval(net, proto, codec, range(a.test_seed0, a.test_seed0 + a.test), a.n_conv, a.tol, a.workers)
    t3 = time.time()
    info = dict(vol=list(proto.vol), shells=proto.shells, accel=proto.accel, block=list(proto.block),
                centre=proto.centre, train_subjects=a.train, n_ref=a.n_ref, epochs=a.epochs, lr=a.lr, seed=a.seed,
                test_subjects=a.test, n_conv=a.n_conv, tol=a.tol, loss_first=losses[0], loss_last=losses[-1],
                pairs_s=round(t1 - t0, 1), train_s=round(t2 - t1, 1), eval_s=round(t3 - t2, 1))
    if a.weights:
        import os
        os.makedirs(os.path.dirname(os.path.abspath(a.weights)), exist_ok=True)
        np.savez(a.weights, channels=np.asarray(net.channels, dtype=np.int32), params=net.params,
                 info=np.asarray(json.dumps(info)))
    net.close()
    return {"protocol": info, **ev}


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
    ap.add_argument("cmd", choices=["train", "protocol"])
    ap.add_argument("--out", default=default_weights_path())
    ap.add_argument("--vol", type=int, nargs=3, default=[96, 96, 48])
    ap.add_argument("--centre", type=int, default=8)
    ap.add_argument("--subjects", type=int, default=32)
    ap.add_argument("--n-ref", type=int, default=600)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=5)
    # protocol: train on --train subjects (--n-ref plain iterations each), judge on --test held-out
    ap.add_argument("--train", type=int, default=200)
    ap.add_argument("--test", type=int, default=20)
    ap.add_argument("--train-seed0", type=int, default=10000)
    ap.add_argument("--test-seed0", type=int, default=20000)
    ap.add_argument("--n-conv", type=int, default=1000)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--workers", type=int, default=0, help="synthesis processes (0: half the host cores, at most 8)")
    ap.add_argument("--weights", default=None, help="protocol: where to write the trained parameters")
    ap.add_argument("--report", default=None, help="protocol: JSON report path")
    a = ap.parse_args(argv)
    if a.cmd == "protocol":
        import os
        if a.workers <= 0:
            a.workers = max(1, min(8, len(os.sched_getaffinity(0)) // 2))
        rep = run_protocol(a)
        txt = json.dumps(rep, indent=1)
        if a.report:
            with open(a.report, "w") as f:
                f.write(txt)
        print(json.dumps({"protocol": rep["protocol"], "summary": rep["summary"]}))
        return
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
