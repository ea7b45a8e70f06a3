#!/usr/bin/env python
"""Benchmark of the LLR reconstruction iteration (iterations per second).

Workload (default ``c2``): 192x192x96 complex64 image x 61 volumes (7 b0 + 54 directions at
b=3000), seeded ellipsoid phantom with smooth phase, 8x variable-density ky-kz line
sampling, complex Gaussian noise at SNR 30, 6x6x6 LLR blocks (Casorati 216 x 61), singular
value soft threshold lambda = 0.02 sigma_max, random block shift per iteration.  One step is
one proximal-gradient iteration (LLR -> A -> hard DC -> A^H) over the whole dataset, with
every input resident in HBM (1.73 GB iterate > 126 MB L2, so no L2 flush is needed).

``--impl reference`` times the reference algorithm's CPU restatement (FP32 numpy/scipy,
all host threads) on a bounded sample per step; the other ranks exit without work.
Multi-GPU runs (torchrun) are independent replicas; value = all ranks' iterations / max
rank time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "llr-reco_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "s to NRMSE≤1e-3 vs FP64 recon: learned+mixed vs plain FP32, 1×B200; it/s"
UNIT = "it/s"


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas only: barrier + max over ranks)
# ---------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(kernel: str, config: str) -> dict | None:
    """DRAM bytes per launch of ``kernel`` at ``config``, as ``--ncu-traffic`` wrote them from an
    ncu capture into profiles/<kernel>_<config>.json (None when no capture was recorded)."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{config}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def _ncu_bytes(value: str, unit: str) -> float:
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12,
             "KB": 1e3, "MB": 1e6, "GB": 1e9, "B": 1.0}
    return float(value.replace(",", "")) * scale.get(unit.strip(), 1.0)


def write_traffic(args) -> None:
    """Sum dram__bytes_read.sum + dram__bytes_write.sum per launch of the kernels matching
    ``--traffic-kernels`` from ``ncu -i <rep> --page raw --csv`` output, scale by
    ``--traffic-scale`` (units processed at the target size / units in the capture) and write
    profiles/<--traffic-name>_<--config>.json."""
    import csv
    with open(args.ncu_traffic) as f:   # ncu's own log lines (==PROF==, ==WARNING==) precede the table
        rows = [r for r in csv.reader([ln for ln in f.read().splitlines() if ln.startswith('"')]) if r]
    head = rows[0]
    units = rows[1]
    ik, ir, iw = head.index("Kernel Name"), head.index("dram__bytes_read.sum"), head.index("dram__bytes_write.sum")
    pat = re.compile(args.traffic_kernels)
    per_kernel: dict[str, list[float]] = {}
    for r in rows[2:]:
        name = r[ik]
        if not pat.search(name):
            continue
        short = re.sub(r"\(.*", "", name).split("::")[-1]
        per_kernel.setdefault(short, []).append(_ncu_bytes(r[ir], units[ir]) + _ncu_bytes(r[iw], units[iw]))
    if not per_kernel:
        raise SystemExit(f"no kernel matching {args.traffic_kernels!r} in {args.ncu_traffic}")
    mean = {k: sum(v) / len(v) for k, v in per_kernel.items()}
    out = {"kernel": args.traffic_name, "config": args.config,
           "captured_on": args.traffic_captured_on or args.config, "scale": args.traffic_scale,
           "per_kernel_captured_bytes": {k: round(v, 1) for k, v in mean.items()},
           "launches_averaged": {k: len(v) for k, v in per_kernel.items()},
           "dram_bytes_per_launch": sum(mean.values()) * args.traffic_scale,
           "source": f"dram__bytes_read.sum + dram__bytes_write.sum from {os.path.basename(args.ncu_traffic)}"}
    path = os.path.join(ROOT, "profiles", f"{args.traffic_name}_{args.config}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out))


# ---------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------
def config_workload(name: str):
    from llr_b200.phantom import CONFIGS
    c = dict(CONFIGS[name])
    return c


def gpu_forward(x: np.ndarray) -> np.ndarray:
    """k-space of the phantom with the library's forward operator (zero corrections)."""
    import llr_b200
    from llr_b200 import DeviceBuffer, _lib as L
    nx, ny, nz, nq = x.shape
    d = DeviceBuffer.from_array(x)
    L.check(L.lib.llr_signal_model_dev(d.ptr, L.i32x3((nx, ny, nz)), nq, None, None, L.LLR_FORWARD, None))
    L.check(L.lib.llr_stream_sync(None))
    out = d.download(np.empty_like(x, order="F"))
    d.close()
    return out


def make_data(name: str, seed: int, use_gpu: bool):
    """Seeded phantom k-space; the b-table is the shared acquisition protocol of the learned
    warm start (so its temporal subspace is the one the network was trained in)."""
    from llr_b200.phantom import PROTOCOL_SEED, make_dataset
    c = config_workload(name)
    return c, make_dataset(c["vol"], c["shells"], c["accel"], seed, centre=16,
                           forward=gpu_forward if use_gpu else None, protocol_seed=PROTOCOL_SEED)


def warm_start_headline(args, c, d) -> dict:
    """Wall (device) time to NRMSE <= 1e-3 against the converged plain recon, from the zero-filled
    start with the FP32 FMA Gram (plain FP32) and from the learned start with the 3xTF32
    tensor-core Gram (learned + mixed), on the same data.  Fixed block partition (with a new
    random shift each iteration there is no single converged image)."""
    import dataclasses
    from llr_b200 import warmstart as W
    from llr_b200.cnn import Cnn
    path = W.default_weights_path()
    if not os.path.exists(path):
        return {"error": "no trained network; run python -m llr_b200.warmstart train"}
    plain = W.Protocol(vol=tuple(c["vol"]), shells=list(c["shells"]), accel=c["accel"], block=tuple(c["block"]),
                       centre=16, gram_mode=1)
    mixed = dataclasses.replace(plain, gram_mode=0)
    x_zf, _, lam, energy, snap = W.reference(plain, d.y, args.ws_ref_iters, snapshot=True)
    codec = W.SubspaceCodec(mixed)
    net = Cnn.load(path)
    W.warm_start_image(net, codec, x_zf, energy, d.y)            # warm-up (workspace, attributes)
    x0, net_ms = W.warm_start_image(net, codec, x_zf, energy, d.y)
    net.close()
    targets = [1e-2, 1e-3]
    rp, cp = W.time_to_targets(plain, d.y, lam, x_zf, snap, targets, args.ws_ref_iters, chunk=10)
    rl, cl = W.time_to_targets(mixed, d.y, lam, x0, snap, targets, args.ws_ref_iters, chunk=10)
    snap.close()
    out = {"metric": "device seconds to NRMSE <= 1e-3 vs the converged plain FP32 recon",
           "reference": f"plain FP32 (FMA Gram), zero-filled start, {args.ws_ref_iters} iterations, fixed partition",
           "start_nrmse": {"zero_filled": round(cp[0][1], 5), "learned": round(cl[0][1], 5)},
           "network_ms": round(net_ms, 3)}
    for t in targets:
        p, l = rp[t], rl[t]
        key = f"to_{t:g}"
        out[key] = {"plain_fp32": None if p is None else {"iterations": p[0], "s": round(p[1] / 1e3, 4)},
                    "learned_mixed": None if l is None else {"iterations": l[0],
                                                             "s": round((l[1] + net_ms) / 1e3, 4)}}
        if p is not None and l is not None:
            out[key]["speedup"] = round(p[1] / (l[1] + net_ms), 3)
    return out


def bench_config(name: str, c: dict, nq: int, world: int) -> dict:
    """The ``config`` object both arms print (identical for the same --config and N)."""
    nx, ny, nz = c["vol"]
    E = nx * ny * nz * nq
    return {"workload": workload_label(name, c, nq), "vol": list(c["vol"]), "nq": nq, "block": list(c["block"]),
            "accel": c["accel"], "lambda_rule": "0.02 x largest block singular value of the zero-filled image, shift 0",
            "l2": f"no flush: the {8 * E / 1e9:.2f} GB iterate exceeds the 126 MB L2" if 8 * E > 126e6 else
                  f"flushed: a 512 MB buffer is written before every timed iteration (the {8 * E / 1e6:.1f} MB "
                  f"iterate fits the 126 MB L2)",
            "parallelism": f"replicas x{world}"}


def workload_label(name: str, c: dict, nq: int) -> str:
    v = c["vol"]
    b = c["block"]
    n = c.get("srank", nq)
    extra = ""
    if "srank" in c:
        where = "subspace coefficient volumes" if c.get("wavelet_space", 0) else "image volumes"
        extra = (f", rank-{c['srank']} temporal subspace (LLR on coefficients), "
                 f"{c['wavelet_levels']}-level db{c['wavelet_moments']} wavelet shrink alpha {c['wavelet_alpha']:g} "
                 f"on the {where}")
    if "stride" in c:
        extra += f", overlapping blocks at stride {c['stride'][0]} (each voxel the mean of its block outputs)"
    return (f"{name}: {v[0]}x{v[1]}x{v[2]} complex64 x {nq} volumes, {b[0]}^3 LLR blocks (Casorati "
            f"{b[0] * b[1] * b[2]}x{n}){extra}, {c['accel']:g}x VD line sampling, soft threshold 0.02 sigma_max, "
            f"FP32, one proximal-gradient iteration per step")


# ---------------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------------
def run_b200(args, dist: Dist) -> None:
    import llr_b200
    from llr_b200 import PinnedBuffer, ReconContext, ReconParams
    if llr_b200.device_count() < 1:
        raise RuntimeError("bench.py needs a CUDA device (the CUDA library is the only implementation)")
    dev = dist.local_rank
    c, d = make_data(args.config, args.seed + dist.rank, use_gpu=True)
    nx, ny, nz = c["vol"]
    nq = d.y.shape[3]
    E = nx * ny * nz * nq
    params = ReconParams(vol_size=(nx, ny, nz), nq=nq, block_size=c["block"], prox_mode=llr_b200.LLR_PROX_SOFT_THRESH,
                         lam=0.0, seed=args.seed, device=dev, gram_mode=args.gram_mode,
                         eig_solver=args.eig_solver, fft_mode=args.fft_mode, block_stride=c.get("stride"))
    if "srank" in c:   # subspace + wavelet configuration: subspace built on the GPU from the b-table
        from llr_b200.phantom import dti_subspace_gpu
        params.subspace_rank = c["srank"]
        params.wavelet_alpha, params.wavelet_moments = c["wavelet_alpha"], c["wavelet_moments"]
        params.wavelet_levels = c["wavelet_levels"]
        params.wavelet_space = c.get("wavelet_space", 0)
    ctx = ReconContext(params)
    if "srank" in c:
        ctx.upload_subspace(dti_subspace_gpu(d.b, d.g, c["srank"], 100000, args.seed)[0])
    ctx.upload_kspace(d.y)
    ctx.init_zero_filled()
    sigma = ctx.sigma_max((0, 0, 0))
    ctx.set_lambda(0.02 * sigma)
    x0 = ctx.download_image() if (dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline) else None

    # warm-up, then the timed region: K iterations, per-stage CUDA events on the context stream.
    # An iterate that fits the 126 MB L2 is evicted before every timed iteration by writing a
    # 512 MB buffer (outside the events), so no iteration starts with its input in L2.
    flush = None
    if 8 * E <= 126e6:
        import torch
        flush = torch.empty(128 << 20, dtype=torch.float32, device=f"cuda:{dev}")
    ctx.iterate_profiled(max(args.warmup, 1))
    dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    if flush is None:
        stage_ms, total_ms = ctx.iterate_profiled(args.steps)
    else:
        stage_ms, total_ms = np.zeros(5), 0.0
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            st, tt = ctx.iterate_profiled(1)
            stage_ms, total_ms = stage_ms + st, total_ms + tt
    clk = clocks.stop()
    dist.barrier()
    t_max = dist.max(total_ms)
    hist = ctx.residual_history(args.steps)
    value = dist.world * args.steps / (t_max / 1e3)

    # roofline of the dominant stage: the LLR proximal step (llr_gram_tc_kernel: gather + 3xTF32
    # tcgen05 Gram; llr_eig_warp_kernel: eigen decomposition; llr_apply_kernel: apply + scatter).
    # Algorithmic bytes = the operator's minimum, one read and one write of every complex64
    # element of the iterate (16 B per voxel-volume element).
    names = ["llr_prox", "wavelet", "fft_fwd", "dc", "fft_inv"]
    per_launch_ms = {n: stage_ms[i] / args.steps for i, n in enumerate(names)}
    prox_bytes = 16.0 * E
    peaks = measured_peaks()
    achieved = prox_bytes / (per_launch_ms["llr_prox"] / 1e3) / 1e9
    prof = profiled_traffic("llr_prox", args.config)
    it_bytes = 16.0 * E * 3 + 24.0 * E / c["accel"]
    prox_label = ("LLR prox stage: llr_subspace_kernel (X <- LR(X S) S^H)" if "srank" in c else
                  "LLR prox stage: llr_gram_tc_kernel + llr_eig_warp_kernel + llr_apply_kernel")
    roofline = {"bound": "hbm", "kernel": prox_label,
                "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "peak_source": peaks["source"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                "algorithmic_bytes_per_launch": prox_bytes,
                "traffic": None if prof is None else prof["dram_bytes_per_launch"],
                "traffic_source": None if prof is None else
                f"profiles/llr_prox_{args.config}.json (captured on {prof['captured_on']}, x{prof['scale']:g})",
                "stage_ms_per_iteration": {k: round(v, 4) for k, v in per_launch_ms.items()},
                "iteration_algorithmic_bytes": it_bytes,
                "iteration_hbm_frac": round(it_bytes / (t_max / args.steps / 1e3) / 1e9 / peaks["hbm_gbs"], 4)}

    # end to end through the host API: H2D of y from pinned memory, zero-filled start,
    # n iterations, D2H of the image and residual history
    e2e = None
    if not args.no_e2e:
        n_e2e = args.e2e_iters
        yp = PinnedBuffer(d.y.shape)
        yp.array[...] = d.y
        xp = PinnedBuffer(d.y.shape)
        dist.barrier()
        t0 = time.perf_counter()
        ctx.upload_kspace(yp.array)
        ctx.init_zero_filled()
        ctx.iterate(n_e2e)
        ctx.download_image(xp.array)
        t_e2e = dist.max(time.perf_counter() - t0)
        e2e = {"value": round(dist.world * n_e2e / t_e2e, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(d.y.nbytes), "d2h_bytes_per_step": int(xp.array.nbytes + 8 * n_e2e),
               "step": f"one reconstruction call sequence: upload k-space, zero-filled start, {n_e2e} iterations, "
                       f"download image", "seconds_per_step": round(t_e2e, 4)}
        yp.close()
        xp.close()

    # learned + mixed against plain FP32: time to NRMSE <= 1e-3 (rank 0, N = 1)
    headline = None
    if dist.rank == 0 and dist.world == 1 and not args.no_warm_start and args.config == "c2":
        try:
            headline = warm_start_headline(args, c, d)
        except Exception as e:  # reported, never fatal to the throughput measurement
            headline = {"error": f"{type(e).__name__}: {e}"}

    # CPU baseline (rank 0, N = 1): FP32 restatement of the reference on a bounded sample
    cpu = None
    if x0 is not None:
        from oracle.cpu_baseline import time_iteration_sample
        from threadpoolctl import threadpool_limits
        with threadpool_limits(1):
            r = time_iteration_sample(x0, d.y, c["block"], "soft", 0, 0.02 * sigma, n_blocks=args.cpu_blocks,
                                      n_vols=args.cpu_vols, seed=args.seed)
        cpu = {"value": round(1.0 / r["seconds_per_iteration"], 5), "unit": UNIT, "cores": r["threads"],
               "kind": "port", "sample": r["sample"], "seconds_per_iteration": round(r["seconds_per_iteration"], 3)}

    n_kernels = ctx.kernel_launches_per_iteration   # the library's own kernels; cuFFT's are not counted
    if dist.rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (FP32)",
            "data": "synthetic (seeded ellipsoid DTI phantom, VD mask, SNR 30 noise)",
            "config": bench_config(args.config, c, nq, dist.world),
            "lambda": 0.02 * sigma, "measured_undersampling": round(ctx.measurement_stats()[1], 3),
            "path": "hybrid (x-transform eliminated: line-structured sampling)",
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "warm_start": headline,
            "gpu_launches": n_kernels * args.steps,
            "jacobi_fallback_blocks_last_iteration": ctx.fallback_blocks,
            "residual_first_last": [float(hist[0]), float(hist[-1])],
        }
        print(json.dumps(out))
    ctx.close()


def run_reference(args, dist: Dist) -> None:
    """The reference's CPU path (FP32 numpy/scipy restatement, all host threads) on the same
    seeded data and threshold rule as the B200 arm.  Imports nothing that maps libllr_b200.so."""
    if dist.rank != 0:
        return
    from oracle.cpu_baseline import sigma_max_all_blocks, time_iteration_sample
    from llr_b200.phantom import PROTOCOL_SEED, make_dataset, centred_fft_unitary
    from threadpoolctl import threadpool_limits
    from oracle import llr_oracle as O
    c = config_workload(args.config)
    d = make_dataset(c["vol"], c["shells"], c["accel"], args.seed, centre=16, mask_fn=O.vd_mask,
                     forward=centred_fft_unitary, protocol_seed=PROTOCOL_SEED)
    nq = d.y.shape[3]
    # zero-filled start A^H y with the CPU restatement
    import scipy.fft as sf
    x0 = np.empty_like(d.y)
    nx, ny, nz = c["vol"]
    ramps = [np.exp(1j * np.pi * (np.arange(n) - n / 2.0)).astype(np.complex64) for n in (nx, ny, nz)]
    pre = ramps[0][:, None, None] * ramps[1][None, :, None] * ramps[2][None, None, :]
    for q in range(nq):
        x0[..., q] = sf.ifftn(d.y[..., q] * pre, norm="ortho", workers=-1) * np.conj(pre)
    bs = c["block"]
    with threadpool_limits(1):
        lam = 0.02 * sigma_max_all_blocks(x0, bs)
        times = []
        for i in range(args.warmup + args.steps):
            r = time_iteration_sample(x0, d.y, bs, "soft", 0, lam, n_blocks=args.cpu_blocks, n_vols=args.cpu_vols,
                                      seed=args.seed + i)
            if i >= args.warmup:
                times.append(r["seconds_per_iteration"])
    sec = sum(times) / len(times)
    value = 1.0 / sec
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (FP32)",
        "data": "synthetic (seeded ellipsoid DTI phantom, VD mask, SNR 30 noise)",
        "config": bench_config(args.config, c, nq, dist.world),
        "lambda": lam,
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": r["threads"], "kind": "port",
                         "sample": r["sample"] + "; the reference (Rust + unvendored git crates) cannot be built "
                                                 "here, so its algorithm is restated in numpy/scipy"},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def cnn_timing(args) -> None:
    """Device time of the warm-start network (forward; loss and gradients) on random channels at
    96^3 and at the config-2 geometry, between stream synchronisations."""
    from llr_b200.cnn import Cnn, DeviceArray
    from llr_b200 import _lib as L
    res = {}
    for dims in ([tuple(args.cnn_dims[::-1])] if args.cnn_dims else [(96, 96, 96), (96, 192, 192)]):
        net = Cnn(seed=1)
        rng = np.random.default_rng(0)
        x = DeviceArray.from_numpy(rng.standard_normal(dims + (14,)).astype(np.float32))
        t = DeviceArray.from_numpy(rng.standard_normal(dims + (14,)).astype(np.float32))
        o = DeviceArray(dims + (14,))
        for _ in range(2):
            net.forward_dev(x, o)
        L.check(L.lib.llr_stream_sync(None))
        t0 = time.perf_counter()
        for _ in range(5):
            net.forward_dev(x, o)
        L.check(L.lib.llr_stream_sync(None))
        fwd = (time.perf_counter() - t0) / 5 * 1e3
        net.loss_grad_dev(x, t)
        t0 = time.perf_counter()
        for _ in range(3):
            net.loss_grad_dev(x, t)
        L.check(L.lib.llr_stream_sync(None))
        fb = (time.perf_counter() - t0) / 3 * 1e3
        flops = 2 * 27 * (14 * 32 + 6 * 32 * 32 + 32 * 14) * dims[0] * dims[1] * dims[2]
        res["x".join(map(str, dims[::-1]))] = {"forward_ms": round(fwd, 3), "forward_tflops": round(flops / fwd / 1e9, 2),
                                               "loss_grad_ms": round(fb, 3),
                                               "loss_grad_tflops": round(3 * flops / fb / 1e9, 2)}
        net.close()
    print(json.dumps({"cnn_timing": res}))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", default="c2")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-iters", type=int, default=100)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-warm-start", action="store_true", help="skip the learned warm-start comparison")
    ap.add_argument("--ws-ref-iters", type=int, default=1200,
                    help="iterations of the converged reference (and the cap of both measured runs)")
    ap.add_argument("--cpu-blocks", type=int, default=2048)
    ap.add_argument("--cpu-vols", type=int, default=8)
    ap.add_argument("--gram-mode", type=int, default=0, help="0: 3xTF32 tensor-core Gram, 1: FP32 FMA Gram")
    ap.add_argument("--fft-mode", type=int, default=0,
                    help="0: fused per-plane FFT + DC + inverse FFT kernel; 1: cuFFT passes")
    ap.add_argument("--eig-solver", type=int, default=0,
                    help="0: tridiagonal, warp per block; 1: Jacobi")
    ap.add_argument("--ncu-traffic", metavar="CSV",
                    help="write profiles/<--traffic-name>_<--config>.json from `ncu -i REP --page raw --csv` output "
                         "and exit")
    ap.add_argument("--traffic-name", default="llr_prox")
    ap.add_argument("--traffic-kernels", default="llr_gram_tc|llr_eig_warp|llr_apply")
    ap.add_argument("--traffic-scale", type=float, default=1.0)
    ap.add_argument("--traffic-captured-on", default=None)
    ap.add_argument("--cnn-timing", action="store_true", help="time the warm-start network and exit")
    ap.add_argument("--cnn-dims", type=int, nargs=3, metavar=("NX", "NY", "NZ"), help="one volume for --cnn-timing")
    args = ap.parse_args(argv)
    if args.cnn_timing:
        cnn_timing(args)
        return
    if args.ncu_traffic:
        write_traffic(args)
        return
    if args.warmup < 3:
        print("note: warm-up raised to 3 (timing rules)", file=sys.stderr)
        args.warmup = 3
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
