"""Benchmark of the distance-driven projector pair on B200.

Workload (one step): forward projection A x followed by backprojection A^T b of
one 2048 x 2048 float32 slice at 1800 angles uniform on [0, 180), 2048 detector
bins, seeded random-ellipse phantom (synthetic data).  Metric: GUPS, i.e.
pixel x angle updates per second (2 * 2048^2 * 1800 updates per step), higher
is better.  Between timed steps L2 is flushed by writing a 256 MiB buffer.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU, each rank projecting its own
slices (independent slices: weak scaling, no collective on the data path);
the step time is the max over ranks.  ``--impl reference`` times the
reference's own C kernel (compiled into oracle/_ref) on the host cores, on a
bounded sample of angles of the same workload.

At N = 1 the line also carries ``blocks``: the other configurations, each
measured after the headline in the same process (C1 SIRT + ray-driven pair,
C2 MLEM / SPS + distance-driven pair against the reference's own results,
C3 ADMM-TV + gridding with the gridding roofline, C4 batched uneven SIRT over
512 slices and a 512 x 2048^2 volume streamed from host memory, C5 learned
warm start trained and evaluated here).  They take a
few minutes; ``--no-blocks`` skips them.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SIDE, N_ANG = 2048, 1800
METRIC = "dd projector pair GUPS (pixel x angle updates per second, forward + adjoint)"
UNIT = "GUPS"
WORKLOAD = "distance-driven pair, 2048x2048 image, 1800 angles [0,180), 2048 bins, float32"
TAU_DD = 2  # gathered operand values per update (distance-driven)
# DRAM bytes per launch of the two main kernels at 2048^2 x 1800, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum)
DRAM_BYTES_PER_LAUNCH = {"forward": 153.6e6 + 10.0e6, "adjoint": 38.0e6 + 0.0064e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-angles", type=int, default=0,
                    help="angles per step of the CPU baseline sample (0: auto)")
    ap.add_argument("--profile", action="store_true",
                    help="run only warm-up + steps of the device path (for ncu captures)")
    ap.add_argument("--n", type=int, default=N_SIDE, help="image side (profiling only)")
    ap.add_argument("--na", type=int, default=N_ANG, help="angle count (profiling only)")
    ap.add_argument("--workload", default="pair",
                    choices=["pair", "batch", "warmstart", "admm", "kinds", "peaks", "volume"],
                    help="pair: the dd pair at 2048^2 x 1800 (default); batch: batched uneven SIRT; "
                         "warmstart: learned warm start, time to the plain SIRT residual")
    ap.add_argument("--train-pairs", type=int, default=2048, help="warmstart: training samples")
    ap.add_argument("--train-steps", type=int, default=2000, help="warmstart: training steps")
    ap.add_argument("--eval-slices", type=int, default=256, help="warmstart: held-out slices")
    ap.add_argument("--compact-pairs", action="store_true",
                    help="warmstart: keep training samples in bf16 without x_ref (for 20k samples)")
    ap.add_argument("--save-net", default=None, help="warmstart: write the trained network's weights here")
    ap.add_argument("--load-net", default=None,
                    help="warmstart: evaluate the network with these weights instead of training one")
    ap.add_argument("--no-blocks", action="store_true",
                    help="pair workload: skip the C1-C5 blocks measured after the headline")
    ap.add_argument("--block-slices", type=int, default=512, help="C4 block: slices")
    ap.add_argument("--block-iters", type=int, default=5, help="C4 block: SIRT iterations timed")
    ap.add_argument("--lam", type=float, default=0.03, help="warmstart: weight of the data-consistency loss")
    ap.add_argument("--slices", type=int, default=64, help="batch workload: number of slices")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="admm workload: skip the host reference sample")
    ap.add_argument("--iters", type=int, default=10, help="batch workload: SIRT iterations per step")
    ap.add_argument("--kinds", default="pd,rd,dd,ss,bspline,grid", help="kinds workload: projectors to time")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region:
    every 25 ms, with nvidia-smi's own timestamps, keeping the samples taken
    between entering and leaving the ``with`` block (the sampler is started
    and given half a second to come up before the block's region begins)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 25

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.t_begin = self.t_end = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)
        except OSError:
            self.proc = None
        self.t_begin = time.time()
        return self

    def __exit__(self, *a):
        self.t_end = time.time()
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def _in_region(self, stamp: str) -> bool:
        import datetime
        try:
            t = datetime.datetime.strptime(stamp.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return False
        margin = self.PERIOD_MS * 1e-3
        return self.t_begin - margin <= t <= self.t_end + margin

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 10 or not self._in_region(f[0]):
                continue
            try:
                sm.append(float(f[2]))
                mx = max(mx, float(f[3]))
            except ValueError:
                continue
            for nm, val in zip(names, f[6:10]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def onchip_peaks():
    """On-chip roofline denominators measured now on the current device
    (tomo_measure_onchip_peaks2): shared-memory 16-byte loads, L1 4-byte and
    16-byte loads (aligned warp requests that hit L1), FP32 FMA.  ``l1_gbs`` is
    the larger L1 rate, the one the gather kernels are measured against."""
    import ctypes
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    v = [ctypes.c_double() for _ in range(4)]
    fn = _lib.lib.tomo_measure_onchip_peaks2
    fn.argtypes = [ctypes.POINTER(ctypes.c_double)] * 4
    _lib.check(fn(*[ctypes.byref(x) for x in v]), "onchip peaks")
    smem, l1_4, l1_16, fp32 = (x.value for x in v)
    return {"smem_gbs": smem, "l1_4_gbs": l1_4, "l1_16_gbs": l1_16, "l1_gbs": max(l1_4, l1_16),
            "fp32_tflops": fp32}


def run_peaks(args, rank, world, local):
    """Only the on-chip probes (for an ncu capture of the probe kernels)."""
    import torch
    torch.cuda.set_device(local)
    for _ in range(max(1, args.steps)):
        pk = onchip_peaks()
    print(json.dumps({"onchip_peaks": pk}), flush=True)


def sample_angle_index(na_total: int, sample_angles: int) -> np.ndarray:
    """``sample_angles`` indices into the reference's (fftshifted) angle order,
    evenly spread over the angles that take the general path: the axis angles
    (|sin| or |cos| < 1e-7, plain row / column sums, radon_dd.c:75-96) are left
    out, so each sampled angle costs what a general angle costs."""
    from oracle.oracle import radon_angles
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import angles_deg
    a = np.fft.fftshift(radon_angles(angles_deg(na_total))).astype(np.float64)
    general = np.nonzero((np.abs(np.sin(a)) >= 1e-7) & (np.abs(np.cos(a)) >= 1e-7))[0]
    return general[np.linspace(0, len(general) - 1, sample_angles).astype(int)]


def cpu_reference_gups(n: int, na_total: int, sample_angles: int, threads: int):
    """Reference dd kernel (oracle/_ref/ref_dd.so) on a sample of the angles.

    Returns (GUPS, seconds, description).  ``threads`` > 1 runs that many
    angle chunks concurrently (ctypes releases the GIL during the C call).
    The rate is that of the general angles; the two axis angles of 1800 (row
    and column sums) are cheaper, so the whole application's rate is higher by
    about 0.1 %.
    """
    from concurrent.futures import ThreadPoolExecutor

    from oracle.oracle import RefLib, radon_angles
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import angles_deg, random_ellipses
    R = RefLib()
    ang_all = radon_angles(angles_deg(na_total))
    idx = sample_angle_index(na_total, sample_angles)
    ang = np.ascontiguousarray(np.fft.fftshift(ang_all)[idx])
    img = random_ellipses(n, seed=0)
    chunks = np.array_split(np.arange(len(ang)), threads)
    import ctypes
    fp = ctypes.POINTER(ctypes.c_float)

    def run(ch, oper):
        a = np.ascontiguousarray(ang[ch])
        if oper == 0:
            out = np.zeros((len(a), n), np.float32)
            R.L["dd"].radon_dd(img.ctypes.data_as(fp), n, a.ctypes.data_as(fp), len(a), 0,
                               out.ctypes.data_as(fp))
        else:
            s = np.ones((len(a), n), np.float32)
            out = np.zeros((n, n), np.float32)
            R.L["dd"].radon_dd(out.ctypes.data_as(fp), n, a.ctypes.data_as(fp), len(a), 1,
                               s.ctypes.data_as(fp))
        return out

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda c: run(c, 0), chunks))
        list(ex.map(lambda c: run(c, 1), chunks))
    dt = time.perf_counter() - t0
    updates = 2.0 * n * n * len(ang)
    desc = (f"reference radon_dd (oracle/_ref, -O3 -ffast-math) forward+adjoint on {len(ang)} of "
            f"{na_total} angles at {n}x{n} (evenly spread over the non-axis angles), {threads} thread(s); "
            f"rate extrapolated to the whole application")
    return updates / dt / 1e9, dt, desc


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample = args.cpu_sample_angles or max(4 * threads, 64)
    vals = []
    for i in range(args.warmup + args.steps):
        g, dt, desc = cpu_reference_gups(N_SIDE, N_ANG, sample, threads)
        if i >= args.warmup:
            vals.append((g, dt))
    gups = float(np.median([v[0] for v in vals]))
    ms = float(np.median([v[1] for v in vals])) * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": gups, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": desc},
            "cpu_baseline": {"value": gups, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": gups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_core(n_slices, iters, steps, warmup, rank, world, dev):
    """Batched uneven SIRT: slices of side 256/512/1024/2048 (weights 4:3:2:1, seeded
    draw), round(1.5 side) angles on [0, 180), ceil(1.5 side) bins (the operator side;
    the phantom is centred in it), noiseless data from the same projector.  All
    slices form one batched plan: every projector application is one persistent
    launch, every iteration one CUDA-graph replay.  A step is ``iters`` SIRT
    iterations of every slice; the metric counts 2 n_op^2 na updates per slice and
    iteration.  With world > 1 the slice list (n_slices per rank) is split across
    ranks by LPT on cost.  Returns the result fields (rank 0) and the step time."""
    import math

    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon import shim_angles
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import embed, random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.sharding import (lpt_partition, max_over_ranks,
                                                                               slice_cost)
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import Solver
    import torch.distributed as dist
    rng = np.random.default_rng(4)
    all_sides = rng.choice([256, 512, 1024, 2048], size=n_slices * world, p=[0.4, 0.3, 0.2, 0.1])
    costs = [slice_cost(int(math.ceil(1.5 * s)), int(round(1.5 * s))) for s in all_sides]
    mine = lpt_partition(costs, world)[rank]
    sides = all_sides[mine]
    geoms, imgs = [], []
    for k, side in zip(mine, sides):
        na, nb = int(round(1.5 * side)), int(math.ceil(1.5 * side))
        ang = shim_angles("dd", (np.linspace(0, 180, na, endpoint=False) * np.pi / 180).astype(np.float32))
        geoms.append((nb, ang))
        imgs.append(torch.from_numpy(embed(random_ellipses(int(side), seed=1000 + int(k)), nb)))
    bp = _lib.BatchPlan(geoms)
    x_true = bp.pack([t.to(dev) for t in imgs])
    b = bp.forward(x_true)
    solver = Solver(bp, "sirt", b)
    x0 = torch.ones(bp.img_total, device=dev)
    for _ in range(max(1, warmup)):
        solver.run(x0, 1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        ev0.record()
        for _ in range(steps):
            x, res = solver.run(x0, iters)
        ev1.record()
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / steps)
    upd = float(sum(2.0 * c for c in costs)) * iters
    out = {"value": upd / (ms * 1e-3) / 1e9, "unit": "GUPS", "ms_per_step": ms,
           "config": {"workload": f"{n_slices * world} slices, sides {{256,512,1024,2048}} weights 4:3:2:1, "
                                  f"na=round(1.5 side), nb=ceil(1.5 side), {iters} SIRT iterations per step",
                      "sides": {int(s): int((all_sides == s).sum()) for s in (256, 512, 1024, 2048)},
                      "slices_total": int(len(all_sides)), "sharding": "LPT on n_op^2 na, no data-path collective",
                      "updates_per_step": upd, "instances": bp.instances},
           "residual_first_last": [float(res[0]), float(res[-1])],
           "tuning": bp.tuning(), "clocks": clk.summary()}
    del solver, bp, x_true, b
    torch.cuda.empty_cache()
    return out


def run_batch(args, rank, world, local):
    """The batched uneven SIRT workload (batch_core) as its own bench line."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    r = batch_core(args.slices, args.iters, args.steps, args.warmup, rank, world, dev)
    if rank == 0:
        line = {"metric": "batched SIRT GUPS (pixel x angle updates per second, uneven slices, one launch per application)",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
        line.update(r)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def oracle_residuals(xs, b, na, threads=None):
    """||A x - b||^2 per slice with the FP64 oracle's distance-driven forward
    (float32 geometry, float64 sums), one angle per call in a thread pool;
    b in the class's row order (sinogram_row_of_angle)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.oracle import Oracle, radon_angles, sinogram_row_of_angle
    orc = Oracle()
    ang = radon_angles(np.linspace(0, 180, na, endpoint=False))
    rows = sinogram_row_of_angle("dd", na)
    out = []
    for x, bb in zip(xs, b):
        x = np.ascontiguousarray(x, np.float32)
        bb = np.asarray(bb, np.float64)

        def one(k):
            r = orc.radon("dd", 0, x, ang[k:k + 1])[0]
            return float(((r - bb[rows[k]]) ** 2).sum())

        with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
            out.append(float(sum(ex.map(one, range(na)))))
    return out


def warmstart_core(train_pairs, train_steps, eval_slices, lam, dev, oracle_slices=2, compact=False,
                   save_net=None, load_net=None):
    """Learned warm start at 512^2 (768 bins), 180 angles on [0, 180), Poisson I0 = 5e3:
    samples (2-iteration SIRT, filtered backprojection, 300-iteration SIRT, phantom)
    generated by the batched solver on seeds 10000 + i, a 4-level, 32-channel U-Net
    trained on them with the tensor-core kernels, then on held-out seeds 100000 + i the
    GPU time plain SIRT needs for its 300 iterations against the time the warm start
    (2 iterations + network + fallback check + SIRT) needs to reach the same data
    residual (summed over the held-out slices).  For ``oracle_slices`` of them the
    final data residuals of both runs are computed again with the FP64 oracle's
    projector beside the GPU's.  Metric: warm / plain time (lower is better)."""
    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import nn, warmstart as ws
    pb = ws.Problem()
    net = nn.UNet(levels=4, base=32, seed=0).to(dev)
    if load_net:  # weights of an earlier run of the same training (save_net)
        net.load_state_dict(torch.load(load_net, map_location=dev))
        t_pairs = t_train = None
        hist = []
    else:
        t0 = time.perf_counter()
        data = ws.make_pairs(pb, [10000 + i for i in range(train_pairs)], compact=compact)
        torch.cuda.synchronize()
        t_pairs = time.perf_counter() - t0
        t0 = time.perf_counter()
        hist = ws.train(net, pb, data, steps=train_steps, batch=4, lam=lam)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        del data
        torch.cuda.empty_cache()
        if save_net:
            torch.save(net.state_dict(), save_net)
    r = ws.time_to_residual(net, pb, [100000 + i for i in range(eval_slices)])
    k = min(oracle_slices, eval_slices)
    bh = r["b"][:k].cpu().numpy()
    tp = r["tp"]
    fp64 = {"slices": k}
    for name in ("plain", "warm"):
        x = r[f"x_{name}"][:k]
        gpu = ((tp.A(x).double() - r["b"][:k].double()) ** 2).sum(dim=(1, 2)).cpu().numpy()
        orc = np.array(oracle_residuals(x.cpu().numpy(), bh, pb.na))
        fp64[name] = {"gpu": gpu.tolist(), "oracle": orc.tolist(),
                      "max_rel_diff": float(np.max(np.abs(gpu - orc) / orc))}
    out = {"value": r["ratio"], "unit": "ratio (warm / plain GPU time)", "higher_is_better": False,
           "config": {"workload": "512^2 phantom in 768 bins, 180 angles, Poisson I0=5e3, dd pair, SIRT from 0; "
                                  "U-Net 4 levels x 32 channels, BF16 weights/activations, FP32 accumulation",
                      "train_pairs": train_pairs, "train_steps": train_steps, "lam": lam,
                      "eval_slices": eval_slices,
                      "stored_samples": "bf16 x2/fbp/x_true, no x_ref" if compact else "f32",
                      "network": f"loaded from {load_net}" if load_net else "trained in this run"},
           "plain_ms": r["plain_ms"], "warm_ms": r["warm_ms"], "warm_iters": r["warm_iters"],
           "plain_iters": r["plain_iters"], "residual_plain": r["residual_plain"],
           "residual_warm": r["residual_warm"], "image_rel_err_plain": r["err_plain"],
           "image_rel_err_warm": r["err_warm"], "image_rel_err_start": r["err_start"],
           "fallback_slices": r["fallback_slices"],
           "fp64_oracle_residual": fp64,
           "pairs_s": t_pairs, "train_s": t_train, "loss_first_last": [hist[0], hist[-1]] if hist else None}
    del r, net
    torch.cuda.empty_cache()
    return out


def run_warmstart(args, rank, world, local):
    """The learned warm start (warmstart_core) as its own bench line."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    r = warmstart_core(args.train_pairs, args.train_steps, args.eval_slices, args.lam, dev,
                       compact=args.compact_pairs, save_net=args.save_net, load_net=args.load_net)
    if rank == 0:
        line = {"metric": "learned warm start: GPU time to reach plain SIRT's 300-iteration data residual, warm / plain",
                "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": r["warm_ms"], "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16 network (fp32 accumulation), f32 projector", "data": "synthetic"}
        line.update(r)
        print(json.dumps(line), flush=True)


def gridding_roofline(n, na, lconv_adj, fwd_ms, adj_ms, pk=None):
    """Roofline figures of one gridding forward and adjoint application: per
    application na * pdim polar samples (both half-planes), each a
    ceil(lconv)^2 window of complex64 taps (8 B and 8 flops a tap), plus the 2-D
    FFT (5 pdim^2 log2(pdim^2) flops), against the L1 16-byte load rate and the
    FP32 FMA rate measured now; and the HBM passes over the complex64 Fourier
    grid (written once by the fill / gather, two read+write passes of the 2-D
    FFT, read once by the gather / deapodisation) plus the na x pdim polar rows
    written and read once, against the measured HBM copy rate.  The forward's
    window width is the reference's fixed 2 * 7 / pi (gridrec_v4_forwproj.c);
    the adjoint's is the plan's (param[6])."""
    from iterative_tomographic_reconstruction_algorithms_b200.gridrec_lut import grid_size
    pk = pk or onchip_peaks()
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    hbm_peak = json.loads(peaks_file.read_text())["hbm_gbs"] if peaks_file.exists() else 6650.0
    pdim = grid_size(n, 2.0)
    roof = {}
    for name, lconv, t_ms in (("forward", 2 * 7.0 / np.pi, fwd_ms), ("adjoint", lconv_adj, adj_ms)):
        taps = float(na) * pdim * math.ceil(lconv) ** 2
        flops = 8.0 * taps + 5.0 * pdim * pdim * math.log2(pdim * pdim)
        gb = 8.0 * taps / (t_ms * 1e-3) / 1e9
        tf = flops / (t_ms * 1e-3) / 1e12
        hbm = 8.0 * (6.0 * pdim * pdim + 2.0 * na * pdim)
        hb = hbm / (t_ms * 1e-3) / 1e9
        roof[name] = {"ms": t_ms, "window": math.ceil(lconv), "gathered_gbs": gb, "frac_of_l1": gb / pk["l1_gbs"],
                      "tflops": tf, "frac_of_fp32": tf / pk["fp32_tflops"],
                      "hbm_bytes_passes": hbm, "hbm_gbs": hb, "frac_of_hbm": hb / hbm_peak}
    return roof


def admm_core(steps, warmup, dev, cpu_baseline=True):
    """ADMM-TV (admm.lasso_tv) with the gridding pair: 1024^2 phantom centred in
    1536 bins, 1500 angles on [0, 180), Kaiser-Bessel W = 6, oversampling 2
    (4096^2 Fourier grid), linear interpolation, b = A x + Gaussian noise of
    sigma 0.01 max(b) (seed 2), lambd1 = 0.1, lambd2 = 1, mu = 20, 5 inner CG
    iterations.  A step is one ADMM outer iteration (6 projector pairs, the
    Gt(G) stencils, shrinkage and multiplier update; one CUDA graph).  Metric:
    outer iterations per second.  The working set (about 0.26 GB with the
    Fourier grid) exceeds L2, so no flush is needed between steps."""
    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import admm as ad
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import embed, random_ellipses
    n, na, side = 1536, 1500, 1024
    deg = np.linspace(0, 180, na, endpoint=False)
    tp = cpg.projectors(n, deg, kernel="kb", oversampl=2.0, W=6.0, errs=1e-3, interp="lin", verbose=False)
    x_true = torch.from_numpy(embed(random_ellipses(side, seed=2), n)).to(dev)
    b = tp.A(x_true)
    g = torch.Generator(device=dev).manual_seed(2)
    b = (b + 0.01 * float(b.max()) * torch.randn(b.shape, generator=g, device=dev)).contiguous()
    l1, l2, mu, n2 = 0.1, 1.0, 20.0, 5
    solver = ad.AdmmSolver(tp, "lasso-tv", b, l1, l2, mu, n2)
    x = torch.ones((1, n, n), device=dev)
    solver.run(x, max(1, warmup), reset=True)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(dev)
    with ClockSampler(dev.index) as clk:
        ev0.record(stream)
        st = solver.run(x, steps, reset=False)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    # the projector pairs alone (6 per outer iteration), same stream
    plan = tp.plan(1, dev.index)
    sino = plan.forward(x)
    img = plan.adjoint(sino)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(6):
        sino = plan.forward(x)
    e1.record(stream)
    for _ in range(6):
        img = plan.adjoint(sino)
    e2.record(stream)
    torch.cuda.synchronize()
    fwd_ms, adj_ms = e0.elapsed_time(e1) / 6, e1.elapsed_time(e2) / 6
    pairs_ms = 6 * (fwd_ms + adj_ms)
    # end to end through the public API: host x and b in, host x out, track=False
    xh = np.ones((1, n, n), np.float32)
    bh = b.cpu().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ad.lasso_tv(xh, bh, tp, ad.Param(lambd1=l1, lambd2=l2, mu=mu, n_iter=steps, n_iter_pcg=n2), track=False)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    rel = float((x[0].double() - x_true.double()).norm() / x_true.double().norm())
    cpu = None
    if cpu_baseline:
        cpu = admm_cpu_baseline(tp, b[0].cpu().numpy(), n, n2)
    upd = 12.0 * n * n * na  # 6 pairs of n^2 na updates per outer iteration
    roof = gridding_roofline(n, na, float(tp.param_nofilt[6]), fwd_ms, adj_ms)
    out = {
        "metric": "ADMM-TV outer iterations per second (gridding pair, 5 inner CG iterations)",
        "value": 1e3 / ms, "unit": "iterations/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 CG r, p)",
        "data": "synthetic",
        "config": {"workload": "ADMM-TV, 1024^2 phantom in 1536 bins, 1500 angles, gridding KB W=6 os=2 lin, "
                               "sigma=0.01 max b, lambd1=0.1 lambd2=1 mu=20, 5 inner CG",
                   "l2": "working set > L2, no flush"},
        "projector_pairs_ms_per_step": pairs_ms, "projector_share": pairs_ms / ms,
        "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
        "pair_gups": upd / (pairs_ms * 1e-3) / 1e9,
        "err_last": float(np.sqrt(st[-1, :, 0].sum())), "image_rel_err_after_all_steps": rel,
        "e2e": {"value": 1e3 / e2e_ms, "unit": "iterations/s", "h2d_bytes_per_step": 4 * (n * n + na * n) / steps,
                "d2h_bytes_per_step": 4 * n * n / steps},
        "gridding_roofline": roof, "clocks": clk.summary()}
    if cpu is not None:
        out["cpu_baseline"] = cpu
    del solver
    torch.cuda.empty_cache()
    return out


def run_admm(args, rank, world, local):
    """The ADMM-TV workload (admm_core) as its own bench line."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    print(json.dumps(admm_core(args.steps, args.warmup, dev, not args.no_cpu_baseline)), flush=True)


def c1_core(dev, cpu=True):
    """C1: SIRT with the ray-driven pair, 256 x 256, 304 angles on [0, 180), 100
    iterations from x0 = 1, on the noiseless sinogram of a random-ellipse phantom
    (seed 0) that the reference projector made (tests/golden/solver_golden.npz).
    GPU: the fused solver's 100 iterations under CUDA events; parity: relative L2
    of x_100 to the reference's own art.sirt result in that fixture.  CPU: the
    reference rd kernel timed once forward and once adjoint at this size, scaled
    to 100 iterations of two forward and one adjoint application each
    (art.py:226-236 and the objective's forward, :326)."""
    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import Solver
    g = np.load(ROOT / "tests" / "golden" / "solver_golden.npz")
    deg, b, xref = g["sirt_rd/angles_deg"], g["sirt_rd/b"], g["sirt_rd/x100"]
    n = b.shape[1]
    tp = cpr.projectors(n, deg, oper="rd")
    solver = Solver(tp, "sirt", b)
    x0 = torch.ones((1, n, n), device=dev)
    solver.run(x0, 1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x, _ = solver.run(x0, 100)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    xh = x[0].cpu().numpy().astype(np.float64)
    rel = float(np.linalg.norm(xh - xref) / np.linalg.norm(xref))
    out = {"gpu_ms_100_iterations": ms, "rel_l2_vs_reference_sirt": rel,
           "config": "SIRT, ray-driven pair, 256x256, 304 angles, 100 iterations, x0 = 1"}
    if cpu:
        from oracle.oracle import RefLib, radon_angles
        R = RefLib()
        ang = radon_angles(deg)
        img = xref.astype(np.float32)
        t0 = time.perf_counter()
        y = R.radon("rd", 0, img, ang)
        t1 = time.perf_counter()
        R.radon("rd", 1, y, ang)
        t2 = time.perf_counter()
        ref_s = 100 * (2 * (t1 - t0) + (t2 - t1))
        out["reference_s_100_iterations"] = ref_s
        out["reference_sample"] = ("reference radon_rd (oracle/_ref) one forward and one adjoint timed on 1 core, "
                                   "x 100 iterations of 2 forward + 1 adjoint")
        out["speedup"] = ref_s / (ms * 1e-3)
    del solver
    return out


def c2_core(dev):
    """C2: MLEM and SPS (no penalty) with the distance-driven pair, 512 x 512
    phantom (seed 1) scaled to mu in [0, 0.02] and centred in 768 bins, 720
    angles on [0, 180), 50 iterations from x0 = 1: MLEM on the noiseless sinogram
    (on the noisy one the reference MLEM diverges), SPS on -log(max(counts,1)/1e4),
    counts ~ Poisson(1e4 exp(-A mu)).  The sinograms and the reference's own 50-
    iteration results and wall times come from tests/golden/solver_c2_<algo>.npz
    (sir.em / sir.sps over the compiled reference projector, one core); the
    GPU time is the fused solver's 50 iterations under CUDA events."""
    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import Solver
    out = {"config": "MLEM / SPS, distance-driven pair, 512^2 phantom in 768 bins, 720 angles, 50 iterations"}
    deg = np.linspace(0, 180, 720, endpoint=False)
    tp = cpr.projectors(768, deg, oper="dd")
    for algo in ("em", "sps"):
        f = ROOT / "tests" / "golden" / f"solver_c2_{algo}.npz"
        if not f.exists():
            out[algo] = {"skipped": "fixture absent"}
            continue
        g = np.load(f)
        solver = Solver(tp, algo, g["b"])
        x0 = torch.ones((1, 768, 768), device=dev)
        solver.run(x0, 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x, _ = solver.run(x0, 50)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        xh, xr = x[0].cpu().numpy().astype(np.float64), g["x50"].astype(np.float64)
        out[algo] = {"gpu_ms_50_iterations": ms, "rel_l2_vs_reference": float(np.linalg.norm(xh - xr) / np.linalg.norm(xr)),
                     "reference_s_50_iterations": float(g["ref_seconds"][0]),
                     "reference_host": "the fixture's build container, 1 core",
                     "speedup": float(g["ref_seconds"][0]) / (ms * 1e-3)}
        del solver
    return out


def volume_core(dev, nslices=512, chunk=16, slots=3):
    """C4 volume: 512 slices of 2048 x 2048 at 1800 angles on [0, 180), 2048
    bins (a 7.55 GB float32 sinogram), held in page-locked host memory and
    streamed through the GPU in chunks of ``chunk`` slices (streaming.
    VolumeStreamer: a copy-in, a compute and a copy-out stream over ``slots``
    buffer sets; one multi-slice distance-driven launch per chunk).  The forward
    projects the image volume, the adjoint backprojects the sinogram volume;
    each is timed end to end on the device (copies included) after a warm-up
    pass, beside the same launches on device-resident chunks (compute only):
    overlap = compute-only time / streamed time.  The phantoms are 8 seeded
    random-ellipse slices repeated."""
    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.streaming import VolumeStreamer
    n, na = N_SIDE, N_ANG
    tp = cpr.projectors(n, np.linspace(0, 180, na, endpoint=False), oper="dd")
    imgs = torch.empty((nslices, n, n), dtype=torch.float32).pin_memory()
    base = [torch.from_numpy(random_ellipses(n, seed=3000 + k)) for k in range(8)]
    for z in range(nslices):
        imgs[z].copy_(base[z % 8])
    sinos = torch.empty((nslices, na, n), dtype=torch.float32).pin_memory()
    back = torch.empty((nslices, n, n), dtype=torch.float32).pin_memory()
    vs = VolumeStreamer(tp, chunk=chunk, slots=slots, device=dev.index)
    vs.project(imgs[:chunk * slots], sinos[:chunk * slots])      # warm-up: plans, tuning
    vs.backproject(sinos[:chunk * slots], back[:chunk * slots])
    with ClockSampler(dev.index) as clk:
        ms_f = vs.project(imgs, sinos)
        ms_a = vs.backproject(sinos, back)
    # compute only: the same per-chunk launches on one resident chunk
    plan = vs._plan(chunk)
    di, ds = vs._buf(0, "img"), vs._buf(0, "sino")
    di.copy_(imgs[:chunk])
    nchunks = (nslices + chunk - 1) // chunk
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    e0.record()
    for _ in range(nchunks):
        plan.forward(di, out=ds)
    e1.record()
    for _ in range(nchunks):
        plan.adjoint(ds, out=di)
    e2.record()
    torch.cuda.synchronize()
    cf, ca = e0.elapsed_time(e1), e1.elapsed_time(e2)
    upd = float(nslices) * n * n * na
    out = {"config": f"{nslices} slices x {n}^2, {na} angles, {n} bins, dd pair, chunk {chunk} slices, "
                     f"copy-in / compute / copy-out streams over {slots} buffer sets, page-locked host volume",
           "sinogram_gb": nslices * na * n * 4 / 1e9, "image_gb": nslices * n * n * 4 / 1e9,
           "forward": {"ms": ms_f, "gups": upd / (ms_f * 1e-3) / 1e9, "compute_only_ms": cf, "overlap": cf / ms_f},
           "adjoint": {"ms": ms_a, "gups": upd / (ms_a * 1e-3) / 1e9, "compute_only_ms": ca, "overlap": ca / ms_a},
           "h2d_bytes": int(imgs.numel() * 4 + sinos.numel() * 4), "d2h_bytes": int(sinos.numel() * 4 + back.numel() * 4),
           "clocks": clk.summary()}
    # spot check: the streamed sinogram of one slice equals the single-slice plan's
    z = nslices // 2
    out["slice_bit_identical"] = bool(torch.equal(sinos[z], tp.A(imgs[z].to(dev)).cpu()))
    del vs, imgs, sinos, back
    torch.cuda.empty_cache()
    return out


def run_blocks(args, dev):
    """The configurations beside the headline, each measured in this process
    (device time by CUDA events): C1 SIRT + rd, C2 MLEM / SPS + dd, C3 ADMM-TV +
    gridding (with the gridding roofline), C4 batched uneven SIRT and the
    streamed 512-slice volume, C5 learned warm start.  A block that fails records its error and the others still run."""
    import torch
    blocks = {}
    jobs = [("c1_sirt_rd", lambda: c1_core(dev)),
            ("c2_mlem_sps_dd", lambda: c2_core(dev)),
            ("c3_admm_tv_grid", lambda: admm_core(3, 1, dev, cpu_baseline=False)),
            ("c4_batched_sirt", lambda: batch_core(args.block_slices, args.block_iters, 1, 1, 0, 1, dev)),
            ("c4_streamed_volume", lambda: volume_core(dev)),
            ("c5_warm_start", lambda: warmstart_core(args.train_pairs, args.train_steps, args.eval_slices,
                                                     args.lam, dev))]
    for name, fn in jobs:
        t0 = time.perf_counter()
        try:
            blocks[name] = fn()
        except Exception as e:  # noqa: BLE001 -- a block's failure is recorded, not fatal
            blocks[name] = {"error": f"{type(e).__name__}: {e}"}
        blocks[name]["seconds"] = time.perf_counter() - t0
        torch.cuda.empty_cache()
    return blocks


# gathered operand bytes per pixel x angle update of each projector (its reference
# arithmetic): 4 B x taps read per update; B-spline 5 taps + 5 LUT values
TAU_BYTES = {"pd": 32.0, "rd": 25.6, "dd": 8.0, "ss": 8.0, "bspline": 40.0}


def run_kinds(args, rank, world, local):
    """Every projector pair through its class API on one seeded random-ellipse
    slice: pd, rd, dd, ss (class_projectors_radon), cubic B-spline
    (class_projectors_bspline, radon_degree 1) and gridding (Kaiser-Bessel W=6,
    os 2, linear interpolation).  Each forward and each adjoint application is
    timed alone with CUDA events after warm-up, L2 flushed (256 MiB write)
    before every application; GUPS = n^2 na / time.  For the gather kernels the
    line also gives the gathered operand bytes per second against the L1 4-byte
    load rate measured in the same run."""
    import ctypes

    import torch
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n, na = args.n, args.na
    deg = np.linspace(0, 180, na, endpoint=False)
    pk = onchip_peaks()
    x = torch.from_numpy(random_ellipses(n, seed=0)).to(dev)
    y = torch.from_numpy(np.random.default_rng(1).standard_normal((na, n)).astype(np.float32)).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {}
    kinds = [k for k in args.kinds.split(",") if k]
    with ClockSampler(local) as clk:
        for kind in kinds:
            if kind in ("pd", "rd", "dd", "ss"):
                tp = cpr.projectors(n, deg, oper=kind)
            elif kind == "bspline":
                tp = cpb.projectors(n, deg, None, bspline_degree=3, proj_support_y=4, radon_degree=1)
            else:
                tp = cpg.projectors(n, deg, kernel="kb", oversampl=2.0, W=6.0, errs=1e-3, interp="lin",
                                    verbose=False)
            res = {}
            for name, fn, arg in (("forward", tp.A, x), ("adjoint", tp.At, y)):
                for _ in range(max(1, args.warmup)):
                    fn(arg)
                times = []
                for _ in range(args.steps):
                    flush.fill_(1.0)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    fn(arg)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1))
                ms = float(np.median(times))
                gups = n * n * na / (ms * 1e-3) / 1e9
                r = {"ms": ms, "gups": gups}
                if kind in TAU_BYTES:
                    gbs = TAU_BYTES[kind] * n * n * na / (ms * 1e-3) / 1e9
                    r["gathered_gbs"] = gbs
                    r["frac_of_l1"] = gbs / pk["l1_gbs"]
                res[name] = r
            if kind == "grid":
                res["roofline"] = gridding_roofline(n, na, float(tp.param_nofilt[6]), res["forward"]["ms"],
                                                    res["adjoint"]["ms"], pk)
            out[kind] = res
            del tp
            torch.cuda.empty_cache()
    print(json.dumps({
        "metric": "per-projector GUPS (pixel x angle updates per second per application)", "unit": "GUPS",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic", "config": {"workload": f"each projector pair, {n}x{n} image, {na} angles [0,180), {n} bins",
                                        "l2": "flushed before every application (256 MiB write)"},
        "kinds": out, "onchip_peaks": pk,
        "clocks": clk.summary()}), flush=True)


def admm_cpu_baseline(tp, b0, n, n2):
    """The reference's outer ADMM-TV iteration on the host, extrapolated from one
    forward + adjoint of the compiled reference gridding C (oracle/_ref, with the
    project's FFT stand-in: FFTW is absent) and one dense Gt(G(.)) (numpy) at full
    size: (n2 + 1) pairs + (n2 + 2) Gt products per outer iteration."""
    from oracle.oracle import RefLib, ref_available
    from oracle import admm_oracle as ao
    if not ref_available():
        return None
    R = RefLib()
    deg = np.asarray(tp.angles, np.float32)
    x = np.ones((n, n), np.float32)
    t0 = time.perf_counter()
    y = R.gridrec(0, x, deg, tp.param_nofilt, tp.lut, tp.deapod)
    R.gridrec(1, y, deg, tp.param_nofilt, tp.lut, tp.deapod)
    t_pair = time.perf_counter() - t0
    t0 = time.perf_counter()
    ao.Gt(ao.G(x.astype(np.float64)))
    t_gt = time.perf_counter() - t0
    per_iter = (n2 + 1) * t_pair + (n2 + 2) * t_gt
    return {"value": 1.0 / per_iter, "unit": "iterations/s", "cores": 1, "kind": "reference",
            "sample": f"one gridding A + A^T ({t_pair:.2f} s) and one dense Gt(G) ({t_gt:.3f} s) at full size, "
                      f"extrapolated to {n2 + 1} pairs + {n2 + 2} Gt per outer iteration; FFT: project stand-in"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batch":
        return run_batch(args, rank, world, local)
    if args.workload == "warmstart":
        return run_warmstart(args, rank, world, local)
    if args.workload == "admm":
        return run_admm(args, rank, world, local)
    if args.workload == "kinds":
        return run_kinds(args, rank, world, local)
    if args.workload == "peaks":
        return run_peaks(args, rank, world, local)
    if args.workload == "volume":
        import torch
        dev = torch.device("cuda", local)
        torch.cuda.set_device(dev)
        print(json.dumps({"metric": "streamed volume GUPS", **volume_core(dev, args.slices)}), flush=True)
        return

    import torch
    import torch.distributed as dist
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import angles_deg, random_ellipses

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    n, na = (args.n, args.na) if args.profile else (N_SIDE, N_ANG)
    deg = angles_deg(na)
    tp = cpr.projectors(n, deg, oper="dd")
    img_np = random_ellipses(n, seed=1000 + rank)
    x = torch.from_numpy(img_np).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    stream = torch.cuda.current_stream(dev)

    if args.profile:
        for _ in range(args.warmup + args.steps):
            flush.fill_(1.0)
            tp.At(tp.A(x))
        torch.cuda.synchronize()
        return

    pk = onchip_peaks()

    def step(events=None):
        flush.fill_(1.0)
        if events is not None:
            events[0].record(stream)
        b = tp.A(x)
        if events is not None:
            events[1].record(stream)
        y = tp.At(b)
        if events is not None:
            events[2].record(stream)
        return b, y

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    fwd_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    adj_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / args.steps
    updates_step = 2.0 * n * n * na  # per rank
    value = updates_step * world / (ms_step * 1e-3) / 1e9

    # end to end through the public API with host arrays (numpy in, numpy out)
    b_np = tp.A(img_np)
    torch.cuda.synchronize()
    e2e_steps = max(2, min(args.steps, 5))
    for _ in range(1):
        tp.At(tp.A(img_np))
    t_e = time.perf_counter()
    for _ in range(e2e_steps):
        b_np = tp.A(img_np)
        g_np = tp.At(b_np)
    e2e_s = (time.perf_counter() - t_e) / e2e_steps
    e2e_val = updates_step * world / e2e_s / 1e9
    h2d = img_np.nbytes + b_np.nbytes
    d2h = b_np.nbytes + g_np.nbytes

    # roofline of the dominant kernel (the projectors are bound by L1/shared-memory gathers)
    dom_ms = max(fwd_ms, adj_ms)
    dom = "adjoint" if adj_ms >= fwd_ms else "forward"
    upd_app = n * n * na
    alg_bytes = 4.0 * TAU_DD * upd_app
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    peak = pk["l1_gbs"]
    roofline = {"bound": "l1", "kernel": f"dd_{dom}", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak,
                "traffic": DRAM_BYTES_PER_LAUNCH.get(dom),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one full-size launch "
                                  "(committed ncu summary of the dd pair)",
                "peak_source": "tomo_measure_onchip_peaks2: larger of the aligned 4-byte and 16-byte L1 load "
                               "rates, this run"}
    hbm_bytes = 4.0 * (n * n + na * n)
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    hbm_peak = json.loads(peaks_file.read_text())["hbm_gbs"] if peaks_file.exists() else 6650.0

    blocks = run_blocks(args, dev) if (world == 1 and not args.no_blocks) else None
    if rank == 0:
        cpu = None
        if world == 1:
            g, dt, desc = cpu_reference_gups(n, na, args.cpu_sample_angles or 16, 1)
            cpu = {"value": g, "unit": UNIT, "cores": 1, "kind": "reference", "sample": desc}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "slices_per_rank_per_step": 1,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"slices x{world}"},
            # per step, forward: row and column prefix sums, corrections, main kernel;
            # adjoint: sinogram expansion, dropped pieces (rows, columns), main kernel
            "gpu_launches": 8 * args.steps,
            "kernel_ms": {"dd_forward (line prefix sums + persistent forward)": fwd_ms,
                          "dd_adjoint (sinogram prefix sums + persistent adjoint)": adj_ms},
            "tuning": _lib.plan_tuning(tp.plan(1, dev.index if hasattr(dev, "index") else 0)),
            "roofline": roofline,
            "roofline_hbm": {"bound": "hbm", "achieved": hbm_bytes / (dom_ms * 1e-3) / 1e9,
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": hbm_bytes / (dom_ms * 1e-3) / 1e9 / hbm_peak},
            "onchip_peaks": pk,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        if blocks is not None:
            line["blocks"] = blocks
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
