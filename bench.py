#!/usr/bin/env python
"""vectors/s of the multi-grid PIV engine on one 6600x4400 image pair.

Workload (one step = one image pair through the whole pipeline): 6600x4400 uint8 pair,
MHE (40 px tiles, 0.91), grid 1 64x64 windows at 32 px spacing for 2 passes, grid 2
32x32 at 16 px for 3 passes, window deformation, bilinear upsampling, normalized
median test (5x5, 2 passes, threshold 2), hole fill, 3x3 smoothing, Nsec_cc = 1.
Synthetic seeded particle images (0.04 particles/px, sigma 0.6 px, Lamb-Oseen vortex
of 10 px peak speed and 600 px core radius plus 0.002 px/px shear).  Final vectors per
pair: 113,300 (412 x 275).

  value  device-resident: frames already in HBM, CUDA events on the engine stream around
         each replay of the captured pair graph; L2 flushed before every step.
  e2e    through the C-ABI with host buffers: upload of both frames from pinned memory
         (piv_queue_images), the pair, readback of the filtered grid-2 field
         (piv_field_async / piv_field_wait), every step, pipelined so that uploads and
         readbacks overlap the computation of the neighbouring pairs.
  learned, learned_split_bf16  the learned form of the same pair (piv_run_pair_learned:
         trained predictor instead of the grid-1 passes, grid-2 passes on FP32 SIMT or
         split-BF16 tensor cores, judge with fallback), per-pair CUDA events.
  batch  64 pairs of uneven size and window shape through piv_batch_run (one persistent
         correlation launch per pass and window shape, one graph), against the same
         engines one pair at a time.
  --impl reference  the reference's own engine (xcorr2d_multi + mhe_gpu, compiled for
         sm_100a from its sources) on the same pair through its public methods.

Multi-GPU: one process per GPU; every rank processes its own pair (replicas, no data
collective); torch.distributed only for the barrier and the max-over-ranks time.
"""
import argparse
import importlib.util
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "piv_xcorr2d_v1.0_b200"
sys.path.insert(0, str(ROOT))

NX, NY = 6600, 4400
METRIC = "vectors/s at 6600x4400 multigrid (64->32 px, 2+3 passes, MHE on)"
UNIT = "vectors/s"


def load_pkg():
    if "piv_b200" in sys.modules:
        return sys.modules["piv_b200"]
    spec = importlib.util.spec_from_file_location("piv_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["piv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# Every value of the parameter file (X/Parameter.dat order) for the workload; both arms
# take their parameters from this one table.
WORKLOAD = dict(
    device_id=0, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, Nx=NX, Ny=NY,
    ws_x1=64, ws_y1=64, spacing_x1=32, spacing_y1=32, Npass1=2,
    ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3, Nsec_cc=1,
    wx1_median=5, wy1_median=5, Npass1_median=2, minNneigh_p1=5, residual_threshold_p1=2.0, insert_threshold_p1=2.0,
    wx1_smooth=3, wy1_smooth=3, Npass1_smooth=1,
    wx2_median=5, wy2_median=5, Npass2_median=2, minNneigh_p2=5, residual_threshold_p2=2.0, insert_threshold_p2=2.0,
    wx2_smooth=3, wy2_smooth=3, Npass2_smooth=1,
    max_dispx_win_percent1=0.4, max_dispy_win_percent1=0.4, max_dispx_win_percent2=0.4, max_dispy_win_percent2=0.4,
    Npeak_save=4, dispx_lim1=-100.0, dispx_lim2=100.0, dispy_lim1=-100.0, dispy_lim2=100.0)
# The seeded pair: 0.04 particles/px, sigma 0.6 px, Lamb-Oseen vortex (10 px, 600 px core) + 0.002 shear.
SYNTH = dict(ppp=0.04, sigma=0.6, field=1, a=10.0, b=600.0, c=0.002)


def workload_params(P, device_id=0, Ny=NY):
    return P.default_params(**{**WORKLOAD, "device_id": device_id, "Ny": Ny})


def workload_synth(P, seed=1):
    return P.synth_params(NX, NY, seed=seed, **SYNTH)


def workload_pair(P, seed=1):
    return P.synth_pair(workload_synth(P, seed))


def bench_config(nvec, world):
    """The `config` of both arms' lines (identical keys and values)."""
    return {"workload": "6600x4400 pair, MHE 40/0.91, grid 64x64@32 x2 -> 32x32@16 x3",
            "vectors_per_pair": nvec, "pairs_per_step_per_gpu": 1, "parallelism": f"replicas x{world}",
            "l2": "each step's working set (58 MB of frames, 117 MB deformed frame, GB-scale FFT buffers in the "
                  "reference) exceeds the 126 MB L2; the device-resident line also flushes L2 (512 MB write) "
                  "before every timed step"}


def accuracy(P, e, s):
    """The filtered grid-2 field against the known synthetic displacement u(x_g) at the
    vector positions: RMS over valid vectors (all, and away from the image border by two
    vector spacings), and the valid fraction."""
    x, y, dx, dy, v = e.field(3)
    u, w = P.synth_field(s, x, y)
    ok = v == 1
    err = np.hypot(dx - u, dy - w)
    sp = e.p.spacing_x2
    inner = ok & (x > 2 * sp) & (x < NX - 2 * sp) & (y > 2 * sp) & (y < NY - 2 * sp)
    return {"rms_px": round(float(np.sqrt(np.mean(err[ok] ** 2))), 4),
            "rms_interior_px": round(float(np.sqrt(np.mean(err[inner] ** 2))), 4),
            "valid_frac": round(float(ok.mean()), 4),
            "truth": "u(x_g) of the generator's Lamb-Oseen vortex + shear at the vector positions"}


def fft_flops(wsx, wsy):
    """Algorithmic FP32 flops of one window correlation: 3 transforms (5 N log2 N) + 8 N."""
    n = wsx * wsy
    return 3 * 5 * n * math.log2(n) + 8 * n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def traffic_from_profile():
    """DRAM bytes per launch of the grid-2 correlation kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "xcorr_grid2_6600x4400.txt"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch_full_size:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


def cpu_baseline(P, f1, f2, rows):
    """The CPU oracle on a bounded band of the same pair (full pipeline), vectors/s."""
    from oracle import oracle as O

    p = workload_params(P, Ny=rows)
    a = np.ascontiguousarray(f1[:rows])
    b = np.ascontiguousarray(f2[:rows])
    t0 = time.perf_counter()
    a = O.mhe(a, 40, 0.91)
    b = O.mhe(b, 40, 0.91)
    r = O.run_pair(a, b, p)
    dt = time.perf_counter() - t0
    nvec = r["geom"]["Nt_vec"][1]
    return {"value": nvec / dt, "unit": UNIT, "cores": O.threads(), "kind": "port",
            "sample": f"CPU oracle (FP64 correlation) on the top {NX}x{rows} band of the pair, full pipeline "
                      f"({nvec} grid-2 vectors in {dt:.2f} s)"}


def learned_form(P, e, ext, flush, args, s, path, plain_ms):
    """The learned form of the same pair (piv_run_pair_learned): the predictor replaces the
    grid-1 passes, grid 2 runs its 3 passes on `path`, and the judge (more than 5 % median
    rejects, or more than 0.5 px RMS between the prediction and the grid-2 field) sends the
    pair back to the plain method.  Timed per pair on the engine stream with CUDA events,
    judge readback and any fallback included, L2 flushed before each pair."""
    import torch

    net = P.PredictorNet(weights=args.weights)
    e.set_xcorr_path(1, path)
    for _ in range(args.warmup):
        e.run_pair_learned(net)
    ms, fb, rej, rms = [], 0, [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        r = e.run_pair_learned(net)
        b.record(ext)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        fb += r["fell_back"]
        rej.append(r["reject_frac"])
        rms.append(r["rms_px"])
    acc = accuracy(P, e, s)
    e.set_xcorr_path(1, P.PIV_XCORR_SIMT)
    net.close()
    t = sum(ms) / len(ms)
    return {"value": round(e.geom["Nt_vec"][1] / (t * 1e-3), 1), "unit": UNIT, "ms_per_step": round(t, 3),
            "vs_plain": round(plain_ms / t, 3), "fallback_rate": fb / len(ms),
            "judge": {"reject_frac": round(float(np.mean(rej)), 5), "rms_px": round(float(np.mean(rms)), 4),
                      "limits": {"reject_frac": 0.05, "rms_px": 0.5}},
            "accuracy": acc, "grid2_path": {P.PIV_XCORR_SIMT: "fp32 simt", P.PIV_XCORR_TC_SPLIT: "split-bf16 tcgen05",
                                            P.PIV_XCORR_TC_BF16: "bf16 tcgen05"}[path],
            "weights": str(Path(args.weights).relative_to(ROOT)) if Path(args.weights).is_relative_to(ROOT)
            else str(args.weights)}


BATCH_SIZES = [(1024, 1024)] * 16 + [(2048, 1536)] * 16 + [(4096, 2160)] * 16 + [(6600, 4400)] * 16


def batch_workload(P, seed=3):
    """64 pairs of uneven size: 16 each at 1024x1024, 2048x1536, 4096x2160 and 6600x4400;
    0.02-0.08 particles/px; sums of 8 Fourier modes (wavelengths 200-2000 px, at most
    12 px); grid-2 windows drawn from {16, 24, 32, 64} at 50 or 75 % overlap, grid 1 at
    min(2 ws, 64) with the same overlap, 2 + 3 passes, MHE on."""
    rng = np.random.default_rng(seed)
    out = []
    for k, (Nx, Ny) in enumerate(BATCH_SIZES):
        ws2 = int(rng.choice([16, 24, 32, 64]))
        ov = float(rng.choice([0.5, 0.75]))
        ws1 = min(2 * ws2, 64)
        sp = lambda ws: int(round(ws * (1 - ov)))
        p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=ws1, ws_y1=ws1,
                             spacing_x1=sp(ws1), spacing_y1=sp(ws1), Npass1=2, ws_x2=ws2, ws_y2=ws2,
                             spacing_x2=sp(ws2), spacing_y2=sp(ws2), Npass2=3, Nsec_cc=1,
                             insert_threshold_p1=2.0, insert_threshold_p2=2.0)
        s = P.synth_params(Nx, Ny, ppp=float(rng.uniform(0.02, 0.08)), field=P.PIV_FIELD_FOURIER, a=200.0,
                           b=2000.0, c=12.0, seed=5000 + k)
        out.append((p, s))
    return out


def batch_form(P, args, flush):
    """The uneven batch: one graph with one persistent correlation launch per pass and window
    shape (piv_batch_run), against the same engines run one pair at a time (each pair's own
    graph, piv_run_pair).  Device time by CUDA events; frames in HBM; L2 flushed first."""
    import torch

    pairs = batch_workload(P)
    b = P.Batch([p for p, _ in pairs])
    frames = []
    for e, (p, s) in zip(b.engines, pairs):
        n = s.Nx * s.Ny
        d1 = torch.empty(n, dtype=torch.uint8, device="cuda")
        d2 = torch.empty_like(d1)
        scratch = torch.empty(2 * n, dtype=torch.float32, device="cuda")
        P.synth_pair_device(s, d1, d2, scratch)
        frames.append((d1, d2))
        del scratch
    torch.cuda.synchronize()
    for e, (d1, d2) in zip(b.engines, frames):
        e.set_device_images(d1.data_ptr(), d2.data_ptr())
    nvec = sum(e.geom["Nt_vec"][1] for e in b.engines)
    ext = torch.cuda.ExternalStream(b.stream())
    for _ in range(args.warmup):
        b.run()
        b.synchronize()
    reps = max(3, min(args.steps, 10))
    ms_b = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(ext)
        b.run()
        t1.record(ext)
        t1.synchronize()
        ms_b.append(t0.elapsed_time(t1))
    b.synchronize()
    se, cnt = 0.0, 0
    for e, (p, s) in zip(b.engines, pairs):
        x, y, dx, dy, v = e.field(3)
        u, w = P.synth_field(s, x, y)
        ok = v == 1
        se += float((((dx - u) ** 2 + (dy - w) ** 2)[ok]).sum())
        cnt += int(ok.sum())
    # the same pairs one at a time, each its own captured graph
    for e in b.engines:
        e.run_pair()
        e.synchronize()
    ms_p = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        tot = 0.0
        for e in b.engines:
            es = torch.cuda.ExternalStream(e.stream())
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(es)
            e.run_pair()
            t1.record(es)
            t1.synchronize()
            tot += t0.elapsed_time(t1)
        ms_p.append(tot)
    groups = b.groups()
    b.close()
    mb, mp = statistics.median(ms_b), statistics.median(ms_p)
    return {"value": round(nvec / (mb * 1e-3), 1), "unit": UNIT, "ms_per_batch": round(mb, 3),
            "pairs": len(pairs), "vectors_per_batch": nvec,
            "one_pair_at_a_time": {"value": round(nvec / (mp * 1e-3), 1), "ms_per_batch": round(mp, 3)},
            "speedup": round(mp / mb, 3), "correlation_launches_per_pass": {
                "grid1_first": sum(1 for g in groups if g["grid"] == 0 and not g["deformed"]),
                "grid1_deformed": sum(1 for g in groups if g["grid"] == 0 and g["deformed"]),
                "grid2": sum(1 for g in groups if g["grid"] == 1)},
            "groups": groups, "accuracy_rms_px": round(float(np.sqrt(se / max(cnt, 1))), 4),
            "workload": "64 uneven pairs: 16 each at 1024x1024, 2048x1536, 4096x2160, 6600x4400; "
                        "ws2 in {16,24,32,64} at 50/75 % overlap, ws1 = min(2 ws2, 64); 2+3 passes; MHE on; "
                        "Fourier fields up to 12 px", "reps": reps}


def replicas():
    load_pkg()
    import piv_b200.replicas as R

    return R


def run_ours(args, rank, world, local):
    import torch

    P = load_pkg()
    torch.cuda.set_device(local)
    p = workload_params(P, device_id=local)
    f1, f2 = workload_pair(P, seed=1 + rank)
    d1 = torch.from_numpy(f1).to(f"cuda:{local}")
    d2 = torch.from_numpy(f2).to(f"cuda:{local}")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")  # > 126 MB L2
    e = P.Engine(p)
    nvec = e.geom["Nt_vec"][1]
    ext = torch.cuda.ExternalStream(e.stream(), device=f"cuda:{local}")
    e.set_device_images(d1.data_ptr(), d2.data_ptr())
    for _ in range(args.warmup):
        e.run_pair()
        e.synchronize()
    R = replicas()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    R.barrier(world)
    torch.cuda.synchronize()
    h1, h2 = e.host_images()
    h1[:] = f1
    h2[:] = f2
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            starts[k].record(ext)
            e.run_pair()
            ends[k].record(ext)
        e.synchronize()
        torch.cuda.synchronize()
        R.barrier(world)
        ms = [starts[k].elapsed_time(ends[k]) for k in range(args.steps)]

        # end to end through the C-ABI with host buffers: every step uploads its pair
        # from pinned memory and reads its filtered field back, pipelined so that the GPU
        # always has the next pair queued -- the upload of pair k+1 (piv_queue_images)
        # and the readback of pair k (piv_field_async) overlap the computation, and the
        # host collects pair k-1's field (piv_field_wait) while pair k runs
        e.queue_images(h1.ctypes.data, h2.ctypes.data)
        e.run_pair()
        e.field(3)
        R.barrier(world)
        t0 = time.perf_counter()
        e.queue_images(h1.ctypes.data, h2.ctypes.data)
        prev = None
        for k in range(args.steps):
            e.run_pair()
            ticket = e.field_async(3)
            if k + 1 < args.steps:
                e.queue_images(h1.ctypes.data, h2.ctypes.data)
            if prev is not None:
                _, _, dx, dy, vv = e.field_wait(prev)
            prev = ticket
        _, _, dx, dy, vv = e.field_wait(prev)
        e2e_local = time.perf_counter() - t0
    total_s = R.max_over_ranks(sum(ms) / 1e3, world)
    value = R.throughput(args.steps * nvec, sum(ms) / 1e3, world)
    e2e_s = R.max_over_ranks(e2e_local, world)
    e2e = {"value": R.sum_over_ranks(args.steps * nvec, world) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * NX * NY,
           "d2h_bytes_per_step": int(dx.nbytes + dy.nbytes + vv.nbytes)}

    acc = accuracy(P, e, workload_synth(P, seed=1 + rank))

    # live roofline of the dominant kernel (grid-2 correlation), on the engine stream
    e.set_device_images(d1.data_ptr(), d2.data_ptr())
    e.run_pair()
    e.synchronize()
    kms = e.time_stage(1, reps=10)
    flops = nvec * fft_flops(p.ws_x2, p.ws_y2)
    peak = P.fp32_peak_tflops()
    achieved = flops / (kms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": round(achieved, 2), "peak": round(peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": traffic_from_profile(),
                "kernel": "xcorr_peak_kernel<32,32> (grid-2 correlation, deformed)",
                "kernel_ms": round(kms, 4), "algorithmic_flops_per_launch": flops,
                "peak_source": "FP32 FMA peak measured live on this GPU by piv_probe_fp32_peak"}
    launches = e.launches_per_pair() * args.steps
    tuned = {f"grid{k + 1}": dict(zip(("windows_per_cta", "threads_per_cta", "tuned_ms"), e.xcorr_config(k)))
             for k in range(2)}
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_s * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded particle images, Lamb-Oseen vortex + shear)",
        "config": bench_config(nvec, world), "xcorr_autotune": tuned,
        "e2e": e2e, "roofline": roofline, "gpu_launches": launches, "clocks": clk.summary(),
        "accuracy": acc,
    }
    # the learned form beside the plain one (same engine, frames and flush)
    plain_ms = total_s * 1e3 / args.steps
    if Path(args.weights).exists():
        e.set_device_images(d1.data_ptr(), d2.data_ptr())
        s_true = workload_synth(P, seed=1 + rank)
        out["learned"] = learned_form(P, e, ext, flush, args, s_true, P.PIV_XCORR_SIMT, plain_ms)
        out["learned_split_bf16"] = learned_form(P, e, ext, flush, args, s_true, P.PIV_XCORR_TC_SPLIT, plain_ms)
    else:
        out["learned"] = {"unavailable": f"no predictor weights at {args.weights}"}
    if not args.no_batch:
        out["batch"] = batch_form(P, args, flush)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(P, f1, f2, args.cpu_rows)
    e.close()
    return out


def run_reference(args, rank, world, local):
    """The reference's own engine (oracle/_ref, compiled for sm_100a from its sources) on the
    same pair, driven through xcorr2d_multi / mhe_gpu in X/main.cpp order.  This process
    loads only the reference library, the CPU oracle (geometry) and the stand-alone
    generator (oracle/libsynth.so): no part of the CUDA engine."""
    if rank != 0:
        return None
    import types

    from oracle import oracle as O
    from oracle import ref as R
    from oracle import synth as S

    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_xcorr2d.so was not built"}
    p = types.SimpleNamespace(**{**WORKLOAD, "device_id": local})
    f1, f2 = S.pair(S.params(NX, NY, seed=1, **SYNTH))
    rc, g = O.geometry(O.params_from(p))
    if rc != 0:
        return {"impl": "reference", "unavailable": f"geometry rejected ({rc})"}
    nvec = g.Nt_vec[1]
    with R.RefEngine(p) as r:
        for _ in range(args.warmup):
            r.run_pair(f1, f2)
            r.filtered(1, nvec)
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                r.run_pair(f1, f2)  # synchronises the device before returning
                dx, dy, vv = r.filtered(1, nvec)
            dt = time.perf_counter() - t0
    value = args.steps * nvec / dt
    n = NX * NY
    # per pair: MHE uploads both raw frames and reads both enhanced frames back
    # (X/main.cpp:267-283); prep_img_data uploads each frame into both grids' buffers
    # (X/xcorr2d_multi_grid.cu:1271-1282); the filtered grid-2 field is read back
    h2d, d2h = 2 * n + 4 * n, 2 * n + int(dx.nbytes + dy.nbytes + vv.nbytes)
    return {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic (seeded particle images, Lamb-Oseen vortex + shear)",
        "config": bench_config(nvec, 1),
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's CUDA engine compiled for sm_100a from its own sources, driven "
                                   "from one host thread through xcorr2d_multi/mhe_gpu in main.cpp order "
                                   "(host frames in, filtered grid-2 field out, wall clock)"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-rows", type=int, default=1024, help="rows of the pair the CPU baseline processes")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-pair uneven batch line")
    ap.add_argument("--weights", default=str(PKG_DIR / "weights" / "predictor.bin"),
                    help="learned-predictor weights (piv_xcorr2d_v1.0_b200/train_predictor.py)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # rank 0 alone runs the reference; the other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        out = run_reference(args, rank, 1, int(os.environ.get("LOCAL_RANK", "0")))
        if out is not None:
            print(json.dumps(out))
        return
    R = replicas()
    rank, world, local = R.init("nccl")
    out = run_ours(args, rank, world, local)
    R.finish(world)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
