#!/usr/bin/env python
"""Benchmark of the helical cone-beam FBP chain on one B200 (or N, weak scaling).

Workload (one step): one full-size scan -- curved detector 888 x 64, 984
views/rotation, pitch 0.984, 20 rotations (19,680 fan views, 4.47 GB FP32) --
rebinned, filtered and backprojected into 512 x 512 x N voxels of 0.9766 x
0.9766 x 0.625 mm, N spanning the fully sampled z range. Synthetic data: an
analytic FP64 projection of a seeded random-ellipsoid phantom (60 ellipsoids
in an elliptic water cylinder), made on the GPU before timing.

Metric: GUPS = voxel-view updates per second (every (voxel, view) in the
clamped [s1, s2] window of the backprojection) for the whole chain; also
seconds per volume. ``value`` is measured with the fan data resident in HBM;
``e2e`` through the C ABI's host-pointer entry (hr_recon_execute_host) with
pinned host buffers, copies inside the timed region.

Multi-GPU (torchrun): every rank reconstructs its own scan (independent
objects, weak scaling); there is no data-path collective.

``--impl reference`` times the reference's own CPU implementation (its C++
rebinning and backprojection compiled from its sources, oracle/_ref/, with the
FP64 filter restatement since the reference has no C/C++ CPU filter) on a
bounded sample of the same workload, on all host cores.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def max_over_ranks(values, world: int, device):
    """Element-wise maximum over the ranks of a job (a multi-GPU step takes as long as its slowest
    rank); the values of a single process are returned unchanged."""
    values = [float(v) for v in values]
    if world <= 1:
        return values
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def sum_over_ranks(values, world: int, device):
    """Element-wise sum over the ranks of a job (byte counts of the ranks' copies)."""
    values = [float(v) for v in values]
    if world <= 1:
        return values
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def job_gups(updates_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job throughput: every rank reconstructs its own scan of the same size (weak scaling)."""
    return updates_per_rank * world / seconds / 1e9
PLAIN_LAUNCHES = 3  # plain chain: rebin, preweight + FFT filter, backprojection
BYTES_PER_UPDATE_FP32 = 16  # four FP32 taps per voxel-view update
BYTES_PER_UPDATE_BF16 = 8   # four BF16 taps per voxel-view update


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["full", "medium", "small", "bigpatient", "batch", "learned"], default="full")
    ap.add_argument("--train-phantoms", type=int, default=2000, help="learned: training phantoms")
    ap.add_argument("--train-steps", type=int, default=2000, help="learned: Adam steps (batch 8)")
    ap.add_argument("--eval-phantoms", type=int, default=100, help="learned: held-out phantoms")
    ap.add_argument("--slab", type=int, default=64, help="slices per slab (bigpatient)")
    ap.add_argument("--rotations", type=int, default=0,
                    help="bigpatient: a shorter helix of this many rotations with the same detector, grid and "
                         "slice thickness (a profiling-size case; 0: the 200-rotation workload)")
    ap.add_argument("--form", choices=["fast", "plain"], default="fast",
                    help="form timed as `value` (the chosen BF16 form by default); the plain FP32 form is "
                         "timed beside it unless --no-plain")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="full config on 1 GPU: skip the big-patient, batch and learned workloads that the line "
                         "otherwise carries as sub-objects")
    ap.add_argument("--extra-steps", type=int, default=5, help="timed steps of each sub-workload")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--e2e-slab", default="128,64",
                    help="fast form: also time e2e through the slab pipeline with slabs of these many slices "
                         "(comma-separated; empty: off); the fastest entry is reported")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"])}, "measured"
    return dict(PEAKS_FALLBACK), "fallback"


def traffic_from_profiles(kernel: str, config: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/<kernel>_<config>.md,
    line 'dram_bytes_per_launch: N'), or None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{config}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9 and (self.uuid is None or self.uuid in parts[0]):
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# CPU baselines (bounded samples; the oracle and the compiled reference are the
# checker and the baseline, never the measured product)
# ---------------------------------------------------------------------------
def cpu_baseline(scan, budget_s: float = 20.0, kind: str = "auto"):
    """Reference CPU path on a bounded sample, extrapolated to one volume.

    rebin: the reference's ParallelRebinningCBCurve_CPU<float> on a block of views;
    filter: the FP64 Toeplitz restatement of the MATLAB filter on a block of rows;
    backprojection: the reference's ParallelFDKHelical3DWeightingCPU on a sub-volume
    of whole columns x a few slices. Each part runs on all host cores (one
    reference call per thread on disjoint blocks). Returns (GUPS, s/volume, detail).
    """
    from concurrent.futures import ThreadPoolExecutor

    import oracle

    use_ref = oracle.ref_available() if kind == "auto" else kind == "reference"
    ncores = os.cpu_count() or 1
    rng = np.random.default_rng(0)
    ra, fa, g = scan.rebin_args(), scan.filter_args(), scan.bp_geom()
    # rebin: a block of views per thread
    nv = max(1, min(64, ra["ViewN"] // ncores))
    blocks = [rng.random((nv + 160, ra["YL"], ra["ZL"]), dtype=np.float32) for _ in range(ncores)]
    a = dict(ra, ViewN=nv + 160)
    fn = oracle.ref_rebin_f32 if use_ref else oracle.rebin_f32
    t = time.perf_counter()
    with ThreadPoolExecutor(ncores) as ex:
        list(ex.map(lambda b: fn(b, **a), blocks))
    t_rebin_sample = time.perf_counter() - t
    t_rebin = t_rebin_sample * ra["ViewN"] / (ncores * (nv + 160))
    # filter: rows of a block of views (OpenMP inside)
    nvf = max(1, min(200, fa["ViewN"]))
    rows = rng.standard_normal((nvf, fa["ZL"], fa["YL"]))
    t = time.perf_counter()
    oracle.filter_f64(rows, **dict(fa, ViewN=nvf), nthreads=ncores)
    t_filter_sample = time.perf_counter() - t
    t_filter = t_filter_sample * fa["ViewN"] / nvf
    # backprojection: whole slices of a z band in the middle of the scan, split by y rows
    w = oracle.weight_table(scan.N_2pi, scan.HSCoef, scan.delta)
    nz = 2
    z0 = scan.ZN // 2
    s0 = int(np.ceil((2 * 3.14159265358979 * ((z0 - g["ZNC"]) * g["dz"]) / g["h"] - g["BetaS"]) / g["DeltaFai"] - .5))
    lo, hi = max(0, s0 - 400), min(g["PN"], s0 + 420)
    fp = rng.standard_normal((hi - lo, g["ZL"], g["YL"]))
    # probe the per-update time on a small block, then size the sample to the budget
    ny_probe = 2
    sub = dict(g, YN=ny_probe, ZN=nz, ZNC=g["ZNC"] - z0, PN=hi - lo, BetaS=g["BetaS"] + lo * g["DeltaFai"])
    t = time.perf_counter()
    (oracle.ref_bp_f64 if use_ref else (lambda f, ww, gg: oracle.bp_f64(f, ww, gg, nthreads=1)))(fp, w, sub)
    t_probe = time.perf_counter() - t
    upd_probe = ny_probe * g["XN"] * nz * 671
    per_upd = t_probe / upd_probe
    ny_per_thread = max(1, min(g["YN"] // ncores, int(budget_s * 0.6 / (per_upd * g["XN"] * nz * 671))))
    subs = []
    for c in range(ncores):
        y0 = c * ny_per_thread
        subs.append(dict(sub, YN=ny_per_thread, YNC=g["YNC"] - y0))
    bp_fn = oracle.ref_bp_f64 if use_ref else (lambda f, ww, gg: oracle.bp_f64(f, ww, gg, nthreads=1))
    t = time.perf_counter()
    with ThreadPoolExecutor(ncores) as ex:
        list(ex.map(lambda gg: bp_fn(fp, w, gg), subs))
    t_bp_sample = time.perf_counter() - t
    upd_sample = ncores * ny_per_thread * g["XN"] * nz * 671
    timed_s = t_rebin_sample + t_filter_sample + t_bp_sample
    t_bp = t_bp_sample * scan.updates() / upd_sample
    total = t_rebin + t_filter + t_bp
    detail = {"rebin_s": t_rebin, "filter_s": t_filter, "bp_s": t_bp,
              "sample": (f"rebin {ncores}x{nv + 160} views, filter {nvf} views x {fa['ZL']} rows, backprojection "
                         f"{ncores}x{ny_per_thread} rows x {g['XN']} x {nz} slices (centre of the scan, "
                         f"{upd_sample:.3g} updates); each extrapolated linearly to the full volume"),
              "kind": "reference" if use_ref else "port", "cores": ncores,
              "sample_updates": upd_sample, "sample_wall_s": timed_s}
    return scan.updates() / total / 1e9, total, detail


def run_reference(args, scan, rank, world):
    if rank != 0:
        return
    steps = []
    detail = None
    for i in range(args.warmup + args.steps):
        gups, spv, detail = cpu_baseline(scan, budget_s=8.0)
        if i >= args.warmup:
            steps.append((gups, spv, detail["sample_wall_s"]))
    gups = statistics.median(s[0] for s in steps)
    spv = statistics.median(s[1] for s in steps)
    line = {"impl": "reference", "metric": "GUPS (voxel-view updates/s, rebin+filter+3D-weighted helical BP)",
            "value": gups, "unit": "GUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": spv * 1e3, "s_per_volume": spv, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": chain_config(scan, args.config, world),
            "extrapolated": True,
            "timed_sample": {"updates_per_step": detail["sample_updates"],
                             "wall_s_per_step": statistics.median(s[2] for s in steps),
                             "note": "each step times a bounded sample of every stage on the host cores and "
                                     "extrapolates it linearly to the whole volume; ms_per_step is that "
                                     "extrapolation, not a timed interval"},
            "cpu_baseline": {"value": gups, "unit": "GUPS", "cores": detail["cores"], "kind": detail["kind"],
                             "sample": detail["sample"]},
            "e2e": {"value": gups, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {k: detail[k] for k in ("rebin_s", "filter_s", "bp_s")}}
    print(json.dumps(line), flush=True)


def chain_config(scan, config, world):
    """The `config` object of the chain's line; the reference arm prints the same one."""
    return {"workload": scan_name(scan, config), "updates_per_volume": scan.updates(),
            "parallelism": f"independent scans x{world}" if world > 1 else "1 GPU",
            "flush": "inputs larger than L2 (fan data 4.47 GB, filtered data 4.4 GB)"}


def scan_name(scan, config):
    return (f"helical {scan.YL}x{scan.ZL} curved detector, {scan.N_2pi} views/rot, pitch {scan.pitch}, "
            f"{scan.rotations:g} rot ({scan.views} fan views, {scan.PN} backprojected) -> "
            f"{scan.XN}x{scan.YN}x{scan.ZN} @ {scan.dx}x{scan.dy}x{scan.dz} mm ({config})")


def measure_form(args, scan, form, fan, dev, world, barrier, with_e2e=True):
    """Stage split, device-resident whole-chain timing and (optionally) e2e for one form."""
    import torch
    import torch.distributed as dist

    from analyticalreconbigpatient_b200 import _lib
    from analyticalreconbigpatient_b200.pipeline import HelicalRecon, StagePlans

    stream = torch.cuda.current_stream(dev)
    st = stream.cuda_stream
    fast = form == _lib.HR_FORM_FAST
    # ---- per-stage timing (warm) ---------------------------------------------
    stages = StagePlans(scan, form)
    rebinned = torch.empty((scan.views, scan.YL, scan.ZL), dtype=torch.float32, device=dev)
    filtered = None if fast else torch.empty((scan.PN, scan.ZL, scan.YL), dtype=torch.float32, device=dev)
    pairs = torch.empty((scan.PN, scan.ZL, scan.YL), dtype=torch.int32, device=dev) if fast else None
    vol = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, device=dev)
    if fast:  # the chain plan autotunes its backprojection at creation; do the same for the stage plans
        stages.rebin(rebinned, fan, st)
        stages.filter_tc(pairs, rebinned, _lib.HR_LAYOUT_REBIN, scan.crop_front, st)
        stages.autotune(vol, pairs, st)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    names = ["rebin", "filter", "backprojection"]
    stage_ms = {k: [] for k in names}
    for i in range(args.warmup + args.steps):
        ev[0].record(stream)
        stages.rebin(rebinned, fan, st)
        ev[1].record(stream)
        if fast:  # tensor-core Toeplitz filter straight to BF16 channel pairs
            stages.filter_tc(pairs, rebinned, _lib.HR_LAYOUT_REBIN, scan.crop_front, st)
        else:
            stages.filter(filtered, rebinned, _lib.HR_LAYOUT_REBIN, scan.crop_front, st)
        ev[2].record(stream)
        stages.backproject(vol, pairs if fast else filtered, st)
        ev[3].record(stream)
        stream.synchronize()
        if i >= args.warmup:
            for k in range(3):
                stage_ms[names[k]].append(ev[k].elapsed_time(ev[k + 1]))
    stages.check()
    del rebinned, filtered, pairs, vol
    stages.close()
    torch.cuda.empty_cache()

    # ---- timed whole chain (device resident) ---------------------------------
    rec = HelicalRecon(scan, form=form, device=dev)
    for _ in range(args.warmup):
        rec.run(fan, stream=st)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        rec.run(fan, stream=st)
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    (ms,) = max_over_ranks([ms], world, dev)
    rec.check()
    out = {"ms_per_step": ms, "stages_ms": {k: statistics.mean(v) for k, v in stage_ms.items() if v},
           "launches_per_step": (3 + fast_launches_per_bp(rec.describe())) if fast else PLAIN_LAUNCHES,
           "kernels": rec.describe()}

    # ---- end to end through the C ABI host entry -----------------------------
    if with_e2e:
        h_fan = torch.empty(fan.shape, dtype=torch.float32, pin_memory=True)
        h_fan.copy_(fan)
        h_vol = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, pin_memory=True)
        rec.run_host(h_fan, h_vol)  # warm
        barrier()
        e2e_t = []
        for _ in range(args.e2e_steps):
            t = time.perf_counter()
            rec.run_host(h_fan, h_vol)
            e2e_t.append(time.perf_counter() - t)
        e2e_s = statistics.median(e2e_t)
        (e2e_s,) = max_over_ranks([e2e_s], world, dev)
        out["e2e_s"] = e2e_s
        out["e2e_entry"] = ("hr_recon_execute_host (C ABI, pinned host buffers; the fan streams in by chunks of "
                            "views under the rebinning, filtering and z-block backprojection of the earlier ones)"
                            if fast else "hr_recon_execute_host (C ABI, pinned host buffers)")
        slab_sizes = [int(x) for x in str(args.e2e_slab).split(",") if x.strip() and int(x) > 0]
        if fast and slab_sizes:
            # the same volume through the slab pipeline: host-to-device copies of later slabs' fan windows
            # overlap the reconstruction of earlier slabs (hr_slab_execute with host buffers)
            from analyticalreconbigpatient_b200.pipeline import SlabRecon

            rec.close()
            torch.cuda.empty_cache()
            out["e2e_chain_s"] = e2e_s
            out["e2e_slab_s"] = {}
            out["slab_device_ms"] = {}
            d_vol = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, device=dev)
            for size in slab_sizes:
                slab = SlabRecon(scan, slab_slices=size, device=dev)
                slab.run(h_fan, h_vol)  # warm (autotunes, captures)
                # the slab pipeline on device-resident buffers (synchronous: all its streams are drained)
                slab.run(fan, d_vol)
                barrier()
                dev_t = []
                for _ in range(args.e2e_steps):
                    t = time.perf_counter()
                    slab.run(fan, d_vol)
                    dev_t.append(time.perf_counter() - t)
                (dev_ms,) = max_over_ranks([statistics.median(dev_t) * 1e3], world, dev)
                out["slab_device_ms"][str(size)] = dev_ms
                barrier()
                slab_t = []
                for _ in range(args.e2e_steps):
                    t = time.perf_counter()
                    slab.run(h_fan, h_vol)
                    slab_t.append(time.perf_counter() - t)
                slab_s = statistics.median(slab_t)
                (slab_s,) = max_over_ranks([slab_s], world, dev)
                out["e2e_slab_s"][str(size)] = slab_s
                slab.close()
                torch.cuda.empty_cache()
                if slab_s < out["e2e_s"]:
                    out["e2e_s"] = slab_s
                    out["e2e_entry"] = f"hr_slab_execute (C ABI, pinned host buffers, z slabs of {size})"
            del d_vol
        del h_fan, h_vol
    rec.close()
    torch.cuda.empty_cache()
    return out


def fast_launches_per_bp(desc: str) -> int:
    """Kernels one fast-form backprojection launches: the backprojection, plus the
    absmax and fill passes of an FP16 texture copy (the fill alone for FP32)."""
    if "texture-fp16" in desc:
        return 3
    if "texture-fp32" in desc:
        return 2
    return 1


def run_bigpatient(args, scan, dev, world, rank, barrier, emit=True):
    """Long scan through the slab pipeline (SlabRecon): fan data resident in HBM
    for `value`, host-resident for `e2e`. With several ranks the scan's z slabs
    are split between them in contiguous blocks (hr_slab_plan_create_part); each
    rank holds, projects and copies only its own fan views and writes only its
    own slices: no data cross between ranks (strong scaling: one scan)."""
    import torch

    from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
    from analyticalreconbigpatient_b200.pipeline import SlabRecon, plain_slab, project, slab_windows

    zlo = scan.h * scan.BetaS / (2 * np.pi)
    zhi = scan.h * (scan.BetaS + scan.views * scan.dBeta) / (2 * np.pi)
    body_half = 0.5 * (zhi - zlo) + 200.0
    objs = P.random_ellipsoids(3000, 400, (zlo, zhi), body=(250.0, 175.0), body_half_length=body_half)
    rec = SlabRecon(scan, slab_slices=args.slab, device=dev, part=rank, nparts=world, assign=_lib.HR_SLAB_BLOCKS)
    f0, nviews, fan_bytes = rec.fan_range()
    # this rank's fan views only: the projection of views [f0, f0 + nviews) of the scan
    sub = G.replace(scan, beta_start=scan.BetaS + f0 * scan.dBeta, rotations=nviews / scan.N_2pi)
    assert sub.views == nviews
    fan = project(sub, objs, device=dev.index)
    vol = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        rec.run(fan, vol, fan_view0=f0)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(None)
    clocks.start()
    stream = torch.cuda.current_stream(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        rec.run(fan, vol, fan_view0=f0)  # synchronous: the slab streams are drained when it returns
    t1.record(stream)
    torch.cuda.synchronize()
    clocks.stop()
    ms = t0.elapsed_time(t1) / args.steps
    (ms,) = max_over_ranks([ms], world, dev)
    desc = rec.describe()
    updates = scan.updates()
    wins = slab_windows(scan, args.slab, rank, world, _lib.HR_SLAB_BLOCKS)
    # per-slab error: the rank's first, middle and last slab against the plain FP32 chain on the same window
    per_slab = []
    for win in (wins[0], wins[len(wins) // 2], wins[-1]):
        a = win["fan_view0"] - f0
        ref = plain_slab(scan, win, fan[a: a + win["fan_views"]])
        got = vol[:, :, win["first_slice"]: win["first_slice"] + win["n_slices"]]
        hu = float(torch.sqrt(torch.mean((got.double() - ref.double()) ** 2))) / G.MU_WATER * 1000.0
        per_slab.append({"slab": win["slab"], "slices": [win["first_slice"], win["first_slice"] + win["n_slices"]],
                         "hu_rmse_vs_plain": hu})
        del ref
    torch.cuda.empty_cache()
    # e2e from host memory (pinned if the host allows it): this rank's fan views in, its slices out
    try:
        h_fan = torch.empty(fan.shape, dtype=torch.float32, pin_memory=True)
        pinned = True
    except RuntimeError:
        h_fan = torch.empty(fan.shape, dtype=torch.float32)
        pinned = False
    h_fan.copy_(fan)
    del fan
    torch.cuda.empty_cache()
    h_vol = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, pin_memory=pinned)
    rec.run(h_fan, h_vol, fan_view0=f0)
    barrier()
    e2e_t = []
    for _ in range(max(1, args.e2e_steps)):
        t = time.perf_counter()
        rec.run(h_fan, h_vol, fan_view0=f0)
        e2e_t.append(time.perf_counter() - t)
    (e2e_s,) = max_over_ranks([statistics.median(e2e_t)], world, dev)
    rec.close()
    my_slices = sum(w["n_slices"] for w in wins)
    h2d, d2h = (float(x) for x in sum_over_ranks([fan_bytes, my_slices * scan.XN * scan.YN * 4], world, dev))
    # backprojection roofline from the autotuner's best measured time per slice (same process)
    import re

    tuned = [float(x) for x in re.findall(r"v\d+=([0-9.]+)", desc)]
    pk, pk_kind = peaks()
    bp_ms_per_slice = min(tuned) if tuned else None
    roof = None
    if bp_ms_per_slice:
        upd_per_slice = updates / scan.ZN
        ach = BYTES_PER_UPDATE_BF16 * upd_per_slice / (bp_ms_per_slice * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": ("bp_tex_seg_kernel" if "segmented" in desc else "bp_tex_kernel")
                if "texture" in desc else "bp_fast_kernel",
                "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": ach / pk["hbm_gbs"], "peak_source": pk_kind, "traffic": None,
                "note": "gather-equivalent (8 B/update) over the autotuner's best time per slice"}
    nslabs = len(wins)
    line = {"metric": "GUPS (voxel-view updates/s, rebin+filter+3D-weighted helical BP)",
            "value": updates / (ms * 1e-3) / 1e9, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "s_per_volume": ms * 1e-3, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (analytic FP64 projections of 400 seeded random ellipsoids in a body cylinder)",
            "form": "fast (slab pipeline)",
            "config": {"workload": scan_name(scan, "bigpatient") + f", z slabs of {args.slab}",
                       "updates_per_volume": updates,
                       "parallelism": (f"one scan, z slabs split in blocks over {world} GPUs (no exchange)"
                                       if world > 1 else "1 GPU"),
                       "flush": "inputs larger than L2 (44.7 GB of fan data)"},
            "roofline": roof,
            "e2e": {"value": updates / e2e_s / 1e9, "unit": "GUPS", "s_per_volume": e2e_s,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "host_memory": "pinned" if pinned else "pageable",
                    "entry": "hr_slab_execute_range (C ABI, host buffers; views shared by consecutive slabs "
                             "are copied once)"},
            "hu_rmse_vs_plain_by_slab": per_slab,
            # per slab: rebin, split, Toeplitz GEMM, then the backprojection's kernels
            "gpu_launches": (3 + fast_launches_per_bp(desc)) * nslabs * args.steps,
            "kernels": desc, "clocks": clocks.summary()}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def run_batch(args, dev, world, rank, barrier, emit=True):
    """Twelve uneven scans (rotations 2..30, rows 16/32/64, three pitches, 256^2 or
    512^2 x 32..400 slices, Poisson noise at I0 = 2e5) through one BatchRecon:
    per-scan rebin + tensor-core filter, one persistent backprojection launch."""
    import torch
    import torch.distributed as dist

    from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
    from analyticalreconbigpatient_b200.pipeline import BatchRecon, HelicalRecon, add_poisson_noise, project

    scans = G.batch_scans()
    fans = []
    for i, sc in enumerate(scans):
        zlo = sc.h * sc.BetaS / (2 * np.pi)
        zhi = sc.h * (sc.BetaS + sc.views * sc.dBeta) / (2 * np.pi)
        f = project(sc, P.random_ellipsoids(5000 + 100 * rank + i, 60, (zlo, zhi)), device=dev.index)
        add_poisson_noise(f, 2e5, 7000 + 100 * rank + i)
        fans.append(f)
    updates = sum(sc.updates() for sc in scans)
    vols = [torch.empty((sc.YN, sc.XN, sc.ZN), dtype=torch.float32, device=dev) for sc in scans]
    rec = BatchRecon(scans, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        rec.run(fans, vols)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(None)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        rec.run(fans, vols)
    t1.record(stream)
    torch.cuda.synchronize()
    clocks.stop()
    ms = t0.elapsed_time(t1) / args.steps
    rec.check()
    # the persistent backprojection alone (roofline)
    t0.record(stream)
    for _ in range(args.steps):
        rec.backproject(vols)
    t1.record(stream)
    torch.cuda.synchronize()
    bp_ms = t0.elapsed_time(t1) / args.steps
    ms, bp_ms = max_over_ranks([ms, bp_ms], world, dev)
    desc = rec.describe()
    batch_vols = [v.cpu() for v in vols]
    # e2e: pinned host fans in, volumes out, every step, through the C ABI's host entry (the fans stream in
    # under the earlier scans' computation, each volume leaves when its scan is done); for comparison the
    # same batch with all copies in, the device entry, then all copies out
    h_fans = [torch.empty(f.shape, dtype=torch.float32, pin_memory=True) for f in fans]
    for h, f in zip(h_fans, fans):
        h.copy_(f)
    h_vols = [torch.empty(v.shape, dtype=torch.float32, pin_memory=True) for v in vols]

    def serial_step():
        for h, f in zip(h_fans, fans):
            f.copy_(h, non_blocking=True)
        rec.run(fans, vols)
        for h, v in zip(h_vols, vols):
            h.copy_(v, non_blocking=True)
        torch.cuda.synchronize()

    def host_step():
        rec.run_host(h_fans, h_vols)

    e2e = {}
    for name, step in (("serial", serial_step), ("host_entry", host_step)):
        step()
        barrier()
        e2e_t = []
        for _ in range(max(1, args.e2e_steps)):
            t = time.perf_counter()
            step()
            e2e_t.append(time.perf_counter() - t)
        (e2e[name],) = max_over_ranks([statistics.median(e2e_t)], world, dev)
    host_max_err = max(float((h - b).abs().max()) for h, b in zip(h_vols, batch_vols))
    e2e_s = e2e["host_entry"]
    del h_fans, h_vols
    rec.close()
    del vols
    torch.cuda.empty_cache()
    # each scan alone: the fast chain (timed, for the batching gain) and the plain FP32 chain (HU reference)
    per_scan, solo_ms = [], 0.0
    for sc, fan, bv in zip(scans, fans, batch_vols):
        fast = HelicalRecon(sc, form=_lib.HR_FORM_FAST, device=dev)
        fast.run(fan)
        torch.cuda.synchronize()
        t0.record(stream)
        for _ in range(args.steps):
            fast.run(fan)
        t1.record(stream)
        torch.cuda.synchronize()
        solo_ms += t0.elapsed_time(t1) / args.steps
        fast.close()
        plain = HelicalRecon(sc, form=_lib.HR_FORM_PLAIN, device=dev)
        ref = plain.run(fan).cpu()
        plain.close()
        torch.cuda.empty_cache()
        hu = float(torch.sqrt(torch.mean((bv.double() - ref.double()) ** 2))) / G.MU_WATER * 1000.0
        per_scan.append({"rotations": sc.rotations, "rows": sc.ZL, "pitch": sc.pitch, "grid": [sc.XN, sc.YN, sc.ZN],
                         "dz_mm": round(sc.dz, 4), "updates": sc.updates(), "hu_rmse_vs_plain_solo": hu})
    pk, pk_kind = peaks()
    ach = BYTES_PER_UPDATE_BF16 * updates / (bp_ms * 1e-3) / 1e9
    n = len(scans)
    if "persistent launch" in desc:
        textured = "FP16 textures" in desc
        bp_kernel = (("bp_tex_seg_batch_kernel" if "segmented" in desc else "bp_tex_batch_spec_kernel"
                      if "specialised" in desc else "bp_tex_batch_kernel") if textured else "bp_fast_batch_kernel")
        how = "one persistent backprojection launch"
        bp_launches = 1 + (2 * n if textured else 0)  # + the FP16 scale and fill kernels per scan
    else:
        solo_v = [int(t) for t in desc.split("variant by scan:")[1].split("(")[0].split()]
        n_tex = sum(v >= 11 for v in solo_v)
        bp_kernel = (("bp_tex_seg_kernel" if any(v >= 16 for v in solo_v) else "bp_tex_kernel") if n_tex
                     else "bp_fast_kernel")
        bp_kernel += " per scan, on parallel streams"
        how = "each scan's backprojection on a stream of its own"
        bp_launches = n + 2 * n_tex
    line = {"metric": "GUPS (voxel-view updates/s, rebin+filter+3D-weighted helical BP)",
            "value": updates * world / (ms * 1e-3) / 1e9, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "s_per_batch": ms * 1e-3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (analytic FP64 projections of 60 seeded random ellipsoids per scan, Poisson noise "
                    "at I0=2e5 before the log)",
            "form": f"fast (uneven batch, {how})",
            "config": {"workload": f"{len(scans)} uneven helical scans (888-channel curved detector, 984 views/rot; "
                                   "rotations 2..30, rows 16/32/64, pitch 0.5/0.9375/1.375, 256^2 or 512^2 x 32..400 "
                                   "slices; seed 6)",
                       "updates_per_batch": updates, "fan_bytes": sum(sc.projection_bytes() for sc in scans),
                       "flush": "inputs larger than L2 (22 GB of fan data)"},
            "roofline": {"bound": "hbm", "kernel": bp_kernel, "achieved": ach, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": ach / pk["hbm_gbs"], "peak_source": pk_kind, "traffic": None,
                         "backprojection_ms": bp_ms,
                         "note": "gather-equivalent bytes (8 B/update) / batch backprojection time"},
            "e2e": {"value": updates * world / e2e_s / 1e9, "unit": "GUPS", "s_per_batch": e2e_s,
                    "h2d_bytes_per_step": sum(sc.projection_bytes() for sc in scans),
                    "d2h_bytes_per_step": sum(sc.volume_bytes() for sc in scans),
                    "entry": "hr_batch_execute_host (C ABI, pinned host buffers; copies overlap the scans' "
                             "computation)",
                    "serial_copies_s": e2e["serial"], "max_abs_diff_vs_device_entry": host_max_err},
            "gpu_launches": (3 * n + bp_launches) * args.steps,
            "solo_fast_sum_ms": solo_ms, "batch_speedup_vs_solo": solo_ms / ms,
            "max_hu_rmse_vs_plain_solo": max(p["hu_rmse_vs_plain_solo"] for p in per_scan),
            "per_scan": per_scan, "kernels": desc, "clocks": clocks.summary()}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def run_learned(args, dev, world, rank, barrier, emit=True):
    """Half-view (492 views/rot) plain reconstruction corrected by the 2.5D CNN,
    trained on pairs the plain method makes from seeded noisy phantoms, against
    the full-view (984 views/rot) plain reconstruction: HU RMSE on held-out
    phantoms, and seconds per 10-rotation volume end to end."""
    import torch
    import torch.distributed as dist

    from analyticalreconbigpatient_b200 import _lib, geometry as G, learned as L, phantom as P
    from analyticalreconbigpatient_b200.pipeline import HelicalRecon, add_poisson_noise, project

    t_start = time.perf_counter()
    train = L.PairSet(range(1, 1 + args.train_phantoms), device=dev.index)
    t_data = time.perf_counter() - t_start
    net = L.Corrector(seed=rank, device=dev)
    t0 = time.perf_counter()
    losses = L.train(net, train, steps=args.train_steps, batch=8, lr=1e-3, seed=rank)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del train
    torch.cuda.empty_cache()
    test = L.PairSet(range(100001, 100001 + args.eval_phantoms), device=dev.index)
    ev = L.evaluate(net, test)
    del test
    torch.cuda.empty_cache()

    # ---- one 10-rotation volume: full-view plain vs half-view plain + CNN ---------
    full = G.Scan(ZL=64, pitch=0.984, rotations=10, N_2pi=984, XN=512, YN=512, ZN=1, dx=0.9766, dy=0.9766,
                  dz=0.625)
    full = G.replace(full, beta_start=full.BetaS)
    half = G.replace(full, N_2pi=492).with_full_z()
    full = G.replace(full, ZN=half.ZN)
    zlo = full.h * full.BetaS / (2 * np.pi)
    zhi = full.h * (full.BetaS + full.views * full.dBeta) / (2 * np.pi)
    fan = project(full, P.random_ellipsoids(200001 + rank, 60, (zlo, zhi)), device=dev.index)
    add_poisson_noise(fan, 1e5, 0x5EED0000 + 200001 + rank)
    h_full = torch.empty(fan.shape, dtype=torch.float32, pin_memory=True)
    h_full.copy_(fan)
    h_half = torch.empty((half.views, half.YL, half.ZL), dtype=torch.float32, pin_memory=True)
    h_half.copy_(fan[::2])
    del fan
    rf = HelicalRecon(full, form=_lib.HR_FORM_PLAIN, device=dev)
    # the half view is reconstructed with the chosen (fast) form; the plain form beside it
    rh = {"fast": HelicalRecon(half, form=_lib.HR_FORM_FAST, device=dev),
          "plain": HelicalRecon(half, form=_lib.HR_FORM_PLAIN, device=dev)}
    v_half = {k: torch.empty((half.YN, half.XN, half.ZN), dtype=torch.float32, device=dev) for k in rh}
    v_out = {k: torch.empty_like(v_half[k]) for k in rh}
    h_out = torch.empty((half.YN, half.XN, half.ZN), dtype=torch.float32, pin_memory=True)
    h_ref = torch.empty_like(h_out, pin_memory=True)

    def learned_step(kind):
        # the C ABI host entry from pinned memory into the device volume the network reads (the fast form
        # streams the fan in under its rebinning, filtering and backprojection)
        rh[kind].run_host(h_half, v_half[kind])
        net.apply_volume(v_half[kind], v_out[kind])
        h_out.copy_(v_out[kind], non_blocking=True)
        torch.cuda.synchronize()

    def full_step():
        rf.run_host(h_full, h_ref)

    for _ in range(args.warmup):
        learned_step("fast")
        learned_step("plain")
        full_step()
    barrier()
    clocks = ClockSampler(None)
    clocks.start()
    tl, tlp, tf, tc = [], [], [], []
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        t = time.perf_counter()
        learned_step("fast")
        tl.append(time.perf_counter() - t)
        t = time.perf_counter()
        learned_step("plain")
        tlp.append(time.perf_counter() - t)
        t = time.perf_counter()
        full_step()
        tf.append(time.perf_counter() - t)
        e0.record(stream)
        net.apply_volume(v_half["fast"], v_out["fast"])
        e1.record(stream)
        torch.cuda.synchronize()
        tc.append(e0.elapsed_time(e1))
    clocks.stop()
    s_learned, s_learned_plain, s_full, cnn_ms = max_over_ranks(
        [statistics.median(tl), statistics.median(tlp), statistics.median(tf), statistics.median(tc)], world, dev)
    ref = h_ref.to(dev)
    hu = {k: (L.hu_rmse(v_out[k], ref), L.hu_rmse(v_half[k], ref)) for k in rh}
    hu_learned, hu_half = hu["fast"]
    net.check()
    rf.close()
    half_desc = rh["fast"].describe()
    for r in rh.values():
        r.close()
    # network FLOPs per slice: 2 * pixels * sum(9 * cin * cout) (padded channels counted)
    flops = 2.0 * half.XN * half.YN * sum(9 * ci * co for ci, co in zip(L.CIN, L.COUT)) * half.ZN
    pk, pk_kind = peaks()
    tflops = flops / (cnn_ms * 1e-3) / 1e12
    upd_half = half.updates()
    line = {"metric": "GUPS (voxel-view updates/s, rebin+filter+3D-weighted helical BP)",
            "value": upd_half * world / s_learned / 1e9, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": s_learned * 1e3, "s_per_volume": s_learned,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
            "data": "synthetic (seeded random-ellipsoid phantoms, Poisson noise at I0=1e5)",
            "form": "learned (half-view fast reconstruction + 2.5D CNN)",
            "config": {"workload": f"helical 888x64, pitch 0.984, 10 rot at 492 views/rot (every second view of "
                                   f"the 984-view scan) -> 512x512x{half.ZN} @ 0.9766x0.9766x0.625 mm",
                       "updates_per_volume": upd_half, "flush": "inputs larger than L2 (1.1 GB of fan data)"},
            "learned": {"train_phantoms": args.train_phantoms, "train_slices": args.train_phantoms * 16,
                        "train_steps": args.train_steps, "batch": 8, "train_s": t_train, "data_s": t_data,
                        "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:])),
                        "held_out_phantoms": args.eval_phantoms, **ev,
                        "volume_hu_rmse_learned": hu_learned, "volume_hu_rmse_half_view": hu_half,
                        "volume_hu_rmse_learned_on_plain_half": hu["plain"][0],
                        "volume_hu_rmse_plain_half_view": hu["plain"][1],
                        "s_per_volume_learned": s_learned, "s_per_volume_learned_on_plain_half": s_learned_plain,
                        "s_per_volume_full_view_plain": s_full,
                        "speedup_vs_full_view_plain": s_full / s_learned, "cnn_ms_per_volume": cnn_ms},
            "roofline": {"bound": "tensor", "kernel": "conv_tc_kernel (8 layers, whole volume)", "achieved": tflops,
                         "peak": pk["bf16_tflops"], "unit": "TFLOP/s", "frac": tflops / pk["bf16_tflops"],
                         "peak_source": pk_kind, "traffic": None,
                         "note": "network FLOPs (padded channels) / CNN time per volume; the conv layers are "
                                 "bound by activation traffic (32 channels: 144 FLOP per byte)"},
            "e2e": {"value": upd_half * world / s_learned / 1e9, "unit": "GUPS", "s_per_volume": s_learned,
                    "h2d_bytes_per_step": half.projection_bytes(), "d2h_bytes_per_step": half.volume_bytes(),
                    "entry": "HelicalRecon.run_host (hr_recon_execute_host, fast form: pinned half-view fan streamed in, "
                             "volume into device memory) + Corrector.apply_volume, volume out to pinned memory"},
            # per learned step: rebin, split, Toeplitz GEMM, the backprojection's kernels; then per 32-slice
            # chunk the input packing and 8 conv layers
            "gpu_launches": (3 + fast_launches_per_bp(half_desc) + 9 * ((half.ZN + 31) // 32)) * args.steps,
            "clocks": clocks.summary()}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    args = parse()
    import torch
    import torch.distributed as dist

    from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
    from analyticalreconbigpatient_b200.pipeline import project

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    scan = G.config("full" if args.config in ("batch", "learned") else args.config)
    if args.config == "bigpatient" and args.rotations > 0:
        scan = G.replace(scan, rotations=args.rotations, ZN=1)
        scan = G.replace(scan, ZN=scan.fully_sampled_slices())
    if args.impl == "reference":
        run_reference(args, scan, rank, world)
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    if args.config in ("bigpatient", "batch", "learned"):
        if args.config == "batch":
            run_batch(args, dev, world, rank, barrier)
        elif args.config == "learned":
            run_learned(args, dev, world, rank, barrier)
        else:
            run_bigpatient(args, scan, dev, world, rank, barrier)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- data (each rank its own seeded phantom) ------------------------------
    zlo = scan.h * scan.BetaS / (2 * np.pi)
    zhi = scan.h * (scan.BetaS + scan.views * scan.dBeta) / (2 * np.pi)
    objs = P.random_ellipsoids(1000 + rank, 60, (zlo, zhi)) if args.config != "small" else P.shepp_logan()
    fan = project(scan, objs, device=local)
    updates = scan.updates()
    chosen = _lib.HR_FORM_FAST if args.form == "fast" else _lib.HR_FORM_PLAIN

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    res = measure_form(args, scan, chosen, fan, dev, world, barrier)
    clocks.stop()
    plain = None
    if chosen != _lib.HR_FORM_PLAIN and not args.no_plain:
        plain = measure_form(args, scan, _lib.HR_FORM_PLAIN, fan, dev, world, barrier, with_e2e=False)
    del fan
    ms = res["ms_per_step"]
    value = updates * world / (ms * 1e-3) / 1e9
    e2e_value = updates * world / res["e2e_s"] / 1e9

    # ---- roofline of the dominant kernel ----------------------------------------
    pk, pk_kind = peaks()
    bp_ms = res["stages_ms"]["backprojection"]
    bytes_per_update = BYTES_PER_UPDATE_BF16 if chosen == _lib.HR_FORM_FAST else BYTES_PER_UPDATE_FP32
    textured = chosen == _lib.HR_FORM_FAST and "texture" in res["kernels"]
    kname = (("bp_tex_seg_kernel" if "segmented" in res["kernels"] else "bp_tex_kernel") if textured
             else "bp_fast_kernel") if chosen == _lib.HR_FORM_FAST else "bp_plain_q_kernel"
    achieved = bytes_per_update * updates / (bp_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "peak_source": pk_kind,
                "algorithmic_bytes_per_launch": bytes_per_update * updates,
                "bytes_per_update": bytes_per_update,
                "traffic": traffic_from_profiles(kname.replace("_kernel", ""), args.config),
                "note": "gather-equivalent bytes (4 taps per update: 16 B FP32, 8 B BF16) / backprojection kernel "
                        "time; the backprojection is gather/issue bound, its compulsory DRAM bytes are only the "
                        "filtered data and the volume"}
    if textured:
        # the taps come from the texture units' bilinear filtering (one sample per update), whose
        # rate on this device the library measures; the backprojection time includes filling the
        # layered FP16 copy of the filtered data
        from analyticalreconbigpatient_b200 import probe

        rate = probe.texture_sample_rate()
        samples = updates / (bp_ms * 1e-3) / 1e9
        roofline["texture"] = {"achieved": samples, "peak": rate / 1e9, "unit": "Gsample/s",
                               "frac": samples * 1e9 / rate if rate > 0 else None,
                               "peak_source": "measured (libhelixprobe.so hr_texture_sample_rate: cache-resident FP16 layered "
                                              "texture, every lane active)"}
        roofline["note"] = ("gather-equivalent bytes (4 FP16 taps = 8 B per update) / backprojection time "
                            "(texture fill included); the taps are bilinear texture samples, so the bound is the "
                            "texture units' sample rate (roofline.texture), not HBM")

    line = {"metric": "GUPS (voxel-view updates/s, rebin+filter+3D-weighted helical BP)", "value": value,
            "unit": "GUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "s_per_volume": ms * 1e-3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16" if chosen == _lib.HR_FORM_FAST else "f32",
            "data": "synthetic (analytic FP64 projections of seeded random-ellipsoid phantoms)",
            "form": args.form,
            "config": chain_config(scan, args.config, world),
            "stages_ms": res["stages_ms"],
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": "GUPS", "s_per_volume": res["e2e_s"],
                    "h2d_bytes_per_step": scan.projection_bytes(), "d2h_bytes_per_step": scan.volume_bytes(),
                    "entry": res["e2e_entry"],
                    **({"chain_s": res["e2e_chain_s"], "slab_s": res["e2e_slab_s"],
                        "slab_device_ms": res["slab_device_ms"]} if "e2e_slab_s" in res else {})},
            "gpu_launches": res["launches_per_step"] * args.steps,
            "kernels": res["kernels"],
            "clocks": clocks.summary()}
    if plain is not None:
        pv = updates * world / (plain["ms_per_step"] * 1e-3) / 1e9
        line["plain"] = {"value": pv, "unit": "GUPS", "ms_per_step": plain["ms_per_step"],
                         "stages_ms": plain["stages_ms"], "speedup_of_chosen": value / pv}
    if rank == 0 and not args.no_cpu_baseline:
        gups, spv, detail = cpu_baseline(scan)
        line["cpu_baseline"] = {"value": gups, "unit": "GUPS", "cores": detail["cores"], "kind": detail["kind"],
                                "sample": detail["sample"], "s_per_volume": spv, "extrapolated": True,
                                "sample_updates": detail["sample_updates"], "sample_wall_s": detail["sample_wall_s"]}
        # beside it, a straight CPU build of the same formulas (the C restatement in oracle/)
        gups_p, spv_p, detail_p = cpu_baseline(scan, budget_s=10.0, kind="port")
        line["cpu_port"] = {"value": gups_p, "unit": "GUPS", "cores": detail_p["cores"], "kind": "port",
                            "sample": detail_p["sample"], "s_per_volume": spv_p}
    if args.config == "full" and world == 1 and not args.no_extra:
        line.update(run_extras(args, dev, world, rank, barrier))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_extras(args, dev, world, rank, barrier):
    """The other workloads, each run after the main one in the same process and
    attached to its line: the 200-rotation big patient (slab pipeline), the
    12-scan uneven batch and the learned half-view correction. Each keeps its
    own value, e2e, error figure, launches and clocks."""
    import torch

    from analyticalreconbigpatient_b200 import geometry as G

    sub = argparse.Namespace(**vars(args))
    sub.steps = max(1, args.extra_steps)
    sub.warmup = min(args.warmup, 3)
    sub.e2e_steps = min(args.e2e_steps, 3)
    out = {}
    for name, fn in (("bigpatient", lambda: run_bigpatient(sub, G.config("bigpatient"), dev, world, rank, barrier,
                                                            emit=False)),
                     ("batch", lambda: run_batch(sub, dev, world, rank, barrier, emit=False)),
                     ("learned", lambda: run_learned(sub, dev, world, rank, barrier, emit=False))):
        t = time.perf_counter()
        try:
            res = fn()
            res = {k: v for k, v in res.items() if k not in ("metric", "unit", "higher_is_better", "vs_baseline")}
        except Exception as e:  # a failing sub-workload is reported, the main line stands
            res = {"error": f"{type(e).__name__}: {e}"}
        res["wall_s"] = time.perf_counter() - t
        out[name] = res
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    main()
