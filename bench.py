#!/usr/bin/env python
"""Benchmark of the B200 SIMPLEC hot path (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one pass of the hot path over one batch of synthetic input (the
workload is named in the line's config). Under torchrun (N > 1) every rank
solves its own independent instances (the path shards by instance: no
collective on the data path); the timed region is bracketed by a barrier and
a device synchronise and the max over ranks is reported.

--impl reference times the reference's CPU implementation of the path, here
the oracle (the FP64 C restatement; the reference itself cannot be built
without AMReX), on the host cores with every thread it can use, on the same
workload, metric and unit.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ----------------------------------------------------------------- clocks ---
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[n] for r in rows for n in range(4) if r[5 + n].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------- workloads ---
class ZlinePhase:
    """The z-line relaxation phase of one SIMPLEC outer iteration on config 1's
    grid (128 x 128 x 64 cells): the five swept fields u, v, w, theta, k at
    their C-grid locations, each `sweeps` z-line Jacobi sweeps of a seeded
    M-matrix system (gust::zline_jacobi, Source/Predictor.cpp:87-127)."""

    name = "zline-relaxation phase, config 1 grid 128x128x64, 5 fields x 4 sweeps, FP64"

    def __init__(self, nx=128, ny=128, nz=64, sweeps=4, seed=1):
        from ablsteadyrans_b200.grid import Grid
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from helpers import random_system
        self.grid = Grid(nx, ny, nz, 25.0, 25.0, 1500.0 / nz, False, True)
        self.sweeps = sweeps
        self.locs = (1, 2, 4, 0, 0)
        self.systems = [random_system(self.grid, loc, seed + n, extra=0.2, xscale=2.0) for n, loc in enumerate(self.locs)]

    @property
    def cells(self):
        return self.grid.cells

    def algorithmic_bytes_per_step(self):
        """10 words per point per sweep (A off-diagonals 6, ap, rhs, delta_old
        read; delta_new written); the first sweep reads no delta_old (9)."""
        total = 0
        for loc in self.locs:
            ni, nj, nk = self.grid.extents(loc)
            pts = ni * nj * nk
            total += pts * 8 * (9 + 10 * (self.sweeps - 1))
        return total

    # device side
    def to_device(self):
        import torch
        self.dev = []
        for (A, ap, rhs) in self.systems:
            self.dev.append(tuple(torch.from_numpy(x).cuda() for x in (A, ap, rhs))
                            + (torch.zeros(self.grid.shape, dtype=torch.float64, device="cuda"),))

    def step(self, ctx):
        import ablsteadyrans_b200 as gb
        for loc, (A, ap, rhs, delta) in zip(self.locs, self.dev):
            gb.zline_jacobi(ctx, self.grid, loc, A, ap, rhs, self.sweeps, delta)

    def launches_per_step(self):
        n = 0
        for loc in self.locs:
            seam = (loc & 1 and self.grid.periodic_x) or (loc & 2 and self.grid.periodic_y)
            n += self.sweeps + (1 if seam else 0)
        return n

    # end-to-end: host inputs each step
    def e2e_setup(self):
        import torch
        self.host = [tuple(torch.from_numpy(x).pin_memory() for x in sysm) for sysm in self.systems]
        self.host_out = [torch.zeros(self.grid.shape, dtype=torch.float64).pin_memory() for _ in self.locs]
        self.h2d = sum(sum(t.numel() * 8 for t in sysm) for sysm in self.host)
        self.d2h = sum(t.numel() * 8 for t in self.host_out)

    def e2e_step(self, ctx):
        import ablsteadyrans_b200 as gb
        for n, loc in enumerate(self.locs):
            A, ap, rhs, delta = self.dev[n]
            hA, hap, hrhs = self.host[n]
            A.copy_(hA, non_blocking=True)
            ap.copy_(hap, non_blocking=True)
            rhs.copy_(hrhs, non_blocking=True)
            gb.zline_jacobi(ctx, self.grid, loc, A, ap, rhs, self.sweeps, delta)
            self.host_out[n].copy_(delta, non_blocking=True)

    # CPU: the oracle on the same systems
    def cpu_step(self, fields=None):
        import oracle
        out = self.grid.np_zeros()
        n = 0
        for idx, (loc, (A, ap, rhs)) in enumerate(zip(self.locs, self.systems)):
            if fields is not None and idx not in fields:
                continue
            oracle.zline_jacobi(self.grid, loc, A, ap, rhs, self.sweeps, out)
            n += 1
        return n


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        return run_reference(args)

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import ablsteadyrans_b200 as gb
    wl = ZlinePhase()
    wl.to_device()
    ctx = gb.Context()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)

    for _ in range(max(args.warmup, 3)):
        wl.step(ctx)
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.profile(True)
    launches0 = ctx.launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the step's events)
        starts[s].record()
        wl.step(ctx)
        stops[s].record()
    torch.cuda.synchronize()
    launches = ctx.launches() - launches0
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, stops)]
    total_ms = sum(step_ms)
    sweep_ms, sweep_n = ctx.profile_read(gb.KERNEL_LINE_SWEEP)
    ctx.profile(False)
    clocks = sampler.stop()
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())

    # end to end through the public API with host buffers
    wl.e2e_setup()
    for _ in range(2):
        wl.e2e_step(ctx)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(args.steps):
        wl.e2e_step(ctx)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    cells_per_step = wl.cells * world
    value = cells_per_step * args.steps / (total_ms / 1e3)
    e2e_value = cells_per_step * args.steps / (e2e_ms / 1e3)
    peak, peak_kind = hbm_peak()
    bytes_total = wl.algorithmic_bytes_per_step() * args.steps
    achieved = (bytes_total / (sweep_ms / 1e3)) / 1e9 if sweep_ms > 0 else None
    bytes_per_launch = bytes_total / max(sweep_n, 1)

    line = {
        "metric": "cell-updates/s",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded M-matrix line systems on config 1's grid)",
        "config": {"workload": wl.name, "cells": wl.cells, "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": wl.h2d,
                "d2h_bytes_per_step": wl.d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "kernel": "zline_sweep_kernel", "peak_kind": peak_kind,
                     "bytes_per_launch": bytes_per_launch, "launch_ms": sweep_ms / max(sweep_n, 1)},
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(wl):
    """The oracle on a bounded sample of the same workload, all host threads."""
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    t0 = time.perf_counter()
    n = 0
    fields = 0
    while True:
        fields += wl.cpu_step()
        n += 1
        if time.perf_counter() - t0 > 10.0 or n >= 5:
            break
    dt = time.perf_counter() - t0
    steps = fields / len(wl.locs)
    return {"value": wl.cells * steps / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{steps:.1f} steps of the same workload ({dt:.1f} s)"}


def run_reference(args):
    import torch  # noqa: F401  (not used for compute: the oracle runs on the host)
    wl = ZlinePhase()
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    for _ in range(max(1, min(args.warmup, 1))):
        wl.cpu_step()
    t0 = time.perf_counter()
    fields = 0
    budget = 60.0
    for s in range(args.steps):
        fields += wl.cpu_step()
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    steps = fields / len(wl.locs)
    value = wl.cells * steps / dt
    line = {
        "impl": "reference",
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": 0,
        "steps": steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded M-matrix line systems on config 1's grid)",
        "config": {"workload": wl.name, "cells": wl.cells},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{steps:.1f} steps ({dt:.1f} s), oracle = FP64 C restatement of the reference"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
