#!/usr/bin/env python
"""Benchmark of the B200 SIMPLEC hot path (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--precision 0|1] [--workload config1]

A step is one SIMPLEC outer iteration of config 1 (a single Gaussian hill,
128 x 128 x 64 cells, dx = 25 m, stretched layers to a 1500 m lid, log-law
inflow from the west, Coriolis, neutral): the local pseudo-time step, the
iteration (ghost fills, FP64 residual, momentum predictor with z-line sweeps,
the terrain pressure correction, theta and k sweeps, norms) and the host
driver's criterion and SER CFL. The metric is cell-updates/s (cells x
iterations / s). Under torchrun (N > 1) every rank iterates its own
independent instance (the path shards by instance: no collective on the data
path); the timed region is bracketed by a barrier and a device synchronise and
the max over ranks is reported.

--impl reference times the reference's CPU implementation of the path, here
the oracle (the FP64 C restatement; the reference itself needs AMReX, which
is not available), on every host thread, on the same workload and metric.
"""
import argparse
import ctypes
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
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None

        def num(s):
            try:
                return float(s)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        smax = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[n] for r in rows for n in range(4) if r[5 + n].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ the workload ---
# algorithmic words of one z-line sweep launch per point: a later sweep reads
# the 4 lateral coefficients, a_ZM, the two kept factors (1/m, c', in place of
# a_P and a_ZP), rhs and the lagged iterate and writes the new iterate (10);
# the first sweep of a solve (zero initial iterate, no lateral terms) reads
# a_P, a_ZM, a_ZP and rhs and writes the iterate (5)
LINE_WORDS_FIRST, LINE_WORDS = 5, 10
LINE_PROFILE = os.path.join(ROOT, "profiles", "zline_fact_multi_kernel_config1_fp64.txt")


def line_traffic_per_point():
    """DRAM bytes per point of the first and the later sweeps from the
    committed ncu capture (None when absent)."""
    vals = {}
    try:
        with open(LINE_PROFILE) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_point_"):
                    key, val = line.split(":")
                    vals[key.strip()[len("traffic_bytes_per_point_"):]] = float(val)
    except OSError:
        return None
    if "first" in vals and "later" in vals:
        return vals["first"], vals["later"]
    return None


class SimplecWorkload:
    def __init__(self, precision=0, sweeps=4):
        from ablsteadyrans_b200 import workloads
        self.inst = workloads.config1(precision=precision, zline_sweeps=sweeps)
        self.precision = precision
        self.sweeps = sweeps
        g = self.inst.grid
        self.name = (f"SIMPLEC outer iteration, config 1: Gaussian hill 150 m, {g.nx}x{g.ny}x{g.nz} cells, dx 25 m, "
                     f"{'plain FP64' if precision == 0 else 'FP32 inner solves in FP64 defect correction'}, "
                     f"zline_sweeps {sweeps}, pressure_reltol 1e-3"
                     f"{', k-L closure and surface layer' if self.inst.physics.closure else ''}")

    @property
    def cells(self):
        return self.inst.cells

    def line_bytes_per_step(self, per_point=None):
        """Bytes of the z-line sweep launches of one iteration (u, v, w,
        theta, k systems, `sweeps` sweeps each): algorithmic, or with
        per_point = (first, later) bytes per point."""
        g = self.inst.grid
        word = 8 if self.precision == 0 else 4
        first, later = per_point if per_point else (LINE_WORDS_FIRST * word, LINE_WORDS * word)
        total = 0
        for loc in (1, 2, 4, 0, 0):
            ni, nj, nk = g.extents(loc)
            total += ni * nj * nk * (first + later * (self.sweeps - 1))
        return total

    def setup(self, ctx):
        import torch

        import ablsteadyrans_b200 as gb
        from ablsteadyrans_b200.driver import Driver
        from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
        inst = self.inst
        g = inst.grid
        z = torch.from_numpy(inst.z).cuda()
        J, ax, ay, az, _ = gb.mesh_metrics(ctx, g, z)
        self.case = DeviceCase(g, z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
        self.stage = SimplecStage(ctx, self.case, inst.bc, inst.physics, inst.options)
        self.stage.fill_ghosts()
        self.driver = Driver(self.stage)
        self.q0 = {f: t.clone() for f, t in self.case.q.items()}

    def step(self):
        return self.driver.step()

    # end to end: one solve through the public API from host memory. The
    # instance's initial state comes from pinned host buffers, the iterations
    # run with the state resident (as a steady solve keeps it), every step
    # reads its residual norms back (gb_iter_info), and the final state
    # returns to pinned host buffers.
    def e2e_setup(self, steps):
        import torch

        from ablsteadyrans_b200 import abi
        self.host_in = {f: t.cpu().pin_memory() for f, t in self.q0.items()}
        self.host_out = {f: torch.empty_like(t).pin_memory() for f, t in self.host_in.items()}
        state_bytes = sum(t.numel() * t.element_size() for t in self.host_in.values())
        info_bytes = ctypes.sizeof(abi.IterInfo)
        self.h2d = int(round(state_bytes / steps))
        self.d2h = int(round(state_bytes / steps)) + info_bytes

    def e2e_solve(self, steps):
        from ablsteadyrans_b200.driver import Driver
        for f, t in self.case.q.items():
            t.copy_(self.host_in[f], non_blocking=True)
        self.stage.fill_ghosts()
        driver = Driver(self.stage)
        status = "running"
        for _ in range(steps):
            status = driver.step()
        for f, t in self.case.q.items():
            self.host_out[f].copy_(t, non_blocking=True)
        return status

    # CPU: the oracle on the same instance
    def cpu_setup(self):
        import oracle
        inst = self.inst
        g = inst.grid
        J, ax, ay, az, _ = oracle.metrics(g, inst.z)
        self.ocase = oracle.Case(g, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.z0map)
        self.ocase.q = {f: a.copy() for f, a in inst.q.items()}
        oracle.fill_ghosts(self.ocase, inst.bc, inst.physics)
        self.ocfl = 1.0

    def cpu_step(self):
        import oracle
        inst = self.inst
        dt = oracle.local_dtau(self.ocase, self.ocfl, phys=inst.physics)
        rc, info, _ = oracle.simplec_iterate(self.ocase, inst.bc, inst.physics, inst.options, dt)
        return rc


def max_over_ranks(dist, x, device):
    """The job's time: the largest of every rank's (x itself on one rank)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank, world, steps, ms):
    """Cell updates per second of the whole job: every rank's instance, every
    step, over the slowest rank's time."""
    return cells_per_rank * world * steps / (ms / 1e3)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1])
    ap.add_argument("--sweeps", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="a context tuning knob (GB_TUNE_*, by number or name without the prefix), repeatable")
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
    wl = SimplecWorkload(precision=args.precision, sweeps=args.sweeps)
    ctx = gb.Context()
    for kv in args.tune:
        key, val = kv.split("=")
        ctx.tune(int(key) if key.isdigit() else getattr(gb, "TUNE_" + key.upper()), int(val))
    wl.setup(ctx)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)

    for _ in range(max(args.warmup, 3)):
        wl.step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # inside the timed region only the roofline kernel's family is bracketed by
    # events (timing every family costs the step about a fifth of its time)
    ctx.profile_mask([gb.KERNEL_LINE_SWEEP])
    ctx.profile(True)
    launches0 = ctx.launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    statuses = []
    for s in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the step's events)
        starts[s].record()
        statuses.append(wl.step())
        stops[s].record()
    torch.cuda.synchronize()
    launches = ctx.launches() - launches0
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, stops)]
    total_ms = sum(step_ms)
    sweep_ms, sweep_n = ctx.profile_read(gb.KERNEL_LINE_SWEEP)
    ctx.profile(False)
    clocks = sampler.stop()

    # per-family breakdown: a separate pass with every family timed
    nb = min(args.steps, 10)
    ctx.profile_mask(range(32))
    ctx.profile(True)
    b0 = torch.cuda.Event(enable_timing=True)
    b1 = torch.cuda.Event(enable_timing=True)
    b0.record()
    for _ in range(nb):
        wl.step()
    b1.record()
    torch.cuda.synchronize()
    families = {"profiled_ms_per_step": b0.elapsed_time(b1) / nb}
    names = ["line_sweep", "poisson_apply", "mg_smooth", "mg_transfer", "residual", "massflux", "coefs", "vector", "bc"]
    for fam, name in enumerate(names):
        ms, n = ctx.profile_read(fam)
        families[name] = {"ms_per_step": ms / nb, "launches_per_step": n / nb}
    ctx.profile(False)
    total_ms = max_over_ranks(dist, total_ms, "cuda")

    # end to end through the public API: one solve of K steps from host memory
    wl.e2e_setup(args.steps)
    wl.e2e_solve(2)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    wl.e2e_solve(args.steps)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(dist, e2e_ms, "cuda")

    value = whole_job_rate(wl.cells, world, args.steps, total_ms)
    e2e_value = whole_job_rate(wl.cells, world, args.steps, e2e_ms)
    peak, peak_kind = hbm_peak()
    line_bytes = wl.line_bytes_per_step() * args.steps
    achieved = (line_bytes / (sweep_ms / 1e3)) / 1e9 if sweep_ms > 0 else None
    tpp = line_traffic_per_point() if args.precision == 0 else None
    traffic = (wl.line_bytes_per_step(tpp) * args.steps / max(sweep_n, 1)) if tpp else None

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
        "dtype": "f64" if args.precision == 0 else "f64 outer, f32 inner",
        "data": ("synthetic (config 1 generated in-project: Gaussian hill, log-law inflow; k-L closure, neutral "
                 "MOST surface layer)" if wl.inst.physics.closure else
                 "synthetic (config 1 generated in-project: Gaussian hill, log-law inflow; frozen mixing-length "
                 "diffusivities, no-slip ground)"),
        "config": {"workload": wl.name, "cells": wl.cells, "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"independent instances x{world}", "driver_status_last": statuses[-1],
                   **({"tune": args.tune} if args.tune else {})},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": wl.h2d,
                "d2h_bytes_per_step": wl.d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "zline_fact_multi_kernel (z-line Thomas sweeps: u, v, w in one launch, theta and k in one)",
                     "peak_kind": peak_kind,
                     "bytes_per_launch": line_bytes / max(sweep_n, 1), "launch_ms": sweep_ms / max(sweep_n, 1)},
        "breakdown": families,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    if rank == 0:
        print(json.dumps(line))
    wl.stage.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(wl):
    """The oracle on a bounded sample of the same workload: one or two
    iterations of config 1 on every host thread."""
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    wl.cpu_setup()
    t0 = time.perf_counter()
    n = 0
    while True:
        wl.cpu_step()
        n += 1
        if time.perf_counter() - t0 > 20.0 or n >= 2:
            break
    dt = time.perf_counter() - t0
    return {"value": wl.cells * n / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{n} SIMPLEC iteration(s) of config 1 ({dt:.1f} s), oracle = FP64 C restatement"}


def run_reference(args):
    wl = SimplecWorkload(precision=0, sweeps=args.sweeps)
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    wl.cpu_setup()
    for _ in range(max(0, min(args.warmup, 3))):   # untimed warm-up iterations
        wl.cpu_step()
    t0 = time.perf_counter()
    n = 0
    budget = 90.0
    for s in range(max(1, args.steps)):
        wl.cpu_step()
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    value = wl.cells * n / dt
    line = {
        "impl": "reference",
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": 0,
        "steps": n, "warmup": max(0, min(args.warmup, 3)), "ms_per_step": dt / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (config 1 generated in-project)",
        "config": {"workload": wl.name, "cells": wl.cells},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{n} SIMPLEC iteration(s) of config 1 ({dt:.1f} s); the oracle, the FP64 C "
                                   "restatement of the reference (the reference needs AMReX)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
