#!/usr/bin/env python
"""Benchmark of the B200 SIMPLEC hot path (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--precision 0|1] [--no-cpu] [--no-steady] [--no-batch] [--no-serve]

A step is one SIMPLEC outer iteration of config 1 (a single Gaussian hill,
128 x 128 x 64 cells, dx = 25 m, stretched layers to a 1500 m lid, log-law
inflow from the west, Coriolis, neutral, the k-L closure and the surface
layer): the local pseudo-time step, the iteration (ghost fills, FP64
residual, momentum predictor with z-line sweeps, the terrain pressure
correction, theta and k sweeps, norms) and the host driver's criterion and
SER CFL. The metric is cell-updates/s (cells x iterations / s). Under
torchrun (N > 1) every rank iterates its own independent instance (the path
shards by instance: no collective on the data path); the timed region is
bracketed by a barrier and a device synchronise and the max over ranks is
reported.

Beside the headline, on one GPU (N = 1): the Poisson kernels' rooflines
(the fine-level terrain operator, one V-cycle in FP64 and FP32), config 1
solved to the steady criterion in plain FP64 and with FP32 inner solves
(steady solves/s, iterations and the per-field difference of the two
steady states), and the batched form on a sample of the batched
configuration's uneven tiles (FP32 inner solves on concurrent streams
against plain FP64 one by one, cell-updates/s), and a bounded sample of the
served configuration (continuous batching against plain FP64 served one at
a time: p50/p99 latency and solves/s).

--impl reference times the reference's CPU implementation of the path, here
the FP64 C restatement of it (the reference itself needs AMReX, which is not
available), built for speed on the host that runs it, on every host thread,
on the same workload and metric.
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
#: B200 HBM3e's nominal rate (DGX figure), beside which fractions are also given
NOMINAL_HBM_GBS = 8000.0


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
LINE_PROFILE = os.path.join(ROOT, "profiles", "zline_seg_multi_kernel_config1_fp64.txt")


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


def bench_config(wl):
    """The `config` object of both arms' lines (the same workload)."""
    return {"workload": wl.name, "cells": wl.cells,
            "l2": "flushed between timed steps (256 MB write); the CPU arm has no flush to make"}


# ------------------------------------------------- the Poisson rooflines ---
# Algorithmic words per cell: the terrain operator apply reads phi, the
# three a beta, J and z_nd and writes y (7); a z-line zebra relaxation of a
# level reads phi, rhs, the three areas, J and z_nd and writes phi (8); the
# residual of a level is an apply (7); restriction reads the fine residual
# and writes a quarter coarse value (1.25 per fine cell), prolongation reads
# a quarter coarse value and phi and writes phi (2.25 per fine cell).
APPLY_WORDS, RELAX_WORDS, RESTRICT_WORDS, PROLONG_WORDS = 7, 8, 1.25, 2.25


def mg_levels(nx, ny, max_levels, min_coarse):
    """The multigrid's levels (nx, ny): x and y halved while both stay even
    and at least min_coarse, at most max_levels."""
    out = [(nx, ny)]
    while len(out) < max_levels:
        cx, cy = out[-1]
        if cx % 2 or cy % 2 or cx // 2 < min_coarse or cy // 2 < min_coarse:
            break
        out.append((cx // 2, cy // 2))
    return out


def vcycle_words(nx, ny, nz, opts):
    """Algorithmic words of one V-cycle per the table above."""
    levels = mg_levels(nx, ny, opts.max_levels, opts.min_coarse)
    words = 0.0
    for n, (lx, ly) in enumerate(levels):
        cells = lx * ly * nz
        if n == len(levels) - 1:
            words += opts.nu_coarse * RELAX_WORDS * cells
        else:
            words += ((opts.nu1 + opts.nu2) * RELAX_WORDS + APPLY_WORDS + RESTRICT_WORDS + PROLONG_WORDS) * cells
    return words, len(levels)


def poisson_rooflines(ctx, wl, flush, peak, reps=12):
    """The fine-level terrain operator (FP64) and one V-cycle (FP64, FP32)
    on config 1's mesh, each launch timed alone by CUDA events on the
    context's stream with a 256 MB L2 flush before it (the level's arrays
    would otherwise sit in the 126 MB L2)."""
    import torch

    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.abi import FACE_INFLOW, FACE_OUTFLOW, FACE_PERIODIC
    g = wl.inst.grid
    case = wl.case
    face = list(wl.inst.bc.face)

    def pbc(t):
        if t == FACE_PERIODIC:
            return gb.POISSON_PERIODIC
        return gb.POISSON_DIRICHLET if t == FACE_OUTFLOW else gb.POISSON_NEUMANN
    bc = tuple(pbc(t) for t in face)
    assert FACE_INFLOW in face
    rng = np.random.default_rng(1)
    r = torch.from_numpy(g.np_zeros()).cuda()
    v = g.valid(0)
    r_host = g.np_zeros()
    r_host[v] = rng.standard_normal(r_host[v].shape)
    r.copy_(torch.from_numpy(r_host))
    out = []
    cells = g.nx * g.ny * g.nz
    stream = ctx.stream
    for prec in (0, 1):
        opts = gb.PoissonOptions.default(precision=prec)
        ps = gb.PoissonSolver(ctx, g, case.z, case.J, bc, opts)
        ps.set_coeffs(case.ax, case.ay, case.az)
        y = torch.zeros_like(r)
        kinds = [("apply", None)] if prec == 0 else []
        kinds.append(("vcycle", None))
        for kind, _ in kinds:
            fn = (lambda: ps.apply(r, out=y)) if kind == "apply" else (lambda: ps.vcycle(r, out=y))
            for _ in range(3):
                fn()
            ms = []
            for _ in range(reps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    fn()
                    e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            t = statistics.median(ms)
            if kind == "apply":
                words, what = APPLY_WORDS * cells, ("k_apply: the terrain operator on the fine level "
                                                   f"({g.nx}x{g.ny}x{g.nz}), FP64; 7 words per cell")
                word = 8
            else:
                words, nlev = vcycle_words(g.nx, g.ny, g.nz, opts)
                word = 8 if prec == 0 else 4
                what = (f"one multigrid V-cycle ({nlev} levels, nu1 = nu2 = {opts.nu1}, {opts.nu_coarse} coarsest "
                        f"relaxations), {'FP64' if prec == 0 else 'FP32'}; 8 words per cell and relaxation, 7 per "
                        "residual, 1.25 restriction, 2.25 prolongation")
            nbytes = words * word
            achieved = nbytes / (t / 1e3) / 1e9
            out.append({"kernel": what, "bound": "hbm", "bytes_per_launch": nbytes, "launch_ms": t,
                        "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak})
        ps.close()
    return out


# ----------------------------------------------------------- the residual ---
# algorithmic words of one residual evaluation per cell: the state (u, v, w,
# p, theta, k), the mesh (z, J and the three areas) read, the six residuals
# written; the closure's and the transport's fields are its intermediates
RESIDUAL_WORDS = 17
RESIDUAL_PROFILE = os.path.join(ROOT, "profiles", "k_fused_residual_fp64_flops_config1.txt")


def residual_flops():
    """FP64 operations of one residual evaluation of config 1 (ncu's FP64
    instruction counters over every launch of one call; committed capture),
    or None."""
    try:
        with open(RESIDUAL_PROFILE) as f:
            for line in f:
                if line.startswith("fp64_flops_per_residual:"):
                    return float(line.split(":")[1])
    except OSError:
        return None
    return None


def fp64_peak(ctx, iters=4096, reps=5):
    """The FP64 pipe's rate on this GPU, measured in-project (gb_probe_fp64:
    chains of dependent FMAs on every SM), best of reps, TFLOP/s."""
    import torch

    import ablsteadyrans_b200 as gb
    sink = torch.zeros(4 * torch.cuda.get_device_properties(0).multi_processor_count * 256, dtype=torch.float64,
                       device="cuda")
    best = 0.0
    stream = ctx.stream
    for _ in range(reps + 1):
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            flops = gb.probe_fp64(ctx, iters, sink)
            e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, flops / (e0.elapsed_time(e1) / 1e3) / 1e12)
    return best


def residual_roofline(ctx, wl, flush, hbm_peak, reps=12):
    """One residual evaluation of config 1 (the closure and the surface
    state at the state, the transport, the stresses, the per-equation
    launches, the forcing, the boundary rows) timed alone by CUDA events on
    the context's stream after a 256 MB L2 flush, against the HBM roofline
    of its algorithmic bytes and the FP64 roofline of its counted FP64
    operations (the FP64 peak measured in-project). One more evaluation runs
    inside the NVTX range "gust_residual", which the ncu capture that counts
    the operations selects."""
    import torch
    g = wl.inst.grid
    cells = g.nx * g.ny * g.nz
    R = [torch.zeros(g.shape, dtype=torch.float64, device="cuda") for _ in range(6)]
    stream = ctx.stream
    for _ in range(3):
        wl.stage.residual(out=R)
    ms = []
    for _ in range(reps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            wl.stage.residual(out=R)
            e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    torch.cuda.nvtx.range_push("gust_residual")
    wl.stage.residual(out=R)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    t = statistics.median(ms)
    nbytes = RESIDUAL_WORDS * 8 * cells
    peak64 = fp64_peak(ctx)
    flops = residual_flops()
    out = {"kernel": (f"one SIMPLEC residual evaluation of config 1 ({g.nx}x{g.ny}x{g.nz}, k-L closure and surface "
                      f"layer), FP64; {RESIDUAL_WORDS} words per cell"),
           "launch_ms": t, "bytes_per_launch": nbytes, "achieved_gbs": nbytes / (t / 1e3) / 1e9,
           "hbm_peak_gbs": hbm_peak, "hbm_frac": nbytes / (t / 1e3) / 1e9 / hbm_peak,
           "fp64_peak_tflops_measured": peak64, "fp64_flops_per_launch": flops}
    if flops is not None:
        tf = flops / (t / 1e3) / 1e12
        out["achieved_tflops"] = tf
        out["fp64_frac"] = tf / peak64
        # the bound: the resource whose roofline time is the longer
        out["bound"] = "fp64" if flops / (peak64 * 1e12) > nbytes / (hbm_peak * 1e9) else "hbm"
    return out


# ------------------------------------------------------------ steady solves ---

def steady_solves(max_iterations=3000, config=1):
    """Config 1 (or config 2: the 256 x 256 x 96 fractal terrain, slopes
    capped at 1) from the mass-consistent initial field to the steady
    criterion (the C++ driver), in plain FP64 and with FP32 inner solves:
    iterations, device seconds, steady solves/s, and the difference of the
    two steady states per field (max |mixed - FP64| / max |FP64|) and of
    the velocity vector in the 2-norm."""
    import torch

    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200 import workloads
    from ablsteadyrans_b200.sequencing import _finest
    from ablsteadyrans_b200.simplec import NativeDriver, run_drivers
    res = {}
    fields = {}
    for prec in (0, 1):
        # config 2 with frozen diffusivities: with the closure it is not steady
        # within 3000 iterations (measured 57.6 s in FP64), so the two forms'
        # difference would compare two transients
        inst = (workloads.config1(precision=prec) if config == 1
                else workloads.config2(precision=prec, turbulence=False))
        ctx = gb.Context()
        case, stage = _finest(ctx, inst)
        stage.initialize()
        stage.fill_ghosts()
        d = NativeDriver(stage)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ctx.stream)
        (verdict, n), = run_drivers([d], max_iterations, 1)
        e1.record(ctx.stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        key = "fp64" if prec == 0 else "fp32_inner"
        res[key] = {"verdict": verdict, "iterations": n, "seconds": sec,
                    "solves_per_s": (1.0 / sec) if verdict == "steady" else None,
                    "cell_updates_per_s": inst.cells * n / sec}
        g = inst.grid
        fields[key] = {f: (case.q[f].cpu().numpy(), loc) for f, loc in zip(("u", "v", "w", "p", "theta", "tke"),
                                                                           (1, 2, 4, 0, 0, 0))}
        fields[key]["grid"] = g
        d.close()
        stage.close()
        ctx.close()
    g = fields["fp64"]["grid"]
    err = {}
    for f in ("u", "v", "w", "p", "theta", "tke"):
        a, loc = fields["fp32_inner"][f]
        b, _ = fields["fp64"][f]
        vv = g.valid(loc)
        scale = float(np.abs(b[vv]).max())
        err[f] = float(np.abs(a[vv] - b[vv]).max()) / (scale if scale > 0 else 1.0)
    res["fp32_inner_vs_fp64_rel_err"] = err
    # the velocity vector's relative error in the 2-norm over all valid points
    # (u, v and w at their faces): ||mixed - FP64|| / ||FP64||
    num = den = 0.0
    for f in ("u", "v", "w"):
        a, loc = fields["fp32_inner"][f]
        b, _ = fields["fp64"][f]
        vv = g.valid(loc)
        num += float(np.sum((a[vv] - b[vv]) ** 2))
        den += float(np.sum(b[vv] ** 2))
    res["fp32_inner_vs_fp64_velocity_rel_l2"] = (num / den) ** 0.5 if den > 0 else None
    res["speedup_fp32_inner"] = res["fp64"]["seconds"] / res["fp32_inner"]["seconds"]
    if config == 1:
        res["workload"] = ("config 1 (128x128x64 hill) from the mass-consistent initial field to the steady criterion "
                           "(4 orders, monitors settled), the C++ driver; device time")
    else:
        g = fields["fp64"]["grid"]
        res["workload"] = (f"config 2 ({g.nx}x{g.ny}x{g.nz} fractal terrain, 120 m rms, node-to-node slopes capped at "
                           f"{workloads.MAX_TILE_SLOPE:g}, u* 0.4 m/s from 225 deg, frozen diffusivities: the closure "
                           f"and the surface layer off) from the mass-consistent initial field to the steady criterion "
                           f"or {max_iterations} iterations; device time")
    return res


def batched_leg(count=16, iterations=10, warmup=2):
    """A sample of the batched configuration (its first `count` uneven tiles
    of the 48, drawn as config 3): every tile's outer iterations with FP32
    inner solves on concurrent streams (the batched form), against the same
    tiles in plain FP64 one by one; cell-updates/s of each (device time)."""
    import torch

    from ablsteadyrans_b200.batch import Batch, config3
    from ablsteadyrans_b200.autotune import Autotuner
    out = {}
    insts = config3(count, 0, precision=1)
    cells = sum(i.cells for i in insts)
    batch = Batch(insts, tuner=Autotuner(iterations=2))
    out["autotuned"] = batch.choices
    batch.run_native(warmup, threads=0)
    ms, _ = batch.run_native(iterations, threads=0)
    out["batched_fp32_inner"] = cells * iterations / (ms / 1e3)
    ms1, _ = batch.run_native(iterations, threads=1)
    out["one_by_one_fp32_inner"] = cells * iterations / (ms1 / 1e3)
    batch.close()
    del batch
    torch.cuda.empty_cache()
    total = 0.0
    for inst in config3(count, 0, precision=0):
        b = Batch([inst])
        b.run_native(warmup, threads=1)
        t, _ = b.run_native(iterations, threads=1)
        total += t
        b.close()
        torch.cuda.empty_cache()
    out["one_by_one_fp64"] = cells * iterations / (total / 1e3)
    out["speedup_batched_fp32_inner_vs_fp64_one_by_one"] = out["batched_fp32_inner"] / out["one_by_one_fp64"]
    out["workload"] = (f"the first {count} of config 3's 48 uneven tiles (n in 64..192, nz in 48..96; {cells} cells), "
                       f"{iterations} outer iterations each after {warmup}; cell-updates/s")
    return out


def batched_sweep_leg(count=48, sweeps=4, reps=3, tune=True):
    """The z-line sweeps of config 3's uneven tiles in one work-list (the
    batched solve, gb_zline_jacobi_batch: one persistent launch per sweep
    and column-height group) against the same systems one call each
    (gb_zline_jacobi, each call reading its system's max |change| back, as
    the batched call reads all of them once) on one stream: the u, v and w
    systems of each of the
    `count` tiles (n x n x nz drawn as config 3), seeded diagonally dominant
    coefficients, `sweeps` sweeps, FP64 and FP32, both forms at the levels
    per warp the autotuner picks for the batch (tune false: the default 5);
    device time per pass, the
    best of `reps` after one untimed pass, and the batched launches' HBM
    rate on the sweep's algorithmic bytes (5 words a point in the first
    sweep, 10 in each later one)."""
    import torch

    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.autotune import Autotuner, tune_batch_sweep
    from ablsteadyrans_b200.batch import CONFIG3_LAYERS, CONFIG3_SIZES
    rng = np.random.default_rng(0)
    shapes = [(int(rng.choice(CONFIG3_SIZES)), int(rng.choice(CONFIG3_LAYERS))) for _ in range(count)]
    peak = hbm_peak()[0]
    out = {"workload": (f"z-line sweeps of the u, v and w systems of config 3's {count} uneven tiles (n in "
                        f"{list(CONFIG3_SIZES)}, nz in {list(CONFIG3_LAYERS)}), {sweeps} sweeps, seeded "
                        f"diagonally dominant coefficients; inputs resident, best of {reps}"), "systems": 3 * count}
    for dtype, key in ((torch.float64, "fp64"), (torch.float32, "fp32")):
        ctx = gb.Context()
        gen = torch.Generator(device="cuda")
        gen.manual_seed(7)
        systems = []
        points = 0
        for n, nz in shapes:
            g = gb.Grid(n, n, nz, 30.0, 30.0, 10.0, False, False)
            for loc in (gb.LOC_XFACE, gb.LOC_YFACE, gb.LOC_ZFACE):
                A = torch.rand((gb.N_COEFS,) + g.shape, dtype=dtype, device="cuda", generator=gen) * 0.9 + 0.1
                ap = A.sum(0) + 0.2
                rhs = torch.rand(g.shape, dtype=dtype, device="cuda", generator=gen) * 2.0 - 1.0
                delta = torch.zeros(g.shape, dtype=dtype, device="cuda")
                systems.append((g, loc, A, ap, rhs, delta))
                ni, nj, nk = g.extents(loc)
                points += ni * nj * nk
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)

        def timed(fn):
            fn()
            best = float("inf")
            for _ in range(reps):
                torch.cuda.synchronize()
                e0.record(ctx.stream)
                fn()
                e1.record(ctx.stream)
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        def batched():
            gb.zline_jacobi_batch(ctx, systems, sweeps)

        def one_by_one():
            for (g, loc, A, ap, rhs, delta) in systems:
                gb.zline_jacobi(ctx, g, loc, A, ap, rhs, sweeps, delta)

        # the levels per warp for these systems (the in-project autotuner),
        # used by both forms below
        seg, seg_ms = tune_batch_sweep(Autotuner(), ctx, systems, sweeps) if tune else (0, None)
        l0 = ctx.launches()
        batched()
        launches_batched = ctx.launches() - l0
        l0 = ctx.launches()
        one_by_one()
        launches_single = ctx.launches() - l0
        ms_b = timed(batched)
        ms_1 = timed(one_by_one)
        elt = torch.finfo(dtype).bits // 8
        bytes_pass = points * (5 + 10 * (sweeps - 1)) * elt
        out[key] = {"points": points, "batched_ms": ms_b, "one_by_one_ms": ms_1, "speedup": ms_1 / ms_b,
                    "levels_per_warp": seg or 5, "autotune_ms": {str(k or 5): v for k, v in (seg_ms or {}).items()},
                    "batched_point_sweeps_per_s": points * sweeps / (ms_b / 1e3),
                    "launches_batched": launches_batched, "launches_one_by_one": launches_single,
                    "hbm": {"achieved_gbs": bytes_pass / (ms_b / 1e3) / 1e9, "peak_gbs": peak,
                            "frac": bytes_pass / (ms_b / 1e3) / 1e9 / peak,
                            "frac_of_nominal": bytes_pass / (ms_b / 1e3) / 1e9 / NOMINAL_HBM_GBS,
                            "bytes_per_pass": bytes_pass}}
        del systems
        ctx.close()
        torch.cuda.empty_cache()
    return out


def served_leg_isolated():
    """served_leg in a child process of its own (bench.py --served-only): the
    served form's latencies depend on the host threads and the device memory
    it finds, so it starts from a fresh process, not after the other legs.
    The parent's cached device memory is released first."""
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    proc = subprocess.run([sys.executable, os.path.abspath(__file__), "--served-only"], capture_output=True,
                          text=True, cwd=ROOT)
    try:
        if proc.returncode != 0:
            raise RuntimeError(f"exit status {proc.returncode}")
        return json.loads(proc.stdout.strip().splitlines()[-1])
    except Exception as e:  # the headline line still prints; the leg reports its failure
        return {"error": f"served leg failed: {e}", "stderr_tail": proc.stderr[-2000:]}


def served_leg(rates=(0.5, 1.0, 2.0, 5.0, 10.0, 20.0)):
    """A bounded sample of the served configuration at each arrival rate of
    `rates`: 12 requests, tiles drawn as config 3 with n in {64, 96} and nz
    in {48, 64}, 70 % mass-consistent only and 30 % full solves (capped at
    1500 iterations); served with continuous batching and FP32 inner solves
    against plain FP64 served one at a time over the same arrivals (its
    service times measured once, the FIFO queue replayed per rate)."""
    from ablsteadyrans_b200.serve import serve_sweep
    points = serve_sweep(rates, count=12, sizes=(64, 96), layers=(48, 64), max_iterations=1500)
    for p in points:
        p["speedup_solves_per_s"] = p["served_fp32_inner"]["solves_per_s"] / p["sequential_fp64"]["solves_per_s"]
    out = dict(points[[p["rate_per_s"] for p in points].index(2.0)]) if 2.0 in rates else dict(points[0])
    out["sweep"] = [{"rate_per_s": p["rate_per_s"], "speedup_solves_per_s": p["speedup_solves_per_s"],
                     "served_p50_s": p["served_fp32_inner"]["p50_s"], "served_p99_s": p["served_fp32_inner"]["p99_s"],
                     "served_solves_per_s": p["served_fp32_inner"]["solves_per_s"],
                     "sequential_p50_s": p["sequential_fp64"]["p50_s"],
                     "sequential_p99_s": p["sequential_fp64"]["p99_s"],
                     "sequential_solves_per_s": p["sequential_fp64"]["solves_per_s"],
                     "peak_concurrent": p["served_fp32_inner"]["peak_concurrent"]} for p in points]
    out["workload"] = ("12 requests, Poisson arrivals at " + ", ".join(f"{r:g}" for r in rates) + " per s, tiles "
                       "drawn as config 3 with n in {64, 96}, nz in {48, 64} (a bounded sample), 70 % "
                       "mass-consistent only, 30 % full solves capped at 1500 iterations; the top-level figures "
                       "are the 2/s point")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1])
    ap.add_argument("--sweeps", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-steady", action="store_true", help="skip the steady-solve legs")
    ap.add_argument("--no-steady2", action="store_true", help="skip the config-2 steady-solve leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the served leg")
    ap.add_argument("--served-only", action="store_true",
                    help="run the served leg alone and print its JSON (the main run's served leg runs this in a "
                         "child process, so no earlier leg's device or host state is shared with it)")
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
    if args.served_only:
        print(json.dumps(served_leg()))
        return 0

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
        "config": bench_config(wl),
        "parallelism": f"independent instances x{world}",
        "driver_status_last": statuses[-1],
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": wl.h2d,
                "d2h_bytes_per_step": wl.d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "zline_seg_multi_kernel (segmented z-line Thomas sweeps: u, v, w in one launch, "
                               "theta and k in one)",
                     "peak_kind": peak_kind,
                     "frac_of_nominal": (achieved / NOMINAL_HBM_GBS) if achieved else None,
                     "nominal_peak": NOMINAL_HBM_GBS,
                     "bytes_per_launch": line_bytes / max(sweep_n, 1), "launch_ms": sweep_ms / max(sweep_n, 1)},
        "breakdown": families,
        "clocks": clocks,
    }
    if args.tune:
        line["tune"] = args.tune
    if world == 1:
        line["rooflines"] = poisson_rooflines(ctx, wl, flush, peak)
        line["residual_roofline"] = residual_roofline(ctx, wl, flush, peak)
    wl.stage.close()
    ctx.close()
    del flush
    torch.cuda.empty_cache()
    if world == 1 and not args.no_steady:
        line["steady"] = steady_solves()
        if not args.no_steady2:
            line["steady_config2"] = steady_solves(max_iterations=3000, config=2)
    if world == 1 and not args.no_batch:
        line["batched"] = batched_leg()
        line["batched_sweeps"] = batched_sweep_leg()
    if world == 1 and not args.no_serve:
        line["served"] = served_leg_isolated()
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(wl, budget=30.0):
    """The FP64 C restatement built for speed on this host, on a bounded
    sample of the same workload: config 1's iterations on every host thread
    (at least one, until `budget` seconds), and one iteration on one thread."""
    import oracle
    path = oracle.use_fast_build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    wl.cpu_setup()
    wl.cpu_step()   # untimed: first touch of the arrays
    t0 = time.perf_counter()
    n = 0
    while True:
        wl.cpu_step()
        n += 1
        if time.perf_counter() - t0 > budget or n >= 3:
            break
    dt = time.perf_counter() - t0
    oracle.set_threads(1)
    t1 = time.perf_counter()
    wl.cpu_step()
    dt1 = time.perf_counter() - t1
    oracle.set_threads(threads)
    return {"value": wl.cells * n / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{n} SIMPLEC iteration(s) of config 1 ({dt:.1f} s) on {threads} threads, after one untimed",
            "single_thread": {"value": wl.cells / dt1, "unit": "cell-updates/s", "cores": 1,
                              "sample": f"1 SIMPLEC iteration of config 1 ({dt1:.1f} s) on one thread"},
            "cpu_model": oracle.cpu_model(), "nproc": threads,
            "build": "the oracle's C sources, gcc -O3 -march=native -fopenmp (" + os.path.basename(path) + ")"}


def run_reference(args):
    wl = SimplecWorkload(precision=0, sweeps=args.sweeps)
    import oracle
    oracle.use_fast_build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    wl.cpu_setup()
    for _ in range(max(0, args.warmup)):   # untimed warm-up iterations
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
        "steps": n, "warmup": max(0, args.warmup), "ms_per_step": dt / n * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": ("synthetic (config 1 generated in-project: Gaussian hill, log-law inflow; k-L closure, neutral "
                 "MOST surface layer)"),
        "config": bench_config(wl),
        "parallelism": f"host threads x{threads}",
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{n} SIMPLEC iteration(s) of config 1 ({dt:.1f} s); the FP64 C restatement of "
                                   "the reference (the reference needs AMReX), gcc -O3 -march=native",
                         "cpu_model": oracle.cpu_model(), "nproc": threads},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
