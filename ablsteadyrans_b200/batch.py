"""Many independent steady solves on one GPU (the batched configuration:
uneven terrain tiles and wind directions).

Each member is one instance with its own CUDA stream, gb_ctx (scratch,
result words), resident state and driver. Members share nothing on the
device. Native threads (gb_driver_run: the C++ steady driver, one thread
per member) step the members, so one member's host-synchronising parts
(the Krylov dot products of its Poisson solve, the result words of its
iteration) overlap the kernels of the others, and the GPU runs the small
kernels of many members at once. A member's arithmetic does not
depend on what else runs: its result is the same alone and in the mix, bit
for bit (deterministic reductions, no shared scratch).

    python -m ablsteadyrans_b200.batch --count 48 --iterations 20

prints one JSON line: the batched and the one-by-one throughput of the same
members (cell-updates/s) and their ratio.
"""
import json
import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

CONFIG3_SIZES = (64, 96, 128, 160, 192)
CONFIG3_LAYERS = (48, 64, 96)


def config3(count=48, seed=0, precision=1, zline_sweeps=4):
    """The batched configuration's instances: n uniform in {64, 96, 128, 160,
    192} (n x n), nz in {48, 64, 96}, dx = 30 m, fractal terrain with rms
    uniform in 20-150 m, wind direction uniform in 0-360 deg, u* in 0.2-0.6
    m/s, z0 in 0.01-0.5 m (workloads.tile, seed = 1000 + instance index)."""
    from . import workloads
    rng = np.random.default_rng(seed)
    out = []
    for n in range(count):
        size = int(rng.choice(CONFIG3_SIZES))
        nz = int(rng.choice(CONFIG3_LAYERS))
        out.append(workloads.tile(size, nz, n, precision=precision, zline_sweeps=zline_sweeps))
    return out


class Member:
    """One instance resident on the device with its own stream and context."""

    def __init__(self, inst, restart=8):
        import torch

        import ablsteadyrans_b200 as gb
        from .driver import Driver
        from .simplec import DeviceCase, SimplecStage
        self.inst = inst
        g = inst.grid
        self.stream = torch.cuda.Stream()
        inst.options.poisson.restart = restart  # the correction needs few Krylov vectors at reltol 1e-3
        with torch.cuda.stream(self.stream):
            self.ctx = gb.Context(self.stream)
            z = torch.from_numpy(inst.z).cuda()
            J, ax, ay, az, _ = gb.mesh_metrics(self.ctx, g, z)
            self.case = DeviceCase(g, z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
            self.stage = SimplecStage(self.ctx, self.case, inst.bc, inst.physics, inst.options)
            self.stage.fill_ghosts()
            self.driver = Driver(self.stage)
            self.driver.dtau = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
        self.stream.synchronize()
        self.status = "running"
        self.iterations = 0
        self._native = None

    @property
    def native(self):
        """This member's C++ driver (gb_driver), made on first use."""
        if self._native is None:
            from .simplec import NativeDriver
            self._native = NativeDriver(self.stage)
        return self._native

    @property
    def cells(self):
        return self.inst.cells

    def step(self):
        import torch
        with torch.cuda.stream(self.stream):
            self.status = self.driver.step()
        self.iterations += 1
        return self.status

    def fields(self):
        """Host copies of the state (u, v, w, p, theta, k)."""
        import torch
        with torch.cuda.stream(self.stream):
            out = {f: t.cpu().numpy() for f, t in self.case.q.items()}
        return out

    def close(self):
        if self._native is not None:
            self._native.close()
        self.stage.close()
        self.ctx.close()


class Batch:
    """Members stepped together (threads over members) or one by one. With
    a tuner (autotune.Autotuner) each member's context takes the knob choice
    of its shape (timed on the first member of each shape)."""

    def __init__(self, instances, restart=8, tuner=None):
        self.members = [Member(inst, restart=restart) for inst in instances]
        self.choices = {}
        if tuner is not None:
            from .autotune import shape_key
            for m in self.members:
                with __import__("torch").cuda.stream(m.stream):
                    choice, _ = tuner.tune(m.stage)
                self.choices[shape_key(m.inst.grid, m.inst.options, m.inst.physics)] = choice

    @property
    def cells(self):
        return sum(m.cells for m in self.members)

    def _run(self, work, concurrent, threads):
        """Runs work(member) for every member; returns the device time (ms)
        from the first member's start event to the last member's end event."""
        import torch
        torch.cuda.synchronize()
        starts = []
        ends = []
        for m in self.members:
            e = torch.cuda.Event(enable_timing=True)
            e.record(m.stream)
            starts.append(e)
        t0 = time.perf_counter()

        def one(m):
            work(m)
            e = torch.cuda.Event(enable_timing=True)
            e.record(m.stream)
            return e

        if concurrent:
            with ThreadPoolExecutor(max_workers=threads or len(self.members)) as ex:
                ends = list(ex.map(one, self.members))
        else:
            ends = [one(m) for m in self.members]
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        ref = starts[0]
        device_ms = max(ref.elapsed_time(e) for e in ends)
        return device_ms, wall

    def run(self, iterations, concurrent=True, threads=None):
        """iterations outer iterations of every member (Python drivers on
        Python threads); returns (device ms, wall ms)."""
        def work(m):
            for _ in range(iterations):
                m.step()
        return self._run(work, concurrent, threads)

    def run_native(self, iterations, threads=0):
        """iterations outer iterations of every member with the C++ drivers on
        native threads (gb_driver_run, one call); returns (device ms, wall ms)."""
        import torch

        from .simplec import run_drivers
        drivers = [m.native for m in self.members]
        torch.cuda.synchronize()
        starts = []
        for m in self.members:
            e = torch.cuda.Event(enable_timing=True)
            e.record(m.stream)
            starts.append(e)
        t0 = time.perf_counter()
        out = run_drivers(drivers, iterations, threads)
        ends = []
        for m, (verdict, n) in zip(self.members, out):
            m.status = verdict
            m.iterations += n
            e = torch.cuda.Event(enable_timing=True)
            e.record(m.stream)
            ends.append(e)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        return max(starts[0].elapsed_time(e) for e in ends), wall

    def close(self):
        for m in self.members:
            m.close()


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--count", type=int, default=48)
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    import torch
    insts = config3(args.count, args.seed, precision=args.precision)
    free0, _ = torch.cuda.mem_get_info()
    batch = Batch(insts)
    free1, _ = torch.cuda.mem_get_info()
    batch.run_native(args.warmup, threads=args.threads)
    seq_ms, seq_wall = batch.run_native(args.iterations, threads=1)
    bat_ms, bat_wall = batch.run_native(args.iterations, threads=args.threads)
    cells = batch.cells * args.iterations
    line = {
        "metric": "cell-updates/s", "unit": "cell-updates/s",
        "workload": f"{args.count} uneven tiles (n in {CONFIG3_SIZES}, nz in {CONFIG3_LAYERS}), "
                    f"{'FP32 inner solves' if args.precision else 'plain FP64'}, {args.iterations} iterations each",
        "cells": batch.cells, "device_bytes": int(free0 - free1),
        "batched": cells / (bat_ms / 1e3), "one_by_one": cells / (seq_ms / 1e3),
        "speedup": seq_ms / bat_ms, "batched_ms": bat_ms, "one_by_one_ms": seq_ms,
        "batched_wall_ms": bat_wall, "one_by_one_wall_ms": seq_wall,
    }
    print(json.dumps(line))
    batch.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
