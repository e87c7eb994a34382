"""Grid sequencing, coarse to fine, over the horizontal grid hierarchy
(gust::sequence_coarse_levels, Source/Sequencing.H:13-56, Sequencing.cpp:
260-400) on the GPU.

With L >= 2 levels: on the coarsest level L-1 the mass-consistent
initializer on that level's mesh, then SIMPLEC under its own native driver
until the loose stop; on each level l = L-2 .. 1 the prolongation from level
l+1 (bilinear per zeta-level, k at the floor, the level's ghost fill, the
projection), then SIMPLEC until the loose stop; on level 0 (the run's mesh)
the prolongation into the run's state, after which the run's driver goes on
to the strict stop. Every finer level starts its residual references from
the coarsest level's (seed_reference), without the reference hold when
steady.sequencing_hold = 0, and with steady.sequencing_cfl_start = previous
at the previous level's CFL. A coarse level that diverges raises, naming the
level; one that reaches max_iterations is prolonged as it is.
"""
from . import abi, hierarchy
from .driver import check_sequencing


class LevelSummary:
    """What sequencing did on one level (gust::LevelSummary)."""

    def __init__(self, level, cells):
        self.level = level
        self.cells = cells
        self.iterations = 0
        self.relative_residual = 0.0
        self.stop = ""
        self.prolonged = False
        self.prolong = None          # abi.ProlongResult into this level
        self.res_ref = None          # the level's residual references after its last iteration

    def __repr__(self):
        return (f"LevelSummary(level={self.level}, cells={self.cells}, iterations={self.iterations}, "
                f"stop={self.stop!r}, prolonged={self.prolonged})")


class LevelSolver:
    """One level's mesh metrics, device state, SIMPLEC stage and native
    driver, built from the run's settings on the level's mesh."""

    def __init__(self, ctx, level, driver_options):
        import torch

        import ablsteadyrans_b200 as gb
        from .simplec import DeviceCase, NativeDriver, SimplecStage
        inst = level.inst
        g = level.grid
        z = torch.from_numpy(inst.z).cuda()
        J, ax, ay, az, _ = gb.mesh_metrics(ctx, g, z)
        self.level = level
        self.case = DeviceCase(g, z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
        self.stage = SimplecStage(ctx, self.case, inst.bc, inst.physics, inst.options)
        self.driver_options = driver_options
        self._driver_cls = NativeDriver
        self.driver = None

    def make_driver(self):
        self.driver = self._driver_cls(self.stage, self.driver_options)
        return self.driver

    def close(self):
        if self.driver is not None:
            self.driver.close()
        self.stage.close()


def start_seeded(driver, ref, seq, cfl_prev):
    """start_seeded (Sequencing.cpp:88-95): the coarsest level's references,
    then no reference hold (sequencing_hold = 0) and the previous level's CFL
    (sequencing_cfl_start = previous)."""
    driver.seed_reference(ref)
    if seq.hold == 0:
        driver.release_hold()
    if seq.cfl_previous:
        driver.start_cfl(cfl_prev)


def _solve_level(lv, seq, max_iterations, label):
    """SIMPLEC on one coarse level until the loose stop, the strict stop or
    max_iterations (Sequencing.cpp:318-345)."""
    from . import GustError
    d = lv.driver
    crit = d.criterion
    s = LevelSummary(lv.level.level, (lv.level.grid.nx, lv.level.grid.ny))
    its = 0
    while its < max_iterations:
        verdict, _, _ = d.step()
        its += 1
        if verdict == "diverged":
            raise GustError(2, f"gust: grid sequencing: level {lv.level.level} diverged ({label})")
        if verdict == "steady":
            s.stop = "steady"
            break
        hold, _, _ = d.status()
        branch, why = crit.loose_stop(seq, hold)
        if branch != abi.LOOSE_NONE:
            s.stop = why
            break
    if not s.stop:
        s.stop = "steady.max_iterations"
    s.iterations = its
    _, _, s.relative_residual = d.status()
    s.res_ref = crit.history()["res_ref"][:6]
    return s


def sequence_coarse_levels(ctx, inst, levels, seq, finest_stage, finest_driver, driver_options=None, passes=1,
                           init_options=None, max_iterations=2000):
    """Steps 1 and 2 of grid sequencing and the prolongation of step 3: the
    coarse levels L-1 .. 1 of inst's hierarchy, then the prolongation from
    level 1 into finest_stage's state (level 0, the run's stage on inst's
    mesh), and finest_driver (no step taken yet) seeded with the coarsest
    level's references. Returns one LevelSummary per level, coarsest first,
    level 0 last (its iterations are the run's driver's)."""
    dopts = driver_options or abi.DriverOptions.make(getattr(inst.options, "line_sweep", 0))
    check_sequencing(seq, dopts, inst.grid.nx, inst.grid.ny, levels)
    if not seq.enabled:
        raise ValueError("gust: sequence_coarse_levels needs steady.sequencing = 1")
    hier = hierarchy.build(inst, levels, passes)
    reltol = inst.options.pressure_reltol
    out = []
    coarse = None
    ref = None
    cfl_prev = 0.0
    try:
        for lev in range(levels - 1, 0, -1):
            lv = LevelSolver(ctx, hier[lev], dopts)
            label = f"level {lev}"
            pr = None
            if coarse is None:
                # the coarsest level: the initializer on its own mesh
                lv.stage.initialize(init_options)
            else:
                pr = lv.stage.prolong(coarse.case, reltol)
                coarse.close()
                coarse = None
            d = lv.make_driver()
            if ref is not None:
                start_seeded(d, ref, seq, cfl_prev)
            s = _solve_level(lv, seq, max_iterations, label)
            if pr is not None:
                s.prolonged, s.prolong = True, pr
            out.append(s)
            if ref is None:
                ref = s.res_ref
            _, cfl_prev, _ = d.status()
            coarse = lv
        s0 = LevelSummary(0, (inst.grid.nx, inst.grid.ny))
        s0.prolong = finest_stage.prolong(coarse.case, reltol)
        s0.prolonged = True
        start_seeded(finest_driver, ref, seq, cfl_prev)
        out.append(s0)
    finally:
        if coarse is not None:
            coarse.close()
    return out


def sequencing_report(levels, finest_iterations, finest_status):
    """The summary table of sequence_coarse_levels (sequencing_report,
    Sequencing.cpp:402-445) without the wall-time and AU columns."""
    lines = ["gust: grid sequencing summary", "  level   cells (x y)  iterations  stop"]
    for s in levels:
        its, stop = s.iterations, s.stop
        if s.level == 0:
            its, stop = finest_iterations, "strict: " + finest_status
        lines.append(f"  {s.level:5d}  {s.cells[0]:5d} {s.cells[1]:5d}  {its:10d}  {stop}")
        if s.prolonged:
            p = s.prolong
            lines.append(f"         prolonged into level {s.level}: divergence {p.divergence_before:.3e} -> "
                         f"{p.divergence_after:.3e}, {p.tke_clipped} k values clipped")
    return "\n".join(lines)


def _finest(ctx, inst):
    import torch

    import ablsteadyrans_b200 as gb
    from .simplec import DeviceCase, SimplecStage
    g = inst.grid
    z = torch.from_numpy(inst.z).cuda()
    J, ax, ay, az, _ = gb.mesh_metrics(ctx, g, z)
    case = DeviceCase(g, z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
    return case, SimplecStage(ctx, case, inst.bc, inst.physics, inst.options)


def compare(inst_fn, levels, max_iterations, seq=None):
    """One steady solve of inst_fn() without and one with grid sequencing
    over `levels` levels (the C++ driver on every level); returns a dict of
    iterations, seconds and the per-field difference of the two solutions."""
    import time

    import numpy as np
    import torch

    import ablsteadyrans_b200 as gb
    from .simplec import NativeDriver, run_drivers
    seq = seq or abi.SequencingOptions.make(enabled=1)
    out = {}
    fields = {}
    for mode in ("plain", "sequenced"):
        inst = inst_fn()
        ctx = gb.Context()
        case, stage = _finest(ctx, inst)
        driver = NativeDriver(stage)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        summary = None
        if mode == "plain":
            stage.initialize()
        else:
            summary = sequence_coarse_levels(ctx, inst, levels, seq, stage, driver, max_iterations=max_iterations)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        (verdict, n), = run_drivers([driver], max_iterations, 1)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        rec = {"verdict": verdict, "level0_iterations": n, "seconds": t2 - t0, "level0_seconds": t2 - t1}
        if summary is not None:
            rec["levels"] = [{"level": s.level, "cells": list(s.cells), "iterations": s.iterations, "stop": s.stop,
                              "divergence": ([s.prolong.divergence_before, s.prolong.divergence_after]
                                             if s.prolonged else None)} for s in summary]
            rec["coarse_seconds"] = t1 - t0
            # work in level-0 iterations: a level-l iteration costs 4^-l of one
            rec["work_level0_iterations"] = n + sum(s.iterations / 4.0 ** s.level for s in summary if s.level > 0)
        out[mode] = rec
        fields[mode] = {f: t.cpu().numpy() for f, t in case.q.items()}
        driver.close()
        stage.close()
        ctx.close()
    g = inst.grid
    valid = {"u": g.valid(1), "v": g.valid(2), "w": g.valid(4), "p": g.valid(0), "theta": g.valid(0),
             "tke": g.valid(0)}
    out["sequenced_vs_plain_rel_difference"] = {
        f: float(np.abs(fields["sequenced"][f][sl] - fields["plain"][f][sl]).max()
                 / max(np.abs(fields["plain"][f][sl]).max(), 1e-300)) for f, sl in valid.items()}
    return out


def main(argv=None):
    """Grid sequencing against a plain solve on config 1 (the 150 m hill):
    python -m ablsteadyrans_b200.sequencing --levels 3 --max-iterations 6000"""
    import argparse
    import json

    from . import workloads
    ap = argparse.ArgumentParser(description="grid sequencing against a plain steady solve")
    ap.add_argument("--levels", type=int, default=3)
    ap.add_argument("--max-iterations", type=int, default=6000)
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--nz", type=int, default=64)
    args = ap.parse_args(argv)
    out = {"workload": f"config 1: 150 m Gaussian hill {args.nx}x{args.nx}x{args.nz}, dx 25 m, the k-L closure and "
                       "the surface layer", "levels": args.levels}
    out.update(compare(lambda: workloads.config1(args.nx, args.nx, args.nz), args.levels, args.max_iterations))
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
