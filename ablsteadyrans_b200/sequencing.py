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
