"""The in-project autotuner of the kernels' shape choices: for an instance's
shape it times a few SIMPLEC iterations under each candidate setting of the
context's tuning knobs and keeps the fastest, per shape.

The knobs it searches choose how columns map onto warps and which kernel
form runs, never what is computed:

  * GB_TUNE_LINE_VARIANT: the segmented z-line sweep (the column's levels
    split among a block's warps) or the sequential factored sweep (one
    thread walks a column);
  * GB_TUNE_LINE_SEGMENT: levels per warp of the segmented sweeps (4 or 8);
  * GB_TUNE_MG_FUSED_RELAX: the zebra relaxation as the residual and the
    column solves in two launches (the default) or as one segmented launch
    per colour.

Every candidate performs the same arithmetic up to rounding (the segmented
and the sequential recurrences differ only in the values carried across a
segment boundary), so the choice changes speed, not results beyond
rounding. Timing runs on a copy of the state, which is restored: tuning
does not advance a solve (the stage's nu_t history, which only
turb.nut_relax < 1 reads, is then the last timed iteration's). Results are
cached per shape key (grid, precision, line-sweep kind, closure) in memory
and, when a path is given, in a JSON file.
"""
import itertools
import json
import os

#: Candidate values per knob name (the ablsteadyrans_b200.TUNE_* names).
CANDIDATES = {
    "LINE_VARIANT": (0, 4),
    "LINE_SEGMENT": (0, 4, 8),
    "MG_FUSED_RELAX": (0, 4),
}


def candidates(space=None):
    """Every combination of the knobs' candidate values, as dicts, the
    defaults (the first value of each) first; combinations that cannot
    differ (a segment length with the sequential sweep and the two-launch
    relaxation) are dropped."""
    space = space or CANDIDATES
    names = list(space)
    out = []
    for values in itertools.product(*[space[n] for n in names]):
        c = dict(zip(names, values))
        seg_default = space.get("LINE_SEGMENT", (0,))[0]
        if c.get("LINE_VARIANT") == 4 and c.get("MG_FUSED_RELAX") == 0 and c.get("LINE_SEGMENT", seg_default) != seg_default:
            continue
        out.append(c)
    return out


def shape_key(grid, options, physics):
    """The cache key of an instance: what the kernels' shapes depend on."""
    return (f"{grid.nx}x{grid.ny}x{grid.nz}:px{int(grid.periodic_x)}py{int(grid.periodic_y)}"
            f":prec{int(options.precision)}:sweep{int(options.line_sweep)}x{int(options.zline_sweeps)}"
            f":closure{int(physics.closure)}")


def best(timings):
    """The candidate with the smallest time from [(candidate, ms)]; ties keep
    the earlier (the defaults first)."""
    if not timings:
        raise ValueError("no timings")
    return min(enumerate(timings), key=lambda t: (t[1][1], t[0]))[1][0]


class Autotuner:
    """Per-shape knob choices, timed on first sight of a shape."""

    def __init__(self, path=None, iterations=3, space=None):
        self.path = path
        self.iterations = iterations
        self.space = space or CANDIDATES
        self.cache = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.cache = json.load(f)

    def save(self):
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)

    @staticmethod
    def apply(ctx, choice):
        import ablsteadyrans_b200 as gb
        for name, value in choice.items():
            ctx.tune(getattr(gb, "TUNE_" + name), int(value))

    def time_candidate(self, stage, choice, dtau):
        """Device milliseconds per iteration of `stage` under `choice`, on a
        copy of its state (restored afterwards)."""
        import torch
        ctx = stage.ctx
        self.apply(ctx, choice)
        saved = {f: t.clone() for f, t in stage.case.q.items()}
        try:
            stage.iterate(dtau)                      # the first iteration under new knobs runs eagerly
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ctx.stream)
            for _ in range(self.iterations):
                stage.iterate(dtau)
            e1.record(ctx.stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / self.iterations
        finally:
            for f, t in stage.case.q.items():
                t.copy_(saved[f])
            stage.fill_ghosts()
            torch.cuda.synchronize()

    def tune(self, stage, cfl=1.0):
        """The knob choice for `stage`'s shape (timed on first sight, then
        cached), applied to its context. Returns (choice, timings or None)."""
        key = shape_key(stage.case.grid, stage.options, stage.physics)
        if key in self.cache:
            choice = self.cache[key]["choice"]
            self.apply(stage.ctx, choice)
            return choice, None
        dtau = stage.local_dtau(cfl)
        timings = [(c, self.time_candidate(stage, c, dtau)) for c in candidates(self.space)]
        choice = best(timings)
        self.cache[key] = {"choice": choice, "ms": {json.dumps(c, sort_keys=True): ms for c, ms in timings}}
        self.save()
        self.apply(stage.ctx, choice)
        return choice, timings


#: Candidate levels per warp of the batched z-line sweep (GB_TUNE_LINE_SEGMENT).
SWEEP_SEGMENTS = (0, 4, 8)


def sweep_key(systems, sweeps):
    """The cache key of a batched sweep: each system's extents at its
    location, the precision and the sweep count."""
    shapes = sorted(tuple(g.extents(loc)) for (g, loc, *_rest) in systems)
    word = systems[0][2].element_size() if systems else 8
    return f"batch-sweep:{word}:{sweeps}:" + ",".join(f"{a}x{b}x{c}" for a, b, c in shapes)


def tune_batch_sweep(tuner, ctx, systems, sweeps, reps=2):
    """The levels per warp of the batched z-line sweep (gb_zline_jacobi_batch)
    over `systems`: each candidate of SWEEP_SEGMENTS timed on the systems
    themselves (the sweep only writes its deltas, so timing changes no
    input), the fastest applied to ctx and cached in `tuner` by sweep_key.
    Returns (segment, {segment: ms} or None when cached)."""
    import torch

    import ablsteadyrans_b200 as gb
    key = sweep_key(systems, sweeps)
    if key in tuner.cache:
        seg = tuner.cache[key]["choice"]["LINE_SEGMENT"]
        ctx.tune(gb.TUNE_LINE_SEGMENT, seg)
        return seg, None
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    timings = []
    for seg in SWEEP_SEGMENTS:
        ctx.tune(gb.TUNE_LINE_SEGMENT, seg)
        gb.zline_jacobi_batch(ctx, systems, sweeps)        # untimed: the scratch at its size
        torch.cuda.synchronize()
        e0.record(ctx.stream)
        for _ in range(reps):
            gb.zline_jacobi_batch(ctx, systems, sweeps, want_change=False)
        e1.record(ctx.stream)
        torch.cuda.synchronize()
        timings.append(({"LINE_SEGMENT": seg}, e0.elapsed_time(e1) / reps))
    choice = best(timings)
    tuner.cache[key] = {"choice": choice, "ms": {str(c["LINE_SEGMENT"]): ms for c, ms in timings}}
    tuner.save()
    ctx.tune(gb.TUNE_LINE_SEGMENT, choice["LINE_SEGMENT"])
    return choice["LINE_SEGMENT"], {c["LINE_SEGMENT"]: ms for c, ms in timings}
