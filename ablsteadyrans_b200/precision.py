"""Mixed precision against plain FP64 on one instance (config 2): both forms
solved from the same mass-consistent initial state to the steady criterion
(or an iteration cap) with the C++ driver; reports each form's iterations,
time and steady solves/s, and the per-field difference of the FP32-inner
result from the FP64 one (max |difference| / max |FP64 field|).

    python -m ablsteadyrans_b200.precision --max-iterations 4000
"""
import json
import time


def solve(inst, max_iterations):
    """One solve; returns (verdict, iterations, seconds, host fields)."""
    import torch

    from .batch import Member
    from .simplec import run_drivers
    m = Member(inst, restart=inst.options.poisson.restart)
    m.stage.initialize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    (verdict, n), = run_drivers([m.native], max_iterations, 1)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    fields = m.fields()
    m.close()
    return verdict, n, dt, fields


def main(argv=None):
    import argparse

    import numpy as np

    from . import workloads
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--max-iterations", type=int, default=4000)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--nz", type=int, default=96)
    ap.add_argument("--max-slope", type=float, default=1.0)
    args = ap.parse_args(argv)
    out = {"workload": f"config 2: fractal terrain {args.n}x{args.n}x{args.nz}, dx 30 m, 120 m rms (slopes capped "
                       f"at {args.max_slope}), u* 0.4 m/s, 225 deg"}
    results = {}
    grid = None
    for prec in (0, 1):
        inst = workloads.config2(precision=prec, n=args.n, nz=args.nz, max_slope=args.max_slope)
        grid = inst.grid
        verdict, n, dt, fields = solve(inst, args.max_iterations)
        results[prec] = fields
        key = "fp64" if prec == 0 else "fp32_inner"
        out[key] = {"verdict": verdict, "iterations": n, "seconds": dt, "ms_per_iteration": dt / max(n, 1) * 1e3,
                    "solves_per_s": 1.0 / dt if verdict == "steady" else None,
                    "cell_updates_per_s": inst.cells * n / dt}
    valid = {"u": grid.valid(1), "v": grid.valid(2), "w": grid.valid(4), "p": grid.valid(0),
             "theta": grid.valid(0), "tke": grid.valid(0)}
    err = {}
    for f, sl in valid.items():
        a, b = results[0][f][sl], results[1][f][sl]
        err[f] = float(np.abs(b - a).max() / max(np.abs(a).max(), 1e-300))
    out["fp32_inner_vs_fp64_rel_error"] = err
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
