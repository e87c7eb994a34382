"""Generate tests/golden/closure_column.npz from the reference's own gold.

The reference's Closure_Column regression (Tests/Discretization/
Closure_Column: inputs_closure_column, Tests/Supporting_Files/Tools/
closure_column.cpp) evaluates, once, the full residual of the wall law's
equilibrium state with the k-L closure: ERF's Neutral_ABL_Flat mesh (8 x 8 x
64 cells over 2560 m x 2560 m x 1000 m, dz 15.625 m, flat, periodic sides),
the surface layer on the ground (z0 0.1 m), a slip top, theta 300 K,
u = (u*/kappa) ln((z + z0)/z0) along 15 degrees with u* = 0.35 m/s,
k = u*^2/Cmu0^2, w = p' = 0, turb.max_geom_lscale 1e12, the logarithmic
face mean. Its plotfile holds the cell fields u (face mean), tke, nut,
length, R_u, R_v, R_w (face means), R_theta, R_tke, Ps, eps and, on the
ground cells, ustar. This script, run once in a container that holds the
reference, writes them as (64, 8, 8) arrays [k, j, i].

Usage: python tests/golden/make_closure_column.py REFERENCE_ROOT
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_poisson_askervein import read_plotfile_level0  # noqa: E402

NAMES = ("u", "tke", "nut", "length", "R_u", "R_v", "R_w", "R_theta", "R_tke", "Ps", "eps", "ustar")


def main(ref):
    plt = os.path.join(ref, "Tests", "Discretization", "Closure_Column", "Gold", "closure_column_plt00000")
    header = open(os.path.join(plt, "Header")).read().split("\n")
    nvar = int(header[1])
    names = header[2:2 + nvar]
    fields = {n: read_plotfile_level0(plt, names.index(n)) for n in NAMES}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "closure_column.npz")
    np.savez_compressed(out, **fields)
    print("wrote", out, {n: (float(f.min()), float(f.max())) for n, f in fields.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
