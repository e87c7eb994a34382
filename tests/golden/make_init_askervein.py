"""Generate tests/golden/init_askervein.npz from the reference's own gold.

The reference's Mass_Consistent_Askervein regression
(Tests/Initialization/Mass_Consistent_Askervein: inputs_init_askervein) builds
the mass-consistent initial field on ERF's Askervein mesh (the mesh of the
Poisson_Askervein case: 30 x 30 x 18 cells of 200 m, 18 layers from 20 m
growing by 1.08, BTF): a log-law first guess along x (u* = 0.6 m/s, z0 = 0.03
m), inflow at xlo, outflow at xhi, slip walls in y and at the top, the
correction with alpha_h = 1, alpha_v = 0.5. Its plotfile stores, per cell,
u, v, w averaged from the two faces (Source/StateIO.cpp:59-74), p, theta, k,
the cell height and detJ. This script, run once in a container that holds the
reference, writes:
  u, v, w, p, theta, tke   the gold fields, shape (18, 30, 30) as [k, j, i];
  info                     Gold/init_askervein.json (iterations, divergence
                           before and after, extrema).
The mesh comes from tests/golden/poisson_askervein.npz (zlevels, ground).

Usage: python tests/golden/make_init_askervein.py REFERENCE_ROOT
"""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_poisson_askervein import read_plotfile_level0  # noqa: E402

NAMES = ("u", "v", "w", "p", "theta", "tke")


def main(ref):
    gold = os.path.join(ref, "Tests", "Initialization", "Mass_Consistent_Askervein", "Gold")
    plt = os.path.join(gold, "init_askervein_plt00000")
    header = open(os.path.join(plt, "Header")).read().split("\n")
    nvar = int(header[1])
    names = header[2:2 + nvar]
    fields = {n: read_plotfile_level0(plt, names.index(n)) for n in NAMES}
    info = json.load(open(os.path.join(gold, "init_askervein.json")))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "init_askervein.npz")
    np.savez_compressed(out, info=json.dumps(info), **fields)
    print("wrote", out, {n: (float(f.min()), float(f.max())) for n, f in fields.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
