"""Generate tests/golden/poisson_askervein.npz from the reference's own gold.

The reference's Poisson_Askervein regression (Tests/Discretization/Poisson_Askervein:
inputs_poisson_askervein, driver Tests/Supporting_Files/Tools/poisson_projection.cpp)
projects a fixed wind on ERF's Askervein terrain, 30 x 30 x 18 cells of 200 m,
18 layers from 20 m growing by 1.08 (BTF, terrain.smoothing = 0), and stores
the potential phi in an AMReX plotfile (Gold/poisson_askervein_plt00000). This
script, run once in a container that holds the reference, writes:
  zlevels   the 19 layer heights (mesh.dz0 = 20, mesh.stretch_ratio = 1.08,
            Source/ZLevels.cpp:117-127);
  ground    the ground height of every node column i, j in [-1, 31] (the ghost
            columns clamped to the edge, Source/TerrainSurface.cpp node_index),
            bilinear in ERF's terrain grid at (x + 1e-3, y + 1e-3)
            (Source/TerrainSurface.cpp:257-307, erf_bilinear);
  phi       the gold potential, shape (18, 30, 30) as [k, j, i];
  info      the gold's iterations and divergence before/after
            (Gold/poisson_askervein.json).
The gold is AMReX's plotfile format: an ASCII FAB header per box, then the
box's doubles in Fortran order, little-endian (the header's byte order
"8 7 6 5 4 3 2 1").

Usage: python tests/golden/make_poisson_askervein.py REFERENCE_ROOT
"""
import json
import os
import re
import sys

import numpy as np


def read_erf_grid(path):
    vals = [float(t) for t in open(path).read().split()]
    nx, ny = int(vals[0]), int(vals[1])
    x = np.array(vals[2:2 + nx])
    y = np.array(vals[2 + nx:2 + nx + ny])
    z = np.array(vals[2 + nx + ny:])
    assert z.size == nx * ny
    return nx, ny, x, y, z


def erf_bilinear(grid, x, y):
    nx, ny, xt, yt, zt = grid
    jf = -1
    for it in range(ny):
        if yt[it] > y:
            jf = it - 1
            break
    else:
        jf = ny - 1
    jf = max(jf, 0)
    iff = -1
    for it in range(nx):
        if xt[it] > x:
            iff = it - 1
            break
    else:
        iff = nx - 1
    iff = max(iff, 0)
    ip1, jp1 = min(iff + 1, nx - 1), min(jf + 1, ny - 1)
    x1, x2, y1, y2 = xt[iff], xt[ip1], yt[jf], yt[jp1]
    i11, i21, i12, i22 = iff * ny + jf, ip1 * ny + jf, iff * ny + jp1, ip1 * ny + jp1
    ix = (ip1 != iff) and (x2 != x1)
    iy = (jp1 != jf) and (y2 != y1)
    if not ix and not iy:
        return zt[i11]
    if ix and not iy:
        return ((x2 - x) * zt[i11] + (x - x1) * zt[i21]) / (x2 - x1)
    if not ix and iy:
        return ((y2 - y) * zt[i11] + (y - y1) * zt[i12]) / (y2 - y1)
    w11 = (x2 - x) * (y2 - y)
    w21 = (x - x1) * (y2 - y)
    w12 = (x2 - x) * (y - y1)
    w22 = (x - x1) * (y - y1)
    return (w11 * zt[i11] + w12 * zt[i12] + w21 * zt[i21] + w22 * zt[i22]) / ((x2 - x1) * (y2 - y1))


def read_plotfile_level0(plt, nvar_index=0):
    lines = open(os.path.join(plt, "Header")).read().split("\n")
    hi = re.findall(r"\(\(0,0,0\) \((\d+),(\d+),(\d+)\)", open(os.path.join(plt, "Header")).read())[0]
    n = [int(v) + 1 for v in hi]
    out = np.full((n[2], n[1], n[0]), np.nan)
    ldir = os.path.join(plt, "Level_0")
    cellh = open(os.path.join(ldir, "Cell_H")).read()
    boxes = re.findall(r"\(\((\d+),(\d+),(\d+)\) \((\d+),(\d+),(\d+)\)", cellh)
    fabs = re.findall(r"FabOnDisk: (\S+) (\d+)", cellh)
    for (lo0, lo1, lo2, hi0, hi1, hi2), (fname, off) in zip(boxes, fabs):
        with open(os.path.join(ldir, fname), "rb") as f:
            f.seek(int(off))
            header = f.readline().decode()
            m = re.search(r"\(\((\d+),(\d+),(\d+)\) \((\d+),(\d+),(\d+)\)", header)
            blo = [int(m.group(i)) for i in (1, 2, 3)]
            bhi = [int(m.group(i)) for i in (4, 5, 6)]
            shape = [bhi[d] - blo[d] + 1 for d in range(3)]
            ncomp = int(header.strip().split()[-1])
            data = np.frombuffer(f.read(8 * shape[0] * shape[1] * shape[2] * ncomp), dtype="<f8")
            data = data.reshape(ncomp, shape[2], shape[1], shape[0])[nvar_index]
            out[blo[2]:bhi[2] + 1, blo[1]:bhi[1] + 1, blo[0]:bhi[0] + 1] = data
    assert not np.isnan(out).any()
    return out


def main(ref):
    nx, ny, nz = 30, 30, 18
    plo, phi_hi = (-3000.0, -3000.0, 0.0), (3000.0, 3000.0, 440.0)
    dx = (phi_hi[0] - plo[0]) / nx
    dy = (phi_hi[1] - plo[1]) / ny
    z = [0.0]
    dz = 20.0
    for k in range(1, nz + 1):
        z.append(z[k - 1] + dz)
        dz *= 1.08
    grid = read_erf_grid(os.path.join(ref, "extern_erf", "askervein.txt"))
    ground = np.zeros((ny + 3, nx + 3))
    for j in range(-1, ny + 2):
        for i in range(-1, nx + 2):
            ii = min(max(i, 0), nx)
            jj = min(max(j, 0), ny)
            x = plo[0] + ii * dx
            y = plo[1] + jj * dy
            ground[j + 1, i + 1] = erf_bilinear(grid, x + 1e-3, y + 1e-3)
    gold = os.path.join(ref, "Tests", "Discretization", "Poisson_Askervein", "Gold")
    phi = read_plotfile_level0(os.path.join(gold, "poisson_askervein_plt00000"))
    info = json.load(open(os.path.join(gold, "poisson_askervein.json")))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "poisson_askervein.npz")
    np.savez_compressed(out, zlevels=np.array(z), ground=ground, phi=phi, info=json.dumps(info),
                        prob_lo=np.array(plo), prob_hi=np.array(phi_hi))
    print("wrote", out, phi.shape, "phi range", phi.min(), phi.max())


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
