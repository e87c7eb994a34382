"""The horizontal grid hierarchy of grid sequencing (gust::MeshHierarchy,
Source/MeshHierarchy.H/.cpp, Source/SmoothSurface.cpp, Source/
SurfaceRoughness.cpp:130-163), built on the host from level 0's instance.

Level l has 2^l times fewer cells in x and y and the same z-levels. Its
ground is level 0's at its nodes (node (I, J) is level 0's node (2^l I,
2^l J)), smoothed on its own grid by passes (2^l - 1) passes of
h <- h + beta (h(i+1) + h(i-1) + h(j+1) + h(j-1) - 4 h) with beta = 1/8
(the neighbour across a non-periodic face is the edge node itself); its node
heights are the basic terrain-following coordinates of that ground; a
per-column roughness map is the geometric mean of the level-0 columns a
coarse column covers (relative to the level-0 map's largest value).

The ground arrays are the node columns -1..n+1 in x and y (shape
(ny + 3, nx + 3)), their ghost nodes the periodic image or the nearest
domain node (fill_surface_ghosts).
"""
import numpy as np

from . import workloads
from .grid import Grid

BETA = 0.125
MAX_LEVELS = 10
MAX_PASSES = 64


def hierarchy_ratio(level):
    if level < 0 or level >= MAX_LEVELS:
        raise ValueError(f"hierarchy level {level} outside [0, {MAX_LEVELS - 1}] (mesh.hierarchy_levels)")
    return 1 << level


def ground_passes(level, passes_per_level):
    """Ground smoothing passes of level l: passes_per_level (2^l - 1)."""
    return passes_per_level * (hierarchy_ratio(level) - 1)


def check_hierarchy_inputs(nx, ny, levels, passes):
    """check_hierarchy_inputs (MeshHierarchy.cpp:68-110): the problems, each
    naming its key (empty: none)."""
    err = []
    if levels < 1 or levels > MAX_LEVELS:
        err.append(f"mesh.hierarchy_levels must be an integer from 1 to {MAX_LEVELS} (got {levels})")
    elif levels > 1:
        r = 1 << (levels - 1)
        if nx % r or ny % r:
            err.append(f"mesh.hierarchy_levels = {levels} needs mesh.n_cell x and y divisible by 2^{levels - 1} = {r} "
                       f"(got {nx} {ny})")
        elif nx // r == 1 and ny // r == 1:
            err.append(f"mesh.hierarchy_levels = {levels} leaves the coarsest level 1 x 1 cells (mesh.n_cell {nx} {ny}); "
                       "use fewer levels")
    if passes < 0 or passes > MAX_PASSES:
        err.append(f"terrain.hierarchy_passes must be an integer from 0 to {MAX_PASSES} (got {passes})")
    return err


def fill_surface_ghosts(h, nx, ny, per_x, per_y):
    """The ghost nodes of a ground array (SmoothSurface.cpp:50-77): the
    periodic images (FillBoundary), then the nearest domain node outside a
    non-periodic face."""
    # FillBoundary: a ghost node takes the node it images across the periodic
    # directions, when that node is a domain node
    for jj in range(ny + 3):
        j = jj - 1
        for ii in range(nx + 3):
            i = ii - 1
            if 0 <= i <= nx and 0 <= j <= ny:
                continue
            si = (i % nx) if per_x else i
            sj = (j % ny) if per_y else j
            if 0 <= si <= nx and 0 <= sj <= ny and (si, sj) != (i, j):
                h[jj, ii] = h[sj + 1, si + 1]
    for jj in range(ny + 3):
        j = jj - 1
        for ii in range(nx + 3):
            i = ii - 1
            ic = i if per_x else min(max(i, 0), nx)
            jc = j if per_y else min(max(j, 0), ny)
            if (ic, jc) != (i, j):
                h[jj, ii] = h[jc + 1, ic + 1]
    return h


def smooth_surface(h, nx, ny, per_x, per_y, passes, beta=BETA):
    """smooth_surface (SmoothSurface.cpp:7-48) of a ground array, in place."""
    if passes < 0 or not (0 <= beta < 0.25):
        raise ValueError("smooth_surface needs passes >= 0 and 0 <= beta < 1/4")
    if passes == 0:
        return h
    ii = np.arange(nx + 1)
    jj = np.arange(ny + 1)
    im = np.where((ii == 0) & (not per_x), ii, ii - 1) + 1
    ip = np.where((ii == nx) & (not per_x), ii, ii + 1) + 1
    jm = np.where((jj == 0) & (not per_y), jj, jj - 1) + 1
    jp = np.where((jj == ny) & (not per_y), jj, jj + 1) + 1
    c_i, c_j = ii + 1, jj + 1
    for _ in range(passes):
        # FillBoundary of the periodic ghosts before each pass
        _periodic_images(h, nx, ny, per_x, per_y)
        old = h.copy()
        hn = old[np.ix_(c_j, c_i)]
        s = old[np.ix_(c_j, ip)] + old[np.ix_(c_j, im)]
        s = s + old[np.ix_(jp, c_i)]
        s = s + old[np.ix_(jm, c_i)]
        s = s - 4.0 * hn
        h[np.ix_(c_j, c_i)] = hn + beta * s
    return fill_surface_ghosts(h, nx, ny, per_x, per_y)


def _periodic_images(h, nx, ny, per_x, per_y):
    for jj in range(ny + 3):
        j = jj - 1
        for ii in range(nx + 3):
            i = ii - 1
            if 0 <= i <= nx and 0 <= j <= ny:
                continue
            si = (i % nx) if per_x else i
            sj = (j % ny) if per_y else j
            if 0 <= si <= nx and 0 <= sj <= ny and (si, sj) != (i, j):
                h[jj, ii] = h[sj + 1, si + 1]


def inject_ground(ground0, r, nxc, nyc, per_x, per_y):
    """inject_ground (MeshHierarchy.cpp:127-147): level 0's ground at the
    coarse nodes, then the coarse ghost nodes."""
    h = np.zeros((nyc + 3, nxc + 3))
    h[1:nyc + 2, 1:nxc + 2] = ground0[1:r * nyc + 2:r, 1:r * nxc + 2:r]
    return fill_surface_ghosts(h, nxc, nyc, per_x, per_y)


def average_roughness(z0map0, grid0, r, gridc):
    """average_roughness_map (SurfaceRoughness.cpp:130-163): each coarse
    column the geometric mean of its r x r level-0 columns relative to the
    level-0 map's largest value; the ghost columns the periodic image or the
    nearest domain column. Planes in gb_mesh_fields.z0's layout."""
    G = grid0.ng
    f = np.asarray(z0map0).reshape(grid0.ny + 1 + 2 * G, grid0.nx + 1 + 2 * G)
    valid = f[G:G + grid0.ny, G:G + grid0.nx]
    ref = valid.max()
    inv = 1.0 / float(r * r)
    cols = np.zeros((gridc.ny, gridc.nx))
    for j in range(gridc.ny):
        for i in range(gridc.nx):
            s = 0.0
            for b in range(r):
                for a in range(r):
                    s += np.log(valid[r * j + b, r * i + a] / ref)
            cols[j, i] = ref * np.exp(s * inv)
    Gc = gridc.ng
    plane = np.zeros((gridc.ny + 1 + 2 * Gc, gridc.nx + 1 + 2 * Gc))
    for j in range(-Gc, gridc.ny + 1 + Gc):
        for i in range(-Gc, gridc.nx + 1 + Gc):
            ic = (i % gridc.nx) if gridc.periodic_x else min(max(i, 0), gridc.nx - 1)
            jc = (j % gridc.ny) if gridc.periodic_y else min(max(j, 0), gridc.ny - 1)
            plane[j + Gc, i + Gc] = cols[jc, ic]
    return plane.reshape(-1)


class Level:
    """One level: its grid, ground (node columns -1..n+1), node heights and
    roughness map (or None), and the instance of the run's settings on it."""

    def __init__(self, level, inst, grid, ground, z0map):
        self.level = level
        self.grid = grid
        self.ground = ground
        self.z0map = z0map
        self.inst = workloads.Instance(f"{inst.name}-level{level}", grid, inst.zlevels, ground, inst.bc, inst.physics,
                                       inst.options, inst.ustar, inst.z0, inst.direction, z0map)


def build(inst, levels, passes=1):
    """The hierarchy of an instance (its grid, ground and roughness map are
    level 0): Level objects 0 .. levels-1."""
    g0 = inst.grid
    err = check_hierarchy_inputs(g0.nx, g0.ny, levels, passes)
    if err:
        raise ValueError("gust: invalid grid hierarchy:\n  " + "\n  ".join(err))
    out = [Level(0, inst, g0, inst.ground, inst.z0map)]
    for lev in range(1, levels):
        r = hierarchy_ratio(lev)
        gc = Grid(g0.nx // r, g0.ny // r, g0.nz, g0.dx * r, g0.dy * r, g0.dzeta, g0.periodic_x, g0.periodic_y)
        ground = inject_ground(inst.ground, r, gc.nx, gc.ny, g0.periodic_x, g0.periodic_y)
        smooth_surface(ground, gc.nx, gc.ny, g0.periodic_x, g0.periodic_y, ground_passes(lev, passes))
        z0map = None if inst.z0map is None else average_roughness(inst.z0map, g0, r, gc)
        out.append(Level(lev, inst, gc, ground, z0map))
    return out
