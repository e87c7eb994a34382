"""Synthetic inputs of the benchmark configurations (one seeded generator for
the GPU path and the CPU baseline): vertical levels, terrain (Gaussian hill,
fractal field), BTF node heights, the per-column roughness, the log-law
inflow state, boundary and physics settings.

Resolved ambiguities of the configurations:
  * "a 2 m first cell at ratio 1.1 up to a 1500 m lid" is over-determined:
    the first cell is 2 m, the lid 1500 m and the ratio is solved
    (1.0927 for nz = 48, 1.0622 for nz = 64, 1.0350 for nz = 96).
  * Wind directions are meteorological ("from"); the inflow direction is the
    one the wind blows towards, CCW from +x: 270 - met.
  * Coriolis f: forcing.latitude = 90 with rotation_period = 4 pi / f; the
    geostrophic wind is the log-law wind at the lid.
  * Physics (turbulence=True, the default): the k-L closure (turb.*
    defaults, max_geom_lscale 30 m) and a neutral surface_layer ground
    (MOST, Dirichlet wall k) with the configuration's z0. With
    turbulence=False the ground is a no-slip wall and the diffusivities are
    frozen at the inflow's equilibrium mixing-length profile, nu = nu_mol +
    kappa u* (h + z0) / (1 + kappa (h + z0) / l_max), gamma_theta = nu / 0.85,
    gamma_k = nu (the given-diffusivity form of the residual).
"""
import math

import numpy as np

from . import abi
from .grid import Grid

KAPPA, CMU0, LMAX, NU_MOL = 0.41, 0.5562, 30.0, 1.5e-5


def geometric_zlevels(nz, dz0=2.0, ztop=1500.0):
    """Levels z_0 = 0 .. z_nz = ztop with a first cell dz0 and a constant
    stretch ratio solved by bisection."""
    def top(r):
        return dz0 * nz if abs(r - 1) < 1e-15 else dz0 * (r ** nz - 1) / (r - 1)
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if top(mid) < ztop:
            lo = mid
        else:
            hi = mid
    r = 0.5 * (lo + hi)
    z = np.zeros(nz + 1)
    dz = dz0
    for k in range(1, nz + 1):
        z[k] = z[k - 1] + dz
        dz *= r
    z[nz] = ztop
    return z, r


def btf_heights(grid, zlevels, ground):
    """Basic terrain-following node heights (ERF_TerrainMetrics.cpp BTF case),
    ground: (ny+3, nx+3) heights of node columns i, j in [-1, n+1]; the rows
    below the ground and above the top extrapolated linearly (Source/Mesh.cpp
    fill_ghost_columns)."""
    g = grid.ng
    z = grid.np_zeros()
    nz = grid.nz
    ztop, z0 = float(zlevels[nz]), float(zlevels[0])
    zs = np.asarray(ground, dtype=np.float64)
    sl = (slice(g - 1, g + grid.ny + 2), slice(g - 1, g + grid.nx + 2))
    z[(g,) + sl] = zs
    for k in range(1, nz + 1):
        z[(g + k,) + sl] = ((zs - z0) * ztop + (ztop - zs) * float(zlevels[k])) / (ztop - z0)
    z[(g - 1,) + sl] = 2.0 * z[(g,) + sl] - z[(g + 1,) + sl]
    for k in range(-2, -grid.ng - 1, -1):
        z[(g + k,) + sl] = z[(g,) + sl] + (0 - k) * (z[(g,) + sl] - z[(g + 1,) + sl])
    for k in range(nz + 1, nz + grid.ng + 1):
        z[(g + k,) + sl] = z[(g + nz,) + sl] + (k - nz) * (z[(g + nz,) + sl] - z[(g + nz - 1,) + sl])
    return z


def node_ground(grid, height_fn):
    """Ground heights of every node column (ghosts: periodic image or the
    clamped edge column, as the reference's terrain fill)."""
    out = np.zeros((grid.ny + 3, grid.nx + 3))
    for j in range(-1, grid.ny + 2):
        for i in range(-1, grid.nx + 2):
            ii = (i % grid.nx) if grid.periodic_x else min(max(i, 0), grid.nx)
            jj = (j % grid.ny) if grid.periodic_y else min(max(j, 0), grid.ny)
            out[j + 1, i + 1] = height_fn(ii * grid.dx, jj * grid.dy)
    return out


def fractal_field(n, seed, rms, slope=3.0, dx=None, max_slope=None):
    """A Gaussian random field on an n x n grid with isotropic power spectrum
    |k|^-slope, standardised, scaled to `rms`, minimum shifted to 0. With
    dx and max_slope the field is scaled down where its steepest node-to-node
    slope would exceed max_slope (beyond a slope of about 2 the terrain-
    following Poisson operator loses definiteness and the solves stagnate)."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n)[:, None]
    ky = np.fft.fftfreq(n)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-slope / 2.0)
    amp[0, 0] = 0.0
    noise = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    f = np.real(np.fft.ifft2(noise * amp))
    f = (f - f.mean()) / f.std() * rms
    if dx is not None and max_slope is not None:
        steepest = max(np.abs(np.diff(f, axis=0)).max(), np.abs(np.diff(f, axis=1)).max()) / dx
        if steepest > max_slope:
            f = f * (max_slope / steepest)
    return f - f.min()


def edge_taper(f, margin):
    """The field brought down to its minimum over the outer `margin` fraction
    of each side with a raised-cosine weight (flat ground at the lateral
    faces, so that the inflow profile and the zero-gradient outflow meet
    level terrain)."""
    if margin <= 0:
        return f
    ny, nx = f.shape

    def w(n):
        s = np.minimum(np.arange(n), np.arange(n)[::-1]) / max((n - 1) * margin, 1e-300)
        return np.where(s < 1.0, 0.5 * (1.0 - np.cos(np.pi * np.minimum(s, 1.0))), 1.0)
    base = f.min()
    return base + (f - base) * w(ny)[:, None] * w(nx)[None, :]


def cap_slope(f, dx, max_slope):
    """f scaled about its minimum so that no node-to-node slope exceeds max_slope."""
    steepest = max(np.abs(np.diff(f, axis=0)).max(), np.abs(np.diff(f, axis=1)).max()) / dx
    if steepest <= max_slope:
        return f
    return f.min() + (f - f.min()) * (max_slope / steepest)


def log_law(h, ustar, z0):
    return ustar / KAPPA * np.log((np.maximum(h, 0.0) + z0) / z0)


class Instance:
    """One solve: grid, host arrays (node heights, diffusivities, initial
    state) and the C ABI settings."""

    def __init__(self, name, grid, zlevels, ground, bc, physics, options, ustar, z0, direction, z0map=None):
        self.name = name
        self.z0map = z0map   # per-column roughness plane (gb_mesh_fields.z0), or None
        self.ground = ground  # node ground heights, columns -1..n+1 (ny + 3, nx + 3)
        self.grid = grid
        self.zlevels = zlevels
        self.z = btf_heights(grid, zlevels, ground)
        self.bc, self.physics, self.options = bc, physics, options
        self.ustar, self.z0, self.direction = ustar, z0, direction
        g = grid
        G = g.ng
        z = self.z
        # cell-centre heights above the ground, from the node heights (mean of 8 nodes)
        zc = 0.125 * sum(z[G + dk:G + dk + g.nz, G + dj:G + dj + g.ny, G + di:G + di + g.nx]
                         for dk in (0, 1) for dj in (0, 1) for di in (0, 1))
        zg = 0.25 * sum(z[G, G + dj:G + dj + g.ny, G + di:G + di + g.nx] for dj in (0, 1) for di in (0, 1))
        h = zc - zg[None]
        self.h = h
        ell = KAPPA * (h + z0) / (1.0 + KAPPA * (h + z0) / LMAX)
        nu_c = NU_MOL + ell * ustar
        self.nu = self._cell_with_ghosts(nu_c)
        self.gamma_theta = self.nu / 0.85
        self.gamma_tke = self.nu.copy()
        self.q = self._initial_state()

    def _cell_with_ghosts(self, c):
        g = self.grid
        G = g.ng
        a = g.np_zeros()
        a[G:G + g.nz, G:G + g.ny, G:G + g.nx] = c
        # one ghost layer: periodic image or the edge value; below/above: the edge
        a[G:G + g.nz, G:G + g.ny, G - 1] = c[:, :, -1] if g.periodic_x else c[:, :, 0]
        a[G:G + g.nz, G:G + g.ny, G + g.nx] = c[:, :, 0] if g.periodic_x else c[:, :, -1]
        a[G:G + g.nz, G - 1, :] = a[G:G + g.nz, G + g.ny - 1, :] if g.periodic_y else a[G:G + g.nz, G, :]
        a[G:G + g.nz, G + g.ny, :] = a[G:G + g.nz, G, :] if g.periodic_y else a[G:G + g.nz, G + g.ny - 1, :]
        a[G - 1] = a[G]
        a[G + g.nz] = a[G + g.nz - 1]
        return a

    def _initial_state(self):
        """The inflow profile at every point's height above the ground."""
        g = self.grid
        G = g.ng
        z = self.z
        dr = math.radians(self.direction)
        q = {f: g.np_zeros() for f in ("u", "v", "w", "p", "theta", "tke")}
        # x-faces: mean of the face's 4 nodes minus its 2 ground nodes
        def face_h(di, dj):
            top = sum(z[G + dk:G + dk + g.nz, G:G + g.ny + dj, G:G + g.nx + di] for dk in (0, 1))
            return top
        hx = (0.25 * (z[G:G + g.nz, G:G + g.ny, G:G + g.nx + 1] + z[G + 1:G + g.nz + 1, G:G + g.ny, G:G + g.nx + 1]
                      + z[G:G + g.nz, G + 1:G + g.ny + 1, G:G + g.nx + 1] + z[G + 1:G + g.nz + 1, G + 1:G + g.ny + 1, G:G + g.nx + 1])
              - 0.5 * (z[G, G:G + g.ny, G:G + g.nx + 1] + z[G, G + 1:G + g.ny + 1, G:G + g.nx + 1])[None])
        hy = (0.25 * (z[G:G + g.nz, G:G + g.ny + 1, G:G + g.nx] + z[G + 1:G + g.nz + 1, G:G + g.ny + 1, G:G + g.nx]
                      + z[G:G + g.nz, G:G + g.ny + 1, G + 1:G + g.nx + 1] + z[G + 1:G + g.nz + 1, G:G + g.ny + 1, G + 1:G + g.nx + 1])
              - 0.5 * (z[G, G:G + g.ny + 1, G:G + g.nx] + z[G, G:G + g.ny + 1, G + 1:G + g.nx + 1])[None])
        q["u"][G:G + g.nz, G:G + g.ny, G:G + g.nx + 1] = log_law(hx, self.ustar, self.z0) * math.cos(dr)
        q["v"][G:G + g.nz, G:G + g.ny + 1, G:G + g.nx] = log_law(hy, self.ustar, self.z0) * math.sin(dr)
        q["theta"][...] = 300.0
        c = 1.0 / (1.0 + KAPPA * (self.h + self.z0) / LMAX)
        q["tke"][G:G + g.nz, G:G + g.ny, G:G + g.nx] = (self.ustar * c) ** 2 / CMU0 ** 2
        return q

    @property
    def cells(self):
        return self.grid.cells


def _faces_for(direction, periodic_y=True, ground=abi.FACE_NO_SLIP_WALL):
    """Inflow on the upwind x face (and y face when not periodic), outflow downwind."""
    c = math.cos(math.radians(direction))
    xlo, xhi = (abi.FACE_INFLOW, abi.FACE_OUTFLOW) if c >= 0 else (abi.FACE_OUTFLOW, abi.FACE_INFLOW)
    if periodic_y:
        ylo = yhi = abi.FACE_PERIODIC
    else:
        s = math.sin(math.radians(direction))
        ylo, yhi = (abi.FACE_INFLOW, abi.FACE_OUTFLOW) if s >= 0 else (abi.FACE_OUTFLOW, abi.FACE_INFLOW)
    return (xlo, ylo, ground, xhi, yhi, abi.FACE_SLIP_WALL)


def _turbulence(turbulence, z0):
    """(ground face type, surface options, physics keywords) of the physics
    switch: the k-L closure and a neutral surface layer, or none."""
    if not turbulence:
        return abi.FACE_NO_SLIP_WALL, None, {}
    return (abi.FACE_SURFACE_LAYER, {"z0": z0},
            dict(closure=1, turb_Cmu0=CMU0, turb_kappa=KAPPA, turb_max_geom_lscale=LMAX))


def lognormal_z0(grid, seed, median, sigma):
    """A per-column roughness plane (gb_mesh_fields.z0's layout): z0 lognormal
    with the median and the log-standard deviation given, on the domain
    columns; the ghost columns the periodic image or the nearest column."""
    rng = np.random.default_rng(seed)
    cols = median * np.exp(sigma * rng.standard_normal((grid.ny, grid.nx)))
    G = grid.ng
    plane = np.zeros((grid.ny + 1 + 2 * G, grid.nx + 1 + 2 * G))
    for j in range(-G, grid.ny + 1 + G):
        for i in range(-G, grid.nx + 1 + G):
            ii = (i % grid.nx) if grid.periodic_x else min(max(i, 0), grid.nx - 1)
            jj = (j % grid.ny) if grid.periodic_y else min(max(j, 0), grid.ny - 1)
            plane[j + G, i + G] = cols[jj, ii]
    return plane.reshape(-1)


def config0(nx=32, ny=32, nz=48, precision=0, zline_sweeps=4, turbulence=True):
    """Plain FP64 over flat ground, the neutral ABL of the oracle case:
    32 x 32 x 48 cells, dx = dy = 40 m, the stretched layers to a 1500 m lid
    (ratio 1.0927); log-law inflow u* = 0.4 m/s, z0 = 0.1 m from the west
    (270 deg), outflow east, periodic in y; the k-L closure and a neutral
    Monin-Obukhov surface layer (turbulence); no Coriolis."""
    dx = 40.0
    zl, _ = geometric_zlevels(nz)
    g = Grid(nx, ny, nz, dx, dx, 1500.0 / nz, False, True)
    ground = np.zeros((ny + 3, nx + 3))
    ustar, z0, direction = 0.4, 0.1, 270.0 - 270.0
    ground_face, surface, turb = _turbulence(turbulence, z0)
    bc = abi.BC.make(_faces_for(direction, ground=ground_face), theta_ref=((0.0, 1500.0), (300.0, 300.0)), ustar=ustar,
                     z0=z0, direction=direction, kappa=KAPPA, Cmu0=CMU0, l_max=LMAX, surface=surface)
    ph = abi.Physics.make(1500.0, gravity=9.81, **turb)
    opts = abi.SimplecOptions.make(zline_sweeps=zline_sweeps, precision=precision)
    return Instance(f"config0-flat-{nx}x{ny}x{nz}", g, zl, ground, bc, ph, opts, ustar, z0, direction)


def config1(nx=128, ny=128, nz=64, precision=0, zline_sweeps=4, turbulence=True):
    """Plain FP64 on the GPU over a single Gaussian hill h = 150 exp(-(r/300)^2)
    centred in a 128 x 128 x 64 grid, dx = dy = 25 m, the stretched layers to a
    1500 m lid; log-law inflow u* = 0.45 m/s, z0 = 0.03 m from 270 deg;
    Coriolis f = 1e-4 1/s with the geostrophic wind at the lid; neutral; the
    k-L closure and the surface layer (turbulence)."""
    dx = 25.0
    zl, _ = geometric_zlevels(nz)
    g = Grid(nx, ny, nz, dx, dx, 1500.0 / nz, False, True)
    xc, yc = nx * dx / 2, ny * dx / 2
    ground = node_ground(g, lambda x, y: 150.0 * math.exp(-(((x - xc) ** 2 + (y - yc) ** 2) / 300.0 ** 2)))
    ustar, z0, direction = 0.45, 0.03, 270.0 - 270.0
    f = 1e-4
    ug = float(log_law(np.array([1500.0]), ustar, z0)[0])
    ground_face, surface, turb = _turbulence(turbulence, z0)
    bc = abi.BC.make(_faces_for(direction, ground=ground_face), theta_ref=((0.0, 1500.0), (300.0, 300.0)), ustar=ustar,
                     z0=z0, direction=direction, kappa=KAPPA, Cmu0=CMU0, l_max=LMAX, surface=surface)
    ph = abi.Physics.make(1500.0, gravity=9.81, coriolis=1, latitude=90.0, rotation_period=4 * math.pi / f,
                          geostrophic=1, ug=ug, vg=0.0, **turb)
    opts = abi.SimplecOptions.make(zline_sweeps=zline_sweeps, precision=precision)
    return Instance("config1-hill-128x128x64", g, zl, ground, bc, ph, opts, ustar, z0, direction)


#: The steepest node-to-node terrain slope of a generated tile (the fractal
#: field is scaled down to it where steeper).
MAX_TILE_SLOPE = 1.0
#: The outer fraction of each side of a tile over which its terrain is
#: tapered to flat (edge_taper).
TILE_EDGE_TAPER = 0.15


def tile(n, nz, seed, rms=None, ustar=None, z0=None, met=None, dx=30.0, precision=1, zline_sweeps=4, turbulence=True):
    """One instance of the batched/served configurations: n x n x nz over
    seeded fractal terrain (|k|^-3, rms uniform 20-150 m unless given), a
    random wind direction, u* and z0 (seed-derived); inflow on the upwind x
    and y faces of the wind's quadrant, outflow on the others. The terrain
    is scaled down where its slope would exceed MAX_TILE_SLOPE and tapered
    to flat over the outer TILE_EDGE_TAPER of each side: without the taper,
    ridges at the outflow faces turn the flow back into the domain there,
    where the zero-gradient outflow is ill-posed, and the solve stalls."""
    rng = np.random.default_rng(1000 + seed)
    rms = rms if rms is not None else rng.uniform(20, 150)
    ustar = ustar if ustar is not None else rng.uniform(0.2, 0.6)
    z0 = z0 if z0 is not None else rng.uniform(0.01, 0.5)
    met = met if met is not None else rng.uniform(0, 360)
    direction = (270.0 - met) % 360.0
    zl, _ = geometric_zlevels(nz)
    g = Grid(n, n, nz, dx, dx, 1500.0 / nz, False, False)
    terrain = cap_slope(edge_taper(fractal_field(n + 1, seed, rms, dx=dx, max_slope=MAX_TILE_SLOPE), TILE_EDGE_TAPER),
                        dx, MAX_TILE_SLOPE)
    ground = node_ground(g, lambda x, y: float(terrain[int(round(y / dx)) % (n + 1), int(round(x / dx)) % (n + 1)]))
    ground_face, surface, turb = _turbulence(turbulence, z0)
    bc = abi.BC.make(_faces_for(direction, periodic_y=False, ground=ground_face), theta_ref=((0.0, 1500.0), (300.0, 300.0)),
                     ustar=ustar, z0=z0, direction=direction, kappa=KAPPA, Cmu0=CMU0, l_max=LMAX, surface=surface)
    ph = abi.Physics.make(1500.0, gravity=9.81, **turb)
    opts = abi.SimplecOptions.make(zline_sweeps=zline_sweeps, precision=precision)
    return Instance(f"tile-{seed}-{n}x{n}x{nz}", g, zl, ground, bc, ph, opts, ustar, z0, direction)


def config2(precision=1, zline_sweeps=4, n=256, nz=96, seed=2, max_slope=1.0, turbulence=True):
    """Mixed precision against plain FP64 on a 256 x 256 x 96 grid, dx = dy =
    30 m, over seeded fractal terrain (|k|^-3, 120 m rms, minimum 0, scaled
    down where steeper than max_slope); log-law inflow u* = 0.4 m/s from
    225 deg (inflow on the x and y faces upwind); the ground's z0 per column
    lognormal with median 0.05 m and sigma 0.7 (the surface layer's map; the
    inflow log law takes the median); the k-L closure (turbulence)."""
    dx = 30.0
    met = 225.0
    direction = (270.0 - met) % 360.0
    zl, _ = geometric_zlevels(nz)
    g = Grid(n, n, nz, dx, dx, 1500.0 / nz, False, False)
    terrain = fractal_field(n + 1, seed, 120.0, dx=dx, max_slope=max_slope)
    ground = node_ground(g, lambda x, y: float(terrain[int(round(y / dx)) % (n + 1), int(round(x / dx)) % (n + 1)]))
    ustar, z0 = 0.4, 0.05
    ground_face, surface, turb = _turbulence(turbulence, z0)
    bc = abi.BC.make(_faces_for(direction, periodic_y=False, ground=ground_face), theta_ref=((0.0, 1500.0), (300.0, 300.0)),
                     ustar=ustar, z0=z0, direction=direction, kappa=KAPPA, Cmu0=CMU0, l_max=LMAX, surface=surface)
    ph = abi.Physics.make(1500.0, gravity=9.81, **turb)
    opts = abi.SimplecOptions.make(zline_sweeps=zline_sweeps, precision=precision)
    z0map = lognormal_z0(g, 5000 + seed, z0, 0.7) if turbulence else None
    return Instance(f"config2-fractal-{n}x{n}x{nz}", g, zl, ground, bc, ph, opts, ustar, z0, direction, z0map)
