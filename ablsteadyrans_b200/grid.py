"""The grid layout of include/gust_b200.h on the Python side (no library
needed): the ctypes mirror of gb_grid and array helpers."""
import ctypes

import numpy as np

LOC_CELL, LOC_XFACE, LOC_YFACE, LOC_ZFACE, LOC_NODE = 0, 1, 2, 4, 7
N_COEFS = 7


class GbGrid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("ng", ctypes.c_int32),
        ("periodic_x", ctypes.c_int32), ("periodic_y", ctypes.c_int32),
        ("sy", ctypes.c_int64), ("sz", ctypes.c_int64),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dzeta", ctypes.c_double),
    ]


class Grid:
    """nx x ny x nz cells with ng ghost layers: every array is
    (nz+1+2ng, ny+1+2ng, nx+1+2ng) indexed [k+ng, j+ng, i+ng]."""

    def __init__(self, nx, ny, nz, dx, dy, dzeta, periodic_x=False, periodic_y=False, ng=2):
        self.nx, self.ny, self.nz, self.ng = int(nx), int(ny), int(nz), int(ng)
        self.dx, self.dy, self.dzeta = float(dx), float(dy), float(dzeta)
        self.periodic_x, self.periodic_y = bool(periodic_x), bool(periodic_y)
        c = GbGrid()
        c.nx, c.ny, c.nz, c.ng = self.nx, self.ny, self.nz, self.ng
        c.periodic_x, c.periodic_y = int(self.periodic_x), int(self.periodic_y)
        c.sy = self.nx + 1 + 2 * self.ng
        c.sz = c.sy * (self.ny + 1 + 2 * self.ng)
        c.dx, c.dy, c.dzeta = self.dx, self.dy, self.dzeta
        self.c = c

    @property
    def shape(self):
        return (self.nz + 1 + 2 * self.ng, self.ny + 1 + 2 * self.ng, int(self.c.sy))

    @property
    def volume(self):
        return int(self.c.sz) * (self.nz + 1 + 2 * self.ng)

    @property
    def cells(self):
        return self.nx * self.ny * self.nz

    def extents(self, loc):
        return (self.nx + (loc & 1), self.ny + ((loc >> 1) & 1), self.nz + ((loc >> 2) & 1))

    def valid(self, loc):
        """Index tuple of the valid points of a location in a (k, j, i) array."""
        ni, nj, nk = self.extents(loc)
        g = self.ng
        return (slice(g, g + nk), slice(g, g + nj), slice(g, g + ni))

    def np_zeros(self, ncomp=None, dtype=np.float64):
        shape = self.shape if ncomp is None else (ncomp,) + self.shape
        return np.zeros(shape, dtype=dtype)

    def coarsened(self):
        """The grid of the next multigrid level: x and y halved, z kept."""
        return Grid(self.nx // 2, self.ny // 2, self.nz, 2 * self.dx, 2 * self.dy, self.dzeta,
                    self.periodic_x, self.periodic_y, self.ng)
