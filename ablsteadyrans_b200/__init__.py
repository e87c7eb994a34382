"""B200-native SIMPLEC hot path of GUST (hgopalan/ablsteadyrans).

The compute lives in libgustb200.so (CUDA for sm_100a behind the C ABI of
include/gust_b200.h). This module is the Python mirror of the reference's
operator interface for the path: it binds the C ABI with ctypes and passes
device memory held by torch tensors (torch is plumbing here: allocation and
the stream). There is no CPU fallback: importing the package without the
built library raises.

Arrays: every field of a grid is a tensor of shape (nz+1+2ng, ny+1+2ng, sy)
indexed [k+ng, j+ng, i+ng] (k-plane-major, i fastest), the same index space
for cells, faces and nodes; multi-component fields add a leading component
axis. See Grid.
"""
import ctypes
import os

import numpy as np

from . import abi as _abi
from .abi import (BC, Diffusivities, IterInfo, MeshFields, Physics, SimplecOptions, State,  # noqa: F401
                  FACE_INFLOW, FACE_NO_SLIP_WALL, FACE_OUTFLOW, FACE_PERIODIC, FACE_SLIP_WALL, LIMITER_UPWIND,
                  LIMITER_VAN_ALBADA, LIMITER_VAN_LEER)
from .grid import Grid, GbGrid, LOC_CELL, LOC_XFACE, LOC_YFACE, LOC_ZFACE, LOC_NODE, N_COEFS  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgustb200.so")
_lib = None

GB_OK = 0
KERNEL_LINE_SWEEP, KERNEL_POISSON_APPLY, KERNEL_MG_SMOOTH, KERNEL_MG_TRANSFER, KERNEL_RESIDUAL, \
    KERNEL_MASSFLUX, KERNEL_COEFS, KERNEL_VECTOR, KERNEL_BC = range(9)
(TUNE_LINE_VARIANT, TUNE_LINE_BLOCK, TUNE_MG_COARSE_KERNEL, TUNE_LINE_DEPTH, TUNE_LINE_BACK, TUNE_MG_FUSED_RELAX,
 TUNE_GRAPHS, TUNE_MG_SOLVE, TUNE_LINE_FIRST, TUNE_LINE_SEGMENT, TUNE_RESIDUAL, TUNE_MG_TAIL,
 TUNE_MG_STENCIL, TUNE_PDL) = range(14)
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "NONFINITE", 3: "NOT_CONVERGED", 4: "TIMEOUT", 5: "OOM", 6: "CUDA"}


class GustError(RuntimeError):
    """A gb_status other than GB_OK, with the library's message."""

    def __init__(self, status, message):
        super().__init__(f"{message} [{STATUS_NAMES.get(status, status)}]")
        self.status = status
        self.message = message


def lib():
    """The loaded libgustb200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libgustb200.so is not built ({LIB_PATH}); run __graft_entry__.build()")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    P = ctypes.c_void_p
    G = ctypes.POINTER(GbGrid)
    i32, i64, f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    L.gb_last_error.restype = ctypes.c_char_p
    L.gb_grid_init.argtypes = [G, i32, i32, i32, i32, f64, f64, f64, i32, i32]
    L.gb_grid_volume.argtypes = [G]
    L.gb_grid_volume.restype = i64
    L.gb_ctx_create.argtypes = [P, ctypes.POINTER(P)]
    L.gb_ctx_destroy.argtypes = [P]
    L.gb_ctx_launches.argtypes = [P]
    L.gb_ctx_launches.restype = i64
    L.gb_ctx_tune.argtypes = [P, i32, i32]
    L.gb_ctx_profile.argtypes = [P, i32]
    L.gb_ctx_profile_read.argtypes = [P, i32, ctypes.POINTER(f64), ctypes.POINTER(i64)]
    L.gb_ctx_profile_mask.argtypes = [P, ctypes.c_uint32]
    L.gb_probe_fp64.argtypes = [P, i32, P, ctypes.POINTER(i64)]
    L.gb_zline_jacobi.argtypes = [P, G, i32, P, P, P, i32, P, ctypes.POINTER(f64)]
    L.gb_zline_jacobi_f32.argtypes = [P, G, i32, P, P, P, i32, P, ctypes.POINTER(ctypes.c_float)]
    L.gb_zline_jacobi_noalloc.argtypes = [G, i32, P, P, P, i32, P, ctypes.POINTER(f64), P]
    L.gb_zline_lusgs.argtypes = [P, G, i32, P, P, P, i32, i32, P, ctypes.POINTER(f64)]
    L.gb_zline_jacobi_batch.argtypes = [P, i32, P, i32, P]
    L.gb_zline_jacobi_batch_f32.argtypes = [P, i32, P, i32, P]


def check(status):
    if status != GB_OK:
        raise GustError(status, lib().gb_last_error().decode())


def _ptr(t):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """A gb_ctx on torch's current CUDA stream (owns the scratch of the calls)."""

    def __init__(self, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()
        self.stream = stream
        self._h = ctypes.c_void_p()
        self._owned = []
        check(lib().gb_ctx_create(ctypes.c_void_p(stream.cuda_stream), ctypes.byref(self._h)))

    def own(self, obj):
        """Record a native object made on this context (a solver, stage or
        driver): close() destroys the live ones first, newest first, since
        their destructors synchronise on the context's stream."""
        import weakref
        self._owned = [r for r in self._owned if r() is not None]
        self._owned.append(weakref.ref(obj))

    @property
    def handle(self):
        return self._h

    def launches(self):
        return int(lib().gb_ctx_launches(self._h))

    def tune(self, key, value):
        check(lib().gb_ctx_tune(self._h, int(key), int(value)))

    def profile(self, enable):
        check(lib().gb_ctx_profile(self._h, int(bool(enable))))

    def profile_mask(self, families):
        """Time only these kernel families while profiling (default: all)."""
        mask = 0
        for f in families:
            mask |= 1 << int(f)
        check(lib().gb_ctx_profile_mask(self._h, mask))

    def profile_read(self, family):
        """(total milliseconds, launches) of one kernel family since profile(True)."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        check(lib().gb_ctx_profile_read(self._h, int(family), ctypes.byref(t), ctypes.byref(n)))
        return float(t.value), int(n.value)

    def close(self):
        if self._h:
            for r in reversed(self._owned):
                obj = r()
                if obj is not None:
                    obj.close()
            self._owned = []
            check(lib().gb_ctx_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def zline_jacobi(ctx, grid, loc, A, ap, rhs, sweeps, delta):
    """gust::zline_jacobi (Source/Predictor.H:267-268): z-line Jacobi sweeps of
    (A, ap) with right-hand side rhs into delta; returns max |change of the last
    sweep|. FP64 or FP32 by the tensors' dtype."""
    import torch
    L = lib()
    if A.dtype == torch.float64:
        out = ctypes.c_double()
        check(L.gb_zline_jacobi(ctx.handle, ctypes.byref(grid.c), loc, _ptr(A), _ptr(ap), _ptr(rhs), sweeps,
                                _ptr(delta), ctypes.byref(out)))
    else:
        out = ctypes.c_float()
        check(L.gb_zline_jacobi_f32(ctx.handle, ctypes.byref(grid.c), loc, _ptr(A), _ptr(ap), _ptr(rhs), sweeps,
                                    _ptr(delta), ctypes.byref(out)))
    return float(out.value)


def zline_jacobi_batch(ctx, systems, sweeps, want_change=True):
    """gust::zline_jacobi over many systems of different grids at once
    (gb_zline_jacobi_batch): systems is a list of (grid, loc, A, ap, rhs,
    delta), all FP64 or all FP32; every delta gets the values
    gb_zline_jacobi gives its system alone. Returns the list of each
    system's max |change of the last sweep| (None when want_change is
    false: nothing waits for the stream)."""
    import torch
    from .abi import LineSystem
    n = len(systems)
    arr = (LineSystem * n)()
    f64 = None
    for q, (grid, loc, A, ap, rhs, delta) in enumerate(systems):
        is64 = A.dtype == torch.float64
        if f64 is None:
            f64 = is64
        elif f64 != is64:
            raise ValueError("zline_jacobi_batch: the systems mix FP64 and FP32")
        arr[q].grid = grid.c
        arr[q].loc = int(loc)
        arr[q].A = A.data_ptr()
        arr[q].ap = ap.data_ptr()
        arr[q].rhs = rhs.data_ptr()
        arr[q].delta = delta.data_ptr()
    out = (ctypes.c_double * n)() if want_change else None
    fn = lib().gb_zline_jacobi_batch if f64 else lib().gb_zline_jacobi_batch_f32
    check(fn(ctx.handle, n, arr, int(sweeps), out))
    return [float(v) for v in out] if want_change else None


def probe_fp64(ctx, iters, sink):
    """gb_probe_fp64: 8 chains of `iters` dependent FP64 FMAs per thread on the
    context's stream (sink: 4 * SMs * 256 doubles); returns the FP64
    operations it executes (2 per FMA)."""
    threads = ctypes.c_int64()
    check(lib().gb_probe_fp64(ctx.handle, int(iters), _ptr(sink), ctypes.byref(threads)))
    return 2 * 8 * int(iters) * threads.value


def implicit_coefficients(ctx, grid, loc, F, gamma, z, J, log_mean, A):
    """gust::implicit_coefficients (Source/ImplicitOperator.H:65-67) at loc:
    the upwind transport of F (three face tensors) and the principal
    diffusion of gamma into A (7 x grid, FP64)."""
    check(_lib_full().gb_implicit_coefficients(ctx.handle, ctypes.byref(grid.c), int(loc), *[_ptr(f) for f in F],
                                         _ptr(gamma), _ptr(z), _ptr(J), int(bool(log_mean)), _ptr(A)))
    return A


def zline_lusgs(ctx, grid, loc, A, ap, rhs, sweeps, delta, alternate=0):
    """gust::zline_lusgs with line_ghosts = lagged (Source/LineSweeps.H:
    159-161): symmetric line LU-SGS passes into delta (FP64); returns max
    |change| over the last backward pass."""
    out = ctypes.c_double()
    check(lib().gb_zline_lusgs(ctx.handle, ctypes.byref(grid.c), loc, _ptr(A), _ptr(ap), _ptr(rhs), int(sweeps),
                               int(alternate), _ptr(delta), ctypes.byref(out)))
    return float(out.value)


def zline_jacobi_noalloc(grid, loc, A, ap, rhs, sweeps, delta, stream=None):
    """The FP64 z-line Jacobi solve without a context and without any device
    allocation (gb_zline_jacobi_noalloc): its scratch is a fixed array in the
    library (grids up to 2^21 padded points); calls that may overlap on one
    device race on it. stream: a torch.cuda.Stream (default: the current
    one). Returns max |change of the last sweep|."""
    import torch
    L = lib()
    if stream is None:
        stream = torch.cuda.current_stream()
    out = ctypes.c_double()
    check(L.gb_zline_jacobi_noalloc(ctypes.byref(grid.c), loc, _ptr(A), _ptr(ap), _ptr(rhs), sweeps, _ptr(delta),
                                    ctypes.byref(out), ctypes.c_void_p(stream.cuda_stream)))
    return float(out.value)


# ------------------------------------------------------------------- mesh ---
POISSON_PERIODIC, POISSON_NEUMANN, POISSON_DIRICHLET = 0, 1, 2


class PoissonOptions(_abi.PoissonOptions):
    """gb_poisson_opts (include/gust_b200.h), with the library's defaults."""

    @classmethod
    def default(cls, **kw):
        o = cls()
        check(lib().gb_poisson_options_default(ctypes.byref(o)))
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class PoissonResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("singular", ctypes.c_int32), ("initial_residual", ctypes.c_double),
                ("final_residual", ctypes.c_double), ("removed_mean", ctypes.c_double)]


def _declare_poisson(L):
    P = ctypes.c_void_p
    G = ctypes.POINTER(GbGrid)
    L.gb_mesh_metrics.argtypes = [P, G, P, P, P, P, P, P]
    L.gb_implicit_coefficients.argtypes = [P, G, ctypes.c_int32, P, P, P, P, P, P, ctypes.c_int32, P]
    L.gb_face_divergence.argtypes = [P, G, P, P, P, P, P, P, P, P]
    from .abi import MeshFields, State
    L.gb_restrict_state.argtypes = [P, G, ctypes.POINTER(State), ctypes.POINTER(MeshFields), G, ctypes.POINTER(State),
                                    ctypes.POINTER(MeshFields), P]
    L.gb_poisson_options_default.argtypes = [ctypes.POINTER(PoissonOptions)]
    L.gb_poisson_create.argtypes = [P, G, ctypes.POINTER(ctypes.c_int32), P, P, ctypes.POINTER(PoissonOptions),
                                    ctypes.POINTER(P)]
    L.gb_poisson_destroy.argtypes = [P]
    L.gb_poisson_set_coeffs.argtypes = [P, P, P, P, P, P, P]
    L.gb_poisson_set_z_cross.argtypes = [P, P, P, P]
    L.gb_poisson_apply.argtypes = [P, P, P]
    L.gb_poisson_vcycle.argtypes = [P, P, P]
    L.gb_poisson_solve.argtypes = [P, P, P, ctypes.POINTER(PoissonResult)]
    L.gb_tucker_wall_distance.argtypes = [P, G, P, ctypes.POINTER(PoissonOptions), P, ctypes.POINTER(PoissonResult)]
    L.gb_poisson_fluxes.argtypes = [P, P, P, P, P, P, P, P]


_declare_hooks = [_declare_poisson]


def _lib_full():
    L = lib()
    if not getattr(L, "_gb_full", False):
        for h in _declare_hooks:
            h(L)
        L._gb_full = True
    return L


def _zeros(grid, dtype=None):
    import torch
    return torch.zeros(grid.shape, dtype=dtype or torch.float64, device="cuda")


def tucker_wall_distance(ctx, grid, z_nd, options=None):
    """gust::tucker_wall_distance (Source/WallDistance.H:14-33): Tucker's
    wall distance on the terrain mesh (a device volume of the grid with its
    ghosts) and the Poisson solve's PoissonResult."""
    L = _lib_full()
    dist = _zeros(grid)
    res = PoissonResult()
    opt = ctypes.byref(options) if options is not None else None
    check(L.gb_tucker_wall_distance(ctx.handle, ctypes.byref(grid.c), _ptr(z_nd), opt, _ptr(dist), ctypes.byref(res)))
    return dist, res


def mesh_metrics(ctx, grid, z_nd):
    """detJ, ax, ay, az, z_cc of the terrain-following mesh (Mesh::make_metrics,
    Source/Mesh.cpp:147-152 -> ERF_TerrainMetrics.cpp:680-808)."""
    out = [_zeros(grid) for _ in range(5)]
    check(_lib_full().gb_mesh_metrics(ctx.handle, ctypes.byref(grid.c), _ptr(z_nd), *[_ptr(t) for t in out]))
    return out


def restrict_state(ctx, fine, coarse):
    """gust::restrict_state (Source/Transfer.H:94-110): the state of a
    DeviceCase `fine` onto the coarser DeviceCase `coarse` (u, v with their
    ghost layer filled); returns the coarse Omega (a device tensor)."""
    L = _lib_full()
    om = _zeros(coarse.grid)
    sf, sc = fine.state(), coarse.state()
    mf, mc = fine.mesh(), coarse.mesh()
    check(L.gb_restrict_state(ctx.handle, ctypes.byref(fine.grid.c), ctypes.byref(sf), ctypes.byref(mf),
                              ctypes.byref(coarse.grid.c), ctypes.byref(sc), ctypes.byref(mc), _ptr(om)))
    return om


def face_divergence(ctx, grid, ax, ay, az, J, fx, fy, fz, out=None):
    """gust::face_divergence (Source/Poisson.cpp:733-764)."""
    div = out if out is not None else _zeros(grid)
    check(_lib_full().gb_face_divergence(ctx.handle, ctypes.byref(grid.c), _ptr(ax), _ptr(ay), _ptr(az), _ptr(J),
                                         _ptr(fx), _ptr(fy), _ptr(fz), _ptr(div)))
    return div


class PoissonSolver:
    """gust::PoissonSolver (Source/Poisson.H:135-161) on the GPU: the terrain
    operator with face coefficients, multigrid-preconditioned FGMRES, fluxes.
    z_nd and detJ are kept by reference (the mesh must outlive the solver)."""

    def __init__(self, ctx, grid, z_nd, detJ, bc, options=None):
        self.ctx = ctx
        self.grid = grid
        self._mesh = (z_nd, detJ)
        self.options = options or PoissonOptions.default()
        self._h = ctypes.c_void_p()
        bcs = (ctypes.c_int32 * 6)(*[int(b) for b in bc])
        check(_lib_full().gb_poisson_create(ctx.handle, ctypes.byref(grid.c), bcs, _ptr(z_nd), _ptr(detJ),
                                            ctypes.byref(self.options), ctypes.byref(self._h)))
        ctx.own(self)

    def set_coeffs(self, ax, ay, az, bx=None, by=None, bz=None):
        self._coeffs = (ax, ay, az, bx, by, bz)
        check(_lib_full().gb_poisson_set_coeffs(self._h, _ptr(ax), _ptr(ay), _ptr(az), _ptr(bx), _ptr(by), _ptr(bz)))

    def set_z_cross(self, az, bz, z_cross):
        """FaceCoeffs::z_cross: the split z-face coefficient (None removes it)."""
        self._cross = (az, bz, z_cross)
        check(_lib_full().gb_poisson_set_z_cross(self._h, _ptr(az), _ptr(bz), _ptr(z_cross)))

    def apply(self, phi, out=None):
        y = out if out is not None else _zeros(self.grid)
        check(_lib_full().gb_poisson_apply(self._h, _ptr(phi), _ptr(y)))
        return y

    def vcycle(self, r, out=None):
        e = out if out is not None else _zeros(self.grid)
        check(_lib_full().gb_poisson_vcycle(self._h, _ptr(r), _ptr(e)))
        return e

    def solve(self, rhs, phi):
        res = PoissonResult()
        check(_lib_full().gb_poisson_solve(self._h, _ptr(rhs), _ptr(phi), ctypes.byref(res)))
        return res

    def fluxes(self, phi, bx=None, by=None, bz=None, out=None):
        f = out if out is not None else [_zeros(self.grid) for _ in range(3)]
        check(_lib_full().gb_poisson_fluxes(self._h, _ptr(phi), _ptr(bx), _ptr(by), _ptr(bz), *[_ptr(t) for t in f]))
        return f

    def close(self):
        if self._h:
            check(_lib_full().gb_poisson_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
