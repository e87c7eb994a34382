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

from .grid import Grid, GbGrid, LOC_CELL, LOC_XFACE, LOC_YFACE, LOC_ZFACE, LOC_NODE, N_COEFS  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgustb200.so")
_lib = None

GB_OK = 0
KERNEL_LINE_SWEEP, KERNEL_POISSON_APPLY, KERNEL_MG_SMOOTH, KERNEL_MG_TRANSFER, KERNEL_RESIDUAL, \
    KERNEL_MASSFLUX, KERNEL_COEFS, KERNEL_VECTOR, KERNEL_BC = range(9)
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
    L.gb_ctx_profile.argtypes = [P, i32]
    L.gb_ctx_profile_read.argtypes = [P, i32, ctypes.POINTER(f64), ctypes.POINTER(i64)]
    L.gb_zline_jacobi.argtypes = [P, G, i32, P, P, P, i32, P, ctypes.POINTER(f64)]
    L.gb_zline_jacobi_f32.argtypes = [P, G, i32, P, P, P, i32, P, ctypes.POINTER(ctypes.c_float)]


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
        check(lib().gb_ctx_create(ctypes.c_void_p(stream.cuda_stream), ctypes.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def launches(self):
        return int(lib().gb_ctx_launches(self._h))

    def profile(self, enable):
        check(lib().gb_ctx_profile(self._h, int(bool(enable))))

    def profile_read(self, family):
        """(total milliseconds, launches) of one kernel family since profile(True)."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        check(lib().gb_ctx_profile_read(self._h, int(family), ctypes.byref(t), ctypes.byref(n)))
        return float(t.value), int(n.value)

    def close(self):
        if self._h:
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
