"""ORACLE -- test infrastructure, not product code.

ctypes bindings of liboracle.so, the FP64 C restatement of the reference's
SIMPLEC hot path (gust_oracle.c). Only the tests, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, as the checker; the product path never
calls it. Arrays are numpy float64, C-contiguous, in the grid layout of
include/gust_b200.h (ablsteadyrans_b200.grid.Grid.shape).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force=False):
    args = ["make", "-C", HERE]
    if force:
        args.append("-B")
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout.decode(errors="replace"))
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    from ablsteadyrans_b200.grid import GbGrid
    G = ctypes.POINTER(GbGrid)
    P = ctypes.c_void_p
    i32, f64 = ctypes.c_int32, ctypes.c_double
    L.og_set_threads.argtypes = [i32]
    L.og_max_threads.restype = i32
    L.og_fill_periodic.argtypes = [G, i32, P, i32]
    L.og_override_sync.argtypes = [G, i32, P]
    L.og_zline_jacobi.argtypes = [G, i32, P, P, P, i32, P]
    L.og_zline_jacobi.restype = f64


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous float64"
    return ctypes.c_void_p(a.ctypes.data)


def set_threads(n):
    lib().og_set_threads(int(n))


def max_threads():
    return int(lib().og_max_threads())


def fill_periodic(grid, loc, f, layers=1):
    lib().og_fill_periodic(ctypes.byref(grid.c), loc, _p(f), layers)


def zline_jacobi(grid, loc, A, ap, rhs, sweeps, delta):
    """Source/Predictor.cpp:87-127 restated; returns the last sweep's change."""
    return float(lib().og_zline_jacobi(ctypes.byref(grid.c), loc, _p(A), _p(ap), _p(rhs), int(sweeps), _p(delta)))
