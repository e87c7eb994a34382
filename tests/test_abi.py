"""The C ABI boundary (include/gust_b200.h): the built library loads without a
GPU and exports every function the header declares; host-only entry points
(grid descriptors, error reporting) work on the CPU; the oracle library loads."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gust_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("gb_zline_jacobi", "gb_poisson_solve", "gb_poisson_apply", "gb_mesh_metrics", "gb_ctx_create"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import ablsteadyrans_b200 as gb
    L = gb.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_grid_init_and_errors_on_the_host():
    import ablsteadyrans_b200 as gb
    L = gb.lib()
    g = gb.GbGrid()
    assert L.gb_grid_init(ctypes.byref(g), 16, 8, 12, 2, 30.0, 30.0, 10.0, 1, 0) == 0
    assert g.sy == 16 + 1 + 4 and g.sz == g.sy * (8 + 1 + 4)
    assert L.gb_grid_volume(ctypes.byref(g)) == g.sz * (12 + 1 + 4)
    py = gb.Grid(16, 8, 12, 30.0, 30.0, 10.0, True, False)
    assert (py.c.sy, py.c.sz) == (g.sy, g.sz)
    bad = gb.GbGrid()
    st = L.gb_grid_init(ctypes.byref(bad), 0, 8, 12, 2, 30.0, 30.0, 10.0, 0, 0)
    assert st == 1
    assert b"grid needs nx, ny >= 1" in L.gb_last_error()


def test_oracle_library_loads():
    import oracle
    assert oracle.max_threads() >= 1
