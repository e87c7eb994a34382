"""The allocation-free z-line solve (gb_zline_jacobi_noalloc): the same
results as gb_zline_jacobi through a context, on two calls in a row that
share the library's fixed scratch array; oversize grids are refused before
any device work. This file is collected last so that it also runs after the
rest of the suite has used the device."""
import ctypes

import numpy as np
import pytest

import ablsteadyrans_b200 as gb
from helpers import LOC_CELL, LOC_XFACE, LOC_ZFACE, Grid, random_system, rel_err, to_dev, to_host

GB_BAD_ARG = 1


def test_refuses_grids_beyond_the_fixed_scratch():
    L = gb.lib()
    big = Grid(160, 160, 80, 10.0, 10.0, 5.0, True, True)  # 165 * 165 * 85 > 2^21 points
    st = L.gb_zline_jacobi_noalloc(ctypes.byref(big.c), LOC_CELL, None, None, None, 2, None, None, None)
    assert st == GB_BAD_ARG
    # The pointer check comes first; with pointers the size check speaks.
    fake = ctypes.c_void_p(256)
    st = L.gb_zline_jacobi_noalloc(ctypes.byref(big.c), LOC_CELL, fake, fake, fake, 2, fake, None, None)
    assert st == GB_BAD_ARG
    assert b"more than the fixed scratch" in L.gb_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("loc,periodic", [(LOC_CELL, (True, True)), (LOC_XFACE, (True, False)),
                                          (LOC_ZFACE, (False, True))])
def test_noalloc_matches_context_path_twice(ctx, loc, periodic):
    import torch
    grid = Grid(40, 24, 20, 10.0, 12.0, 4.0, *periodic)
    A, ap, rhs = random_system(grid, loc, seed=11 + loc)
    dA, dap, drhs = to_dev(A), to_dev(ap), to_dev(rhs)
    ref = torch.empty_like(drhs)
    ch_ref = gb.zline_jacobi(ctx, grid, loc, dA, dap, drhs, 3, ref)
    v = grid.valid(loc)
    expect = to_host(ref)
    for _ in range(2):
        out = torch.full_like(drhs, np.nan)  # every point is written: the solve zeroes delta first
        ch = gb.zline_jacobi_noalloc(grid, loc, dA, dap, drhs, 3, out)
        got = to_host(out)
        assert np.isfinite(got).all()
        assert rel_err(got, expect, v) <= 1e-12
        assert np.abs(got - expect).max() <= 1e-12 * max(np.abs(expect).max(), 1.0)
        assert abs(ch - ch_ref) <= 1e-12 * max(abs(ch_ref), 1e-300)


@pytest.mark.gpu
def test_noalloc_on_a_side_stream(ctx):
    import torch
    grid = Grid(33, 17, 12, 10.0, 10.0, 3.0, False, False)
    A, ap, rhs = random_system(grid, LOC_CELL, seed=5)
    dA, dap, drhs = to_dev(A), to_dev(ap), to_dev(rhs)
    ref = torch.empty_like(drhs)
    gb.zline_jacobi(ctx, grid, LOC_CELL, dA, dap, drhs, 2, ref)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    out = torch.empty_like(drhs)
    with torch.cuda.stream(side):
        gb.zline_jacobi_noalloc(grid, LOC_CELL, dA, dap, drhs, 2, out, stream=side)
        gb.zline_jacobi_noalloc(grid, LOC_CELL, dA, dap, drhs, 2, out, stream=side)
    side.synchronize()
    assert rel_err(to_host(out), to_host(ref), grid.valid(LOC_CELL)) <= 1e-12
