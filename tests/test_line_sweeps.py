"""z-line relaxation (gust::zline_jacobi, Source/Predictor.cpp:87-127; column
kernel Source/LineSolve_K.H:22-45).

CPU tests pin the oracle to the reference's own known answers
(test_Predictor.cpp:378-442: the sweeps converge to the dense solve, the error
falls with the sweep count; test_LineSweeps.cpp: M-matrix systems at every
location, periodic seams). GPU tests compare the CUDA path through the C ABI
with the oracle on the same seeded systems: FP64 to 1e-12 relative (one
sweep and several), FP32 to 2e-5 relative.
"""
import numpy as np
import pytest

import oracle
from helpers import LOCS, Grid, dense_line_system_solve, random_system, rel_err, to_dev, to_host

CASES = [
    # nx, ny, nz, periodic_x, periodic_y
    (5, 4, 6, False, False),
    (6, 5, 7, True, True),
    (4, 7, 5, True, False),
    (1, 1, 12, True, True),
]


@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("case", CASES)
def test_oracle_converges_to_dense_solve(loc, case):
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=7 + loc, extra=0.3)
    exact = dense_line_system_solve(g, loc, A, ap, rhs)
    scale = np.abs(exact).max()
    v = g.valid(loc)
    # the error falls with the sweeps (every 4 sweeps in the max norm: a random
    # M-matrix's Jacobi error need not fall at every single sweep)
    prev = np.inf
    for sweeps in (1, 4, 16):
        d = g.np_zeros()
        oracle.zline_jacobi(g, loc, A, ap, rhs, sweeps, d)
        err = np.abs(d - exact)[v].max() / scale
        if prev > 1e-14:
            assert err < prev, (sweeps, err, prev)
        prev = err
    d = g.np_zeros()
    change = oracle.zline_jacobi(g, loc, A, ap, rhs, 400, d)
    assert np.abs(d - exact)[v].max() / scale < 1e-12
    assert change / scale < 1e-12
    # the ghosts below the ground and above the top stay 0
    assert np.all(d[: g.ng] == 0) and np.all(d[g.ng + g.extents(loc)[2]:] == 0)


def test_oracle_single_sweep_is_the_column_solve():
    """One sweep from delta = 0 is the exact tridiagonal solve of each column."""
    g = Grid(3, 2, 9, 25.0, 25.0, 5.0, False, False)
    A, ap, rhs = random_system(g, 0, seed=3)
    d = g.np_zeros()
    change = oracle.zline_jacobi(g, 0, A, ap, rhs, 1, d)
    G = g.ng
    for j in range(2):
        for i in range(3):
            nk = 9
            M = np.zeros((nk, nk))
            for k in range(nk):
                M[k, k] = ap[k + G, j + G, i + G]
                if k > 0:
                    M[k, k - 1] = -A[5, k + G, j + G, i + G]
                if k < nk - 1:
                    M[k, k + 1] = -A[6, k + G, j + G, i + G]
            x = np.linalg.solve(M, rhs[G:G + nk, j + G, i + G])
            np.testing.assert_allclose(d[G:G + nk, j + G, i + G], x, rtol=1e-13, atol=1e-14)
    assert change == pytest.approx(np.abs(d).max(), rel=0, abs=0)


@pytest.mark.gpu
@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("case", CASES + [(37, 29, 17, True, False), (64, 48, 48, False, True)])
@pytest.mark.parametrize("sweeps", [1, 2, 5])
def test_gpu_zline_jacobi_matches_oracle_fp64(ctx, loc, case, sweeps):
    import torch
    import ablsteadyrans_b200 as gb
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=11 + 3 * loc + sweeps, extra=0.2, xscale=3.0)
    d_ref = g.np_zeros()
    ch_ref = oracle.zline_jacobi(g, loc, A, ap, rhs, sweeps, d_ref)
    dA, dap, drhs = to_dev(A), to_dev(ap), to_dev(rhs)
    dd = torch.full(g.shape, 7.0, dtype=torch.float64, device="cuda")  # overwritten: delta starts at 0
    ch = gb.zline_jacobi(ctx, g, loc, dA, dap, drhs, sweeps, dd)
    d = to_host(dd)
    assert rel_err(d, d_ref, g.valid(loc)) < 1e-12
    assert abs(ch - ch_ref) <= 1e-12 * max(abs(ch_ref), 1e-300)
    # ghosts outside the domain are 0
    G = g.ng
    assert np.all(d[:G] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("variant,segment,first", [(4, 0, 0), (5, 4, 0), (5, 5, 0), (5, 8, 0), (6, 8, 0), (6, 5, 0),
                                                    (5, 8, 2), (6, 4, 2)],
                         ids=["factored", "segmented4", "segmented5", "segmented8", "split8", "split5", "hybrid8",
                              "hybrid-split4"])
@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("case", [(37, 29, 17, True, False), (64, 48, 65, False, True), (33, 20, 128, True, True)])
def test_gpu_zline_jacobi_kernels_match_oracle(ctx, variant, segment, first, loc, case):
    """The sequential factored sweep (GB_TUNE_LINE_VARIANT 4), the segmented
    one with 4, 5 or 8 levels per warp (5, the default), the segmented one
    with the later sweeps split into the fold and the column solves (6),
    and either segmented form after a first sweep (the factorisation) by the
    factored kernel (GB_TUNE_LINE_FIRST 2) agree with the oracle's column
    solves to 1e-12, on columns of 17 to 129 levels."""
    import torch
    import ablsteadyrans_b200 as gb
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=5 + loc, extra=0.2, xscale=3.0)
    d_ref = g.np_zeros()
    ch_ref = oracle.zline_jacobi(g, loc, A, ap, rhs, 3, d_ref)
    ctx.tune(gb.TUNE_LINE_VARIANT, variant)
    ctx.tune(gb.TUNE_LINE_SEGMENT, segment)
    ctx.tune(gb.TUNE_LINE_FIRST, first)
    try:
        dd = torch.full(g.shape, 7.0, dtype=torch.float64, device="cuda")
        ch = gb.zline_jacobi(ctx, g, loc, to_dev(A), to_dev(ap), to_dev(rhs), 3, dd)
    finally:
        ctx.tune(gb.TUNE_LINE_VARIANT, 0)
        ctx.tune(gb.TUNE_LINE_SEGMENT, 0)
        ctx.tune(gb.TUNE_LINE_FIRST, 0)
    assert rel_err(to_host(dd), d_ref, g.valid(loc)) < 1e-12
    assert abs(ch - ch_ref) <= 1e-12 * max(abs(ch_ref), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("loc", LOCS)
def test_gpu_zline_jacobi_fp32(ctx, loc):
    import torch
    import ablsteadyrans_b200 as gb
    g = Grid(40, 33, 24, 30.0, 30.0, 10.0, True, False)
    A, ap, rhs = random_system(g, loc, seed=99 + loc, extra=0.5)
    d_ref = g.np_zeros()
    oracle.zline_jacobi(g, loc, A, ap, rhs, 3, d_ref)
    dd = torch.zeros(g.shape, dtype=torch.float32, device="cuda")
    gb.zline_jacobi(ctx, g, loc, to_dev(A, torch.float32), to_dev(ap, torch.float32), to_dev(rhs, torch.float32), 3, dd)
    assert rel_err(to_host(dd), d_ref, g.valid(loc)) < 2e-5


BATCH = [
    # nx, ny, nz, periodic_x, periodic_y, loc: uneven tiles, columns of 6 to 97
    # levels (several warps-a-block groups), periodic seams
    (37, 29, 17, True, False, 1),
    (64, 48, 48, False, True, 0),
    (5, 4, 6, False, False, 4),
    (33, 20, 96, True, True, 4),
    (40, 33, 64, False, False, 2),
    (1, 1, 12, True, True, 0),
    (24, 24, 48, False, False, 4),
]


def _batch_case(dtype, segment, seed0):
    import torch
    import ablsteadyrans_b200 as gb
    systems, refs = [], []
    for q, (nx, ny, nz, px, py, loc) in enumerate(BATCH):
        g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
        A, ap, rhs = random_system(g, loc, seed=seed0 + q, extra=0.2, xscale=3.0)
        dA, dap, drhs = to_dev(A, dtype), to_dev(ap, dtype), to_dev(rhs, dtype)
        dd = torch.full(g.shape, 7.0, dtype=dtype, device="cuda")  # overwritten: delta starts at 0
        systems.append((g, loc, dA, dap, drhs, dd))
        refs.append((g, loc, A, ap, rhs))
    return gb, systems, refs


@pytest.mark.gpu
@pytest.mark.parametrize("segment", [0, 4, 8])
@pytest.mark.parametrize("sweeps", [1, 3])
def test_gpu_zline_jacobi_batch_equals_single_systems(ctx, segment, sweeps):
    """The batched solve (one column work-list over uneven systems, one
    persistent launch per sweep and warps-a-block group) gives every system
    the values of gb_zline_jacobi on that system alone, bit for bit (the same
    segmented column solves; a block's warps above a column's top are
    identity maps), in FP64 and FP32, with each system's max |change|; the
    FP64 values are within 1e-12 of the oracle's."""
    import torch
    import ablsteadyrans_b200 as gb
    ctx.tune(gb.TUNE_LINE_SEGMENT, segment)
    try:
        for dtype in (torch.float64, torch.float32):
            gb, systems, refs = _batch_case(dtype, segment, 300 + sweeps)
            changes = gb.zline_jacobi_batch(ctx, systems, sweeps)
            for (g, loc, dA, dap, drhs, dd), (_, _, A, ap, rhs), ch in zip(systems, refs, changes):
                alone = torch.full(g.shape, -3.0, dtype=dtype, device="cuda")
                ch1 = gb.zline_jacobi(ctx, g, loc, dA, dap, drhs, sweeps, alone)
                assert torch.equal(dd, alone), (g.nx, g.ny, g.nz, loc)
                assert ch == pytest.approx(ch1, rel=1e-7 if dtype == torch.float32 else 0.0, abs=0.0)
                if dtype == torch.float64:
                    d_ref = g.np_zeros()
                    ch_ref = oracle.zline_jacobi(g, loc, A, ap, rhs, sweeps, d_ref)
                    assert rel_err(to_host(dd), d_ref, g.valid(loc)) < 1e-12
                    assert abs(ch - ch_ref) <= 1e-12 * max(abs(ch_ref), 1e-300)
    finally:
        ctx.tune(gb.TUNE_LINE_SEGMENT, 0)


@pytest.mark.gpu
def test_gpu_zline_jacobi_batch_repeat_and_refusals(ctx):
    """A second batched call on the same context (the scratch and work-list
    reused) gives the same values; a system whose columns are taller than
    the segmented sweep holds, and a bad sweep count, are refused."""
    import torch
    gb, systems, _ = _batch_case(torch.float64, 0, 500)
    gb.zline_jacobi_batch(ctx, systems, 2, want_change=False)
    first = [s[5].clone() for s in systems]
    gb.zline_jacobi_batch(ctx, systems, 2)
    for a, s in zip(first, systems):
        assert torch.equal(a, s[5])
    with pytest.raises(gb.GustError, match="sweeps must be >= 1"):
        gb.zline_jacobi_batch(ctx, systems, 0)
    with pytest.raises(gb.GustError, match="n must be >= 1"):
        gb.zline_jacobi_batch(ctx, [], 1)
    tall = Grid(2, 2, 400, 1.0, 1.0, 1.0)
    z = torch.zeros((7,) + tall.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(gb.GustError, match="z-levels"):
        gb.zline_jacobi_batch(ctx, [(tall, 0, z, z[0], z[0], z[1])], 1)


@pytest.mark.gpu
def test_gpu_zline_jacobi_batch_many_small_systems(ctx):
    """More systems than one launch's parameter block holds (120): 130 small
    uneven systems (1 to 5 columns a side, 3 to 14 levels, every location,
    periodic seams) split over several launches per sweep, each system's
    values still bit for bit those of gb_zline_jacobi alone."""
    import torch
    import ablsteadyrans_b200 as gb
    rng = np.random.default_rng(77)
    systems = []
    for q in range(130):
        nx, ny, nz = (int(v) for v in rng.integers((1, 1, 3), (6, 6, 15)))
        px, py = bool(rng.integers(2)), bool(rng.integers(2))
        loc = int(rng.choice(LOCS))
        g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
        A, ap, rhs = random_system(g, loc, seed=900 + q, extra=0.2, xscale=3.0)
        systems.append((g, loc, to_dev(A), to_dev(ap), to_dev(rhs),
                        torch.full(g.shape, 5.0, dtype=torch.float64, device="cuda")))
    changes = gb.zline_jacobi_batch(ctx, systems, 3)
    for (g, loc, dA, dap, drhs, dd), ch in zip(systems, changes):
        alone = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
        assert gb.zline_jacobi(ctx, g, loc, dA, dap, drhs, 3, alone) == ch
        assert torch.equal(dd, alone), (g.nx, g.ny, g.nz, loc)


@pytest.mark.gpu
def test_gpu_zline_jacobi_refusals(ctx):
    import torch
    import ablsteadyrans_b200 as gb
    g = Grid(4, 4, 4, 1.0, 1.0, 1.0)
    z = torch.zeros((7,) + g.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(gb.GustError, match="sweeps must be >= 1"):
        gb.zline_jacobi(ctx, g, 0, z, z[0], z[0], 0, z[1])
    with pytest.raises(gb.GustError, match="loc must be"):
        gb.zline_jacobi(ctx, g, 3, z, z[0], z[0], 1, z[1])


# ------------------------------------------------------------------ LU-SGS
# gust::zline_lusgs (Source/LineSweeps.cpp:38-428) with line_ghosts = lagged.

@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("alternate", [0, 1])
@pytest.mark.parametrize("case", CASES)
def test_oracle_lusgs_diagonal_equals_sequential(loc, alternate, case):
    """The wavefront order performs the sequential order's operations on the
    same values: bit-identical results (the reference's
    LineSweeps.DiagonalOrderingEqualsTheSequentialSweep, test_LineSweeps.cpp:483)."""
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=21 + loc, extra=0.3)
    d0, d1 = g.np_zeros(), g.np_zeros()
    c0 = oracle.zline_lusgs(g, loc, A, ap, rhs, 3, d0, order=0, alternate=alternate)
    c1 = oracle.zline_lusgs(g, loc, A, ap, rhs, 3, d1, order=1, alternate=alternate)
    assert np.array_equal(d0, d1) and c0 == c1


@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("case", CASES)
def test_oracle_lusgs_converges_to_dense_solve(loc, case):
    """Symmetric line Gauss-Seidel converges to the same system's dense solve,
    in fewer sweeps than the z-line Jacobi iteration."""
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=7 + loc, extra=0.3)
    exact = dense_line_system_solve(g, loc, A, ap, rhs)
    scale = np.abs(exact).max()
    v = g.valid(loc)
    d = g.np_zeros()
    change = oracle.zline_lusgs(g, loc, A, ap, rhs, 200, d)
    assert np.abs(d - exact)[v].max() / scale < 1e-12
    assert change / scale < 1e-12
    dl, dj = g.np_zeros(), g.np_zeros()
    oracle.zline_lusgs(g, loc, A, ap, rhs, 4, dl)
    oracle.zline_jacobi(g, loc, A, ap, rhs, 8, dj)
    assert np.abs(dl - exact)[v].max() <= np.abs(dj - exact)[v].max() * (1 + 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("loc", LOCS)
@pytest.mark.parametrize("case", CASES + [(37, 29, 17, True, False), (24, 40, 33, False, True)])
@pytest.mark.parametrize("alternate", [0, 1])
def test_gpu_zline_lusgs_matches_oracle(ctx, loc, case, alternate):
    import torch
    import ablsteadyrans_b200 as gb
    nx, ny, nz, px, py = case
    g = Grid(nx, ny, nz, 30.0, 30.0, 10.0, px, py)
    A, ap, rhs = random_system(g, loc, seed=31 + 3 * loc + alternate, extra=0.2, xscale=3.0)
    d_ref = g.np_zeros()
    ch_ref = oracle.zline_lusgs(g, loc, A, ap, rhs, 3, d_ref, alternate=alternate)
    dd = torch.full(g.shape, 7.0, dtype=torch.float64, device="cuda")  # overwritten: delta starts at 0
    ch = gb.zline_lusgs(ctx, g, loc, to_dev(A), to_dev(ap), to_dev(rhs), 3, dd, alternate=alternate)
    d = to_host(dd)
    assert rel_err(d, d_ref, g.valid(loc)) < 1e-12
    assert abs(ch - ch_ref) <= 1e-11 * max(abs(ch_ref), 1e-300)
    G = g.ng
    assert np.all(d[:G] == 0)


@pytest.mark.gpu
def test_gpu_zline_lusgs_refusals(ctx):
    import torch
    import ablsteadyrans_b200 as gb
    g = Grid(4, 4, 4, 1.0, 1.0, 1.0)
    z = torch.zeros((7,) + g.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(gb.GustError, match="sweeps must be >= 1"):
        gb.zline_lusgs(ctx, g, 0, z, z[0], z[0], 0, z[1])
    with pytest.raises(gb.GustError, match="steady.line_alternate = 2"):
        gb.zline_lusgs(ctx, g, 0, z, z[0], z[0], 1, z[1], alternate=2)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_batched_sweep_back_substitution_placement_is_bitwise_neutral(ctx, precision):
    """The batched factored sweeps keep c' and e' for the back substitution in
    shared memory (TUNE_LINE_BACK = 1), in the global arrays (2), or e' in
    shared memory with c' read again (3): the same arithmetic in the same
    order, so three SIMPLEC iterations (u, v, w and theta, k swept in batched
    launches) give identical fields."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200 import workloads
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    out = []
    ctx.tune(gb.TUNE_LINE_VARIANT, 4)   # the factored kernel, where the placement applies
    for back in (1, 2, 3):
        inst = workloads.tile(40, 24, 3, precision=precision)
        ctx.tune(gb.TUNE_LINE_BACK, back)
        J, ax, ay, az, _ = oracle.metrics(inst.grid, inst.z)
        dc = DeviceCase(inst.grid, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
        st = SimplecStage(ctx, dc, inst.bc, inst.physics, inst.options)
        st.fill_ghosts()
        for _ in range(3):
            st.iterate(st.local_dtau(2.0))
        out.append({f: dc.host(f) for f in ("u", "v", "w", "p", "theta", "tke")})
        st.close()
    ctx.tune(gb.TUNE_LINE_BACK, 0)
    ctx.tune(gb.TUNE_LINE_VARIANT, 0)
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f
        assert np.array_equal(out[0][f], out[2][f]), f


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_fused_zebra_relaxation_is_bitwise_neutral(ctx, precision):
    """The multigrid's zebra relaxation as one launch per colour (the
    residual kept in shared memory) or as the residual and the sequential
    column solve (GB_TUNE_MG_SOLVE 1) in two launches: the same arithmetic
    in the same order, so three SIMPLEC iterations give identical fields.
    (The default segmented column solve carries e' and x across segments
    and is held to the oracle's V-cycle with a tolerance instead.)"""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200 import workloads
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    out = []
    for mode in (2, 1):
        inst = workloads.tile(40, 24, 3, precision=precision)
        ctx.tune(gb.TUNE_MG_FUSED_RELAX, mode)
        ctx.tune(gb.TUNE_MG_SOLVE, 1)
        J, ax, ay, az, _ = oracle.metrics(inst.grid, inst.z)
        dc = DeviceCase(inst.grid, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
        st = SimplecStage(ctx, dc, inst.bc, inst.physics, inst.options)
        st.fill_ghosts()
        for _ in range(3):
            st.iterate(st.local_dtau(2.0))
        out.append({f: dc.host(f) for f in ("u", "v", "w", "p", "theta", "tke")})
        st.close()
    ctx.tune(gb.TUNE_MG_FUSED_RELAX, 0)
    ctx.tune(gb.TUNE_MG_SOLVE, 0)
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f
