"""The terrain-following Poisson layer (Source/Poisson.cpp, extern_erf/
ERF_TerrainPoisson*): mesh, operator, fluxes, ghosts, multigrid, solve.

The oracle is pinned to the reference's gold: the Poisson_Askervein potential
(Tests/Discretization/Poisson_Askervein, gold plotfile) at 1e-8 relative, the
reference's own tolerance for both its back ends (README: "The potential
matches Gold/poisson_askervein_plt00000 at relative 1e-8"), and to its unit
tests' properties (test_Poisson.cpp: OperatorMatchesFluxDivergence :321,
ProjectedFieldIsDivergenceFree :364, SingularProblemRemovesTheMean :514).
GPU tests compare the CUDA operator, fluxes and V-cycle with the oracle.
"""
import numpy as np
import pytest

import oracle
from helpers import (DIRICHLET, NEUMANN, PERIODIC, Grid, askervein_case, rel_err, smooth_terrain_case, to_dev,
                     to_host)


def test_oracle_askervein_matches_reference_gold():
    c = askervein_case()
    g = c["grid"]
    fx, fy, fz = c["U"]
    rhs = oracle.face_divergence(g, c["ax"], c["ay"], c["az"], c["J"], fx, fy, fz)
    div0 = np.sqrt((rhs[g.valid(0)] ** 2).sum())
    assert div0 == pytest.approx(c["info"]["div_before"], rel=1e-9)
    mg = oracle.Multigrid(g, c["bc"], c["z"], c["J"], c["ax"], c["ay"], c["az"])
    phi, it, r0, r1, mean = mg.solve(rhs.copy(), reltol=1e-12, max_iter=200)
    assert it > 0
    gold = c["phi_gold"]
    v = g.valid(0)
    err = np.abs(phi[v] - gold).max() / np.abs(gold).max()
    assert err < 1e-8, err
    # the projected field is divergence free to the solver tolerance
    F = oracle.poisson_fluxes(g, c["bc"], c["z"], phi)
    U1 = [c["U"][d] + F[d] for d in range(3)]
    div1 = oracle.face_divergence(g, c["ax"], c["ay"], c["az"], c["J"], *U1)
    assert np.sqrt((div1[v] ** 2).sum()) < 1e-10 * div0


@pytest.mark.parametrize("per", [(False, False), (True, True), (True, False)])
def test_oracle_operator_matches_flux_divergence(per):
    """A phi = -face_divergence(fluxes(phi)) for beta = 1 (test_Poisson.cpp:321)."""
    g, z, J, ax, ay, az, _ = smooth_terrain_case(12, 10, 8, *per)
    bc = (PERIODIC if per[0] else NEUMANN, PERIODIC if per[1] else NEUMANN, NEUMANN,
          PERIODIC if per[0] else DIRICHLET, PERIODIC if per[1] else NEUMANN, DIRICHLET)
    rng = np.random.default_rng(4)
    phi = g.np_zeros()
    phi[g.valid(0)] = rng.standard_normal(phi[g.valid(0)].shape)
    y = oracle.poisson_apply(g, bc, ax, ay, az, J, z, phi)
    F = oracle.poisson_fluxes(g, bc, z, phi)
    d = oracle.face_divergence(g, ax, ay, az, J, *F)
    v = g.valid(0)
    assert np.abs(y[v] + d[v]).max() < 1e-11 * np.abs(y[v]).max()


def test_oracle_vcycle_contracts_and_solve_converges():
    g, z, J, ax, ay, az, _ = smooth_terrain_case(32, 32, 24, True, True, hill=120.0)
    bc = (PERIODIC, PERIODIC, NEUMANN, PERIODIC, PERIODIC, DIRICHLET)
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az)
    assert mg.levels >= 4
    rng = np.random.default_rng(1)
    b = g.np_zeros()
    b[g.valid(0)] = rng.standard_normal(b[g.valid(0)].shape)
    r = b.copy()
    x = g.np_zeros()
    norms = [np.sqrt((r[g.valid(0)] ** 2).sum())]
    for _ in range(6):
        x += mg.vcycle(r)
        r = b - oracle.poisson_apply(g, bc, ax, ay, az, J, z, x)
        norms.append(np.sqrt((r[g.valid(0)] ** 2).sum()))
    factor = (norms[-1] / norms[0]) ** (1 / 6)
    assert factor < 0.35, norms
    phi, it, r0, r1, _ = mg.solve(b.copy(), reltol=1e-10)
    assert 0 < it <= 15 and r1 <= 1e-10 * r0 * 1.01


def test_oracle_singular_problem_removes_the_mean():
    """Neumann everywhere: the J-weighted mean of rhs is removed and phi has
    zero J-weighted mean (test_Poisson.cpp:514)."""
    g, z, J, ax, ay, az, _ = smooth_terrain_case(16, 16, 12, True, True)
    bc = (PERIODIC, PERIODIC, NEUMANN, PERIODIC, PERIODIC, NEUMANN)
    rng = np.random.default_rng(2)
    b = g.np_zeros()
    b[g.valid(0)] = rng.standard_normal(b[g.valid(0)].shape) + 0.3
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az)
    rhs = b.copy()
    phi, it, r0, r1, mean = mg.solve(rhs, reltol=1e-10)
    assert mean == pytest.approx(oracle.weighted_mean(g, b, J), rel=1e-12)
    assert abs(oracle.weighted_mean(g, phi, J)) < 1e-12 * np.abs(phi).max()
    assert it > 0 and r1 <= 1e-10 * r0 * 1.01


# ------------------------------------------------------------------ GPU parity
def _gpu_case(g, z, J, ax, ay, az):
    import ablsteadyrans_b200 as gb
    return [to_dev(a) for a in (z, J, ax, ay, az)]


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(False, False), (True, True), (True, False)])
def test_gpu_metrics_bit_exact(ctx, per):
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, zcc = smooth_terrain_case(20, 14, 9, *per, hill=150.0)
    out = gb.mesh_metrics(ctx, g, to_dev(z))
    for ref, dev in zip((J, ax, ay, az, zcc), out):
        assert np.array_equal(to_host(dev), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(False, False), (True, True), (False, True)])
def test_gpu_apply_and_fluxes_match_oracle(ctx, per):
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(24, 18, 12, *per, hill=150.0)
    bc = (PERIODIC if per[0] else NEUMANN, PERIODIC if per[1] else NEUMANN, NEUMANN,
          PERIODIC if per[0] else DIRICHLET, PERIODIC if per[1] else DIRICHLET, DIRICHLET)
    rng = np.random.default_rng(9)
    beta = [g.np_zeros() + rng.uniform(0.5, 2.0, g.shape) for _ in range(3)]
    AX, AY, AZ = ax * beta[0], ay * beta[1], az * beta[2]
    phi = g.np_zeros()
    phi[g.valid(0)] = rng.standard_normal(phi[g.valid(0)].shape)
    y_ref = oracle.poisson_apply(g, bc, AX, AY, AZ, J, z, phi.copy())
    F_ref = oracle.poisson_fluxes(g, bc, z, phi.copy(), *beta)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    ps = gb.PoissonSolver(ctx, g, dz, dJ, bc)
    db = [to_dev(b) for b in beta]
    ps.set_coeffs(dax, day, daz, *db)
    y = to_host(ps.apply(to_dev(phi)))
    assert rel_err(y, y_ref, g.valid(0)) < 1e-12
    F = [to_host(f) for f in ps.fluxes(to_dev(phi), *db)]
    for loc, f, fr in zip((1, 2, 4), F, F_ref):
        assert rel_err(f, fr, g.valid(loc)) < 1e-12
    d = to_host(gb.face_divergence(ctx, g, dax, day, daz, dJ, *[to_dev(f) for f in F_ref]))
    d_ref = oracle.face_divergence(g, ax, ay, az, J, *F_ref)
    assert rel_err(d, d_ref, g.valid(0)) < 1e-12
    ps.close()


@pytest.mark.gpu
@pytest.mark.parametrize("solve", [0, 1])
@pytest.mark.parametrize("relax", [0, 4])
@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("per", [(True, True), (False, False), (True, False)])
def test_gpu_vcycle_matches_oracle_fp64(ctx, per, kernel, relax, solve):
    """One V-cycle of the FP64 multigrid agrees with the oracle's to 1e-12,
    with the coarsest level's relaxations in one single-block launch (kernel
    0, the default) and launched one by one (kernel 1), and the zebra
    relaxation as the residual and the column solves in two launches (relax
    0, the default; the column solves segmented, solve 0, or one thread per
    column, solve 1) or as one segmented launch per colour (relax 4)."""
    import ablsteadyrans_b200 as gb
    ctx.tune(gb.TUNE_MG_COARSE_KERNEL, kernel)
    ctx.tune(gb.TUNE_MG_FUSED_RELAX, relax)
    ctx.tune(gb.TUNE_MG_SOLVE, solve)
    g, z, J, ax, ay, az, _ = smooth_terrain_case(32, 24, 16, *per, hill=150.0)
    bc = (PERIODIC if per[0] else NEUMANN, PERIODIC if per[1] else NEUMANN, NEUMANN,
          PERIODIC if per[0] else DIRICHLET, PERIODIC if per[1] else NEUMANN, DIRICHLET)
    rng = np.random.default_rng(3)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az, max_levels=12, min_coarse=2, nu1=1, nu2=1, nu_coarse=8)
    e_ref = mg.vcycle(r)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    opts = gb.PoissonOptions.default(precision=0, nu1=1, nu2=1, nu_coarse=8, max_levels=12, min_coarse=2)
    ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, opts)
    ps.set_coeffs(dax, day, daz)
    e = to_host(ps.vcycle(to_dev(r)))
    ctx.tune(gb.TUNE_MG_COARSE_KERNEL, 0)
    ctx.tune(gb.TUNE_MG_FUSED_RELAX, 0)
    ctx.tune(gb.TUNE_MG_SOLVE, 0)
    ctx.tune(gb.TUNE_MG_TAIL, 0)
    assert rel_err(e, e_ref, g.valid(0)) < 1e-12
    ps.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tail", [1024, 0, 64], ids=["tail-1024-columns", "per-level", "tail-64-columns"])
@pytest.mark.parametrize("case", [(32, 24, 16, False, False), (64, 48, 24, True, False), (40, 32, 70, False, True),
                                  (16, 16, 129, True, True)])
def test_gpu_vcycle_tail_matches_oracle_fp64(ctx, case, tail):
    """The V-cycle's coarse levels as one thread-block-cluster launch
    (GB_TUNE_MG_TAIL N: the levels of at most N columns) agree with the
    oracle's V-cycle to 1e-12, as the per-level launches (0, the default)
    do: the whole hierarchy in the tail, part of it, 16 to 70
    z-levels (one to three levels a lane), and a column of 129 levels,
    which keeps the per-level launches."""
    import ablsteadyrans_b200 as gb
    nx, ny, nz, px, py = case
    g, z, J, ax, ay, az, _ = smooth_terrain_case(nx, ny, nz, px, py, hill=150.0)
    bc = (PERIODIC if px else NEUMANN, PERIODIC if py else NEUMANN, NEUMANN,
          PERIODIC if px else DIRICHLET, PERIODIC if py else NEUMANN, DIRICHLET)
    rng = np.random.default_rng(8)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az, max_levels=12, min_coarse=2, nu1=1, nu2=1, nu_coarse=8)
    e_ref = mg.vcycle(r)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    opts = gb.PoissonOptions.default(precision=0, nu1=1, nu2=1, nu_coarse=8, max_levels=12, min_coarse=2)
    ctx.tune(gb.TUNE_MG_TAIL, tail)
    try:
        ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, opts)
        ps.set_coeffs(dax, day, daz)
        es = [to_host(ps.vcycle(to_dev(r))) for _ in range(2)]
        ps.close()
    finally:
        ctx.tune(gb.TUNE_MG_TAIL, 0)
    for e in es:
        assert rel_err(e, e_ref, g.valid(0)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(True, False), (False, True)])
def test_gpu_vcycle_tail_fp32_tracks_per_level_launches(ctx, per):
    """In FP32 the cluster tail and the per-level launches give the same
    V-cycle to FP32 rounding (1e-5 relative)."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(64, 48, 24, *per, hill=150.0)
    bc = (PERIODIC if per[0] else NEUMANN, PERIODIC if per[1] else NEUMANN, NEUMANN,
          PERIODIC if per[0] else DIRICHLET, PERIODIC if per[1] else DIRICHLET, DIRICHLET)
    rng = np.random.default_rng(9)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    out = []
    try:
        for tail in (1024, 0):
            ctx.tune(gb.TUNE_MG_TAIL, tail)
            dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
            ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(precision=1))
            ps.set_coeffs(dax, day, daz)
            out.append(to_host(ps.vcycle(to_dev(r))))
            ps.close()
    finally:
        ctx.tune(gb.TUNE_MG_TAIL, 0)
    assert rel_err(out[0], out[1], g.valid(0)) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("per", [(True, False), (False, True)])
def test_gpu_coarse_kernel_equals_per_relaxation_launches(ctx, precision, per):
    """The single-block coarsest-level kernel performs the per-relaxation
    launches' arithmetic: a V-cycle on a 64 x 48 x 24 hill (coarsest level
    4 x 3 ... down to the last even split) agrees with the launch-by-launch
    V-cycle to rounding, in FP64 and FP32."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(64, 48, 24, *per, hill=150.0)
    bc = (PERIODIC if per[0] else NEUMANN, PERIODIC if per[1] else NEUMANN, NEUMANN,
          PERIODIC if per[0] else DIRICHLET, PERIODIC if per[1] else DIRICHLET, DIRICHLET)
    rng = np.random.default_rng(4)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    out = []
    for kernel in (0, 1):
        ctx.tune(gb.TUNE_MG_COARSE_KERNEL, kernel)
        dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
        opts = gb.PoissonOptions.default(precision=precision, nu1=1, nu2=1, nu_coarse=8, max_levels=12, min_coarse=2)
        ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, opts)
        ps.set_coeffs(dax, day, daz)
        out.append(to_host(ps.vcycle(to_dev(r))))
        ps.close()
    ctx.tune(gb.TUNE_MG_COARSE_KERNEL, 0)
    ctx.tune(gb.TUNE_MG_TAIL, 0)
    assert rel_err(out[0], out[1], g.valid(0)) < (1e-13 if precision == 0 else 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_askervein_solve_matches_reference_gold(ctx, precision):
    """The GPU solve of the reference's Poisson_Askervein projection matches the
    gold potential at the reference's 1e-8 relative, in FP64 and with the FP32
    multigrid inside the FP64 Krylov solve."""
    import ablsteadyrans_b200 as gb
    c = askervein_case()
    g = c["grid"]
    dz, dJ, dax, day, daz = _gpu_case(g, c["z"], c["J"], c["ax"], c["ay"], c["az"])
    rhs = gb.face_divergence(ctx, g, dax, day, daz, dJ, *[to_dev(u) for u in c["U"]])
    ps = gb.PoissonSolver(ctx, g, dz, dJ, c["bc"], gb.PoissonOptions.default(reltol=1e-12, precision=precision))
    ps.set_coeffs(dax, day, daz)
    phi = to_dev(g.np_zeros())
    res = ps.solve(rhs, phi)
    assert res.iterations > 0 and not res.singular
    assert res.final_residual <= 1e-12 * res.initial_residual * 1.01
    err = np.abs(to_host(phi)[g.valid(0)] - c["phi_gold"]).max() / np.abs(c["phi_gold"]).max()
    assert err < 1e-8, err
    ps.close()


@pytest.mark.gpu
def test_gpu_singular_solve_removes_the_mean(ctx):
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(32, 32, 16, True, True)
    bc = (PERIODIC, PERIODIC, NEUMANN, PERIODIC, PERIODIC, NEUMANN)
    rng = np.random.default_rng(5)
    b = g.np_zeros()
    b[g.valid(0)] = rng.standard_normal(b[g.valid(0)].shape) + 0.25
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az)
    phi_ref, *_ , mean_ref = mg.solve(b.copy(), reltol=1e-12)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(reltol=1e-12))
    ps.set_coeffs(dax, day, daz)
    phi = to_dev(g.np_zeros())
    res = ps.solve(to_dev(b), phi)
    assert res.singular and res.removed_mean == pytest.approx(mean_ref, rel=1e-12)
    assert rel_err(to_host(phi), phi_ref, g.valid(0)) < 1e-9
    ps.close()


@pytest.mark.gpu
def test_gpu_poisson_refusals(ctx):
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(8, 8, 6, True, False)
    dz, dJ = to_dev(z), to_dev(J)
    with pytest.raises(gb.GustError, match="periodic exactly when"):
        gb.PoissonSolver(ctx, g, dz, dJ, (NEUMANN, NEUMANN, NEUMANN, NEUMANN, NEUMANN, NEUMANN))
    with pytest.raises(gb.GustError, match="solver.poisson_reltol"):
        gb.PoissonSolver(ctx, g, dz, dJ, (PERIODIC, NEUMANN, NEUMANN, PERIODIC, NEUMANN, DIRICHLET),
                         gb.PoissonOptions.default(reltol=2.0))


@pytest.mark.gpu
@pytest.mark.parametrize("top", [NEUMANN, DIRICHLET])
def test_gpu_split_operator_fluxes_and_solve_match_oracle(ctx, top):
    """FaceCoeffs::z_cross (beta_h = 1 on x, y and the cross part, beta_z =
    0.25): the GPU operator and fluxes equal the oracle's to 1e-12 relative
    (the top face's cross term counted when the top is not Neumann), and the
    split solve's potential agrees to 1e-9."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(24, 20, 12, False, False, hill=200.0)
    bc = (DIRICHLET, NEUMANN, NEUMANN, DIRICHLET, NEUMANN, top)
    bh = np.ones_like(ax)
    bv = np.full_like(ax, 0.25)
    rng = np.random.default_rng(12)
    phi = g.np_zeros()
    phi[g.valid(0)] = rng.standard_normal(phi[g.valid(0)].shape)
    y_ref = oracle.poisson_apply_split(g, bc, ax, ay, az, J, z, phi.copy(), bh, bh, bv, bh)
    F_ref = oracle.poisson_fluxes_split(g, bc, z, phi.copy(), bh, bh, bv, bh)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    dbh, dbv = to_dev(bh), to_dev(bv)
    ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(reltol=1e-12))
    ps.set_coeffs(dax, day, daz, dbh, dbh, dbv)
    ps.set_z_cross(daz, dbv, dbh)
    y = to_host(ps.apply(to_dev(phi)))
    v = g.valid(0)
    assert np.abs(y[v] - y_ref[v]).max() <= 1e-12 * np.abs(y_ref[v]).max()
    F = [to_host(f) for f in ps.fluxes(to_dev(phi), dbh, dbh, dbv)]
    for d in range(3):
        vf = g.valid(1 << d)
        assert np.abs(F[d][vf] - F_ref[d][vf]).max() <= 1e-12 * np.abs(F_ref[d][vf]).max(), d
    # the split solve against the oracle's
    b = g.np_zeros()
    b[v] = rng.standard_normal(b[v].shape)
    mg = oracle.Multigrid(g, bc, z, J, ax * bh, ay * bh, az * bv)
    mg.set_cross(az, bv, bh)
    phi_ref, it_ref, *_ = mg.solve(b.copy(), reltol=1e-12, max_iter=200)
    assert it_ref > 0
    out = to_dev(g.np_zeros())
    res = ps.solve(to_dev(b), out)
    assert res.final_residual <= 1e-12 * res.initial_residual * 1.01
    got = to_host(out)
    assert np.abs(got[v] - phi_ref[v]).max() <= 1e-9 * np.abs(phi_ref[v]).max()
    # removing the split gives back the plain operator
    ps.set_z_cross(None, None, None)
    y0 = to_host(ps.apply(to_dev(phi)))
    y0_ref = oracle.poisson_apply(g, bc, ax * bh, ay * bh, az * bv, J, z, phi.copy())
    assert np.abs(y0[v] - y0_ref[v]).max() <= 1e-12 * np.abs(y0_ref[v]).max()
    ps.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_vcycle_graph_equals_eager_launches(ctx, precision):
    """From its second call on the V-cycle runs as a CUDA graph captured once
    per solver; it performs the eager launches' kernels in their order, so
    three V-cycles through the graph give the eager V-cycle's result bit for
    bit (GB_TUNE_GRAPHS = 1 runs every kernel alone)."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(64, 48, 24, False, True, hill=150.0)
    bc = (NEUMANN, PERIODIC, NEUMANN, DIRICHLET, PERIODIC, DIRICHLET)
    rng = np.random.default_rng(6)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    out = []
    for graphs in (1, 0):
        ctx.tune(gb.TUNE_GRAPHS, graphs)
        dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
        ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(precision=precision))
        ps.set_coeffs(dax, day, daz)
        es = [to_host(ps.vcycle(to_dev(r))) for _ in range(3)]
        out.append(es)
        ps.close()
    ctx.tune(gb.TUNE_GRAPHS, 0)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", [(64, 48, 24, False, True), (37, 29, 17, True, False), (40, 32, 70, True, True),
                                  (96, 40, 9, False, False)])
def test_gpu_tma_tiles_match_one_thread_per_cell(ctx, case, precision):
    """The operator from TMA-staged tiles (GB_TUNE_MG_STENCIL 2: every
    level) equals the one-thread-per-cell kernels (1) on the apply, one
    V-cycle and the colour residuals inside it: the same values in the same
    operations (1e-13 in FP64, 1e-5 in FP32; the compiler's contractions may
    differ), periodic and mirrored faces, odd extents, 9 to 70 levels."""
    import ablsteadyrans_b200 as gb
    nx, ny, nz, px, py = case
    g, z, J, ax, ay, az, _ = smooth_terrain_case(nx, ny, nz, px, py, hill=150.0)
    bc = (PERIODIC if px else NEUMANN, PERIODIC if py else NEUMANN, NEUMANN,
          PERIODIC if px else DIRICHLET, PERIODIC if py else DIRICHLET, DIRICHLET)
    rng = np.random.default_rng(12)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    phi = g.np_zeros() + rng.standard_normal(g.shape)
    out = []
    try:
        for knob in (1, 2):
            ctx.tune(gb.TUNE_MG_STENCIL, knob)
            dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
            ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(precision=precision))
            ps.set_coeffs(dax, day, daz)
            y = to_host(ps.apply(to_dev(phi)))
            e = to_host(ps.vcycle(to_dev(r)))
            e2 = to_host(ps.vcycle(to_dev(r)))
            out.append((y, e, e2))
            ps.close()
    finally:
        ctx.tune(gb.TUNE_MG_STENCIL, 0)
    v = g.valid(0)
    tol = 1e-13 if precision == 0 else 1e-5
    assert rel_err(out[1][0], out[0][0], v) < 1e-13
    assert rel_err(out[1][1], out[0][1], v) < tol
    assert rel_err(out[1][2], out[0][2], v) < tol


@pytest.mark.gpu
def test_gpu_tma_tiles_solve_matches_oracle(ctx):
    """A full FP64 Poisson solve (FGMRES with the V-cycle) with the tiles on
    every level meets the oracle's solution of the same system to 1e-9."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, _ = smooth_terrain_case(64, 48, 24, False, True, hill=150.0)
    bc = (NEUMANN, PERIODIC, NEUMANN, DIRICHLET, PERIODIC, DIRICHLET)
    rng = np.random.default_rng(13)
    rhs = g.np_zeros()
    rhs[g.valid(0)] = rng.standard_normal(rhs[g.valid(0)].shape)
    dz, dJ, dax, day, daz = _gpu_case(g, z, J, ax, ay, az)
    ctx.tune(gb.TUNE_MG_STENCIL, 2)
    try:
        ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, gb.PoissonOptions.default(precision=0, reltol=1e-12))
        ps.set_coeffs(dax, day, daz)
        phi = to_dev(g.np_zeros())
        ps.solve(to_dev(rhs), phi)
        got = to_host(phi)
        ps.close()
    finally:
        ctx.tune(gb.TUNE_MG_STENCIL, 0)
    y_ref = oracle.poisson_apply(g, bc, ax, ay, az, J, z, got.copy())
    v = g.valid(0)
    assert np.abs(y_ref[v] - rhs[v]).max() <= 1e-9 * np.abs(rhs[v]).max()
