"""Tucker's differential wall distance (Source/WallDistance.cpp:78-94,
turb.wall_distance = tucker) and the terrain Poisson problem it solves, with
phi = 0 on the ground (tucker_bc, Source/WallDistance.cpp:65-76).

Over flat ground the Poisson solution is phi = H z - z^2 / 2 and Tucker's
formula returns the height above the ground exactly, so the oracle's
discrete distance is pinned to the height (the discretisation error of the
stretched mesh, 3e-3 relative). The GPU's Dirichlet-ground operator, V-cycle
and solve, its wall distance, and a closure residual that reads that distance
are compared with the oracle.
"""
import numpy as np
import pytest

import oracle
from helpers import rel_err, smooth_terrain_case, to_dev, to_host


def _height_above_ground(g, zcc, z):
    """Cell-centre height above the column's ground (the mean of the four
    ground nodes of the column)."""
    G = g.ng
    zg = 0.25 * (z[G, G:G + g.ny, G:G + g.nx] + z[G, G:G + g.ny, G + 1:G + g.nx + 1]
                 + z[G, G + 1:G + g.ny + 1, G:G + g.nx] + z[G, G + 1:G + g.ny + 1, G + 1:G + g.nx + 1])
    return zcc[G:G + g.nz, G:G + g.ny, G:G + g.nx] - zg[None]


def _cells(g, a):
    G = g.ng
    return a[G:G + g.nz, G:G + g.ny, G:G + g.nx]


@pytest.mark.parametrize("per", [(True, True), (False, False)])
def test_oracle_flat_ground_distance_is_the_height(per):
    g, z, J, ax, ay, az, zcc = smooth_terrain_case(12, 10, 24, *per, hill=0.0)
    d, it = oracle.tucker_wall_distance(g, z)
    h = _height_above_ground(g, zcc, z)
    assert it < 40
    assert np.abs(_cells(g, d) - h).max() <= 3e-3 * h.max()
    assert np.all(np.abs(_cells(g, d) - h) <= 3e-3 * h + 1e-9 * h.max())


def test_oracle_hill_distance_properties():
    """Over a hill: the distance is positive, grows up every column, is
    mirror-symmetric about the summit as the terrain is, and stays near the
    height above the ground (Tucker's local one-dimensional model
    overestimates above the convex summit: by up to 18 % on this mesh)."""
    g, z, J, ax, ay, az, zcc = smooth_terrain_case(16, 12, 16, False, True, hill=150.0)
    d, _ = oracle.tucker_wall_distance(g, z, reltol=1e-13)
    h = _height_above_ground(g, zcc, z)
    dc = _cells(g, d)
    assert np.all(dc > 0.0)
    assert np.all(np.diff(dc, axis=0) > 0.0)
    assert np.abs(dc - dc[:, :, ::-1]).max() <= 1e-9 * dc.max()
    assert np.abs(dc - dc[:, ::-1, :]).max() <= 1e-9 * dc.max()
    assert np.all(np.abs(dc / h - 1.0) < 0.2)


def _tucker_case(per, hill=150.0):
    g, z, J, ax, ay, az, zcc = smooth_terrain_case(24, 16, 12, *per, hill=hill)
    return g, z, J, ax, ay, az, oracle.tucker_bc(g)


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(True, True), (False, False), (True, False)])
def test_gpu_dirichlet_ground_apply_and_vcycle_match_oracle(ctx, per):
    """With phi = 0 on the ground (the odd ghost and ERF's one-sided ground
    flux), the GPU operator and one FP64 V-cycle equal the oracle's to
    1e-12."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, bc = _tucker_case(per)
    rng = np.random.default_rng(5)
    phi = g.np_zeros()
    phi[g.valid(0)] = rng.standard_normal(phi[g.valid(0)].shape)
    y_ref = oracle.poisson_apply(g, bc, ax, ay, az, J, z, phi.copy())
    mg = oracle.Multigrid(g, bc, z, J, ax, ay, az, max_levels=12, min_coarse=2, nu1=1, nu2=1, nu_coarse=8)
    e_ref = mg.vcycle(phi)
    mg.close()
    dz, dJ, dax, day, daz = [to_dev(a) for a in (z, J, ax, ay, az)]
    opts = gb.PoissonOptions.default(precision=0, nu1=1, nu2=1, nu_coarse=8, max_levels=12, min_coarse=2)
    ps = gb.PoissonSolver(ctx, g, dz, dJ, bc, opts)
    ps.set_coeffs(dax, day, daz)
    y = to_host(ps.apply(to_dev(phi)))
    e = to_host(ps.vcycle(to_dev(phi)))
    ps.close()
    assert rel_err(y, y_ref, g.valid(0)) < 1e-12
    assert rel_err(e, e_ref, g.valid(0)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(True, True), (False, False), (False, True)])
def test_gpu_tucker_wall_distance_matches_oracle(ctx, per):
    """gb_tucker_wall_distance over a hill: the distance on every cell and
    every ghost equals the oracle's (both Poisson solves converged to 1e-12
    relative; 1e-9 relative on the distance)."""
    import ablsteadyrans_b200 as gb
    g, z, J, ax, ay, az, bc = _tucker_case(per)
    d_ref, _ = oracle.tucker_wall_distance(g, z, reltol=1e-13)
    G = g.ng
    opts = gb.PoissonOptions.default(reltol=1e-13, abstol=0.0, max_iter=200)
    d, res = gb.tucker_wall_distance(ctx, g, to_dev(z), opts)
    d = to_host(d)
    assert res.iterations < 60
    scale = np.abs(d_ref).max()
    assert np.abs(_cells(g, d) - _cells(g, d_ref)).max() <= 1e-9 * scale
    box = d[G - 1:G + g.nz + 1, G - 1:G + g.ny + 1, G - 1:G + g.nx + 1]
    box_ref = d_ref[G - 1:G + g.nz + 1, G - 1:G + g.ny + 1, G - 1:G + g.nx + 1]
    assert np.abs(box - box_ref).max() <= 1e-9 * scale


@pytest.mark.gpu
def test_gpu_tucker_refuses_short_columns(ctx):
    import ablsteadyrans_b200 as gb
    g, z, *_ = smooth_terrain_case(8, 8, 2, True, True, hill=10.0)
    with pytest.raises(gb.GustError):
        gb.tucker_wall_distance(ctx, g, to_dev(z))


@pytest.mark.gpu
def test_gpu_closure_with_tucker_distance_matches_oracle(ctx):
    """The k-L closure and all six residuals with the Tucker distance in
    place of the height above the ground: the GPU stage given the GPU's
    distance equals the oracle given the oracle's (1e-9 relative per field,
    the distances' own agreement)."""
    import ablsteadyrans_b200 as gb
    from test_turbulence import FIELDS, LOCS, _hill_case, _stage
    case, bc, ph = _hill_case()
    g = case.grid
    d_ref, _ = oracle.tucker_wall_distance(g, case.z, reltol=1e-13)
    case.wall_dist = d_ref
    dc, st = _stage(ctx, case, bc, ph)
    try:
        opts = gb.PoissonOptions.default(reltol=1e-13, abstol=0.0, max_iter=200)
        d, _ = gb.tucker_wall_distance(ctx, g, to_dev(case.z), opts)
        st.set_wall_distance(d)
        oracle.fill_ghosts(case, bc, ph)
        R_ref, cf_ref, _ = oracle.residual(case, bc, ph, fields=True)
        st.fill_ghosts()
        R = [r.cpu().numpy() for r in st.residual()]
        cf, _ = st.turbulence()
    finally:
        st.close()
    for f in ("nu", "nut", "length"):
        ref, got = _cells(g, cf_ref[f]), _cells(g, cf[f])
        assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), f
    for n, loc in enumerate(LOCS):
        v = g.valid(loc)
        ref, got = R_ref[n][v], R[n][v]
        assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), FIELDS[n]
    # the distance changed the closure: the mixing length differs from the
    # height-above-ground run
    case.wall_dist = None
    _, cf_h, _ = oracle.residual(case, bc, ph, fields=True)
    assert np.abs(_cells(g, cf_h["length"]) - _cells(g, cf_ref["length"])).max() > 0.0
