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
