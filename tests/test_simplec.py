"""The SIMPLEC outer iteration (Source/Simplec.cpp:452-506) with given
diffusivities: the oracle is pinned to the reference's known answers
(test_Simplec.cpp: PoiseuilleToMachinePrecision :344-403, the uniform state's
fixed point :482, one correction removes the divergence :173)."""
import numpy as np
import pytest

import oracle
from ablsteadyrans_b200.abi import BC, FACE_NO_SLIP_WALL, FACE_PERIODIC, FACE_SLIP_WALL, Physics, SimplecOptions
from helpers import flat_case, seam_sync


def laminar(case, ground, top, H):
    g = case.grid
    faces = (FACE_PERIODIC if g.periodic_x else FACE_SLIP_WALL, FACE_PERIODIC if g.periodic_y else FACE_SLIP_WALL,
             ground, FACE_PERIODIC if g.periodic_x else FACE_SLIP_WALL,
             FACE_PERIODIC if g.periodic_y else FACE_SLIP_WALL, top)
    bc = BC.make(faces, theta_ref=((-1000.0, 5000.0), (300.0, 300.0)))
    return bc


def test_oracle_poiseuille_to_machine_precision():
    """Laminar Poiseuille flow between no-slip walls driven by a constant force:
    the discrete steady solution is u_k = F/(2 nu) (z_k (H - z_k) + dz^2/4),
    reached to machine precision; w, v, p' stay 0; theta and k untouched; a
    converged state is a fixed point of one more iteration."""
    H, F, nu, nz = 500.0, 1e-4, 10.0, 16
    case = flat_case(2, 2, nz, 1000.0, 1000.0, H, True, True, nu)
    bc = laminar(case, FACE_NO_SLIP_WALL, FACE_NO_SLIP_WALL, H)
    phys = Physics.make(H, gravity=0.0, pressure_gradient=(F, 0.0, 0.0))
    opts = SimplecOptions.make(zline_sweeps=2)
    opts.poisson.reltol = 0.1
    case.q["theta"][...] = 300.0
    case.q["tke"][...] = 0.5
    oracle.fill_ghosts(case, bc)
    umax = F * H * H / (8 * nu)
    its = 0
    for its in range(400):
        dtau = oracle.local_dtau(case, 10.0)
        st, info, _ = oracle.simplec_iterate(case, bc, phys, opts, dtau)
        assert st == 0
        if its > 5 and info.max_du < 1e-15 * umax:
            break
    assert its < 399
    g = case.grid
    G = g.ng
    dz = H / nz
    zc = (np.arange(nz) + 0.5) * dz
    exact = F / (2 * nu) * (zc * (H - zc) + dz * dz / 4)
    u = case.q["u"][G:G + nz, G:G + g.ny, G:G + g.nx + 1]
    assert np.abs(u - exact[:, None, None]).max() < 1e-13 * umax
    v = g.valid
    assert np.abs(case.q["w"][v(4)]).max() == 0
    assert np.abs(case.q["v"][v(2)]).max() == 0
    assert np.abs(case.q["p"][v(0)]).max() < 1e-14 * umax * umax
    assert case.q["theta"][v(0)].min() == 300.0 and case.q["theta"][v(0)].max() == 300.0
    assert case.q["tke"][v(0)].min() == 0.5
    q0 = case.copy()
    dtau = oracle.local_dtau(case, 10.0)
    st, info, _ = oracle.simplec_iterate(case, bc, phys, opts, dtau)
    assert np.abs(case.q["u"][v(1)] - q0.q["u"][v(1)]).max() < 1e-14 * umax
    assert np.abs(case.q["w"][v(4)] - q0.q["w"][v(4)]).max() == 0
    assert max(info.residual_norms) < 1e-12


def test_oracle_uniform_state_is_a_fixed_point():
    """A uniform wind over flat ground with slip walls has R = 0: an iteration
    changes nothing (test_Simplec.cpp:482)."""
    case = flat_case(8, 4, 6, 1000.0, 800.0, 500.0, True, True, 1.0)
    bc = laminar(case, FACE_SLIP_WALL, FACE_SLIP_WALL, 500.0)
    phys = Physics.make(500.0, gravity=9.81)
    opts = SimplecOptions.make()
    case.q["u"][...] = 6.0
    case.q["v"][...] = -2.0
    case.q["theta"][...] = 300.0
    case.q["tke"][...] = 0.1
    oracle.fill_ghosts(case, bc)
    q0 = case.copy()
    dtau = oracle.local_dtau(case, 5.0)
    st, info, R = oracle.simplec_iterate(case, bc, phys, opts, dtau)
    assert st == 0
    assert max(info.residual_norms) < 1e-14
    for f in ("u", "v", "w", "p", "theta", "tke"):
        assert np.abs(case.q[f] - q0.q[f])[case.grid.valid(0)].max() < 1e-13


def test_oracle_one_correction_reduces_the_divergence():
    """One pressure correction of a predicted random velocity leaves a
    divergence below the Poisson tolerance times the predicted one."""
    case = flat_case(8, 4, 6, 1000.0, 800.0, 500.0, True, True, 1.0)
    bc = laminar(case, FACE_SLIP_WALL, FACE_SLIP_WALL, 500.0)
    phys = Physics.make(500.0, gravity=0.0)
    opts = SimplecOptions.make(pressure_reltol=1e-10)
    rng = np.random.default_rng(21)
    g = case.grid
    for f, loc, lo, hi in (("u", 1, 5, 10), ("v", 2, -2, 2), ("w", 4, -0.5, 0.5)):
        case.q[f][g.valid(loc)] = rng.uniform(lo, hi, case.q[f][g.valid(loc)].shape)
        seam_sync(g, loc, case.q[f])
    case.q["theta"][...] = 300.0
    oracle.fill_ghosts(case, bc)
    dtau = oracle.local_dtau(case, 5.0)
    st, info, _ = oracle.simplec_iterate(case, bc, phys, opts, dtau)
    assert st == 0
    assert info.divergence_after < 1e-8 * info.divergence_before


def test_workload_mesh_matches_oracle_bit_for_bit():
    """The product's host mesh construction (BTF from the ground, ghost rows)
    equals the oracle's restatement bit for bit; the stretched levels have
    the solved ratios the configurations need."""
    from ablsteadyrans_b200 import workloads
    for nz, ratio in ((48, 1.0927), (64, 1.0622), (96, 1.0350)):
        zl, r = workloads.geometric_zlevels(nz)
        assert abs(r - ratio) < 5e-5 and zl[1] == 2.0 and abs(zl[-1] - 1500.0) < 1e-9
    inst = workloads.config1(nx=24, ny=20, nz=16)
    g = inst.grid
    ground = workloads.node_ground(g, lambda x, y: 150.0 * np.exp(-(((x - 300) ** 2 + (y - 250) ** 2) / 300.0 ** 2)))
    zl, _ = workloads.geometric_zlevels(16)
    a = workloads.btf_heights(g, zl, ground)
    b = oracle.btf_heights(g, zl, ground)
    G = g.ng
    sl = (slice(G - 1, G + g.nz + 2), slice(G - 1, G + g.ny + 2), slice(G - 1, G + g.nx + 2))
    assert np.array_equal(a[sl], b[sl])


def test_driver_ser_law():
    """ser_cfl (Source/PseudoTime.cpp:53-61): the cap, the growth limit and cfl0 r^-p."""
    from ablsteadyrans_b200.driver import ser_cfl
    assert ser_cfl(1.0, 1.0, 1.0, 10.0, 1.0, 2.0) == 1.0
    assert ser_cfl(1.0, 0.1, 1.0, 10.0, 1.0, 2.0) == 2.0
    assert ser_cfl(8.0, 0.01, 1.0, 10.0, 1.0, 2.0) == 10.0
    assert ser_cfl(4.0, 0.2, 1.0, 10.0, 1.0, 2.0) == pytest.approx(5.0)
    assert ser_cfl(4.0, 0.2, 1.0, 10.0, 0.0, 2.0) == 1.0


# ----------------------------------------------------- mass-consistent init
# gust::initialize_state with init.first_guess = profile (Source/Initializer.cpp).

INIT_FACES = {
    "periodic": (True, True, (0, 0, 4, 0, 0, 3)),
    "inflow_x": (False, True, (1, 0, 4, 2, 0, 3)),
}


def _init_case(name, seed=3):
    from ablsteadyrans_b200.abi import BC
    from helpers import terrain_simplec_case
    px, py, faces = INIT_FACES[name]
    case = terrain_simplec_case(20, 14, 10, px, py, seed=seed)
    bc = BC.make(faces, theta_ref=((0.0, 500.0, 1500.0), (300.0, 301.5, 305.0)), ustar=0.4, z0=0.1)
    return case, bc


@pytest.mark.parametrize("name", list(INIT_FACES))
def test_oracle_initializer_is_mass_consistent(name):
    """The projection removes the first guess's divergence (Mass_Consistent_*:
    divergence after at most solver.poisson_reltol times before, Tests/
    Initialization/Mass_Consistent_Askervein/README.md); theta is the
    sounding, p' = 0, k > 0, and the ground faces carry no flux."""
    from ablsteadyrans_b200.abi import InitOptions
    case, bc = _init_case(name)
    io = InitOptions.make()
    io.poisson.reltol = 1e-11
    rc, info = oracle.initialize(case, bc, io)
    assert rc == 0
    before, after, iters = info[0], info[1], info[2]
    assert before > 1e-3 and after <= 1e-10 * before
    assert 1 <= iters <= 30
    g = case.grid
    v = g.valid(0)
    assert np.all(case.q["p"] == 0)
    assert np.all(case.q["tke"][v] > 0)
    assert np.all((case.q["theta"][v] >= 300.0) & (case.q["theta"][v] <= 305.0))
    # no flux through the ground: Omega = 0 on the ground faces
    om = oracle.omega_from_w(g, case.q["u"], case.q["v"], case.q["w"], case.z)
    G = g.ng
    assert np.abs(om[G, G:G + g.ny, G:G + g.nx]).max() <= 1e-12 * np.abs(case.q["u"]).max()


def test_oracle_initializer_askervein_matches_reference_gold():
    """The reference's Mass_Consistent_Askervein regression: the split
    projection (alpha_h = 1, alpha_v = 0.5; FaceCoeffs::z_cross) on ERF's
    Askervein mesh gives the gold u, v, w, k, theta (cell values, faces
    averaged) at 1e-8 relative, with the gold's divergence before the
    projection and p' = 0."""
    from helpers import gold_cell_fields, init_askervein_case
    case, bc, io, gold = init_askervein_case()
    rc, info = oracle.initialize(case, bc, io)
    assert rc == 0
    assert info[0] == pytest.approx(gold["info"]["div_before"], rel=1e-9)
    assert info[1] <= io.poisson.reltol * info[0]
    got = gold_cell_fields(case.grid, case.q)
    for f in ("u", "v", "w", "tke", "theta"):
        err = np.abs(got[f] - gold[f]).max() / np.abs(gold[f]).max()
        assert err < 1e-8, (f, err)
    assert np.all(got["p"] == 0) and np.all(gold["p"] == 0)


def test_oracle_split_operator_matches_split_flux_divergence():
    """With z_cross the operator stays minus the divergence of its own fluxes
    (test_Poisson.cpp:321's property, on the split coefficient): A phi =
    -face_divergence(F(phi)) with F_z = -(beta_z dphi/dz - z_cross cross)."""
    from helpers import init_askervein_case
    case, bc, io, gold = init_askervein_case()
    g = case.grid
    pbc = (2, 1, 1, 2, 1, 1)
    rng = np.random.default_rng(11)
    phi = g.np_zeros()
    phi[g.valid(0)] = rng.standard_normal(phi[g.valid(0)].shape)
    bh = np.full_like(case.ax, 1.0)
    bv = np.full_like(case.ax, 0.25)
    y = oracle.poisson_apply_split(g, pbc, case.ax, case.ay, case.az, case.J, case.z, phi, bh, bh, bv, bh)
    F = oracle.poisson_fluxes_split(g, pbc, case.z, phi, bh, bh, bv, bh)
    div = oracle.face_divergence(g, case.ax, case.ay, case.az, case.J, *F)
    v = g.valid(0)
    assert np.abs(y[v] + div[v]).max() <= 1e-10 * np.abs(y[v]).max()
    # the split changes the operator (the cross part carries beta_h, not beta_z)
    y0 = oracle.poisson_apply_split(g, pbc, case.ax, case.ay, case.az, case.J, case.z, phi, bh, bh, bv, None)
    assert np.abs(y0[v] - y[v]).max() > 1e-6 * np.abs(y[v]).max()


def _obrien_case(seed=3):
    from ablsteadyrans_b200.abi import BC
    from helpers import terrain_simplec_case
    case = terrain_simplec_case(16, 12, 10, False, True, hill=150.0, seed=seed)
    bc = BC.make((1, 0, 4, 2, 0, 3), theta_ref=((0.0, 500.0, 1500.0), (300.0, 301.5, 305.0)), ustar=0.4, z0=0.1,
                 direction=30.0)
    return case, bc


def test_oracle_obrien_column_correction():
    """O'Brien (Initializer.OBrienColumnCorrection, test_Initializer.cpp:662-737):
    Omega vanishes at the ground and the top exactly, each cell keeps the
    weight difference times its column's residual E, the column sum of J D is
    the residual flux, the worst |E| is the one reported; through the
    initializer the field differs and the projection still converges."""
    from ablsteadyrans_b200.abi import InitOptions
    case, bc = _obrien_case()
    rc, _ = oracle.initialize(case, bc, InitOptions.make(projection=0))
    assert rc == 0
    g = case.grid
    om, E = oracle.obrien_omega(case)
    assert E > 1e-3
    G = g.ng
    zero = g.np_zeros()
    u, v = case.q["u"], case.q["v"]
    d = oracle.face_divergence(g, case.ax, case.ay, case.az, case.J, u, v, om)
    d0 = oracle.face_divergence(g, case.ax, case.ay, case.az, case.J, u, v, zero)
    nz, dzeta = g.nz, g.dzeta
    z = case.z
    worst = 0.0
    for j in range(g.ny):
        for i in range(g.nx):
            I, Jc = i + G, j + G
            assert om[G, Jc, I] == 0 and om[G + nz, Jc, I] == 0
            Jk = case.J[G:G + nz, Jc, I]
            Ecol = -(Jk * d0[G:G + nz, Jc, I] * dzeta).sum() / case.az[G + nz, Jc, I]
            worst = max(worst, abs(Ecol))
            zf = 0.25 * (z[G:G + nz + 1, Jc, I] + z[G:G + nz + 1, Jc, I + 1] + z[G:G + nz + 1, Jc + 1, I]
                         + z[G:G + nz + 1, Jc + 1, I + 1])
            depth = zf[-1] - zf[0]
            assert zf[1] - zf[0] < 0.9 * depth / nz   # stretched: the index weight would differ
            f = (zf - zf[0]) / depth
            azc = case.az[G:G + nz + 1, Jc, I]
            want = -(f[1:] ** 2 * azc[1:] - f[:-1] ** 2 * azc[:-1]) * Ecol / (Jk * dzeta)
            got = d[G:G + nz, Jc, I]
            assert np.all(np.abs(got - want) <= 1e-11 * (np.abs(d0[G:G + nz, Jc, I]) + np.abs(want)))
            total = (Jk * got).sum()
            assert total == pytest.approx(-Ecol * azc[-1] / dzeta, rel=1e-11)
    assert worst == pytest.approx(E, rel=1e-12)
    # through the initializer
    co, _ = _obrien_case()
    cp, _ = _obrien_case()
    io = InitOptions.make(obrien=1)
    io.poisson.reltol = 1e-11
    ro, info_o = oracle.initialize(co, bc, io)
    io.obrien = 0
    rp, info_p = oracle.initialize(cp, bc, io)
    assert ro == 0 and rp == 0
    assert info_o[4] == pytest.approx(E, rel=1e-12) and info_p[4] == 0
    assert info_o[0] != info_p[0]
    assert info_o[1] < 10 * 1e-11 * info_o[0]
    assert np.abs(co.q["w"] - cp.q["w"]).max() > 1e-3


def test_oracle_initializer_projection_off_keeps_the_first_guess():
    from ablsteadyrans_b200.abi import InitOptions
    case, bc = _init_case("inflow_x")
    rc, info = oracle.initialize(case, bc, InitOptions.make(projection=0))
    assert rc == 0 and info[0] == info[1] and info[2] == 0
    # w is 0 above the ground faces
    g = case.grid
    G = g.ng
    assert np.all(case.q["w"][G + 1:G + g.nz + 1, G:G + g.ny, G:G + g.nx] == 0)
