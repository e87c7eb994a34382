"""The k-L closure and the surface layer (the wall model): the oracle's
restatement (oracle/turbulence.c) pinned to the reference's Closure_Column
gold (Tests/Discretization/Closure_Column: "The plotfile matches
Gold/closure_column_plt00000 at relative 1e-10") and to that test's closed
forms (check_closure.py), the stratified branches of the closure against the
AL01 relations, and the heat-flux MOST solve; GPU tests compare the CUDA
closure, wall model, residual and SIMPLEC iterations with the oracle."""
import math

import numpy as np
import pytest

import oracle
from helpers import GOLDEN, closure_column_case, closure_column_outputs

KAPPA, CMU0 = 0.41, 0.5562


def _gold():
    d = np.load(f"{GOLDEN}/closure_column.npz")
    return {k: d[k] for k in d.files}


def test_oracle_closure_column_matches_reference_gold():
    case, bc, ph = closure_column_case()
    oracle.fill_ghosts(case, bc, ph)
    R, cf, ss = oracle.residual(case, bc, ph, fields=True)
    got = closure_column_outputs(case.grid, case.q, R, cf, ss)
    gold = _gold()
    for f, ref in gold.items():
        scale = np.abs(ref).max()
        err = np.abs(got[f] - ref).max()
        if scale == 0:
            assert err <= 1e-13, f
        else:
            assert err <= 1e-10 * scale, (f, err / scale)


def test_oracle_closure_column_closed_forms():
    """check_closure.py: nu_t = kappa u* (z + z0) and L = kappa (z + z0) (1e-9),
    u* recovered (1e-10), eps = u*^3/(kappa (z + z0)) (1e-9), R_u, R_v zero
    below the top cell (1e-10 of u*^2/dz) and u*^2/dz (cos, sin) there (1e-8), R_w =
    R_theta = 0, the first cell's R_k 0 (the wall-k row at k = k_w)."""
    us, z0, deg = 0.35, 0.1, 15.0
    case, bc, ph = closure_column_case(us, z0, deg)
    oracle.fill_ghosts(case, bc, ph)
    R, cf, ss = oracle.residual(case, bc, ph, fields=True)
    g = case.grid
    out = closure_column_outputs(g, case.q, R, cf, ss)
    dz = g.dzeta
    zc = (np.arange(g.nz) + 0.5) * dz
    nut_ref = KAPPA * us * (zc + z0)
    assert np.abs(out["nut"] - nut_ref[:, None, None]).max() <= 1e-9 * nut_ref.max()
    L_ref = KAPPA * (zc + z0)
    assert np.abs(out["length"] - L_ref[:, None, None]).max() <= 1e-9 * L_ref.max()
    assert np.abs(out["ustar"][0] - us).max() <= 1e-10 * us
    eps_ref = us ** 3 / (KAPPA * (zc + z0))
    assert np.abs(out["eps"] - eps_ref[:, None, None]).max() <= 1e-9 * eps_ref.max()
    s = us * us / dz
    a = math.radians(deg)
    assert np.abs(out["R_u"][:-1]).max() <= 1e-10 * s and np.abs(out["R_v"][:-1]).max() <= 1e-10 * s
    assert np.abs(out["R_u"][-1] - s * math.cos(a)).max() <= 1e-8 * s
    assert np.abs(out["R_v"][-1] - s * math.sin(a)).max() <= 1e-8 * s
    assert np.abs(out["R_w"]).max() <= 1e-12 and np.abs(out["R_theta"]).max() <= 1e-12
    assert np.abs(out["R_tke"][0]).max() <= 1e-15


def _al01(k, N2, l_g, Cb=0.35, Rt_crit=-1.0, Rt_min=-3.0):
    """AL01 (Axell and Liungman 2001) relations as ERF_RANSClosure.H states them."""
    c3 = CMU0 ** 3

    def smooth(rt):
        if rt >= Rt_crit:
            return rt
        x, aa = rt - Rt_crit, Rt_min - Rt_crit
        return Rt_crit + aa * x / (x + aa)

    if abs(N2) <= np.finfo(float).eps:
        L = l_g
    elif N2 > 0:
        L = math.sqrt(1.0 / (1.0 / (l_g * l_g) + N2 / (Cb * Cb) / k))
    else:
        L = l_g * math.sqrt(1.0 - c3 * c3 / (Cb * Cb) * smooth(l_g * l_g * N2 / (k * c3 * c3)))
    rt = smooth(L * L * N2 / (k * c3 * c3))
    cmu = (CMU0 + 0.108 * rt) / (1 + 0.308 * rt + 0.00837 * rt * rt)
    cmup = CMU0 / (1 + 0.277 * rt)
    nut = cmu * math.sqrt(k) * L
    return L, rt, nut, cmup / cmu * nut, c3 * k ** 1.5 / L


@pytest.mark.parametrize("dtdz", [0.02, -0.02, -2.0])
def test_oracle_closure_stratified_branches(dtdz):
    """A stable, an unstable and a strongly unstable (Rt smoothed) column:
    the length, Rt, nu_t, gamma_theta and eps of every cell against the AL01
    relations, with N^2 = (g/theta_0) dtheta/dz and the capped l_g."""
    case, bc, ph = closure_column_case()
    g = case.grid
    G = g.ng
    zc = (np.arange(-G, g.nz + 1 + G) + 0.5) * g.dzeta
    case.q["theta"][...] = (300.0 + dtdz * zc)[:, None, None]
    ph.turb_max_geom_lscale = 30.0
    case.q["tke"][...] = 0.05
    oracle.fill_ghosts(case, bc, ph)
    cf = oracle.closure_fields(case, bc, ph)
    N2 = 9.81 / 300.0 * dtdz
    kk = 0.05
    smoothed = 0
    for k in range(1, g.nz - 1):   # the ground gradient and the top differ from dtheta/dz
        d = (k + 0.5) * g.dzeta
        lraw = KAPPA * (d + 0.1)
        l_g = 30.0 * lraw / (30.0 + lraw)
        L, rt, nut, nutp, eps = _al01(kk, N2, l_g)
        smoothed += rt < -1.0
        o = (G + k, G + 3, G + 4)
        assert cf["length"][o] == pytest.approx(L, rel=1e-12)
        assert cf["Rt"][o] == pytest.approx(rt, rel=1e-11, abs=1e-14)
        assert cf["nut"][o] == pytest.approx(nut, rel=1e-11)
        assert cf["gamma_theta"][o] == pytest.approx(nutp, rel=1e-11)
        assert cf["eps"][o] == pytest.approx(eps, rel=1e-12)
    if dtdz == -2.0:
        assert smoothed > 0


@pytest.mark.parametrize("q", [0.1, -0.02])
def test_oracle_surface_layer_heat_flux(q):
    """bc.surface_stability = heat_flux: u* solves the MOST relation
    u* = kappa U / max(ln((d + z0)/z0) - psi_m(d/L), m), 1/L = -kappa g q /
    (u*^3 theta_0), to round-off; an upward flux raises u* above the neutral
    value and k_w to (u*^3 + kappa g q d0/theta_0)^(2/3)/Cmu0^2, a downward one
    lowers u*."""
    from ablsteadyrans_b200.abi import SURFACE_HEAT_FLUX
    case, bc, ph = closure_column_case()
    oracle.fill_ghosts(case, bc, ph)
    neutral, bad0 = oracle.surface_state(case, bc, ph)
    bc.surface_stability, bc.surface_heat_flux = SURFACE_HEAT_FLUX, q
    ss, bad = oracle.surface_state(case, bc, ph)
    assert bad0 == 0 and bad == 0
    g = case.grid
    p = (g.ng + 2) * int(g.c.sy) + g.ng + 3
    us, U, d0, invL = ss["ustar"][p], ss["speed"][p], ss["d0"][p], ss["inv_L"][p]
    z0 = 0.1
    zeta = max(min(d0 * invL, 100.0), -100.0)
    if zeta > 0:
        psi = -5.0 * zeta
    else:
        x = (1 - 16 * zeta) ** 0.25
        psi = 2 * math.log(0.5 * (1 + x)) + math.log(0.5 * (1 + x * x)) - 2 * math.atan(x) + math.pi / 2
    lz = math.log((d0 + z0) / z0)
    assert us == pytest.approx(KAPPA * U / max(lz - psi, min(lz, 1.0)), rel=1e-12)
    assert invL == pytest.approx(-KAPPA * 9.81 * q / (300.0 * us ** 3), rel=1e-12)
    if q > 0:
        assert us > neutral["ustar"][p]
        kw = (us ** 3 + KAPPA * 9.81 / 300.0 * q * d0) ** (2.0 / 3.0) / CMU0 ** 2
        assert ss["kwall"][p] == pytest.approx(kw, rel=1e-12)
    else:
        assert us < neutral["ustar"][p]
        assert ss["kwall"][p] == pytest.approx(us * us / CMU0 ** 2, rel=1e-12)


def test_oracle_stage_with_closure_and_wall_model():
    """SIMPLEC iterations with the closure and the surface layer over a hill:
    every field stays finite, u* stays positive, and the momentum residual
    falls over 30 iterations from the log-law start."""
    from ablsteadyrans_b200.abi import FACE_SURFACE_LAYER, SimplecOptions
    case, bc, ph = _hill_case()
    so = SimplecOptions.make()
    norms = []
    for _ in range(30):
        dt = oracle.local_dtau(case, 2.0, phys=ph)
        rc, info, R = oracle.simplec_iterate(case, bc, ph, so, dt)
        assert rc == 0
        norms.append(info.residual_norms[0])
    assert bc.face[2] == FACE_SURFACE_LAYER
    for f in case.FIELDS:
        assert np.all(np.isfinite(case.q[f])), f
    assert norms[-1] < 0.5 * norms[0], norms
    ss, bad = oracle.surface_state(case, bc, ph)
    assert bad == 0


def _hill_case(seed=1):
    """A 16 x 12 x 16 Gaussian hill (periodic in y) with inflow and outflow in
    x, the surface layer on the ground (per-column z0 around 0.1 m), the
    closure, and the log-law state with k from the inflow profile."""
    from ablsteadyrans_b200.abi import BC, FACE_INFLOW, FACE_OUTFLOW, FACE_SLIP_WALL, FACE_SURFACE_LAYER, Physics
    from helpers import terrain_simplec_case
    case = terrain_simplec_case(16, 12, 16, False, True, hill=60.0, seed=seed)
    rng = np.random.default_rng(seed)
    z0 = case.plane()
    z0[:] = 0.1 * np.exp(0.3 * rng.standard_normal(z0.shape))
    case.z0map = z0
    bc = BC.make((FACE_INFLOW, 0, FACE_SURFACE_LAYER, FACE_OUTFLOW, 0, FACE_SLIP_WALL),
                 theta_ref=((0.0, 1500.0), (300.0, 300.0)), ustar=0.4, z0=0.1, surface={"z0": 0.1})
    ph = Physics.make(1500.0, closure=1, log_mean=1)
    case.q["tke"][...] = np.abs(case.q["tke"]) + 0.2
    case.q["theta"][...] = 300.0
    case.q["w"][...] = 0.0
    return case, bc, ph


# ---------------------------------------------------------------- GPU ---

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)


def _stage(ctx, case, bc, ph, **opts):
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    dc = DeviceCase.from_oracle(case)
    return dc, SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(**opts))


def _cells(g, a):
    G = g.ng
    return a[G:G + g.nz, G:G + g.ny, G:G + g.nx]


def _columns(g, a):
    G = g.ng
    return np.asarray(a).reshape(-1, int(g.c.sy))[G - 1:G + g.ny + 1, G - 1:G + g.nx + 1]


@pytest.mark.gpu
def test_gpu_closure_column_matches_reference_gold(ctx):
    """The reference's Closure_Column regression on the B200: the closure,
    the surface layer and the full residual give the gold plotfile's fields
    at the reference's 1e-10 relative."""
    case, bc, ph = closure_column_case()
    dc, st = _stage(ctx, case, bc, ph)
    st.fill_ghosts()
    R = [r.cpu().numpy() for r in st.residual()]
    cf, ss = st.turbulence()
    q = {f: dc.host(f) for f in FIELDS}
    got = closure_column_outputs(case.grid, q, R, cf, ss)
    for f, ref in _gold().items():
        scale = np.abs(ref).max()
        err = np.abs(got[f] - ref).max()
        assert err <= (1e-13 if scale == 0 else 1e-10 * scale), (f, err / max(scale, 1e-300))
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("heat", [0.0, 0.05])
def test_gpu_wall_model_and_closure_match_oracle(ctx, heat):
    """Over a hill with a per-column z0: the ghost fill (the wall law's
    ground gradient), the surface state, the closure's fields and all six
    residuals of the GPU equal the oracle's (1e-11 relative per field; the
    MOST Newton and pow/log of the two libraries differ in the last bits)."""
    from ablsteadyrans_b200.abi import SURFACE_HEAT_FLUX
    case, bc, ph = _hill_case()
    if heat:
        bc.surface_stability, bc.surface_heat_flux = SURFACE_HEAT_FLUX, heat
    dc, st = _stage(ctx, case, bc, ph)
    ss_ref = oracle.fill_ghosts(case, bc, ph)
    R_ref, cf_ref, _ = oracle.residual(case, bc, ph, fields=True)
    st.fill_ghosts()
    R = [r.cpu().numpy() for r in st.residual()]
    cf, ss = st.turbulence()
    g = case.grid
    for f in FIELDS:
        ref, got = case.q[f], dc.host(f)
        assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max(), f
    for f in ("ustar", "speed", "d0", "inv_L", "tau_x", "tau_y", "drag", "kwall", "area"):
        ref, got = _columns(g, ss_ref[f]), _columns(g, ss[f])
        assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300), f
    for f in ("nu", "gamma_theta", "gamma_tke", "nut", "length", "Ps", "Pb", "eps", "dSdk"):
        ref, got = _cells(g, cf_ref[f]), _cells(g, cf[f])
        assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300), f
    for n, loc in enumerate(LOCS):
        v = g.valid(loc)
        ref, got = R_ref[n][v], R[n][v]
        assert np.abs(got - ref).max() <= 1e-10 * max(np.abs(ref).max(), 1e-300), n
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("heat", [0.0, 0.05])
def test_gpu_fused_residual_with_wall_and_closure(ctx, heat):
    """With the closure's k sources and the wall's ground fluxes (stress on
    u and v, the heat flux on theta, none on k), the fused residual
    launches equal the separate flux and divergence launches to 1e-13."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.abi import SURFACE_HEAT_FLUX
    case, bc, ph = _hill_case()
    if heat:
        bc.surface_stability, bc.surface_heat_flux = SURFACE_HEAT_FLUX, heat
        rng = np.random.default_rng(3)
        case.q["theta"][...] = 300.0 + rng.uniform(-0.5, 0.5, case.q["theta"].shape)
    dc, st = _stage(ctx, case, bc, ph)
    try:
        st.fill_ghosts()
        ctx.tune(gb.TUNE_RESIDUAL, 1)
        R1 = [r.cpu().numpy() for r in st.residual()]
        ctx.tune(gb.TUNE_RESIDUAL, 0)
        R0 = [r.cpu().numpy() for r in st.residual()]
    finally:
        ctx.tune(gb.TUNE_RESIDUAL, 0)
        st.close()
    g = case.grid
    for n, loc in enumerate(LOCS):
        v = g.valid(loc)
        scale = max(np.abs(R1[n][v]).max(), 1e-300)
        assert np.abs(R0[n][v] - R1[n][v]).max() <= 1e-13 * scale, n


@pytest.mark.gpu
def test_gpu_iterations_with_closure_and_wall_model_match_oracle(ctx):
    """Five SIMPLEC iterations with the closure and the surface layer (the
    local dtau from the last iteration's nu, 0 at first) agree with the
    oracle's to 1e-9 relative per field."""
    from ablsteadyrans_b200.abi import SimplecOptions
    case, bc, ph = _hill_case()
    opts = dict(pressure_reltol=1e-11, zline_sweeps=3)
    dc, st = _stage(ctx, case, bc, ph, **opts)
    so = SimplecOptions.make(**opts)
    for it in range(5):
        dt_ref = oracle.local_dtau(case, 2.0, phys=ph)
        dt = st.local_dtau(2.0)
        v0 = case.grid.valid(0)
        assert np.abs(dt.cpu().numpy()[v0] - dt_ref[v0]).max() <= 1e-10 * dt_ref[v0].max(), it
        rc, info_ref, _ = oracle.simplec_iterate(case, bc, ph, so, dt_ref)
        assert rc == 0
        info = st.iterate(dt)
        for n in range(6):
            assert info.residual_norms[n] == pytest.approx(info_ref.residual_norms[n], rel=1e-9, abs=1e-14), (it, n)
        for f, loc in zip(FIELDS, LOCS):
            v = case.grid.valid(loc)
            ref, got = case.q[f][v], dc.host(f)[v]
            assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), (it, f)
    st.close()


@pytest.mark.gpu
def test_gpu_turbulence_refusals(ctx):
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.abi import FACE_SURFACE_LAYER
    case, bc, ph = _hill_case()
    for mutate, msg in ((lambda b, p: setattr(b, "surface_z0", 0.0), "bc.surface_z0"),
                        (lambda b, p: b.face.__setitem__(5, FACE_SURFACE_LAYER), "the ground's only"),
                        (lambda b, p: setattr(b, "surface_heat_flux", 0.1), "stability is neutral"),
                        (lambda b, p: setattr(p, "turb_Rt_min", -4.0), "turb.Rt_min"),
                        (lambda b, p: setattr(p, "turb_Cb", 0.0), "turb.Cb"),
                        # a QNSE coefficient set under Businger-Dyer would be ignored (SurfaceLayer.cpp:282-288)
                        (lambda b, p: setattr(b, "surface_qnse_bm", 0.3), "qnse_bm is set but stable_functions")):
        case, bc, ph = _hill_case()
        mutate(bc, ph)
        with pytest.raises(gb.GustError, match=msg):
            _stage(ctx, case, bc, ph)


# ------------------------------------------------------------ damping ---

def _profile_u(h, ustar=0.35, z0=0.1):
    return ustar / KAPPA * np.log((np.maximum(h, 0.0) + z0) / z0)


def test_oracle_rayleigh_layer_closed_form():
    """The Rayleigh layer (BoundaryConditions::add_damping): R_u gains
    c(z) (u - u_profile(h)) with c = coef sin^2(pi/2 (z - z_d)/(z_top - z_d))
    above z_d, R_w gains c w; the u rows' diagonal gains c; nothing below
    z_d. A field excluded from bc.rayleigh_fields is left alone."""
    case, bc, ph = closure_column_case()
    g = case.grid
    G = g.ng
    case.q["w"][G + 1:G + g.nz, G:G + g.ny, G:G + g.nx] = 0.01
    oracle.fill_ghosts(case, bc, ph)
    R0 = oracle.residual(case, bc, ph)
    A0 = oracle.implicit_rows(case, bc, ph, 0)
    bc.rayleigh_zdamp, bc.rayleigh_dampcoef, bc.rayleigh_fields = 500.0, 0.2, 0b00011   # u and v only
    R1 = oracle.residual(case, bc, ph)
    A1 = oracle.implicit_rows(case, bc, ph, 0)
    zc = (np.arange(g.nz) + 0.5) * g.dzeta
    c = np.where(zc > 500.0, 0.2 * np.sin(0.5 * np.pi * (zc - 500.0) / (1000.0 - 500.0)) ** 2, 0.0)
    u = case.q["u"][G:G + g.nz, G:G + g.ny, G:G + g.nx + 1]
    want = c[:, None, None] * (u - _profile_u(zc)[:, None, None])
    got = (R1[0] - R0[0])[G:G + g.nz, G:G + g.ny, G:G + g.nx + 1]
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    dA = (A1[0] - A0[0])[G:G + g.nz, G:G + g.ny, G:G + g.nx + 1]
    assert np.abs(dA - c[:, None, None]).max() <= 1e-15
    assert np.array_equal(R1[2], R0[2])   # w not in bc.rayleigh_fields
    bc.rayleigh_fields = 0b00100           # w alone: towards 0
    R2 = oracle.residual(case, bc, ph)
    zf = np.arange(g.nz + 1) * g.dzeta
    cw = np.where(zf > 500.0, 0.2 * np.sin(0.5 * np.pi * (zf - 500.0) / 500.0) ** 2, 0.0)
    w = case.q["w"][G:G + g.nz + 1, G:G + g.ny, G:G + g.nx]
    dRw = (R2[2] - R0[2])[G + 1:G + g.nz, G:G + g.ny, G:G + g.nx]   # the top and ground rows are boundary rows
    assert np.abs(dRw - (cw[:, None, None] * w)[1:g.nz]).max() <= 1e-15


def test_oracle_sponge_closed_form():
    """The lateral sponge: within sponge_width of an inflow or outflow face,
    R_k gains strength (1 - s/width)^2 (k - k_profile(h)); beyond it, and
    along the periodic y faces, nothing."""
    case, bc, ph = _hill_case()
    g = case.grid
    G = g.ng
    oracle.fill_ghosts(case, bc, ph)
    R0 = oracle.residual(case, bc, ph)
    bc.sponge_width, bc.sponge_strength = 100.0, 0.05
    R1 = oracle.residual(case, bc, ph)
    dk = (R1[5] - R0[5])[G:G + g.nz, G:G + g.ny, G:G + g.nx]
    x = (np.arange(g.nx) + 0.5) * g.dx
    s = np.minimum(x, g.nx * g.dx - x)
    cs = np.where(s < 100.0, 0.05 * (1 - s / 100.0) ** 2, 0.0)
    assert np.all(dk[:, :, cs == 0] == 0)
    inside = np.nonzero(cs > 0)[0]
    assert inside.size >= 2
    # k_ref: the inflow profile's k at the cell's height above the ground,
    # (u* c)^2 / Cmu0^2 with c = 1 / (1 + kappa (h + z0) / l_max)
    h = oracle.height_above_ground(case)[G:G + g.nz, G:G + g.ny, G:G + g.nx]
    ul = 0.4 / (1.0 + KAPPA * (h + 0.1) / 30.0)
    kref = ul * ul / CMU0 ** 2
    k = case.q["tke"][G:G + g.nz, G:G + g.ny, G:G + g.nx]
    want = cs[None, None, :] * (k - kref)
    assert np.abs(dk - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_gpu_damping_matches_oracle(ctx):
    """The Rayleigh layer and the sponge on the GPU: the residual and five
    SIMPLEC iterations (with the closure and the surface layer) equal the
    oracle's."""
    from ablsteadyrans_b200.abi import SimplecOptions
    case, bc, ph = _hill_case()
    bc.rayleigh_zdamp, bc.rayleigh_dampcoef, bc.rayleigh_fields = 400.0, 0.1, 31
    bc.sponge_width, bc.sponge_strength = 120.0, 0.05
    opts = dict(pressure_reltol=1e-11, zline_sweeps=3)
    dc, st = _stage(ctx, case, bc, ph, **opts)
    oracle.fill_ghosts(case, bc, ph)
    R_ref = oracle.residual(case, bc, ph)
    st.fill_ghosts()
    R = [r.cpu().numpy() for r in st.residual()]
    for n, loc in enumerate(LOCS):
        v = case.grid.valid(loc)
        assert np.abs(R[n][v] - R_ref[n][v]).max() <= 1e-10 * max(np.abs(R_ref[n][v]).max(), 1e-300), n
    so = SimplecOptions.make(**opts)
    for it in range(5):
        dt_ref = oracle.local_dtau(case, 2.0, phys=ph)
        rc, info_ref, _ = oracle.simplec_iterate(case, bc, ph, so, dt_ref)
        assert rc == 0
        st.iterate(st.local_dtau(2.0))
        for f, loc in zip(FIELDS, LOCS):
            v = case.grid.valid(loc)
            ref, got = case.q[f][v], dc.host(f)[v]
            assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), (it, f)
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("damping", [False, True])
def test_gpu_implicit_rows_match_oracle(ctx, damping):
    """implicit_rows of u, v, w, theta and k with the closure, the wall rows
    and (with damping) the Rayleigh layer and the sponge on the diagonal:
    every coefficient equal to the oracle's (1e-11 relative)."""
    case, bc, ph = _hill_case()
    if damping:
        bc.rayleigh_zdamp, bc.rayleigh_dampcoef, bc.rayleigh_fields = 400.0, 0.1, 31
        bc.sponge_width, bc.sponge_strength = 120.0, 0.05
    dc, st = _stage(ctx, case, bc, ph)
    oracle.fill_ghosts(case, bc, ph)
    _, cf, ss = oracle.residual(case, bc, ph, fields=True)
    st.fill_ghosts()
    st.residual()
    for eq, loc in ((0, 1), (1, 2), (2, 4), (4, 0), (5, 0)):
        A_ref = oracle.implicit_rows(case, bc, ph, eq, cf, ss)
        A = st.implicit_rows(eq).cpu().numpy()
        v = case.grid.valid(loc)
        for c in range(7):
            ref, got = A_ref[c][v], A[c][v]
            assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300), (eq, c, np.abs(got - ref).max())
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 3])
def test_gpu_tile_layout_iterations_match_oracle(ctx, seed):
    """The served tiles' layout (inflow on the upwind x and y faces, outflow
    on the others, fractal terrain tapered at the edges, the closure and the
    wall law with the tile's u* and z0): three SIMPLEC iterations on the GPU
    equal the oracle's, from the oracle's mass-consistent initial state."""
    from ablsteadyrans_b200 import workloads
    from helpers import case_from_instance
    inst = workloads.tile(16, 12, seed, precision=0, zline_sweeps=3)
    case = case_from_instance(inst)
    bc, ph, so = inst.bc, inst.physics, inst.options
    so.pressure_reltol = 1e-11
    from ablsteadyrans_b200.abi import InitOptions
    rc, _ = oracle.initialize(case, bc, InitOptions.make())
    assert rc == 0
    dc, st = _stage(ctx, case, bc, ph, pressure_reltol=1e-11, zline_sweeps=3)
    oracle.fill_ghosts(case, bc, ph)
    st.fill_ghosts()
    try:
        for it in range(3):
            dt_ref = oracle.local_dtau(case, 2.0, phys=ph)
            rc, _, _ = oracle.simplec_iterate(case, bc, ph, so, dt_ref)
            assert rc == 0
            st.iterate(st.local_dtau(2.0))
            for f, loc in zip(FIELDS, LOCS):
                v = case.grid.valid(loc)
                ref, got = case.q[f][v], dc.host(f)[v]
                assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), (it, f)
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_confidence_share_and_height(ctx):
    """SimplecStage::confidence on the last iteration's residual: every cell
    passes thresholds far above the residuals (share 1, no failing height),
    no cell passes zero thresholds (share 0, the failing height is the
    highest cell's height above the ground), and the share grows with the
    thresholds."""
    case, bc, ph = _hill_case()
    dc, st = _stage(ctx, case, bc, ph)
    st.fill_ghosts()
    try:
        info = st.iterate(st.local_dtau(2.0))
        s1, h1 = st.confidence([1e30] * 6)
        assert s1 == 1.0 and h1 == 0.0
        s0, h0 = st.confidence([0.0] * 6)
        assert s0 == 0.0
        agl = oracle.height_above_ground(case)
        assert abs(h0 - agl[case.grid.valid(0)].max()) <= 1e-9 * h0
        norms = list(info.residual_norms)
        shares = [st.confidence([f * n for n in norms])[0] for f in (0.3, 1.0, 3.0, 10.0)]
        assert shares == sorted(shares) and 0.0 < shares[1] < 1.0
    finally:
        st.close()


@pytest.mark.parametrize("dtdz", [0.02, -0.02])
def test_oracle_closure_gate_and_cap(dtdz):
    """turb.ri_gate: the length, Rt, nu_t and the heat diffusivity follow the
    AL01 relations at N^2 N^4 / (N^4 + Ri_0^2 S^4) while P_b keeps the ungated
    N^2 (gate_stratification, Closure.cpp:337-354); a neutral column is the
    same bits with the gate on. turb.realizability: nu_t = min(nu_t,
    C_r max(k, floor) / S) (ClosureWake.cpp:8-29)."""
    case, bc, ph = closure_column_case()
    g = case.grid
    G = g.ng
    zc = (np.arange(-G, g.nz + 1 + G) + 0.5) * g.dzeta
    case.q["theta"][...] = (300.0 + dtdz * zc)[:, None, None]
    ph.turb_max_geom_lscale = 30.0
    case.q["tke"][...] = 0.05
    oracle.fill_ghosts(case, bc, ph)
    plain = oracle.closure_fields(case, bc, ph)
    ri0 = 0.25
    ph.turb_ri_gate = ri0
    gated = oracle.closure_fields(case, bc, ph)
    N2 = 9.81 / 300.0 * dtdz
    kk = 0.05
    changed = 0
    for k in range(1, g.nz - 1):
        o = (G + k, G + 3, G + 4)
        S2 = plain["Ps"][o] / plain["nut"][o]
        N2c = N2 * (N2 * N2) / (N2 * N2 + ri0 * ri0 * S2 * S2 + np.finfo(float).tiny)
        d = (k + 0.5) * g.dzeta
        lraw = KAPPA * (d + 0.1)
        l_g = 30.0 * lraw / (30.0 + lraw)
        L, rt, nut, nutp, eps = _al01(kk, N2c, l_g)
        assert gated["length"][o] == pytest.approx(L, rel=1e-11)
        assert gated["nut"][o] == pytest.approx(nut, rel=1e-10)
        assert gated["gamma_theta"][o] == pytest.approx(nutp, rel=1e-10)
        assert gated["Pb"][o] == pytest.approx(-nutp * N2, rel=1e-10)
        changed += abs(gated["nut"][o] - plain["nut"][o]) > 1e-6 * plain["nut"][o]
    assert changed > 0
    # neutral: the gate changes nothing
    case.q["theta"][...] = 300.0
    oracle.fill_ghosts(case, bc, ph)
    ph.turb_ri_gate = 0.0
    n0 = oracle.closure_fields(case, bc, ph)
    ph.turb_ri_gate = ri0
    n1 = oracle.closure_fields(case, bc, ph)
    for f in ("nu", "nut", "length", "Rt", "eps"):
        assert np.array_equal(n0[f], n1[f]), f
    # the realizability cap on the neutral column
    ph.turb_ri_gate = 0.0
    cr = 0.2
    ph.turb_realizability = cr
    capped = oracle.closure_fields(case, bc, ph)
    floor = max(ph.turb_tke_floor, np.finfo(float).eps)
    n_capped = 0
    for k in range(0, g.nz - 1):
        o = (G + k, G + 3, G + 4)
        S2 = n0["Ps"][o] / n0["nut"][o]
        cap = cr * max(case.q["tke"][o], floor) / math.sqrt(S2)
        assert capped["nut"][o] == pytest.approx(min(n0["nut"][o], cap), rel=1e-12)
        n_capped += cap < n0["nut"][o]
    assert n_capped > 0


@pytest.mark.gpu
def test_gpu_closure_gate_and_cap_match_oracle(ctx):
    """The stratification gate and the realizability cap on the GPU over a
    stratified hill: the closure's fields and the residuals equal the
    oracle's (1e-11 relative)."""
    case, bc, ph = _hill_case()
    g = case.grid
    G = g.ng
    case.q["theta"][...] = 300.0 + 0.01 * np.arange(case.q["theta"].shape[0])[:, None, None] * 40.0
    ph.turb_ri_gate, ph.turb_realizability = 0.25, 0.3
    dc, st = _stage(ctx, case, bc, ph)
    try:
        oracle.fill_ghosts(case, bc, ph)
        R_ref, cf_ref, _ = oracle.residual(case, bc, ph, fields=True)
        st.fill_ghosts()
        R = [r.cpu().numpy() for r in st.residual()]
        cf, _ = st.turbulence()
        for f in ("nu", "gamma_theta", "gamma_tke", "nut", "length", "Ps", "Pb", "eps", "dSdk"):
            ref, got = _cells(g, cf_ref[f]), _cells(g, cf[f])
            assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300), f
        for n, loc in enumerate(LOCS):
            v = g.valid(loc)
            assert np.abs(R[n][v] - R_ref[n][v]).max() <= 1e-10 * max(np.abs(R_ref[n][v]).max(), 1e-300), n
    finally:
        st.close()


def test_oracle_nut_relaxation_blends_with_the_history():
    """turb.nut_relax = w: after an iteration the closure's nu_t is w times
    the new one plus 1 - w times the last iteration's (Closure.cpp:407-436),
    and the diffusivities follow it; before the first iteration there is no
    history and the weight is 1."""
    from ablsteadyrans_b200.abi import SimplecOptions
    case, bc, ph = _hill_case()
    ph.turb_nut_relax = 0.4
    oracle.fill_ghosts(case, bc, ph)
    first = oracle.closure_fields(case, bc, ph)
    ph.turb_nut_relax = 1.0
    plain = oracle.closure_fields(case, bc, ph)
    assert np.array_equal(first["nut"], plain["nut"])      # no history yet
    ph.turb_nut_relax = 0.4
    oracle.simplec_iterate(case, bc, ph, SimplecOptions.make(), oracle.local_dtau(case, 2.0, phys=ph))
    hist = case.nut_hist.copy()
    oracle.fill_ghosts(case, bc, ph)
    relaxed = oracle.closure_fields(case, bc, ph)
    ph.turb_nut_relax = 1.0
    case.nut_hist = None
    new = oracle.closure_fields(case, bc, ph)
    v = case.grid.valid(0)
    expect = 0.4 * new["nut"][v] + (1 - 0.4) * hist[v]
    assert np.abs(relaxed["nut"][v] - expect).max() <= 1e-14 * np.abs(expect).max()
    assert np.abs(relaxed["nu"][v] - (ph.turb_nu_molecular + relaxed["nut"][v])).max() == 0


@pytest.mark.gpu
def test_gpu_nut_relaxation_iterations_match_oracle(ctx):
    """turb.nut_relax = 0.5 on the GPU: three SIMPLEC iterations (each
    blending the closure's nu_t with the last one's) equal the oracle's."""
    from ablsteadyrans_b200.abi import SimplecOptions
    case, bc, ph = _hill_case()
    ph.turb_nut_relax = 0.5
    opts = dict(pressure_reltol=1e-11, zline_sweeps=3)
    dc, st = _stage(ctx, case, bc, ph, **opts)
    oracle.fill_ghosts(case, bc, ph)
    st.fill_ghosts()
    so = SimplecOptions.make(**opts)
    try:
        for it in range(3):
            rc, _, _ = oracle.simplec_iterate(case, bc, ph, so, oracle.local_dtau(case, 2.0, phys=ph))
            assert rc == 0
            st.iterate(st.local_dtau(2.0))
            for f, loc in zip(FIELDS, LOCS):
                v = case.grid.valid(loc)
                ref, got = case.q[f][v], dc.host(f)[v]
                assert np.abs(got - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1e-300), (it, f)
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_initialize_clears_the_nut_history(ctx):
    """A stage that iterated with turb.nut_relax < 1 and is then initialized
    again starts without a nu_t history, as a fresh stage does (each level's
    closure is new when its state is initialized in the reference): its next
    iteration equals a fresh stage's bit for bit."""
    import torch
    from ablsteadyrans_b200.abi import InitOptions
    case, bc, ph = _hill_case()
    ph.turb_nut_relax = 0.5
    opts = dict(pressure_reltol=1e-8, zline_sweeps=2)
    q0 = {f: a.copy() for f, a in case.q.items()}
    dc1, st1 = _stage(ctx, case, bc, ph, **opts)
    dc2, st2 = _stage(ctx, case, bc, ph, **opts)
    try:
        st1.fill_ghosts()
        for _ in range(2):
            st1.iterate(st1.local_dtau(2.0))
        for dc, st in ((dc1, st1), (dc2, st2)):
            for f in q0:
                dc.q[f].copy_(torch.from_numpy(q0[f]))
            st.initialize(InitOptions.make())
            st.fill_ghosts()
            st.iterate(st.local_dtau(2.0))
        for f, loc in zip(FIELDS, LOCS):
            v = case.grid.valid(loc)
            assert np.array_equal(dc1.host(f)[v], dc2.host(f)[v]), f
    finally:
        st1.close()
        st2.close()


def test_oracle_surface_layer_qnse_stable_side():
    """bc.surface_stable_functions = qnse under a downward heat flux: u*
    solves the MOST relation with QNSE's stable psi_m = -((a - b)/b)
    ln(1 + b zeta) (StabilityFunctions.H), which lowers u* less than
    Businger-Dyer's -5 zeta; the range checks refuse b <= 0 and a < b."""
    from ablsteadyrans_b200.abi import SURFACE_HEAT_FLUX
    case, bc, ph = closure_column_case()
    bc.surface_stability, bc.surface_heat_flux = SURFACE_HEAT_FLUX, -0.02
    oracle.fill_ghosts(case, bc, ph)
    bd, _ = oracle.surface_state(case, bc, ph)
    bc.surface_qnse = 1
    ss, bad = oracle.surface_state(case, bc, ph)
    assert bad == 0
    g = case.grid
    p = (g.ng + 2) * int(g.c.sy) + g.ng + 3
    us, U, d0, invL = ss["ustar"][p], ss["speed"][p], ss["d0"][p], ss["inv_L"][p]
    zeta = max(min(d0 * invL, 100.0), -100.0)
    assert zeta > 0
    am, bm = bc.surface_qnse_am, bc.surface_qnse_bm
    psi = -((am - bm) / bm) * math.log(1 + bm * zeta)
    lz = math.log((d0 + 0.1) / 0.1)
    assert us == pytest.approx(KAPPA * U / max(lz - psi, min(lz, 1.0)), rel=1e-12)
    assert us > bd["ustar"][p]


@pytest.mark.gpu
def test_gpu_qnse_wall_model_matches_oracle(ctx):
    """QNSE's stable side under a downward heat flux on the GPU: the surface
    state, the wall law's ghost fill and the residuals equal the oracle's."""
    from ablsteadyrans_b200.abi import SURFACE_HEAT_FLUX
    case, bc, ph = _hill_case()
    bc.surface_stability, bc.surface_heat_flux, bc.surface_qnse = SURFACE_HEAT_FLUX, -0.02, 1
    dc, st = _stage(ctx, case, bc, ph)
    try:
        ss_ref = oracle.fill_ghosts(case, bc, ph)
        R_ref = oracle.residual(case, bc, ph)
        st.fill_ghosts()
        R = [r.cpu().numpy() for r in st.residual()]
        _, ss = st.turbulence()
        g = case.grid
        for f in FIELDS:
            ref, got = case.q[f], dc.host(f)
            assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max(), f
        for f in ("ustar", "inv_L", "tau_x", "tau_y", "kwall"):
            ref, got = _columns(g, ss_ref[f]), _columns(g, ss[f])
            assert np.abs(got - ref).max() <= 1e-11 * max(np.abs(ref).max(), 1e-300), f
        for n, loc in enumerate(LOCS):
            v = g.valid(loc)
            assert np.abs(R[n][v] - R_ref[n][v]).max() <= 1e-10 * max(np.abs(R_ref[n][v]).max(), 1e-300), n
    finally:
        st.close()
