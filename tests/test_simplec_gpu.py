"""GPU SIMPLEC stage against the oracle: ghost fills, the FP64 residual, full
iterations, and the reference's Poiseuille known answer on the B200."""
import numpy as np
import pytest

import oracle
from ablsteadyrans_b200.abi import (BC, FACE_INFLOW, FACE_NO_SLIP_WALL, FACE_OUTFLOW, FACE_PERIODIC, FACE_SLIP_WALL,
                                    LIMITER_UPWIND, LIMITER_VAN_ALBADA, LIMITER_VAN_LEER, Physics, SimplecOptions)
from helpers import flat_case, terrain_simplec_case

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)

CONFIGS = {
    # periodic box over a hill, no-slip ground, slip top
    "periodic": dict(px=True, py=True, faces=(FACE_PERIODIC, FACE_PERIODIC, FACE_NO_SLIP_WALL, FACE_PERIODIC,
                                              FACE_PERIODIC, FACE_SLIP_WALL)),
    # log-law inflow from the west, outflow east, periodic in y (the bench's layout)
    "inflow": dict(px=False, py=True, faces=(FACE_INFLOW, FACE_PERIODIC, FACE_NO_SLIP_WALL, FACE_OUTFLOW,
                                             FACE_PERIODIC, FACE_SLIP_WALL)),
    # walls all round, a moving no-slip lid
    "walls": dict(px=False, py=False, faces=(FACE_INFLOW, FACE_SLIP_WALL, FACE_NO_SLIP_WALL, FACE_OUTFLOW,
                                             FACE_SLIP_WALL, FACE_NO_SLIP_WALL)),
}


def make(name, nx=20, ny=14, nz=10, seed=0):
    c = CONFIGS[name]
    case = terrain_simplec_case(nx, ny, nz, c["px"], c["py"], seed=seed)
    bc = BC.make(c["faces"], theta_ref=((0.0, 500.0, 1500.0), (300.0, 301.5, 305.0)), ustar=0.4, z0=0.1,
                 direction=0.0, zhi_theta_grad=0.003, wall_velocity={5: (2.0, 0.5, 0.0)})
    return case, bc


def physics(case, **kw):
    return Physics.make(1500.0, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_gpu_fill_ghosts_matches_oracle(ctx, name):
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(name)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, physics(case), SimplecOptions.make())
    oracle.fill_ghosts(case, bc)
    st.fill_ghosts()
    for f in FIELDS:
        ref = case.q[f]
        got = dc.host(f)
        scale = max(np.abs(ref).max(), 1.0)
        assert np.abs(got - ref).max() <= 1e-13 * scale, f
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("opts", [dict(limiter=LIMITER_VAN_LEER), dict(limiter=LIMITER_VAN_ALBADA, log_mean=1),
                                  dict(limiter=LIMITER_UPWIND, coriolis=1, latitude=45.0, geostrophic=1, ug=8.0,
                                       vg=0.0, pressure_gradient=(1e-4, -2e-5, 0.0))])
def test_gpu_residual_matches_oracle(ctx, name, opts):
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(name, seed=3)
    ph = physics(case, **opts)
    oracle.fill_ghosts(case, bc)
    R_ref = oracle.residual(case, bc, ph)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make())
    R = [r.cpu().numpy() for r in st.residual()]
    g = case.grid
    for n, (a, b) in enumerate(zip(R, R_ref)):
        v = g.valid(LOCS[n])
        scale = max(np.abs(b[v]).max(), 1e-300)
        assert np.abs(a[v] - b[v]).max() <= 1e-11 * scale, (FIELDS[n], np.abs(a[v] - b[v]).max(), scale)
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("levels", [0, 3, 64], ids=["8-levels", "3-levels", "one-block-column"])
def test_gpu_fused_residual_matches_separate_launches(ctx, name, levels):
    """The residual's convection, diffusion and pressure gradient as one
    launch per equation (GB_TUNE_RESIDUAL 0, or N levels per block) equal
    the separate flux and divergence launches (GB_TUNE_RESIDUAL 1) to 1e-13
    relative per field: the same face fluxes by the same device functions
    (the compiler's contractions may differ between the two kernels)."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(name, nx=37, ny=19, nz=11, seed=3)
    ph = physics(case, limiter=LIMITER_VAN_ALBADA, log_mean=1, coriolis=1, latitude=45.0)
    oracle.fill_ghosts(case, bc, ph)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make())
    try:
        ctx.tune(gb.TUNE_RESIDUAL, 1)
        R1 = [r.cpu().numpy() for r in st.residual()]
        ctx.tune(gb.TUNE_RESIDUAL, levels)
        R0 = [r.cpu().numpy() for r in st.residual()]
    finally:
        ctx.tune(gb.TUNE_RESIDUAL, 0)
        st.close()
    g = case.grid
    for n, (a, b) in enumerate(zip(R0, R1)):
        v = g.valid(LOCS[n])
        scale = max(np.abs(b[v]).max(), 1e-300)
        assert np.abs(a[v] - b[v]).max() <= 1e-13 * scale, (FIELDS[n], np.abs(a[v] - b[v]).max(), scale)


@pytest.mark.gpu
@pytest.mark.parametrize("sweep", [(0, 0), (1, 1)], ids=["zjacobi", "lusgs-alternate"])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_gpu_iterations_match_oracle(ctx, name, sweep):
    """Three SIMPLEC iterations (gravity, Coriolis, VNN cap on) agree with the
    oracle's to 1e-9 relative per field (the Poisson solves to 1e-11), with
    z-line Jacobi sweeps and with line LU-SGS sweeps (steady.sweep = lusgs,
    steady.line_alternate = 1)."""
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(name, seed=5)
    ph = physics(case, coriolis=1, latitude=40.0, geostrophic=1, ug=7.0, vg=-1.0)
    opts = SimplecOptions.make(pressure_reltol=1e-11, zline_sweeps=3, w_vnn_cap=16.0, tke_floor=1e-3,
                               line_sweep=sweep[0], line_alternate=sweep[1])
    oracle.fill_ghosts(case, bc)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, opts)
    for it in range(3):
        dt_ref = oracle.local_dtau(case, 4.0)
        dt = st.local_dtau(4.0)
        assert np.abs(dt.cpu().numpy()[case.grid.valid(0)] - dt_ref[case.grid.valid(0)]).max() <= 1e-12 * dt_ref.max()
        rc, info_ref, _ = oracle.simplec_iterate(case, bc, ph, opts, dt_ref)
        assert rc == 0
        info = st.iterate(dt)
        for n in range(6):
            assert info.residual_norms[n] == pytest.approx(info_ref.residual_norms[n], rel=1e-9, abs=1e-14)
        for f, loc in zip(FIELDS, LOCS):
            v = case.grid.valid(loc)
            ref = case.q[f][v]
            got = dc.host(f)[v]
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(got - ref).max() <= 1e-9 * scale, (it, f, np.abs(got - ref).max() / scale)
    st.close()


@pytest.mark.gpu
def test_gpu_poiseuille_to_machine_precision(ctx):
    """The reference's PoiseuilleToMachinePrecision (test_Simplec.cpp:344-403)
    run on the B200."""
    import torch
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    H, F, nu, nz = 500.0, 1e-4, 10.0, 16
    case = flat_case(2, 2, nz, 1000.0, 1000.0, H, True, True, nu)
    bc = BC.make((FACE_PERIODIC, FACE_PERIODIC, FACE_NO_SLIP_WALL, FACE_PERIODIC, FACE_PERIODIC, FACE_NO_SLIP_WALL),
                 theta_ref=((-1000.0, 5000.0), (300.0, 300.0)))
    ph = Physics.make(H, gravity=0.0, pressure_gradient=(F, 0.0, 0.0))
    opts = SimplecOptions.make(zline_sweeps=2)
    opts.poisson.reltol = 0.1
    case.q["theta"][...] = 300.0
    case.q["tke"][...] = 0.5
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, opts)
    st.fill_ghosts()
    umax = F * H * H / (8 * nu)
    for its in range(400):
        info = st.iterate(st.local_dtau(10.0))
        if its > 5 and info.max_du < 1e-15 * umax:
            break
    assert its < 399
    G = case.grid.ng
    dz = H / nz
    zc = (np.arange(nz) + 0.5) * dz
    exact = F / (2 * nu) * (zc * (H - zc) + dz * dz / 4)
    u = dc.host("u")[G:G + nz, G:G + 2, G:G + 3]
    assert np.abs(u - exact[:, None, None]).max() < 1e-13 * umax
    assert np.abs(dc.host("w")[case.grid.valid(4)]).max() == 0
    assert max(info.residual_norms) < 1e-12
    st.close()


@pytest.mark.gpu
def test_gpu_mixed_precision_tracks_fp64(ctx):
    """FP32 inner solves (sweeps and multigrid) inside the FP64 defect
    correction follow the plain FP64 path: after 10 iterations the velocity
    differs by less than 1e-4 relative."""
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make("inflow", nx=24, ny=16, nz=12, seed=7)
    ph = physics(case)
    oracle.fill_ghosts(case, bc)
    runs = {}
    for prec in (0, 1):
        dc = DeviceCase.from_oracle(case)
        st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(precision=prec, pressure_reltol=1e-6))
        for _ in range(10):
            st.iterate(st.local_dtau(5.0))
        runs[prec] = {f: dc.host(f) for f in FIELDS}
        st.close()
    for f, loc in (("u", 1), ("v", 2), ("w", 4)):
        v = case.grid.valid(loc)
        a, b = runs[1][f][v], runs[0][f][v]
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max(), f


@pytest.mark.gpu
def test_gpu_line_sweep_option_refusals(ctx):
    """steady.sweep / steady.line_alternate checks with the reference's
    messages (Source/Driver.cpp:99-118)."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(list(CONFIGS)[0], seed=5)
    ph = physics(case)
    oracle.fill_ghosts(case, bc)
    dc = DeviceCase.from_oracle(case)
    for kw, msg in (({"line_sweep": 2}, "steady.sweep = 2"),
                    ({"line_alternate": 1}, "has no effect unless steady.sweep = lusgs"),
                    ({"line_sweep": 1, "line_alternate": 1, "zline_sweeps": 1}, "needs steady.zline_sweeps >= 2")):
        with pytest.raises(gb.GustError, match=msg):
            SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(**kw))


# ----------------------------------------------------- mass-consistent init

@pytest.mark.gpu
@pytest.mark.parametrize("alpha", [(1.0, 1.0), (0.5, 0.5), (1.0, 0.5)])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_gpu_initializer_matches_oracle(ctx, name, alpha):
    """gust::initialize_state (init.first_guess = profile, projection on) on
    the B200 against the oracle: every field to 1e-9 relative (the
    projections to 1e-11), the divergence removed, the same iteration count;
    Sigma = diag(alpha_h^2, alpha_h^2, alpha_v^2), the split z-face
    coefficient where alpha_v != alpha_h."""
    from ablsteadyrans_b200.abi import InitOptions
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(name, seed=5)
    ph = physics(case)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make())
    io = InitOptions.make(alpha_h=alpha[0], alpha_v=alpha[1], k_decay_height=600.0, z_agl_min=1.0)
    io.poisson.reltol = 1e-11
    rc, info = oracle.initialize(case, bc, io)
    assert rc == 0
    res = st.initialize(io)
    assert res.divergence_before == pytest.approx(info[0], rel=1e-11)
    assert res.divergence_after <= 1e-10 * res.divergence_before
    assert res.poisson_iterations == int(info[2])
    for f, loc in zip(FIELDS, LOCS):
        ref = case.q[f]
        got = dc.host(f)
        scale = max(np.abs(ref).max(), 1e-300)
        # every point the initializer writes, ghosts included
        assert np.abs(got - ref).max() <= 1e-9 * scale, (f, np.abs(got - ref).max() / scale)
    st.close()


@pytest.mark.gpu
def test_gpu_initializer_refusals(ctx):
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.abi import InitOptions
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc = make(list(CONFIGS)[0], seed=5)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, physics(case), SimplecOptions.make())
    for kw, msg in (({"obrien": 2}, "init.obrien must be 0 or 1"),
                    ({"z_agl_min": -1.0}, "init.z_agl_min"), ({"alpha_h": 0.0, "alpha_v": 0.0}, "init.alpha_h")):
        with pytest.raises(gb.GustError, match=msg):
            st.initialize(InitOptions.make(**kw))
    st.close()


@pytest.mark.gpu
def test_gpu_initializer_askervein_matches_reference_gold(ctx):
    """The reference's Mass_Consistent_Askervein regression on the B200: the
    split projection (alpha_h = 1, alpha_v = 0.5) gives the gold u, v, w, k
    and theta (cell values, faces averaged) at 1e-8 relative."""
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    from helpers import gold_cell_fields, init_askervein_case
    case, bc, io, gold = init_askervein_case()
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, physics(case), SimplecOptions.make())
    res = st.initialize(io)
    assert res.divergence_before == pytest.approx(gold["info"]["div_before"], rel=1e-9)
    assert res.divergence_after <= io.poisson.reltol * res.divergence_before
    got = gold_cell_fields(case.grid, {f: dc.host(f) for f in FIELDS})
    for f in ("u", "v", "w", "tke", "theta"):
        err = np.abs(got[f] - gold[f]).max() / np.abs(gold[f]).max()
        assert err < 1e-8, (f, err)
    st.close()


@pytest.mark.gpu
def test_gpu_initializer_obrien_matches_oracle(ctx):
    """init.obrien = 1 on the B200 against the oracle: the column pass's top
    residual to 1e-12, every field to 1e-9 after the projection."""
    from ablsteadyrans_b200.abi import BC, InitOptions
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    from helpers import terrain_simplec_case
    case = terrain_simplec_case(16, 12, 10, False, True, hill=150.0, seed=3)
    bc = BC.make((1, 0, 4, 2, 0, 3), theta_ref=((0.0, 500.0, 1500.0), (300.0, 301.5, 305.0)), ustar=0.4, z0=0.1,
                 direction=30.0)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, physics(case), SimplecOptions.make())
    io = InitOptions.make(obrien=1, alpha_v=0.5)
    io.poisson.reltol = 1e-11
    rc, info = oracle.initialize(case, bc, io)
    assert rc == 0 and info[4] > 1e-3
    res = st.initialize(io)
    assert res.obrien_top_residual == pytest.approx(info[4], rel=1e-12)
    assert res.divergence_before == pytest.approx(info[0], rel=1e-11)
    assert res.poisson_iterations == int(info[2])
    for f in FIELDS:
        ref = case.q[f]
        got = dc.host(f)
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got - ref).max() <= 1e-9 * scale, (f, np.abs(got - ref).max() / scale)
    st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_iteration_graphs_equal_eager_launches(ctx, precision):
    """From its second iteration a stage runs the launch sequences before and
    after the Krylov solve as CUDA graphs (and the V-cycle as one): the same
    kernels in the same order, so five iterations with graphs give the eager
    iterations' fields bit for bit (GB_TUNE_GRAPHS = 1 launches every kernel
    alone); the nu_t history's appearance after the first iteration and a
    new dtau array rebuild the graphs."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200 import workloads
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    out = []
    for graphs in (1, 0):
        ctx.tune(gb.TUNE_GRAPHS, graphs)
        inst = workloads.tile(40, 24, 3, precision=precision)
        inst.physics.coriolis, inst.physics.latitude, inst.physics.rotation_period = 1, 45.0, 86164.0
        inst.physics.turb_nut_relax = 0.7
        J, ax, ay, az, _ = oracle.metrics(inst.grid, inst.z)
        dc = DeviceCase(inst.grid, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
        st = SimplecStage(ctx, dc, inst.bc, inst.physics, inst.options)
        st.fill_ghosts()
        infos = []
        for it in range(5):
            dt = st.local_dtau(2.0)          # a new dtau array each iteration
            infos.append(list(st.iterate(dt).residual_norms))
        out.append(({f: dc.host(f) for f in FIELDS}, infos))
        st.close()
    ctx.tune(gb.TUNE_GRAPHS, 0)
    for f in FIELDS:
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
    assert out[0][1] == out[1][1]
