"""Parity at the configurations' sizes and at convergence: the GPU's SIMPLEC
solve against the oracle's on the flat neutral ABL of the oracle case (32 x
32 x 48, 300 outer iterations), on a small hill run to the steady criterion,
and on the 128 x 128 x 64 hill at full size (one iteration, one residual
evaluation, one V-cycle, one line solve). The mixed-precision form (FP32
inner solves) is compared with the oracle's FP64 steady state field by
field. The GPU's converged neutral ABL is checked against the physics the
reference's Neutral_ABL_Flat regression checks
(Tests/Canonical_RANS/Neutral_ABL_Flat/README.md:17-22)."""
import math

import numpy as np
import pytest

import oracle
from ablsteadyrans_b200 import workloads

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)


def oracle_case(inst):
    """The oracle's copy of an instance (metrics from its node heights), ghosts filled."""
    g = inst.grid
    J, ax, ay, az, _ = oracle.metrics(g, inst.z)
    oc = oracle.Case(g, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.z0map)
    oc.q = {f: a.copy() for f, a in inst.q.items()}
    oracle.fill_ghosts(oc, inst.bc, inst.physics)
    return oc


def gpu_stage(ctx, oc, inst, options=None):
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    dc = DeviceCase.from_oracle(oc)
    st = SimplecStage(ctx, dc, inst.bc, inst.physics, options if options is not None else inst.options)
    st.fill_ghosts()
    return dc, st


def field_errors(grid, got, ref):
    """Per field: max |got - ref| over the valid points over the field's
    scale: the velocity magnitude max(|u|, |v|, |w|) for u, v and w (a
    component that is zero up to rounding, such as v over flat ground with
    a wind along x, has no scale of its own), max |ref| for the others (1
    for a field that is zero everywhere)."""
    vel = max(float(np.abs(ref[f][grid.valid(loc)]).max()) for f, loc in zip(FIELDS[:3], LOCS[:3]))
    out = {}
    for f, loc in zip(FIELDS, LOCS):
        v = grid.valid(loc)
        scale = vel if f in ("u", "v", "w") else float(np.abs(ref[f][v]).max())
        out[f] = float(np.abs(got[f][v] - ref[f][v]).max()) / (scale if scale > 0 else 1.0)
    return out


def run_oracle(oc, inst, cfls):
    """The oracle's SIMPLEC iterations at the given CFL per iteration (the
    GPU driver's sequence, so both take the same pseudo-time steps)."""
    for cfl in cfls:
        dt = oracle.local_dtau(oc, cfl, phys=inst.physics)
        rc, info, _ = oracle.simplec_iterate(oc, inst.bc, inst.physics, inst.options, dt)
        assert rc == 0
    return info


def closure_length(oc, inst):
    oracle.fill_ghosts(oc, inst.bc, inst.physics)
    return oracle.closure_fields(oc, inst.bc, inst.physics)["length"]


def gpu_closure_length(st):
    st.fill_ghosts()
    st.residual()
    cf, _ = st.turbulence(closure=True, surface=False)
    return cf["length"]


@pytest.mark.gpu
def test_gpu_config0_300_iterations_match_oracle(ctx):
    """The oracle case itself (flat, 32 x 32 x 48, log-law inflow u* = 0.4
    m/s, z0 = 0.1 m, the k-L closure and neutral MOST, no Coriolis): 300
    outer iterations of the SER driver on the GPU, and the oracle's 300 at
    the same CFL per iteration; U, V, W, p, k, theta and the closure's
    length L agree within 1e-6 relative."""
    from ablsteadyrans_b200.driver import Driver
    inst = workloads.config0()
    oc = oracle_case(inst)
    dc, st = gpu_stage(ctx, oc, inst)
    try:
        drv = Driver(st)
        for _ in range(300):
            assert drv.step() != "diverged"
        cfls = [h[0] for h in drv.history]
        oracle.set_threads(oracle.max_threads())
        run_oracle(oc, inst, cfls)
        got = {f: dc.host(f) for f in FIELDS}
        err = field_errors(inst.grid, got, oc.q)
        v = inst.grid.valid(0)
        Lg, Lo = gpu_closure_length(st), closure_length(oc, inst)
        err["L"] = float(np.abs(Lg[v] - Lo[v]).max() / np.abs(Lo[v]).max())
        print("config 0, 300 iterations, GPU vs oracle:", err)
        for f, e in err.items():
            assert e <= 1e-6, (f, e)
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_config0_steady_meets_the_neutral_abl_checks(ctx):
    """Config 0 run to the steady criterion on the GPU meets the physics the
    reference's Neutral_ABL_Flat regression checks on its steady state
    (Tests/Canonical_RANS/Neutral_ABL_Flat/README.md:17-22, the --physics
    set): u* within 0.35 +- 0.15 m/s, the wall cell's k within 5 % of
    u*^2 / Cmu0^2, the speed in the lowest four cells within 10 % of the log
    law u*/kappa ln((z + z0)/z0), and the eddy viscosity of the second cell
    within 30 % of kappa u* (z + z0); planar means over the domain's
    columns."""
    from ablsteadyrans_b200.simplec import NativeDriver, run_drivers
    inst = workloads.config0()
    oc = oracle_case(inst)
    dc, st = gpu_stage(ctx, oc, inst)
    try:
        d = NativeDriver(st)
        (verdict, n), = run_drivers([d], 8000, 1)
        d.close()
        assert verdict == "steady", (verdict, n)
        _, mon = st.norms()
        ustar = mon[2]
        st.fill_ghosts()
        st.residual()
        cf, _ = st.turbulence(closure=True, surface=False)
        g = inst.grid
        G = g.ng
        u = dc.host("u")[G:G + g.nz, G:G + g.ny, G:G + g.nx + 1]
        v = dc.host("v")[G:G + g.nz, G:G + g.ny + 1, G:G + g.nx]
        k = dc.host("tke")[G:G + g.nz, G:G + g.ny, G:G + g.nx]
        nut = cf["nut"][G:G + g.nz, G:G + g.ny, G:G + g.nx]
        uc = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
        vc = 0.5 * (v[:, :-1, :] + v[:, 1:, :])
        speed = np.sqrt(uc * uc + vc * vc).mean(axis=(1, 2))
        zc = 0.5 * (inst.zlevels[:-1] + inst.zlevels[1:])
        z0, kappa, cmu0 = inst.z0, workloads.KAPPA, workloads.CMU0
        report = {"iterations": n, "ustar": ustar, "k_wall_ratio": k[0].mean() / ustar ** 2 * cmu0 ** 2,
                  "log_law": [float(speed[m] / (ustar / kappa * math.log((zc[m] + z0) / z0))) for m in range(4)],
                  "nut_ratio": float(nut[1].mean() / (kappa * ustar * (zc[1] + z0)))}
        print("config 0 steady, the Neutral_ABL_Flat checks:", report)
        assert abs(ustar - 0.35) <= 0.15
        assert abs(report["k_wall_ratio"] - 1.0) <= 0.05
        for r in report["log_law"]:
            assert abs(r - 1.0) <= 0.10
        assert abs(report["nut_ratio"] - 1.0) <= 0.30
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_config1_full_size_steps_match_oracle(ctx):
    """Config 1 at its full size (128 x 128 x 64, the hill, Coriolis, the
    closure and the surface layer) from its initial state: one residual
    evaluation within 1e-12 relative per field, one SIMPLEC outer iteration
    within 1e-9 (the Poisson solve to 1e-11), and one z-line solve of the
    iteration's u system (four sweeps) within 1e-12."""
    import torch

    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.abi import SimplecOptions
    inst = workloads.config1()
    oracle.set_threads(oracle.max_threads())
    oc = oracle_case(inst)
    opts = SimplecOptions.make(zline_sweeps=4, pressure_reltol=1e-11)
    dc, st = gpu_stage(ctx, oc, inst, opts)
    g = inst.grid
    try:
        R_ref = oracle.residual(oc, inst.bc, inst.physics)
        R = [r.cpu().numpy() for r in st.residual()]
        for n, (a, b) in enumerate(zip(R, R_ref)):
            v = g.valid(LOCS[n])
            scale = max(float(np.abs(b[v]).max()), 1e-300)
            assert float(np.abs(a[v] - b[v]).max()) <= 1e-12 * scale, (FIELDS[n], float(np.abs(a[v] - b[v]).max()) / scale)
        # the u system of the first iteration, solved alone
        A = st.implicit_rows(0)
        Ah = A.cpu().numpy()
        rng = np.random.default_rng(1)
        ap = Ah[0] + 1.0 / 5.0
        rhs = g.np_zeros()
        v = g.valid(1)
        rhs[v] = rng.uniform(-1, 1, rhs[v].shape)
        d_ref = g.np_zeros()
        oracle.zline_jacobi(g, 1, Ah, ap, rhs, 4, d_ref)
        dd = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
        gb.zline_jacobi(ctx, g, 1, A, torch.from_numpy(ap).cuda(), torch.from_numpy(rhs).cuda(), 4, dd)
        got = dd.cpu().numpy()
        assert float(np.abs(got[v] - d_ref[v]).max()) <= 1e-12 * float(np.abs(d_ref[v]).max())
        # one outer iteration
        dt_ref = oracle.local_dtau(oc, 1.0, phys=inst.physics)
        dt = st.local_dtau(1.0)
        rc, info_ref, _ = oracle.simplec_iterate(oc, inst.bc, inst.physics, opts, dt_ref)
        assert rc == 0
        info = st.iterate(dt)
        got = {f: dc.host(f) for f in FIELDS}
        err = field_errors(g, got, oc.q)
        print("config 1, one iteration, GPU vs oracle:", err)
        for f, e in err.items():
            assert e <= 1e-9, (f, e)
        for n in range(6):
            assert info.residual_norms[n] == pytest.approx(info_ref.residual_norms[n], rel=1e-9, abs=1e-14)
    finally:
        st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_config1_full_size_vcycle_matches_oracle(ctx, precision):
    """One V-cycle of the pressure-correction multigrid on config 1's mesh
    (128 x 128 x 64, the hill): FP64 within 1e-12 of the oracle's; the FP32
    hierarchy within 1e-5 of the oracle's FP64 V-cycle."""
    import torch

    import ablsteadyrans_b200 as gb
    inst = workloads.config1()
    g = inst.grid
    J, ax, ay, az, _ = oracle.metrics(g, inst.z)
    bc = (gb.POISSON_NEUMANN, gb.POISSON_PERIODIC, gb.POISSON_NEUMANN, gb.POISSON_DIRICHLET, gb.POISSON_PERIODIC,
          gb.POISSON_NEUMANN)
    rng = np.random.default_rng(3)
    r = g.np_zeros()
    r[g.valid(0)] = rng.standard_normal(r[g.valid(0)].shape)
    opts = gb.PoissonOptions.default(precision=precision)
    oracle.set_threads(oracle.max_threads())
    mg = oracle.Multigrid(g, bc, inst.z, J, ax, ay, az, max_levels=opts.max_levels, min_coarse=opts.min_coarse,
                          nu1=opts.nu1, nu2=opts.nu2, nu_coarse=opts.nu_coarse)
    e_ref = mg.vcycle(r)
    mg.close()
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    ps = gb.PoissonSolver(ctx, g, dev(inst.z), dev(J), bc, opts)
    ps.set_coeffs(dev(ax), dev(ay), dev(az))
    e = ps.vcycle(dev(r)).cpu().numpy()
    ps.close()
    v = g.valid(0)
    err = float(np.abs(e[v] - e_ref[v]).max()) / float(np.abs(e_ref[v]).max())
    print(f"config 1 V-cycle, precision {precision}: {err:.3e}")
    assert err <= (1e-12 if precision == 0 else 1e-5)


CONVERGED_CASE = dict(nx=8, ny=8, nz=48)


@pytest.mark.gpu
def test_gpu_converged_states_match_oracle(ctx):
    """The flat neutral ABL of config 0 on an 8 x 8 x 48 grid run to the
    steady criterion on the GPU in plain FP64 and with FP32 inner solves
    (mixed precision), and the oracle's FP64 iterations at the FP64 run's
    CFL per iteration, as many: the converged U, V, W, p, k, theta and L of
    the plain FP64 GPU run agree with the oracle's within 1e-6 relative;
    the mixed-precision run's converged velocity within 1e-4 of the
    oracle's (the per-field table is printed)."""
    from ablsteadyrans_b200.driver import Driver
    runs = {}
    for prec in (0, 1):
        inst = workloads.config0(precision=prec, **CONVERGED_CASE)
        oc = oracle_case(inst)
        dc, st = gpu_stage(ctx, oc, inst)
        try:
            drv = Driver(st)
            status, n = drv.run(6000)
            assert status == "steady", (prec, status, n)
            runs[prec] = {"fields": {f: dc.host(f) for f in FIELDS}, "cfls": [h[0] for h in drv.history],
                          "L": gpu_closure_length(st), "iterations": n}
        finally:
            st.close()
    inst = workloads.config0(precision=0, **CONVERGED_CASE)
    oc = oracle_case(inst)
    oracle.set_threads(oracle.max_threads())
    run_oracle(oc, inst, runs[0]["cfls"])
    g = inst.grid
    v = g.valid(0)
    Lo = closure_length(oc, inst)
    table = {}
    for prec, name in ((0, "fp64"), (1, "fp32_inner")):
        err = field_errors(g, runs[prec]["fields"], oc.q)
        err["L"] = float(np.abs(runs[prec]["L"][v] - Lo[v]).max() / np.abs(Lo[v]).max())
        table[name] = err
    print("converged (config 0 at 8x8x48), GPU vs oracle, iterations", runs[0]["iterations"], runs[1]["iterations"],
          table)
    for f, e in table["fp64"].items():
        assert e <= 1e-6, ("fp64", f, e)
    for f in ("u", "v", "w"):
        assert table["fp32_inner"][f] <= 1e-4, ("fp32_inner", f, table["fp32_inner"][f])
