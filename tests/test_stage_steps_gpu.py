"""The SIMPLEC iteration's steps through their own C-ABI entry points
(gb_momentum_predictor, gb_pressure_correction, gb_scalar_sweep,
gb_implicit_coefficients), each against the oracle's same step: the pieces
the reference's Newton preconditioner and grid-sequencing transfer call
outside SimplecStage::iterate (Source/Predictor.H:242-252,
Source/Simplec.H:139-163, Source/ImplicitOperator.H:65-67)."""
import numpy as np
import pytest

import oracle
from ablsteadyrans_b200.abi import SimplecOptions

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)


def _cases():
    from test_simplec_gpu import make, physics
    from test_turbulence import _hill_case
    case, bc = make("inflow", seed=5)
    yield "inflow-coriolis", case, bc, physics(case, coriolis=1, latitude=40.0, geostrophic=1, ug=7.0, vg=-1.0)
    case, bc, ph = _hill_case()
    yield "hill-closure-wall", case, bc, ph


def _rel(got, ref, v):
    scale = max(float(np.abs(ref[v]).max()), 1e-300)
    return float(np.abs(got[v] - ref[v]).max()) / scale


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1], ids=["inflow-coriolis", "hill-closure-wall"])
def test_gpu_stage_steps_match_oracle(ctx, which):
    """fill_ghosts, residual, momentum_predictor, pressure_correction and the
    two scalar sweeps taken one at a time on the GPU equal the oracle's same
    steps: the predicted velocity, a_P and d, the corrected u, v, w, p, then
    theta and k, with every result struct, to 1e-9 relative (the Poisson
    solve to 1e-11)."""
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    name, case, bc, ph = list(_cases())[which]
    opts = SimplecOptions.make(pressure_reltol=1e-11, zline_sweeps=3, w_vnn_cap=16.0, tke_floor=1e-3)
    oracle.fill_ghosts(case, bc, ph)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, opts)
    g = case.grid
    try:
        st.fill_ghosts()
        dt = st.local_dtau(2.0)
        dt_ref = oracle.local_dtau(case, 2.0, phys=ph)
        assert _rel(dt.cpu().numpy(), dt_ref, g.valid(0)) <= 1e-12
        ref = oracle.stage_steps(case, bc, ph, opts, dt_ref)
        assert ref["status"] == 0
        R = st.residual()
        for n in range(6):
            assert _rel(R[n].cpu().numpy(), ref["R"][n], g.valid(LOCS[n])) <= 1e-11, FIELDS[n]
        pres, ap, d = st.momentum_predictor(R, dt, with_fields=True)
        for c, f in enumerate(("u", "v", "w")):
            v = g.valid(LOCS[c])
            assert _rel(dc.host(f), ref["pred"][f], v) <= 1e-9, ("predictor", f)
            assert _rel(ap[c].cpu().numpy(), ref["ap"][c], v) <= 1e-11, ("ap", f)
            assert _rel(d[c].cpu().numpy(), ref["d"][c], v) <= 1e-11, ("d", f)
        pi = ref["pred_info"]
        got = (pres.max_du, pres.max_dv, pres.max_dw, pres.last_sweep_du, pres.last_sweep_dv, pres.last_sweep_dw)
        for a, b in zip(got, pi):
            assert a == pytest.approx(b, rel=1e-9, abs=1e-15)
        pc = st.pressure_correction()
        for c, f in enumerate(("u", "v", "w", "p")):
            assert _rel(dc.host(f), ref["pc"][f], g.valid(LOCS[c])) <= 1e-9, ("correction", f)
        ci = ref["pc_info"]
        assert pc.divergence_before == pytest.approx(ci[0], rel=1e-9)
        assert pc.divergence_after == pytest.approx(ci[1], rel=1e-6, abs=1e-12)
        assert pc.max_dp == pytest.approx(ci[2], rel=1e-9)
        for a, b in zip((pc.max_du, pc.max_dv, pc.max_dw), ci[3:6]):
            assert a == pytest.approx(b, rel=1e-9, abs=1e-15)
        assert abs(pc.poisson_iterations - int(ci[7])) <= 1
        th = st.scalar_sweep(4, R[4], dt)
        k = st.scalar_sweep(5, R[5], dt)
        for f in ("theta", "tke"):
            assert _rel(dc.host(f), case.q[f], g.valid(0)) <= 1e-9, f
        si = ref["scalar_info"]
        assert th.max_dq == pytest.approx(si[0], rel=1e-9, abs=1e-15)
        assert k.max_dq == pytest.approx(si[2], rel=1e-9, abs=1e-15)
        assert k.clipped == int(si[4])
    finally:
        st.close()


@pytest.mark.gpu
@pytest.mark.parametrize("log_mean", [0, 1])
@pytest.mark.parametrize("loc", [0, 1, 2, 4])
def test_gpu_implicit_coefficients_match_oracle(ctx, loc, log_mean):
    """gb_implicit_coefficients (upwind transport plus the principal
    diffusion with the metric) equals the oracle's coefficients<C> at every
    location, with arithmetic and logarithmic face means, to 1e-13."""
    import torch
    import ablsteadyrans_b200 as gb
    from helpers import terrain_simplec_case
    case = terrain_simplec_case(18, 14, 10, False, True, seed=2)
    g = case.grid
    rng = np.random.default_rng(7 + loc)
    F = [g.np_zeros() + rng.standard_normal(g.shape) for _ in range(3)]
    gamma = g.np_zeros() + rng.uniform(0.5, 3.0, g.shape)
    C = {0: -1, 1: 0, 2: 1, 4: 2}[loc]
    ref = oracle.implicit_coefficients(g, C, F, gamma, case.z, case.J, logz=bool(log_mean))
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    A = torch.zeros((7,) + tuple(g.shape), dtype=torch.float64, device="cuda")
    gb.implicit_coefficients(ctx, g, loc, [dev(f) for f in F], dev(gamma), dev(case.z), dev(case.J), log_mean, A)
    got = A.cpu().numpy()
    v = g.valid(loc)
    for n in range(7):
        scale = max(float(np.abs(ref[n][v]).max()), 1e-300)
        assert float(np.abs(got[n][v] - ref[n][v]).max()) <= 1e-13 * scale, n


@pytest.mark.gpu
@pytest.mark.parametrize("levels", [0, 5])
@pytest.mark.parametrize("loc", [0, 1, 2, 4])
def test_gpu_implicit_coefficients_per_block_faces_match_per_point(ctx, loc, levels):
    """The implicit coefficients with each face's conductance and transport
    evaluated once per block (GB_TUNE_RESIDUAL 0, or N levels per block)
    equal the one-thread-per-point form (GB_TUNE_RESIDUAL 1), which
    evaluates every face from both sides, to 1e-14 relative."""
    import torch
    import ablsteadyrans_b200 as gb
    from helpers import terrain_simplec_case
    case = terrain_simplec_case(41, 13, 12, False, True, seed=4)
    g = case.grid
    rng = np.random.default_rng(11 + loc)
    F = [g.np_zeros() + rng.standard_normal(g.shape) for _ in range(3)]
    gamma = g.np_zeros() + rng.uniform(0.5, 3.0, g.shape)
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    out = []
    try:
        for knob in (1, levels):
            ctx.tune(gb.TUNE_RESIDUAL, knob)
            A = torch.zeros((7,) + tuple(g.shape), dtype=torch.float64, device="cuda")
            gb.implicit_coefficients(ctx, g, loc, [dev(f) for f in F], dev(gamma), dev(case.z), dev(case.J), 1, A)
            out.append(A.cpu().numpy())
    finally:
        ctx.tune(gb.TUNE_RESIDUAL, 0)
    v = g.valid(loc)
    for n in range(7):
        scale = max(float(np.abs(out[0][n][v]).max()), 1e-300)
        assert float(np.abs(out[1][n][v] - out[0][n][v]).max()) <= 1e-14 * scale, n
