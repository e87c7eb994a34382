"""The Newton-Krylov finishing stage: the continuation's line search, SER
ramp and retries on known answers (test_Continuation.cpp), the option checks,
and on the GPU the jvp against the oracle's residual difference, Poiseuille
in one Newton step (test_Newton.cpp) and continuation steps that reduce |R|
over a hill with the closure and the wall law."""
import math
import sys

import numpy as np
import pytest

import oracle
from ablsteadyrans_b200 import GustError
from ablsteadyrans_b200.abi import LIMITER_VAN_ALBADA, LIMITER_VAN_LEER
from ablsteadyrans_b200.driver import ser_cfl
from ablsteadyrans_b200.newton import (ContinuationOptions, ContinuationState, NewtonOptions, armijo_accepts,
                                       armijo_line_search, check_continuation_options, check_newton_options,
                                       continuation_after_accept, continuation_after_failure, line_search_growth)

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = (1, 2, 4, 0, 0, 0)


@pytest.mark.parametrize("K,c,beta,lmin,lam,nb,acc", [(3, 1e-4, 0.5, 1e-2, 0.25, 2, True),
                                                      (3, 1e-4, 0.3, 1e-2, 0.3, 1, True),
                                                      (0.5, 1e-4, 0.5, 1e-2, 1, 0, True),
                                                      (1.5, 0.4, 0.5, 1e-2, 0.25, 2, True),
                                                      (9, 1e-4, 0.5, 1e-2, 0.0625, 4, True),
                                                      (100, 1e-4, 0.5, 0.05, 0.0625, 4, False)])
def test_armijo_on_known_quadratic(K, c, beta, lmin, lam, nb, acc):
    o = ContinuationOptions(armijo_c=c, backtrack=beta, lambda_min=lmin)
    r = 7.0
    calls = []
    ls = armijo_line_search(lambda l: calls.append(l) or r * (1 - l + K * l * l), r, o)
    lstar = (1 - c) / K
    expect, n = 1.0, 0
    while expect > lstar and expect * beta >= lmin:
        expect *= beta
        n += 1
    assert ls.accepted == acc == (expect <= lstar)
    assert abs(ls.lam - lam) < 1e-15 and abs(ls.lam - expect) < 1e-15
    assert ls.backtracks == nb == n and len(calls) == n + 1


def test_armijo_non_finite_trials_and_growth_bound():
    o = ContinuationOptions()
    nan, inf = float("nan"), float("inf")
    ls = armijo_line_search(lambda l: nan if l > 0.3 else (inf if l > 0.2 else 1.0), 2.0, o)
    assert ls.accepted and ls.lam == 0.125 and ls.backtracks == 3
    assert not armijo_accepts(nan, 1, 1, 1e-4) and not armijo_accepts(inf, 1, 1, 1e-4)
    assert armijo_accepts(0.5, 1, 1, 0.5) and not armijo_accepts(math.nextafter(0.5, 1), 1, 1, 0.5)
    g = ContinuationOptions(lambda_min=0.05)
    r = 2.0
    for growth in (100.0, math.nextafter(100.0, 0.0), 1.0):
        calls = []
        lg = armijo_line_search(lambda l: calls.append(l) or r * (1 - l + 100 * l * l), r, g, growth)
        accept = growth >= 100.0
        assert lg.accepted == accept and lg.by_growth == accept and lg.backtracks == 4
        assert len(calls) == (6 if accept else 5) and calls[-1] == (1.0 if accept else 0.0625)
        if accept:
            assert lg.lam == 1 and lg.residual == 100 * r
    assert not armijo_line_search(lambda l: nan, r, g, 1e30).accepted


def test_dtau_ramp_follows_ser():
    """continuation_after_accept: the SER law from |R_n| / |R_0|, growth
    capped, the switch to infinite dtau at cfl_max (and cfl_max as the base
    while infinite); a failure cuts the CFL and leaves infinite dtau."""
    o = ContinuationOptions(cfl0=1.0, cfl_max=50.0, ser_exponent=1.0, ser_max_growth=2.0)
    st = ContinuationState(o.cfl0)
    st.r0 = 1.0
    cfl = o.cfl0
    for n, rn in enumerate([0.9, 0.5, 0.2, 0.05, 0.01, 1e-3, 1e-4]):
        expect = ser_cfl(cfl, rn, o.cfl0, o.cfl_max, o.ser_exponent, o.ser_max_growth)
        st = continuation_after_accept(o, st, rn)
        assert st.steps == n + 1 and st.r_last == rn and st.cfl == expect
        assert st.infinite == (expect >= o.cfl_max)
        cfl = expect
    assert st.infinite
    f = continuation_after_failure(o, st)
    assert not f.infinite and f.cfl == o.cfl_cut * o.cfl_max
    st2 = ContinuationState(1e-307)
    for _ in range(5):
        st2 = continuation_after_failure(o, st2)
    assert st2.cfl == sys.float_info.min
    assert line_search_growth(ContinuationOptions(ptc_growth=3.0), st) == 1.0
    assert line_search_growth(ContinuationOptions(ptc_growth=3.0), f) == 3.0


@pytest.mark.parametrize("key,kw", [("steady.newton_armijo_c", {"armijo_c": 0.5}),
                                    ("steady.newton_backtrack", {"backtrack": 1.0}),
                                    ("steady.newton_lambda_min", {"lambda_min": float("nan")}),
                                    ("steady.newton_cfl_cut", {"cfl_cut": 0.0}),
                                    ("steady.newton_max_retries", {"max_retries": 0}),
                                    ("steady.newton_dtau_inf_at_cap", {"dtau_inf_at_cap": 2}),
                                    ("steady.newton_ptc_growth", {"ptc_growth": 0.5}),
                                    ("steady.cfl_max", {"cfl_max": 0.5})])
def test_continuation_range_checks_name_their_keys(key, kw):
    assert check_continuation_options(ContinuationOptions()) == []
    err = check_continuation_options(ContinuationOptions(**kw))
    assert len(err) == 1 and key in err[0]


@pytest.mark.parametrize("key,kw", [("steady.newton_gmres_restart", {"gmres_restart": 4}),
                                    ("steady.newton_gmres_restart", {"gmres_restart": 201}),
                                    ("steady.newton_gmres_max_iters", {"gmres_max_iters": 0}),
                                    ("steady.newton_fd_eps_scale", {"fd_eps_scale": 1e-13}),
                                    ("steady.newton_fd_eps_scale", {"fd_eps_scale": 0.02}),
                                    ("steady.newton_krylov_rtol", {"krylov_rtol": 1.0})])
def test_newton_option_checks_name_their_keys(key, kw):
    check_newton_options(NewtonOptions.make())
    with pytest.raises(GustError, match=key.replace(".", r"\.")):
        check_newton_options(NewtonOptions.make(**kw))


# ------------------------------------------------------------------ GPU ---

@pytest.mark.parametrize("case,want", [
    # the criterion first: steady or diverged ends the run whatever the stage asks
    (dict(verdict="steady", idle=9, status="accepted", converged_now=True, differs=True, failures=0), "steady"),
    (dict(verdict="diverged", idle=0, status="failed", converged_now=False, differs=False, failures=5), "diverged"),
    # converged on equations that differ from the run's: the final SIMPLEC pass
    (dict(verdict="running", idle=0, status="accepted", converged_now=True, differs=True, failures=0), "hand_back"),
    # converged on the run's own equations: no hand-back, the window fills
    (dict(verdict="running", idle=0, status="accepted", converged_now=True, differs=False, failures=0), "continue"),
    # converged and idle past the monitor window: hand back
    (dict(verdict="running", idle=6, status="accepted", converged_now=False, differs=False, failures=0), "hand_back"),
    (dict(verdict="running", idle=5, status="accepted", converged_now=False, differs=False, failures=0), "continue"),
    # failed steps: the fall-back (not for good)
    (dict(verdict="running", idle=0, status="failed", converged_now=False, differs=True, failures=2), "fallback"),
    (dict(verdict="running", idle=0, status="failed", converged_now=False, differs=True, failures=1), "continue"),
])
def test_newton_stage_action_follows_the_reference_order(case, want):
    """The two-stage driver's decision after a Newton-stage iteration
    (Driver.cpp:403-468, NewtonStage.cpp:127-178), monitor window 5, two
    failures to fall back."""
    from ablsteadyrans_b200.newton import newton_stage_action
    action, reason = newton_stage_action(monitor_window=5, fallback_failures=2, **case)
    assert action == want, (action, reason)
    if action == "hand_back":
        assert reason


@pytest.mark.parametrize("limiter,closure,relax,want", [(0, 0, 1.0, True), (1, 0, 1.0, False), (2, 0, 1.0, False),
                                                        (1, 1, 0.5, True), (1, 1, 1.0, False)])
def test_newton_equations_differ_with_the_smooth_limiter(limiter, closure, relax, want):
    """NewtonStage::differs (NewtonStage.cpp:196-205): van Leer's smooth
    counterpart makes the Newton stage's equations differ from the run's;
    van Albada and upwind are their own counterparts; turb.nut_relax < 1
    with the closure differs too."""
    from types import SimpleNamespace
    from ablsteadyrans_b200.newton import newton_equations_differ
    stage = SimpleNamespace(physics=SimpleNamespace(limiter=limiter, closure=closure, turb_nut_relax=relax))
    assert newton_equations_differ(stage) is want


def _hill():
    from test_turbulence import _hill_case
    return _hill_case()


@pytest.mark.gpu
def test_gpu_jvp_matches_the_oracle_difference(ctx):
    """J v on the GPU equals the oracle's (R(fill(q + eps v)) - R(fill(q))) /
    eps at the GPU's eps (the closure and the wall law, refilled ghosts),
    R with the Newton stage's smooth limiter."""
    import torch
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.newton import NewtonKrylov
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    from helpers import seam_sync
    case, bc, ph = _hill()
    g = case.grid
    rng = np.random.default_rng(3)
    v = []
    for f, loc in zip(FIELDS, LOCS):
        a = g.np_zeros()
        a[g.valid(loc)] = rng.standard_normal(a[g.valid(loc)].shape) * (0.3 if f != "p" else 3.0)
        seam_sync(g, loc, a)
        v.append(a)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make())
    nk = NewtonKrylov(st)
    try:
        Jv, eps = nk.jvp([torch.from_numpy(a).cuda() for a in v])
        assert eps > 0
        # the Newton stage's residual inputs: van Leer's smooth counterpart
        # (Smoothness.cpp:54-67)
        phs = type(ph).from_buffer_copy(ph)
        if phs.limiter == LIMITER_VAN_LEER:
            phs.limiter = LIMITER_VAN_ALBADA
        oracle.fill_ghosts(case, bc, phs)
        R0 = oracle.residual(case, bc, phs)
        qp = case.copy()
        for n, f in enumerate(FIELDS):
            qp.q[f] = case.q[f] + eps * v[n]
        oracle.fill_ghosts(qp, bc, phs)
        Rp = oracle.residual(qp, bc, phs)
        for n, loc in enumerate(LOCS):
            vv = g.valid(loc)
            ref = (Rp[n][vv] - R0[n][vv]) / eps
            got = Jv[n].cpu().numpy()[vv]
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(got - ref).max() <= 1e-4 * scale, (FIELDS[n], np.abs(got - ref).max() / scale)
    finally:
        nk.close()
        st.close()


@pytest.mark.gpu
def test_gpu_newton_residuals_take_the_smooth_limiter(ctx):
    """Every residual of the Newton stage takes van Leer's smooth counterpart
    (Smoothness.cpp:54-67): its norm on a van Leer stage equals the norm on
    the same state of a stage built with van Albada, bit for bit; the
    stage's own residual afterwards is its van Leer residual again, which
    differs from van Albada's on this hill."""
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.newton import NewtonKrylov
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc, ph = _hill()
    assert ph.limiter == LIMITER_VAN_LEER
    pha = type(ph).from_buffer_copy(ph)
    pha.limiter = LIMITER_VAN_ALBADA
    stages = []
    try:
        for p in (ph, pha, ph):
            st = SimplecStage(ctx, DeviceCase.from_oracle(case), bc, p, SimplecOptions.make())
            st.fill_ghosts()
            stages.append(st)
        leer, albada, fresh = stages
        before, _ = leer.norms()
        nk_leer, nk_albada = NewtonKrylov(leer), NewtonKrylov(albada)
        assert nk_leer.residual_norm() == nk_albada.residual_norm()
        after, _ = leer.norms()
        own, _ = fresh.norms()
        other, _ = albada.norms()
        assert list(after) == list(before) == list(own)
        assert list(after) != list(other)
    finally:
        for st in reversed(stages):
            st.close()


@pytest.mark.gpu
def test_gpu_poiseuille_in_one_newton_step(ctx):
    """Laminar Poiseuille flow (R linear in the column): one plain Newton
    step from rest with GMRES to 1e-12 gives the discrete solution to 1e-9 of
    the peak; v and w stay 0 and theta unchanged (Newton.PoiseuilleInOneStep)."""
    from ablsteadyrans_b200.abi import (BC, FACE_NO_SLIP_WALL, FACE_PERIODIC, Physics, SimplecOptions)
    from ablsteadyrans_b200.newton import NewtonKrylov
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    from helpers import flat_case
    H, F, nu, nz = 500.0, 1e-4, 10.0, 16
    case = flat_case(2, 2, nz, 1000.0, 1000.0, H, True, True, nu)
    bc = BC.make((FACE_PERIODIC, FACE_PERIODIC, FACE_NO_SLIP_WALL, FACE_PERIODIC, FACE_PERIODIC, FACE_NO_SLIP_WALL),
                 theta_ref=((-1000.0, 5000.0), (300.0, 300.0)))
    ph = Physics.make(H, gravity=0.0, pressure_gradient=(F, 0.0, 0.0))
    case.q["theta"][...] = 300.0
    case.q["tke"][...] = 0.5
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make())
    nk = NewtonKrylov(st, NewtonOptions.make(gmres_restart=100, krylov_rtol=1e-12))
    try:
        info = nk.step(None)
        assert info.gmres_status == 0 and info.jvp_calls > 0 and info.applied
        G = case.grid.ng
        dz = H / nz
        zc = (np.arange(nz) + 0.5) * dz
        exact = F / (2 * nu) * (zc * (H - zc) + dz * dz / 4)
        umax = F * H * H / (8 * nu)
        u = dc.host("u")[G:G + nz, G:G + 2, G:G + 3]
        assert np.abs(u - exact[:, None, None]).max() < 1e-9 * umax
        assert np.abs(dc.host("v")[case.grid.valid(2)]).max() < 1e-12 * umax
        assert np.abs(dc.host("w")[case.grid.valid(4)]).max() < 1e-12 * umax
        th = dc.host("theta")[case.grid.valid(0)]
        assert th.min() == 300.0 and th.max() == 300.0
    finally:
        nk.close()
        st.close()


@pytest.mark.gpu
def test_gpu_continuation_reduces_the_residual(ctx):
    """Over the hill with the closure and the wall law, after SIMPLEC
    iterations: every accepted continuation step lowers |R| (the Armijo
    condition), and five steps take it well below where they started. The
    run takes van Albada, so SIMPLEC and the Newton stage (which replaces
    van Leer by it) iterate on the same equations."""
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.newton import Continuation
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc, ph = _hill()
    ph.limiter = LIMITER_VAN_ALBADA
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(pressure_reltol=1e-6))
    st.fill_ghosts()
    for _ in range(40):
        st.iterate(st.local_dtau(2.0))
    cont = Continuation(st, ContinuationOptions(cfl0=2.0, cfl_max=50.0),
                        NewtonOptions.make(gmres_restart=60, krylov_rtol=1e-3))
    try:
        r_start = cont.nk.residual_norm()
        status, converged, steps = cont.run(5, 1e-12)
        acc = [r for r in cont.records if r["outcome"] == "accepted"]
        assert status == "accepted" and steps == 5 and len(acc) == 5
        for r in acc:
            assert r["residual_new"] <= (1 - 1e-4 * r["lam"]) * r["residual"]
        assert cont.st.r_last < 0.5 * r_start
        for f, loc in zip(FIELDS, LOCS):
            assert np.isfinite(dc.host(f)[case.grid.valid(loc)]).all(), f
    finally:
        cont.close()
        st.close()


@pytest.mark.gpu
def test_gpu_simplec_newton_reaches_the_strict_criterion(ctx):
    """steady.stage = simplec_newton over the hill: SIMPLEC until r_n has
    stayed at or below the switch residual, then the continuation; the run
    ends steady by the driver's own criterion, with Newton iterations."""
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.newton import SwitchOptions, solve_simplec_newton
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc, ph = _hill()
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(pressure_reltol=1e-6))
    st.fill_ghosts()
    try:
        from ablsteadyrans_b200.abi import DriverOptions
        verdict, its, newton_its = solve_simplec_newton(
            st, 3000, driver_options=DriverOptions.make(monitor_window=5), switch=SwitchOptions(1e-2, 5),
            newton_options=NewtonOptions.make(gmres_restart=60, gmres_max_iters=300))
        assert verdict == "steady", (verdict, its, newton_its)
        assert newton_its > 0
        res, _ = st.norms()
        assert max(res) < 5e-5
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_newton_hands_back_when_nut_relax_blends_the_history(ctx):
    """With turb.nut_relax < 1 the Newton stage's equations blend nu_t with a
    frozen SIMPLEC history, so they are not the run's: once the continuation
    has converged on them the stage hands the run back to SIMPLEC for good
    (NewtonStage::differs, NewtonStage.cpp:196-205 and 169-177) unless the
    criterion holds at that iteration (the driver checks it first); the run
    ends steady, and after a hand-back it never switches to Newton again."""
    from ablsteadyrans_b200.abi import DriverOptions, SimplecOptions
    from ablsteadyrans_b200.newton import SwitchOptions, newton_equations_differ, solve_simplec_newton
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc, ph = _hill()
    ph.turb_nut_relax = 0.5
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(pressure_reltol=1e-6))
    st.fill_ghosts()
    assert newton_equations_differ(st)
    events = []
    try:
        verdict, its, newton_its = solve_simplec_newton(
            st, 4000, driver_options=DriverOptions.make(monitor_window=5), switch=SwitchOptions(1e-2, 5),
            newton_options=NewtonOptions.make(gmres_restart=60, gmres_max_iters=300), events=events)
        assert verdict == "steady", (verdict, its, events)
        assert newton_its > 0
        to_newton = [e for e in events if e[2] == "newton"]
        back = [e for e in events if e[2] == "simplec" and "differ" in e[3]]
        assert len(back) <= 1, events
        if back:
            # no switch to Newton after the hand-back: the run ends on SIMPLEC
            assert all(e[0] < back[0][0] for e in to_newton), events
            assert events[-1] == back[0], events
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_simplec_preconditioner_apply_is_one_simplec_iteration(ctx):
    """With the stage's SIMPLEC denominators the preconditioner applied to
    r = -R(q) is the increment of one iteration of the stage from q, off the
    Dirichlet rows of u, v, w (NewtonPreconditioner.ApplyIsOneSimplecIteration):
    the same predictor rows, the pressure correction of du* after the
    homogeneous fill against that of u* = q + du* after the full fill (the
    fills are linear without a wall law), theta's coupling and the scalar
    steps on the corrected transport. Inflow, outflow, Coriolis and
    gravity; the Poisson solves to 1e-11."""
    import torch
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    from test_simplec_gpu import make, physics
    case, bc = make("inflow", seed=5)
    ph = physics(case, coriolis=1, latitude=40.0, geostrophic=1, ug=7.0, vg=-1.0)
    case.q["tke"][...] = np.abs(case.q["tke"]) + 0.3
    opts = SimplecOptions.make(pressure_reltol=1e-11, zline_sweeps=3, tke_floor=1e-6)
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, opts)
    g = case.grid
    try:
        st.fill_ghosts()
        dt = st.local_dtau(2.0)
        R = st.residual()
        r = [-x for x in R]
        q0 = {f: dc.host(f) for f in FIELDS}
        dq = [t.cpu().numpy() for t in st.precondition(r, dtau=dt, denominators=2)]
        for f in FIELDS:     # the preconditioner leaves the state alone
            assert np.array_equal(dc.host(f), q0[f]), f
        st.iterate(dt)
        G = g.ng
        for n, (f, loc) in enumerate(zip(FIELDS, LOCS)):
            v = list(g.valid(loc))
            # off the Dirichlet rows: the boundary points of the normal velocity
            if loc in (1, 2, 4):
                d = {1: 2, 2: 1, 4: 0}[loc]
                sl = v[d]
                v[d] = slice(sl.start + 1, sl.stop - 1)
            v = tuple(v)
            inc = dc.host(f)[v] - q0[f][v]
            scale = max(float(np.abs(inc).max()), 1e-300)
            err = float(np.abs(dq[n][v] - inc).max()) / scale
            assert err <= 1e-7, (f, err)
    finally:
        st.close()


@pytest.mark.gpu
def test_gpu_simplec_preconditioner_cuts_the_gmres_iterations(ctx):
    """Over the hill with the closure and the wall law, after SIMPLEC
    iterations: one Newton direction at CFL 10 with the SIMPLEC
    preconditioner (the SIMPLE denominators, the default) converges to the
    Krylov tolerance and is usable, in fewer FGMRES iterations than the
    identity takes (which may reach its cap of 600)."""
    from ablsteadyrans_b200.abi import SimplecOptions
    from ablsteadyrans_b200.newton import NewtonKrylov
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    case, bc, ph = _hill()
    dc = DeviceCase.from_oracle(case)
    st = SimplecStage(ctx, dc, bc, ph, SimplecOptions.make(pressure_reltol=1e-6))
    try:
        st.fill_ghosts()
        for _ in range(30):
            st.iterate(st.local_dtau(2.0))
        dt = st.local_dtau(10.0)
        its = {}
        for pre in (NewtonOptions.IDENTITY, NewtonOptions.SIMPLEC):
            nk = NewtonKrylov(st, NewtonOptions.make(gmres_restart=60, gmres_max_iters=600, krylov_rtol=1e-2,
                                                     preconditioner=pre))
            try:
                dq = nk._zeros()
                info = nk.direction(st.case.state(), dt, dq)
                its[pre] = (info.gmres_iterations, info.gmres_status, info.applied)
            finally:
                nk.close()
        print("GMRES iterations (iterations, status, applied):", its)
        s_its, s_status, s_applied = its[NewtonOptions.SIMPLEC]
        assert s_status == 0 and s_applied, its
        # the identity may stop at the cap (600) without converging
        assert s_its < its[NewtonOptions.IDENTITY][0], its
    finally:
        st.close()
