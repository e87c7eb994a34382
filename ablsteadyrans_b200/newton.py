"""The Newton-Krylov finishing stage on the GPU: the Newton core
(gust::NewtonKrylov, Source/Newton.H, through gb_newton) and the
pseudo-transient continuation around it (gust::Continuation,
Source/Continuation.H, Continuation.cpp), host logic over the native core.

One continuation step from q: dtau = local_dtau(q, CFL_n) (or no pseudo-time
term once the CFL reached cfl_max with newton_dtau_inf_at_cap = 1); the Newton
direction dq from (D + J) dq = -R(q); an Armijo backtracking line search on
|R| = |T^-1 R(fill(q))|_2 (trial point q + lambda dq with k clipped at the
floor): accepted when |R(q + lambda dq)| <= (1 - c lambda) |R(q)|, lambda =
1, backtrack, backtrack^2, ... down to lambda_min; accepted: the SER law for
the next CFL from |R_n| / |R_0|; a skipped update or a rejected search leaves
q as it was, cuts the CFL by newton_cfl_cut and retries, up to
newton_max_retries times, then fails.
"""
import ctypes
import math
import sys

from . import abi
from .driver import ser_cfl


class NewtonOptions(ctypes.Structure):
    """gb_newton_opts: steady.newton_* of the Newton core."""
    _fields_ = [("gmres_restart", ctypes.c_int32), ("gmres_max_iters", ctypes.c_int32),
                ("fd_eps_scale", ctypes.c_double), ("krylov_rtol", ctypes.c_double),
                ("scale_pressure", ctypes.c_double), ("preconditioner", ctypes.c_int32),
                ("inf_cfl", ctypes.c_double)]

    #: steady.newton_preconditioner values
    IDENTITY, SIMPLEC, SIMPLEC_STAGE = 0, 1, 2

    @classmethod
    def make(cls, **kw):
        o = cls(gmres_restart=30, gmres_max_iters=2000, fd_eps_scale=math.sqrt(sys.float_info.epsilon),
                krylov_rtol=1e-2, scale_pressure=100.0, preconditioner=1, inf_cfl=10.0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class NewtonStepInfo(ctypes.Structure):
    _fields_ = [("gmres_iterations", ctypes.c_int32), ("gmres_status", ctypes.c_int32),
                ("residual_norm", ctypes.c_double), ("krylov_residual", ctypes.c_double),
                ("krylov_relative", ctypes.c_double), ("eps_min", ctypes.c_double), ("eps_max", ctypes.c_double),
                ("jvp_calls", ctypes.c_int32), ("applied", ctypes.c_int32)]


def _declare(L):
    if getattr(L, "_gb_newton", False):
        return
    P = ctypes.c_void_p
    PP = ctypes.POINTER(ctypes.c_void_p)
    S = ctypes.POINTER(abi.State)
    L.gb_newton_options_default.argtypes = [ctypes.POINTER(NewtonOptions)]
    L.gb_newton_check.argtypes = [ctypes.POINTER(NewtonOptions)]
    L.gb_newton_create.argtypes = [P, ctypes.POINTER(NewtonOptions), ctypes.POINTER(P)]
    L.gb_newton_destroy.argtypes = [P]
    L.gb_newton_jvp.argtypes = [P, S, PP, PP, ctypes.POINTER(ctypes.c_double)]
    L.gb_newton_step.argtypes = [P, S, P, ctypes.POINTER(NewtonStepInfo)]
    L.gb_newton_direction.argtypes = [P, S, P, PP, ctypes.POINTER(NewtonStepInfo)]
    L.gb_newton_residual_norm.argtypes = [P, S, ctypes.POINTER(ctypes.c_double)]
    L.gb_newton_trial.argtypes = [P, S, PP, ctypes.c_double, S]
    L._gb_newton = True


FIELDS = ("u", "v", "w", "p", "theta", "tke")


def check_newton_options(o):
    """check_newton_options through the library: raises GustError naming
    each offending steady.newton_* key."""
    from . import _lib_full, check
    L = _lib_full()
    _declare(L)
    check(L.gb_newton_check(ctypes.byref(o)))


def _ptrs(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


class NewtonKrylov:
    """gust::NewtonKrylov on a SimplecStage (gb_newton)."""

    def __init__(self, stage, options=None):
        from . import _lib_full, check
        self.stage = stage
        self._L = _lib_full()
        _declare(self._L)
        self.options = options or NewtonOptions.make()
        self._h = ctypes.c_void_p()
        check(self._L.gb_newton_create(stage._h, ctypes.byref(self.options), ctypes.byref(self._h)))
        stage.ctx.own(self)
        stage.own(self)

    def _zeros(self):
        import torch
        return [torch.zeros(self.stage.case.grid.shape, dtype=torch.float64, device="cuda") for _ in FIELDS]

    def jvp(self, v):
        """(J v, eps) at the stage's state, v six device tensors (ghosts 0)."""
        from . import check
        Jv = self._zeros()
        eps = ctypes.c_double()
        st = self.stage.case.state()
        check(self._L.gb_newton_jvp(self._h, ctypes.byref(st), _ptrs(v), _ptrs(Jv), ctypes.byref(eps)))
        return Jv, eps.value

    def step(self, dtau=None):
        from . import check
        info = NewtonStepInfo()
        st = self.stage.case.state()
        check(self._L.gb_newton_step(self._h, ctypes.byref(st), None if dtau is None else ctypes.c_void_p(dtau.data_ptr()),
                                     ctypes.byref(info)))
        return info

    def direction(self, state, dtau, dq):
        from . import check
        info = NewtonStepInfo()
        check(self._L.gb_newton_direction(self._h, ctypes.byref(state),
                                          None if dtau is None else ctypes.c_void_p(dtau.data_ptr()), _ptrs(dq),
                                          ctypes.byref(info)))
        return info

    def residual_norm(self, state=None):
        from . import check
        st = state if state is not None else self.stage.case.state()
        r = ctypes.c_double()
        check(self._L.gb_newton_residual_norm(self._h, ctypes.byref(st), ctypes.byref(r)))
        return r.value

    def trial(self, q0, dq, lam, out):
        from . import check
        check(self._L.gb_newton_trial(self._h, ctypes.byref(q0), _ptrs(dq), float(lam), ctypes.byref(out)))

    def close(self):
        if self._h:
            self._L.gb_newton_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ continuation ---

class ContinuationOptions:
    """steady.* of the continuation (gust::ContinuationOptions,
    Source/Continuation.H:63-80): the driver's SER keys and the new ones."""

    def __init__(self, cfl0=1.0, cfl_max=10.0, ser_exponent=1.0, ser_max_growth=2.0, armijo_c=1e-4, backtrack=0.5,
                 lambda_min=1e-2, cfl_cut=0.25, max_retries=4, dtau_inf_at_cap=1, ptc_growth=1.0):
        self.cfl0, self.cfl_max, self.ser_exponent, self.ser_max_growth = cfl0, cfl_max, ser_exponent, ser_max_growth
        self.armijo_c, self.backtrack, self.lambda_min, self.cfl_cut = armijo_c, backtrack, lambda_min, cfl_cut
        self.max_retries, self.dtau_inf_at_cap, self.ptc_growth = max_retries, dtau_inf_at_cap, ptc_growth


def check_continuation_options(o):
    """check_continuation_options (Continuation.cpp:101-140): one message per
    violation naming steady.<key>."""
    err = []

    def bad(x):
        return x is None or math.isnan(x) or math.isinf(x)
    if bad(o.cfl0) or not o.cfl0 > 0:
        err.append(f"steady.cfl0 = {o.cfl0}: must be finite and > 0")
    if bad(o.cfl_max) or not o.cfl_max >= o.cfl0:
        err.append(f"steady.cfl_max = {o.cfl_max}: must be finite and >= steady.cfl0")
    if bad(o.ser_exponent) or not o.ser_exponent >= 0:
        err.append(f"steady.ser_exponent = {o.ser_exponent}: must be finite and >= 0")
    if bad(o.ser_max_growth) or not o.ser_max_growth >= 1:
        err.append(f"steady.ser_max_growth = {o.ser_max_growth}: must be finite and >= 1")
    for key, x, hi in (("newton_armijo_c", o.armijo_c, 0.5), ("newton_backtrack", o.backtrack, 1.0),
                       ("newton_lambda_min", o.lambda_min, 1.0), ("newton_cfl_cut", o.cfl_cut, 1.0)):
        if x is None or math.isnan(x) or not (0 < x < hi):
            err.append(f"steady.{key} = {x}: must be > 0 and < {hi:g}")
    if o.max_retries < 1:
        err.append(f"steady.newton_max_retries = {o.max_retries}: must be an integer >= 1")
    if o.dtau_inf_at_cap not in (0, 1):
        err.append(f"steady.newton_dtau_inf_at_cap = {o.dtau_inf_at_cap}: must be 0 or 1")
    if o.ptc_growth is None or math.isnan(o.ptc_growth) or math.isinf(o.ptc_growth) or not o.ptc_growth >= 1:
        err.append(f"steady.newton_ptc_growth = {o.ptc_growth}: must be finite and >= 1")
    return err


def armijo_accepts(r_trial, r, lam, c):
    """Continuation.cpp:175-178: r_trial finite and <= (1 - c lambda) r."""
    return math.isfinite(r_trial) and r_trial <= (1.0 - c * lam) * r


class LineSearchResult:
    def __init__(self):
        self.accepted, self.lam, self.backtracks, self.residual, self.by_growth = False, 1.0, 0, 0.0, False


def armijo_line_search(phi, r, o, growth=1.0):
    """armijo_line_search (Continuation.cpp:180-206): lambda = 1, backtrack,
    ... while >= lambda_min; with growth > 1 a full step whose |R| grew by at
    most that factor is accepted (phi(1) evaluated again last)."""
    ls = LineSearchResult()
    r_full = 0.0
    while True:
        ls.residual = phi(ls.lam)
        if ls.lam == 1:
            r_full = ls.residual
        if armijo_accepts(ls.residual, r, ls.lam, o.armijo_c):
            ls.accepted = True
            return ls
        nxt = o.backtrack * ls.lam
        if not nxt >= o.lambda_min:
            break
        ls.lam = nxt
        ls.backtracks += 1
    if growth > 1 and math.isfinite(r_full) and r_full <= growth * r:
        ls.lam = 1.0
        ls.residual = phi(ls.lam)
        ls.accepted = True
        ls.by_growth = True
    return ls


class ContinuationState:
    def __init__(self, cfl):
        self.steps, self.cfl, self.infinite, self.r0, self.r_last = 0, cfl, False, 0.0, 0.0

    def copy(self):
        s = ContinuationState(self.cfl)
        s.steps, s.infinite, s.r0, s.r_last = self.steps, self.infinite, self.r0, self.r_last
        return s


def continuation_after_accept(o, st, r_new):
    """Continuation.cpp:208-217."""
    st = st.copy()
    st.steps += 1
    st.r_last = r_new
    r = r_new / st.r0 if st.r0 > 0 else 0.0
    frm = o.cfl_max if st.infinite else st.cfl
    st.cfl = ser_cfl(frm, r, o.cfl0, o.cfl_max, o.ser_exponent, o.ser_max_growth)
    st.infinite = o.dtau_inf_at_cap == 1 and st.cfl >= o.cfl_max
    return st


def continuation_after_failure(o, st):
    """Continuation.cpp:219-226: the CFL cut (from infinite dtau: cfl_cut
    cfl_max), floored at the smallest normal double."""
    st = st.copy()
    st.cfl = max(o.cfl_cut * (o.cfl_max if st.infinite else st.cfl), sys.float_info.min)
    st.infinite = False
    return st


def line_search_growth(o, st):
    return 1.0 if st.infinite else o.ptc_growth


class Continuation:
    """gust::Continuation on a SimplecStage: step() and run(); the stage's
    state (its DeviceCase) is q."""

    def __init__(self, stage, options=None, newton_options=None, verbose=0):
        import torch
        from . import GustError
        self.o = options or ContinuationOptions()
        err = check_continuation_options(self.o)
        if err:
            raise GustError(1, "gust: Continuation: invalid inputs:\n  " + "\n  ".join(err))
        self.stage = stage
        self.nk = NewtonKrylov(stage, newton_options)
        self.st = ContinuationState(self.o.cfl0)
        self.records = []
        self.verbose = verbose
        g = stage.case.grid
        z = lambda: torch.zeros(g.shape, dtype=torch.float64, device="cuda")     # noqa: E731
        self._qb = {f: z() for f in FIELDS}
        self._qt = {f: z() for f in FIELDS}
        self._dq = [z() for _ in FIELDS]
        self._dtau = z()

    def _state(self, d):
        return abi.State(*[d[f].data_ptr() for f in FIELDS], self.stage.case.z.data_ptr())

    def set_reference_residual(self, r0):
        if not (math.isfinite(r0) and r0 > 0):
            from . import GustError
            raise GustError(1, "gust: Continuation::set_reference_residual: needs a finite |R_0| > 0")
        self.st.r0 = r0

    def step(self):
        """One continuation step with its retries: 'accepted' or 'failed'."""
        q = self.stage.case.q
        for attempt in range(self.o.max_retries + 1):
            rec = {"step": self.st.steps, "attempt": attempt, "cfl": self.st.cfl, "infinite": self.st.infinite}
            for f in FIELDS:
                self._qb[f].copy_(q[f])
            qb = self._state(self._qb)
            self.stage._fill_state(qb)
            dtau = None
            if not self.st.infinite:
                self.stage.local_dtau_of(qb, self.st.cfl, self._dtau)
                dtau = self._dtau
            info = self.nk.direction(qb, dtau, self._dq)
            rec.update(residual=info.residual_norm, residual_new=info.residual_norm,
                       gmres_iterations=info.gmres_iterations, gmres_status=info.gmres_status,
                       krylov_relative=info.krylov_relative)
            finite_r = math.isfinite(info.residual_norm)
            if self.st.r0 == 0 and finite_r:
                self.st.r0 = info.residual_norm
            if finite_r and info.residual_norm == 0:
                rec["outcome"] = "accepted"
                self.records.append(rec)
                self.st = continuation_after_accept(self.o, self.st, 0.0)
                return "accepted"
            if info.applied:
                r = info.residual_norm
                qt = self._state(self._qt)

                def phi(lam):
                    self.nk.trial(qb, self._dq, lam, qt)
                    return self.nk.residual_norm(qt)
                ls = armijo_line_search(phi, r, self.o, line_search_growth(self.o, self.st))
                rec.update(lam=ls.lam, backtracks=ls.backtracks, residual_new=ls.residual, by_growth=ls.by_growth)
                if ls.accepted:
                    for f in FIELDS:
                        q[f].copy_(self._qt[f])
                    rec["outcome"] = "accepted"
                    self.records.append(rec)
                    self._log(rec)
                    self.st = continuation_after_accept(self.o, self.st, ls.residual)
                    return "accepted"
                rec["outcome"] = "rejected"
            else:
                rec["outcome"] = "skipped"
            self.records.append(rec)
            self._log(rec)
            self.st = continuation_after_failure(self.o, self.st)
        return "failed"

    def run(self, max_steps, rel_tol):
        """Steps until |R| <= rel_tol |R_0| (checked before each step), a
        failed step or max_steps steps: (status, converged, steps)."""
        status, steps = "accepted", 0
        for _ in range(max_steps):
            if self.st.steps > 0 and self.st.r_last <= rel_tol * self.st.r0:
                return status, True, steps
            status = self.step()
            if status == "failed":
                return status, False, steps
            steps += 1
        return status, self.st.steps > 0 and self.st.r_last <= rel_tol * self.st.r0, steps

    def _log(self, rec):
        if self.verbose:
            print("gust: PTC", rec)

    def close(self):
        self.nk.close()


# ------------------------------------------------------------ the stage ---

class SwitchOptions:
    """steady.switch_* and newton_fallback_failures of the two-stage driver
    (Source/Driver.H:60-80): forward to Newton after switch_window
    iterations with r_n <= switch_residual; back to SIMPLEC after
    fallback_failures consecutive failed continuation steps."""

    def __init__(self, switch_residual=1e-4, switch_window=20, fallback_failures=2):
        self.switch_residual, self.switch_window, self.fallback_failures = switch_residual, switch_window, fallback_failures


def newton_equations_differ(stage):
    """NewtonStage::differs (NewtonStage.cpp:196-205) for what this build
    has. (1) The Newton stage's residuals take the smooth counterpart of the
    van Leer limiter, van Albada (gb_newton; Smoothness.cpp:54-67), so with
    van Leer the stage solves other equations than the run's. (2) With the
    closure and turb.nut_relax < 1 the residual blends nu_t with the history
    of the last SIMPLEC iteration, which the Newton stage does not update.
    (The frozen k-floor switches, the reference's third reason, are not
    built: the Newton stage runs live floor decisions.) The stage always has
    a history here: SIMPLEC iterated for the switch window before the Newton
    stage began."""
    from .abi import LIMITER_VAN_LEER
    ph = stage.physics
    if int(ph.limiter) == LIMITER_VAN_LEER:
        return True
    return bool(ph.closure) and ph.turb_nut_relax < 1.0


def newton_stage_action(verdict, idle, monitor_window, status, converged_now, differs, failures, fallback_failures):
    """What the two-stage driver does after one Newton-stage iteration, in the
    reference's order: the criterion's verdict first (Driver::step,
    Driver.cpp:403-468: a steady or diverged verdict ends the run whatever
    the stage asks), then the stage's requests (NewtonStage::iterate,
    NewtonStage.cpp:127-178): a hand-back for good after sitting converged
    for more than steady.monitor_window iterations (idle) or after
    converging on equations that differ from the run's (differs), the
    fall-back after steady.newton_fallback_failures failed steps. verdict:
    "steady", "diverged" or "running"; status: the continuation step's
    outcome. Returns (action, reason): action "steady", "diverged",
    "hand_back", "fallback" or "continue"."""
    if verdict in ("steady", "diverged"):
        return verdict, ""
    if idle > monitor_window:
        return "hand_back", "Newton converged but the steady criterion did not hold for steady.monitor_window iterations"
    if failures >= fallback_failures:
        return "fallback", f"{failures} consecutive failed Newton steps"
    if status == "accepted" and converged_now and differs:
        return "hand_back", ("Newton converged on its own equations, which differ from the run's (the smooth limiter, "
                             "or turb.nut_relax < 1): the final SIMPLEC pass")
    return "continue", ""


def solve_simplec_newton(stage, max_iterations, driver_options=None, switch=None, newton_options=None,
                         continuation_options=None, events=None):
    """steady.stage = simplec_newton on one stage: the native SIMPLEC driver
    until the switch rule holds, then one continuation step per iteration
    (started afresh at cfl_max, as the reference's Newton stage starts its
    continuation), the run's norms and monitors at each new state into the
    driver's criterion, back to SIMPLEC after the failures. As the reference's
    NewtonStage::iterate (NewtonStage.cpp:127-178), the stage hands the run
    back to SIMPLEC for good (no later switch, so the run ends on SIMPLEC)
    when it has converged on equations that differ from the run's
    (newton_equations_differ), or when it has converged but the criterion
    has not held for steady.monitor_window further iterations. `events`, a
    list, receives (iteration, from, to, reason) per switch. Returns
    (verdict, iterations, newton_iterations)."""
    from .simplec import NativeDriver
    d = NativeDriver(stage, driver_options)
    crit = d.criterion
    sw = switch or SwitchOptions()
    o = d.options
    copt = continuation_options or ContinuationOptions(cfl0=o.cfl_max, cfl_max=o.cfl_max,
                                                       ser_exponent=o.ser_exponent, ser_max_growth=o.ser_max_growth)
    mode, below, failures, newton_its = "simplec", 0, 0, 0
    handed_back, idle = False, 0
    cont = None
    n_mon = 3 if stage.bc.face[2] == abi.FACE_SURFACE_LAYER else 2
    drop = 10.0 ** (-o.residual_drop_orders)

    def switch_to(it, to, reason):
        if events is not None:
            events.append((it + 1, mode, to, reason))
        return to

    try:
        for it in range(max_iterations):
            if mode == "simplec":
                verdict, _, _ = d.step()
                if verdict != "running":
                    return verdict, it + 1, newton_its
                _, _, r = d.status()
                below = below + 1 if r <= sw.switch_residual else 0
                if below >= sw.switch_window and not handed_back:
                    mode, failures, idle = switch_to(it, "newton", "switch_residual held"), 0, 0
                    if cont is not None:
                        cont.close()
                    cont = Continuation(stage, copt, newton_options)
                continue
            # once the continuation has converged on the run's equations
            # (|R| <= 10^-residual_drop_orders |R_0|) no step is taken: the
            # norms fill the criterion's monitor window (NewtonStage.H)
            done = cont.st.steps > 0 and cont.st.r0 > 0 and cont.st.r_last <= drop * cont.st.r0
            if done:
                idle += 1
                status = "accepted"
            else:
                status = cont.step()
                newton_its += 1
            failures = failures + 1 if status == "failed" else 0
            res, mon = stage.norms()
            crit.add(res, mon[:n_mon])
            v = crit.verdict()
            verdict = "diverged" if v.status == abi.DIVERGED else ("steady" if v.status == abi.STEADY else "running")
            converged_now = (not done and status == "accepted" and cont.st.steps > 0 and cont.st.r0 > 0
                             and cont.st.r_last <= drop * cont.st.r0)
            action, reason = newton_stage_action(verdict, idle, o.monitor_window, status, converged_now,
                                                 newton_equations_differ(stage), failures, sw.fallback_failures)
            if action in ("steady", "diverged"):
                return action, it + 1, newton_its
            if action == "hand_back":
                handed_back = True
                mode, below = switch_to(it, "simplec", reason), 0
            elif action == "fallback":
                mode, below = switch_to(it, "simplec", reason), 0
        return "running", max_iterations, newton_its
    finally:
        if cont is not None:
            cont.close()
        d.close()


def main(argv=None):
    """SIMPLEC alone against SIMPLEC with the Newton finishing stage on the
    config-1 hill, both to the strict criterion:
    python -m ablsteadyrans_b200.newton --nx 64 --nz 32"""
    import argparse
    import json
    import time

    import torch

    import ablsteadyrans_b200 as gb
    from . import workloads
    from .sequencing import _finest
    from .simplec import NativeDriver, run_drivers
    ap = argparse.ArgumentParser(description="the Newton finishing stage against SIMPLEC alone")
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--max-iterations", type=int, default=4000)
    ap.add_argument("--switch-residual", type=float, default=1e-4)
    ap.add_argument("--switch-window", type=int, default=20)
    ap.add_argument("--restart", type=int, default=60)
    N = NewtonOptions
    ap.add_argument("--preconditioner", type=int, default=N.SIMPLEC, choices=[N.IDENTITY, N.SIMPLEC, N.SIMPLEC_STAGE],
                    help="0 identity, 1 SIMPLEC (a_P denominators, the default), 2 SIMPLEC (the stage's)")
    args = ap.parse_args(argv)
    names = {N.IDENTITY: "identity", N.SIMPLEC: "SIMPLEC (a_P denominators)",
             N.SIMPLEC_STAGE: "SIMPLEC (stage denominators)"}
    out = {"workload": f"config 1: 150 m Gaussian hill {args.nx}x{args.nx}x{args.nz}, dx 25 m, the k-L closure and "
                       f"the surface layer; the Newton stage's preconditioner: {names[args.preconditioner]}"}
    for mode in ("simplec", "simplec_newton"):
        inst = workloads.config1(args.nx, args.nx, args.nz)
        ctx = gb.Context()
        case, stage = _finest(ctx, inst)
        stage.initialize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if mode == "simplec":
            d = NativeDriver(stage)
            (verdict, n), = run_drivers([d], args.max_iterations, 1)
            nn = 0
            d.close()
        else:
            verdict, n, nn = solve_simplec_newton(
                stage, args.max_iterations, switch=SwitchOptions(args.switch_residual, args.switch_window),
                newton_options=NewtonOptions.make(gmres_restart=args.restart, preconditioner=args.preconditioner))
        torch.cuda.synchronize()
        out[mode] = {"verdict": verdict, "iterations": n, "newton_iterations": nn, "seconds": time.perf_counter() - t0}
        res, _ = stage.norms()
        out[mode]["final_residual_norms"] = res
        stage.close()
        ctx.close()
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
