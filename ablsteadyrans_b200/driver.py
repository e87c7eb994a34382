"""The pseudo-time driver of a SIMPLEC solve on the host (gust::Driver::step,
Source/Driver.cpp:403-468), the steady criterion (gust::SteadyCriterion,
Source/SteadyCriterion.cpp, through the native gb_criterion) and the loose
stop of grid sequencing (gust::loose_stop, Source/Sequencing.cpp:172-222).

Per iteration: local dtau at the current CFL, one SimplecStage iteration,
the scaled residual norms and the monitors into the criterion; r_n = max
over equations of res / max(res_ref, residual_tol) after the reference hold
(res_ref: each residual's largest value over the first
residual_ref_iterations, or the seed they raise); steady when every residual
is below residual_tol and has dropped residual_drop_orders orders below its
reference and every monitor has settled over its window; otherwise the next
CFL: cfl0 during the hold, then the SER law.
"""
import ctypes
import math

from . import abi

NONFINITE = 2  # gb_status GB_NONFINITE

RESIDUAL_NAMES = ("u", "v", "w", "p", "theta", "tke")


def ser_cfl(cfl, r, cfl0, cfl_max, p, growth):
    """Source/PseudoTime.cpp:53-61: min(cfl_max, growth cfl, cfl0 r^-p)."""
    capped = min(cfl_max, growth * cfl)
    if p == 0:
        return min(capped, cfl0)
    r_min = (cfl0 / cfl_max) ** (1.0 / p)
    if not (r > r_min):
        return capped
    return min(capped, cfl0 * r ** (-p))


def _declare(L):
    if getattr(L, "_gb_criterion", False):
        return
    P = ctypes.c_void_p
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.POINTER(ctypes.c_int32)
    S = ctypes.POINTER(ctypes.c_char_p)
    L.gb_criterion_create.argtypes = [ctypes.POINTER(abi.DriverOptions), ctypes.c_int32, S, ctypes.c_int32, S, D,
                                      ctypes.POINTER(P)]
    L.gb_criterion_destroy.argtypes = [P]
    L.gb_criterion_add.argtypes = [P, D, D]
    L.gb_criterion_seed_reference.argtypes = [P, D]
    L.gb_criterion_verdict.argtypes = [P, I, I, I, ctypes.c_char_p, ctypes.c_int32]
    L.gb_criterion_history.argtypes = [P, ctypes.POINTER(abi.SteadyHistory)]
    L.gb_criterion_monitor_window.argtypes = [P, ctypes.c_int32, D, ctypes.c_int32, I]
    L.gb_sequencing_check.argtypes = [ctypes.POINTER(abi.SequencingOptions), ctypes.POINTER(abi.DriverOptions),
                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.gb_loose_stop.argtypes = [P, ctypes.POINTER(abi.SequencingOptions), ctypes.c_int32, I, ctypes.c_char_p,
                                ctypes.c_int32]
    L._gb_criterion = True


def _L():
    from . import _lib_full
    L = _lib_full()
    _declare(L)
    return L


def _darr(values):
    vals = [float(x) for x in values]
    return (ctypes.c_double * max(len(vals), 1))(*vals)


class Verdict:
    def __init__(self, status, residuals_met, monitors_met, reasons):
        self.status = status                  # abi.NOT_STEADY, STEADY or DIVERGED
        self.residuals_met = residuals_met
        self.monitors_met = monitors_met
        self.reasons = reasons

    @property
    def steady(self):
        return self.status == abi.STEADY


class SteadyCriterion:
    """gust::SteadyCriterion (gb_criterion): params from a DriverOptions
    (residual_* and monitor_*), residual names, monitors as (name, scale)."""

    def __init__(self, options=None, residuals=RESIDUAL_NAMES, monitors=(), handle=None, owner=None):
        from . import check
        self._L = _L()
        self._owner = owner
        if handle is not None:
            # a driver's criterion (the driver owns it)
            self._h = handle
            self._own = False
            return
        o = options or abi.DriverOptions.make()
        rn = (ctypes.c_char_p * max(len(residuals), 1))(*[n.encode() for n in residuals])
        mn = (ctypes.c_char_p * max(len(monitors), 1))(*[m[0].encode() for m in monitors])
        ms = _darr([m[1] for m in monitors])
        self._h = ctypes.c_void_p()
        check(self._L.gb_criterion_create(ctypes.byref(o), len(residuals), rn, len(monitors), mn, ms,
                                          ctypes.byref(self._h)))
        self._own = True
        self.n_residuals, self.n_monitors = len(residuals), len(monitors)

    def add(self, residuals, monitors=()):
        from . import check
        check(self._L.gb_criterion_add(self._h, _darr(residuals), _darr(monitors)))

    def seed_reference(self, ref):
        from . import check
        check(self._L.gb_criterion_seed_reference(self._h, _darr(ref)))

    def verdict(self):
        from . import check
        st, rm, mm = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        buf = ctypes.create_string_buffer(8192)
        check(self._L.gb_criterion_verdict(self._h, ctypes.byref(st), ctypes.byref(rm), ctypes.byref(mm), buf,
                                           len(buf)))
        text = buf.value.decode()
        return Verdict(st.value, bool(rm.value), bool(mm.value), text.split("\n") if text else [])

    def history(self):
        """(count, nonfinite, res_ref, res_last, monitor windows)."""
        from . import check
        h = abi.SteadyHistory()
        check(self._L.gb_criterion_history(self._h, ctypes.byref(h)))
        windows = []
        for m in range(h.n_monitors):
            n = ctypes.c_int32()
            buf = (ctypes.c_double * max(h.monitor_values[m], 1))()
            check(self._L.gb_criterion_monitor_window(self._h, m, buf, len(buf), ctypes.byref(n)))
            windows.append(list(buf)[:n.value])
        return {"count": h.count, "nonfinite": bool(h.nonfinite), "res_ref": list(h.res_ref)[:h.n_residuals],
                "res_last": list(h.res_last)[:h.n_residuals], "monitors": windows}

    @property
    def iterations(self):
        return self.history()["count"]

    def loose_stop(self, seq, hold_iterations):
        """loose_stop (Sequencing.cpp:172-222): (branch, reason); branch
        abi.LOOSE_NONE, LOOSE_RESIDUALS or LOOSE_MONITORS."""
        from . import check
        b = ctypes.c_int32()
        buf = ctypes.create_string_buffer(512)
        check(self._L.gb_loose_stop(self._h, ctypes.byref(seq), int(hold_iterations), ctypes.byref(b), buf, len(buf)))
        return b.value, buf.value.decode()

    def close(self):
        if self._own and self._h:
            self._L.gb_criterion_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def check_sequencing(seq, strict, nx, ny, levels):
    """check_sequencing_options (Sequencing.cpp:120-169): raises GustError
    naming each offending key."""
    from . import check
    check(_L().gb_sequencing_check(ctypes.byref(seq), ctypes.byref(strict), int(nx), int(ny), int(levels)))


def default_cfl_max(line_sweep):
    """Source/Driver.cpp:133-136 (default_cfl_max): 8 with steady.sweep =
    lusgs, 10 with zjacobi."""
    return 8.0 if line_sweep == 1 else 10.0


def stage_monitors(stage):
    """stage_monitor_specs (Simplec.cpp:365-371): (name, scale) of the
    monitors a stage reports."""
    ph = stage.physics
    mon = [("max_speed", ph.scale_velocity), ("mean_tke", ph.scale_tke)]
    if stage.bc.face[2] == abi.FACE_SURFACE_LAYER:
        mon.append(("mean_ustar", 0.1))
    return mon


def info_monitors(info, n):
    return [info.max_speed, info.mean_tke, info.mean_ustar][:n]


class Driver:
    """Drives one SimplecStage to the steady criterion from Python (steady.*
    defaults: cfl0 1, cfl_max the sweep's default, ser_exponent 1,
    ser_max_growth 2); the C++ driver (simplec.NativeDriver) does the same
    with no Python in the loop."""

    def __init__(self, stage, cfl0=1.0, cfl_max=None, ser_exponent=1.0, growth=2.0, options=None):
        self.stage = stage
        if cfl_max is None:
            opts = getattr(stage, "options", None)
            cfl_max = default_cfl_max(getattr(opts, "line_sweep", 0))
        self.cfl0, self.cfl_max, self.p, self.growth = cfl0, cfl_max, ser_exponent, growth
        self.options = options or abi.DriverOptions.make(cfl0=cfl0, cfl_max=cfl_max)
        self.cfl = cfl0
        self.monitors = stage_monitors(stage)
        self.criterion = SteadyCriterion(self.options, RESIDUAL_NAMES, self.monitors)
        self.hold = -1
        self.history = []
        self.dtau = None

    def hold_iterations(self):
        return self.options.residual_ref_iterations if self.hold < 0 else self.hold

    def step(self):
        """One iteration; returns 'steady', 'diverged' or 'running'. An
        iteration that produced non-finite values (GB_NONFINITE) ends the
        solve as diverged, as the criterion's non-finite residual does."""
        from . import GustError
        self.dtau = self.stage.local_dtau(self.cfl, out=self.dtau)
        try:
            info = self.stage.iterate(self.dtau)
        except GustError as e:
            if e.status != NONFINITE:
                raise
            self.history.append((self.cfl, float("nan"), [float("nan")] * 6))
            return "diverged"
        res = list(info.residual_norms)
        self.criterion.add(res, info_monitors(info, len(self.monitors)))
        h = self.criterion.history()
        if h["nonfinite"]:
            self.history.append((self.cfl, float("nan"), res))
            return "diverged"
        r = 1.0
        if h["count"] > self.hold_iterations():
            tol = self.options.residual_tol
            r = max(abs(x) / max(ref, tol) for x, ref in zip(res, h["res_ref"]))
        self.history.append((self.cfl, r, res))
        if self.criterion.verdict().steady:
            return "steady"
        if h["count"] <= self.hold_iterations():
            self.cfl = self.cfl0
        else:
            self.cfl = ser_cfl(self.cfl, r, self.cfl0, self.cfl_max, self.p, self.growth)
        return "running"

    def run(self, max_iterations):
        status = "running"
        for _ in range(max_iterations):
            status = self.step()
            if status != "running":
                break
        return status, len(self.history)
