"""The pseudo-time driver of a SIMPLEC solve on the host (gust::Driver::step,
Source/Driver.cpp:403-468; gust::SteadyCriterion, Source/SteadyCriterion.cpp:
96-224; the SER law gust::ser_cfl, Source/PseudoTime.cpp:53-61).

Per iteration: local dtau at the current CFL, one SimplecStage iteration,
the scaled residual norms into the criterion; r_n = max over equations of
res / max(res_ref, residual_tol) after the reference hold (res_ref: each
residual's largest value over the first residual_ref_iterations); steady when
every residual is below residual_tol and has dropped residual_drop_orders
orders below its reference; otherwise the next CFL from the SER law.
The monitor window test of the reference's criterion is not applied here.
"""
import math

NONFINITE = 2  # gb_status GB_NONFINITE


def ser_cfl(cfl, r, cfl0, cfl_max, p, growth):
    """Source/PseudoTime.cpp:53-61: min(cfl_max, growth cfl, cfl0 r^-p)."""
    capped = min(cfl_max, growth * cfl)
    if p == 0:
        return min(capped, cfl0)
    r_min = (cfl0 / cfl_max) ** (1.0 / p)
    if not (r > r_min):
        return capped
    return min(capped, cfl0 * r ** (-p))


class SteadyCriterion:
    def __init__(self, residual_tol=5e-5, drop_orders=4.0, ref_iterations=5):
        self.residual_tol = residual_tol
        self.drop = 10.0 ** (-drop_orders)
        self.ref_iterations = ref_iterations
        self.res_ref = None
        self.iterations = 0
        self.nonfinite = False

    def add(self, res):
        self.iterations += 1
        if any(not math.isfinite(x) for x in res):
            self.nonfinite = True
            return
        if self.res_ref is None:
            self.res_ref = list(res)
        elif self.iterations <= self.ref_iterations:
            self.res_ref = [max(a, b) for a, b in zip(self.res_ref, res)]

    def relative(self, res):
        if self.iterations <= self.ref_iterations:
            return 1.0
        return max(abs(r) / max(ref, self.residual_tol) for r, ref in zip(res, self.res_ref))

    def steady(self, res):
        if self.nonfinite or self.iterations <= self.ref_iterations:
            return False
        for r, ref in zip(res, self.res_ref):
            if not (r < self.residual_tol) or not (r <= max(ref, self.residual_tol) * self.drop):
                return False
        return True


def default_cfl_max(line_sweep):
    """Source/Driver.cpp:133-136 (default_cfl_max): 8 with steady.sweep =
    lusgs, 10 with zjacobi."""
    return 8.0 if line_sweep == 1 else 10.0


class Driver:
    """Drives one SimplecStage to the steady criterion (steady.* defaults:
    cfl0 1, cfl_max the sweep's default, ser_exponent 1, ser_max_growth 2)."""

    def __init__(self, stage, cfl0=1.0, cfl_max=None, ser_exponent=1.0, growth=2.0, criterion=None):
        self.stage = stage
        if cfl_max is None:
            opts = getattr(stage, "options", None)
            cfl_max = default_cfl_max(getattr(opts, "line_sweep", 0))
        self.cfl0, self.cfl_max, self.p, self.growth = cfl0, cfl_max, ser_exponent, growth
        self.cfl = cfl0
        self.criterion = criterion or SteadyCriterion()
        self.history = []
        self.dtau = None

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
            self.criterion.nonfinite = True
            self.history.append((self.cfl, float("nan"), [float("nan")] * 6))
            return "diverged"
        res = list(info.residual_norms)
        self.criterion.add(res)
        if self.criterion.nonfinite:
            self.history.append((self.cfl, float("nan"), res))
            return "diverged"
        r = self.criterion.relative(res)
        self.history.append((self.cfl, r, res))
        if self.criterion.steady(res):
            return "steady"
        self.cfl = ser_cfl(self.cfl, r, self.cfl0, self.cfl_max, self.p, self.growth)
        return "running"

    def run(self, max_iterations):
        status = "running"
        for _ in range(max_iterations):
            status = self.step()
            if status != "running":
                break
        return status, len(self.history)
