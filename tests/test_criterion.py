"""The native steady criterion (gb_criterion) and the loose stop of grid
sequencing on synthetic histories, pinned to the iterations the reference's
own tests give (test_SteadyCriterion.cpp, test_Sequencing.cpp): converging,
stalling and oscillating histories, divergence, near-zero monitors, the
window boundary, the residual reference and its seed, the released hold,
the parameter and input checks. Host only."""
import math

import pytest

from ablsteadyrans_b200 import GustError, abi
from ablsteadyrans_b200.driver import SteadyCriterion, check_sequencing


def params(**kw):
    return abi.DriverOptions.make(**kw)


def first_steady(c, res, mon, n_max):
    for n in range(n_max):
        c.add([f(n) for f in res], [f(n) for f in mon])
        if c.verdict().status == abi.STEADY:
            return n
    return -1


def mentions(v, s):
    return any(s in r for r in v.reasons)


CONV_RES = [lambda n: 2.0 * 0.8 ** n, lambda n: 0.5 * 0.85 ** n]
CONV_MON = [lambda n: 0.3 + 0.05 * 0.9 ** n, lambda n: 0.4 * (1 - 0.5 * 0.93 ** n)]
CONV_SPEC = [("speedup", 1.0), ("ustar", 1e-6)]


def test_converging_history_is_steady_at_the_pinned_iteration():
    c = SteadyCriterion(params(), ("u", "p"), CONV_SPEC)
    assert first_steady(c, CONV_RES, CONV_MON, 1000) == 136


def test_stalling_history_is_never_steady():
    c = SteadyCriterion(params(), ("u",), [("speedup", 1.0)])
    assert first_steady(c, [lambda n: max(1e-3, 0.8 ** n)], [lambda n: 0.3], 2000) == -1
    v = c.verdict()
    assert v.status == abi.NOT_STEADY
    assert mentions(v, "residual 'u' = 0.001 is not below steady.residual_tol")
    assert mentions(v, "dropped 3 orders")


def test_residual_at_the_tolerance_is_not_below_it():
    p = params()
    at = SteadyCriterion(p, ("u",), [])
    at.add([1.0])
    for _ in range(10):
        at.add([p.residual_tol])
    assert at.verdict().status == abi.NOT_STEADY
    below = SteadyCriterion(p, ("u",), [])
    below.add([1.0])
    below.add([0.98 * p.residual_tol])
    assert below.verdict().status == abi.STEADY


def test_oscillating_monitor_and_residual_are_never_steady():
    c = SteadyCriterion(params(), ("u",), [("speedup", 1.0)])
    assert first_steady(c, [lambda n: 0.8 ** n], [lambda n: 1.0 + 0.005 * math.sin(2 * math.pi * n / 37.0)], 2000) == -1
    v = c.verdict()
    assert len(v.reasons) == 1 and mentions(v, "monitor 'speedup' changed by")
    c2 = SteadyCriterion(params(), ("u",), [])
    assert first_steady(c2, [lambda n: 1e-3 * (1.5 + math.sin(0.3 * n))], [], 2000) == -1


def test_non_finite_values_mean_diverged():
    c = SteadyCriterion(params(), ("u", "k"), [("speedup", 1.0)])
    c.add([1.0, 1.0], [0.3])
    c.add([0.5, float("nan")], [0.3])
    v = c.verdict()
    assert v.status == abi.DIVERGED and mentions(v, "residual 'k' became NaN or infinite")
    for _ in range(200):
        c.add([0.0, 0.0], [0.3])
    assert c.verdict().status == abi.DIVERGED
    d = SteadyCriterion(params(), ("u",), [("ustar", 1.0)])
    d.add([1.0], [float("inf")])
    assert d.verdict().status == abi.DIVERGED and mentions(d.verdict(), "monitor 'ustar'")


def test_near_zero_monitor_uses_its_scale():
    res = [lambda n: 0.0]
    mon = [lambda n: (1.0 if n % 2 else -1.0) * 1e-17]
    assert first_steady(SteadyCriterion(params(), ("u",), [("speedup", 1.0)]), res, mon, 200) == 50
    assert first_steady(SteadyCriterion(params(), ("u",), [("speedup", 1e-20)]), res, mon, 200) == -1


def test_window_needs_all_its_values():
    c = SteadyCriterion(params(), ("u",), [("m", 1.0)])
    for _ in range(50):
        c.add([0.0], [1.0])
    v = c.verdict()
    assert v.status == abi.NOT_STEADY and mentions(v, "50 of the 51 values")
    c.add([0.0], [1.0])
    assert c.verdict().status == abi.STEADY
    # a change of exactly the tolerance passes, one ulp-scale step above does not
    p = params(monitor_window=2, monitor_rel_tol=1.0 / 1024.0)
    at = 1.0 + 1.0 / 1024.0
    above = at + 1.0 / (1024.0 * 1024.0)
    edge = SteadyCriterion(p, ("u",), [("m", 1.0)])
    for x in (at, 1.0, 1.0):
        edge.add([0.0], [x])
    assert edge.verdict().status == abi.STEADY
    over = SteadyCriterion(p, ("u",), [("m", 1.0)])
    for x in (above, 1.0, 1.0):
        over.add([0.0], [x])
    assert over.verdict().status == abi.NOT_STEADY


def test_drop_is_measured_from_the_early_peak():
    res = [lambda n: 1e-2 * 10.0 ** n if n < 3 else 10.0 * 0.7 ** (n - 3)]
    assert first_steady(SteadyCriterion(params(), ("u",), []), res, [], 500) == 38
    assert first_steady(SteadyCriterion(params(residual_ref_iterations=1), ("u",), []), res, [], 500) == 49


@pytest.mark.parametrize("key,kw", [("steady.residual_tol", {"residual_tol": 0.0}),
                                    ("steady.residual_drop_orders", {"residual_drop_orders": -1.0}),
                                    ("steady.residual_ref_iterations", {"residual_ref_iterations": 0}),
                                    ("steady.monitor_rel_tol", {"monitor_rel_tol": float("nan")}),
                                    ("steady.monitor_window", {"monitor_window": 1}),
                                    ("steady.residual_drop_orders", {"residual_drop_orders": 309.0})])
def test_parameter_checks_name_their_keys(key, kw):
    with pytest.raises(GustError, match=key.replace(".", r"\.")):
        SteadyCriterion(params(**kw), ("u",), [])


def test_monitor_scales_and_sizes_are_checked():
    with pytest.raises(GustError, match="scale must be finite and > 0"):
        SteadyCriterion(params(), ("u",), [("m", 0.0)])
    with pytest.raises(GustError, match="residuals"):
        SteadyCriterion(params(), (), [])


def test_slow_monitor_stops_near_its_limit():
    A, r = 0.1, 0.999
    c = SteadyCriterion(params(), ("u",), [("ustar", 1.0)])
    n = first_steady(c, [lambda k: 0.5 ** k], [lambda k: 1.0 + A * r ** k], 10000)
    assert n == 4602
    assert A * r ** n <= 1e-3 * (1.0 + A * r ** n)


@pytest.mark.parametrize("period", [37.0, 100.0, 200.0])
def test_oscillations_up_to_four_windows_are_never_steady(period):
    c = SteadyCriterion(params(), ("u",), [("speedup", 1.0)])
    assert first_steady(c, [lambda k: 0.5 ** k], [lambda k: 1.0 + 0.01 * math.sin(2 * math.pi * k / period)], 5000) == -1


def test_zero_residual_reference_does_not_block():
    c = SteadyCriterion(params(), ("theta",), [("m", 1.0)])
    assert first_steady(c, [lambda k: 0.0 if k < 5 else 1e-16], [lambda k: 1.0], 500) == 50


def test_slowly_growing_monitor_is_not_steady():
    c = SteadyCriterion(params(), ("u",), [("k", 1.0)])
    assert first_steady(c, [lambda k: 0.0], [lambda k: 1.0 + 1e-6 * 1.05 ** k], 120) == -1
    assert mentions(c.verdict(), "is not converging over the window")


# ------------------------------------------------------------ sequencing ---

def seq_params():
    return params(residual_tol=1e-12, residual_drop_orders=4.0, residual_ref_iterations=5, monitor_rel_tol=1e-3,
                  monitor_window=50)


NOISY = [lambda n: 1.1 if n % 2 == 0 else 0.9]
ONE_MON = [("speed", 1.0)]


def first_loose(c, p, seq, res, mon, n_max, hold=-1):
    if hold < 0:
        hold = p.residual_ref_iterations
    for n in range(n_max):
        c.add([f(n) for f in res], [f(n) for f in mon])
        branch, why = c.loose_stop(seq, hold)
        if branch != abi.LOOSE_NONE:
            return n, why
    return -1, ""


def test_loose_residual_branch_stops_at_the_pinned_iteration():
    p = seq_params()
    o = abi.SequencingOptions.make(enabled=1)
    c = SteadyCriterion(p, ("u", "k", "p"), ONE_MON)
    res = [lambda n: 2.0 * 0.9 ** n, lambda n: 1.0 + n if n < 2 else 3.0 * 0.95 ** (n - 2), lambda n: 1e-13]
    n, why = first_loose(c, p, o, res, NOISY, 1000)
    assert n == 92 and "orders below its reference" in why
    assert c.history()["res_ref"][1] == 3.0
    assert c.verdict().status == abi.NOT_STEADY
    o3 = abi.SequencingOptions.make(enabled=1, drop_orders=3.0)
    assert first_loose(SteadyCriterion(p, ("u", "k", "p"), ONE_MON), p, o3, res, NOISY, 1000)[0] == 137


def test_loose_residual_branch_waits_for_the_reference():
    p = seq_params()
    o = abi.SequencingOptions.make(enabled=1)
    c = SteadyCriterion(p, ("u",), ONE_MON)
    assert first_loose(c, p, o, [lambda n: 1.0 if n == 0 else 1e-6], NOISY, 100)[0] == 4


def test_loose_monitor_branch_stops_at_the_pinned_iteration():
    p = seq_params()
    specs = [("speedup", 1.0), ("ustar", 0.1)]
    res = [lambda n: 1.0]
    mon = [lambda n: 1 + 0.5 * 0.9 ** n, lambda n: 0.002 * 0.95 ** n]
    off = abi.SequencingOptions.make(enabled=1)
    assert first_loose(SteadyCriterion(p, ("u",), specs), p, off, res, mon, 2000)[0] == -1
    on = abi.SequencingOptions.make(enabled=1, monitor_tol=0.01)
    n, why = first_loose(SteadyCriterion(p, ("u",), specs), p, on, res, mon, 2000)
    assert n == 88 and "every monitor within" in why
    flat = [lambda n: 1.0, lambda n: 0.0]
    assert first_loose(SteadyCriterion(p, ("u",), specs), p, on, res, flat, 200)[0] == 50
    q = params(residual_tol=1e-12, monitor_window=10, residual_ref_iterations=30)
    assert first_loose(SteadyCriterion(q, ("u",), specs), q, on, res, flat, 200)[0] == 29


def test_non_finite_history_never_stops():
    p = seq_params()
    o = abi.SequencingOptions.make(enabled=1)
    res = [lambda n: 1.0 if n < 5 else 0.0, lambda n: float("inf") if n == 7 else 0.0]
    mon = [lambda n: 1.0]
    assert first_loose(SteadyCriterion(p, ("u", "v"), ONE_MON), p, o, res, mon, 6)[0] == 5
    c2 = SteadyCriterion(p, ("u", "v"), ONE_MON)
    for n in range(200):
        c2.add([res[0](n), res[1](n)], [1.0])
        if n >= 7:
            assert c2.loose_stop(o, p.residual_ref_iterations)[0] == abi.LOOSE_NONE
    assert c2.verdict().status == abi.DIVERGED


def test_seeded_reference_is_the_drop_origin():
    p = seq_params()
    o = abi.SequencingOptions.make(enabled=1)
    res = [lambda n: 1e-2]
    own = SteadyCriterion(p, ("u",), ONE_MON)
    seeded = SteadyCriterion(p, ("u",), ONE_MON)
    seeded.seed_reference([1.0])
    assert first_loose(own, p, o, res, NOISY, 100)[0] == -1
    assert first_loose(seeded, p, o, res, NOISY, 100)[0] == 4
    assert seeded.history()["res_ref"][0] == 1.0
    raised = SteadyCriterion(p, ("u",), ONE_MON)
    raised.seed_reference([1.0])
    raised.add([5.0], [1.0])
    assert raised.history()["res_ref"][0] == 5.0
    with pytest.raises(GustError, match="before the first iteration"):
        raised.seed_reference([1.0])


def test_released_hold_stops_from_the_first_iterations():
    p = seq_params()
    o = abi.SequencingOptions.make(enabled=1)
    res = [lambda n: 1e-2]

    def seeded(pp=p):
        c = SteadyCriterion(pp, ("u",), ONE_MON)
        c.seed_reference([1.0])
        return c

    assert first_loose(seeded(), p, o, res, NOISY, 100, hold=5)[0] == 4
    assert first_loose(seeded(), p, o, res, NOISY, 100, hold=0)[0] == 2
    p1 = params(residual_tol=1e-12, residual_ref_iterations=1)
    assert first_loose(seeded(p1), p1, o, res, NOISY, 100, hold=0)[0] == 0
    falling = [lambda n: 3e-2 if n < 3 else 1e-2]
    assert first_loose(seeded(), p, o, falling, NOISY, 100, hold=0)[0] == 3
    rising = [lambda n: 5.0 if n == 0 else (0.1 if n <= 2 else 4e-2)]
    assert first_loose(seeded(), p, o, rising, NOISY, 100, hold=0)[0] == 3
    om = abi.SequencingOptions.make(enabled=1, monitor_tol=0.01)
    for hold in (0, 5):
        n, why = first_loose(seeded(), p, om, [lambda n: 1.0], [lambda n: 2.0], 100, hold=hold)
        assert n == 50 and "every monitor" in why
    ps = params(residual_tol=1e-12, monitor_window=2)
    assert first_loose(seeded(ps), ps, om, [lambda n: 1.0], [lambda n: 2.0], 100, hold=0)[0] == 4


def test_sequencing_input_checks_name_their_keys():
    p = seq_params()
    ok = abi.SequencingOptions.make(enabled=1)
    check_sequencing(ok, p, 32, 16, 3)
    check_sequencing(ok, p, 32, 16, 4)
    with pytest.raises(GustError, match="at least 2 cells in x and in y on the coarsest level"):
        check_sequencing(ok, p, 32, 16, 5)
    for d in (0.0, -1.0, 4.5, float("nan")):
        with pytest.raises(GustError, match="steady.sequencing_drop_orders"):
            check_sequencing(abi.SequencingOptions.make(enabled=1, drop_orders=d), p, 32, 16, 3)
    check_sequencing(abi.SequencingOptions.make(enabled=1, drop_orders=4.0), p, 32, 16, 3)
    check_sequencing(abi.SequencingOptions.make(enabled=1, monitor_tol=0.0), p, 32, 16, 3)
    for t in (1.0, -0.1, float("nan"), float("inf")):
        with pytest.raises(GustError, match="steady.sequencing_monitor_tol"):
            check_sequencing(abi.SequencingOptions.make(enabled=1, monitor_tol=t), p, 32, 16, 3)
    with pytest.raises(GustError, match="needs mesh.hierarchy_levels >= 2"):
        check_sequencing(ok, p, 32, 16, 1)
    # off, the defaults are not range-checked
    for strict_orders in (1.0, 0.0):
        check_sequencing(abi.SequencingOptions.make(), params(residual_drop_orders=strict_orders), 32, 16, 1)
    for hold in (0, 1):
        check_sequencing(abi.SequencingOptions.make(enabled=1, hold=hold), p, 32, 16, 3)
        o = abi.SequencingOptions.make(enabled=1, hold=hold, cfl_previous=1)
        if hold == 1:
            with pytest.raises(GustError, match="steady.sequencing_cfl_start = previous needs steady.sequencing_hold = 0"):
                check_sequencing(o, p, 32, 16, 3)
        else:
            check_sequencing(o, p, 32, 16, 3)
