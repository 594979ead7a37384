"""Properties of the host clock (``rbsim.scheduler``) and the scheme selector, on the CPU.

These restate solver/test_scheduler.py:83-290 and solver/core/test_schemes.py:11-30.
The equal-step fill never lengthens the scheme's step and never leaves a remainder.
Sync points, frames and slow-process activations are pure schedule arithmetic that
no fast step can move. Re-quantisation inside a span stays within its 1/n bound. Bad
inputs fail loudly. tests/test_host_modules.py already replays the reference
scheduler's own tick sequences exactly. These are the invariants behind them.
"""

from __future__ import annotations

import itertools
import math

import pytest

from rbsim.scheduler import EPS_T, MultiRateScheduler, SlowProcess, fill_span

_EVENTS = [300.0, 137.5, 900.0]  # forcing knots, unsorted as a run passes them
_DTS = [73.3, 41.0, 210.0]


def _const(v):
    return lambda: v


def _cycle(values):
    it = itertools.cycle(values)
    return lambda: next(it)


def _sched(**kw):
    kw.setdefault("end_time", 1200.0)
    kw.setdefault("output_every", 300.0)
    kw.setdefault("events", _EVENTS)
    return MultiRateScheduler(**kw)


def test_the_scheduler_never_lengthens_the_step_the_scheme_asked_for():
    raws = []
    it = itertools.cycle(_DTS)

    def dt_fn():
        raws.append(next(it))
        return raws[-1]

    for tick in _sched().ticks(dt_fn):
        assert tick.dt <= raws[-1] + 1e-12


def test_steps_are_equal_inside_every_span():
    sched = _sched(end_time=1000.0, output_every=250.0, events=[137.0])
    ticks = list(sched.ticks(_const(97.0)))
    syncs = sorted(set(sched.sync_times))
    for a, b in zip(ticks, ticks[1:], strict=False):
        if not any(abs(a.t1 - s) < EPS_T for s in syncs):
            assert b.dt == pytest.approx(a.dt, rel=1e-9), a.t1


def test_the_sync_points_and_frames_do_not_depend_on_the_steps():
    sched = _sched()
    outs = [t.t1 for t in sched.ticks(_cycle(_DTS)) if t.is_output]
    assert outs == pytest.approx([300.0, 600.0, 900.0, 1200.0])
    assert sched.n_frames == 5
    assert sched.sync_times == [300.0, 600.0, 900.0, 1200.0, *_EVENTS, 1200.0]


def test_the_schedule_is_reproducible():
    a = [(t.t0, t.dt, t.t1, t.is_output) for t in _sched().ticks(_cycle(_DTS))]
    b = [(t.t0, t.dt, t.t1, t.is_output) for t in _sched().ticks(_cycle(_DTS))]
    assert a == b


@pytest.mark.parametrize(("span", "dt_raw"),
                         [(100.0, 100.0), (100.0, 250.0), (100.0, 50.0), (100.0, 99.9), (100.0, 51.0),
                          (100.0, 33.4), (100.0, 0.0007)])  # fmt: skip
def test_a_span_is_filled_with_equal_steps_none_longer_than_asked(span, dt_raw):
    ticks = list(MultiRateScheduler(end_time=span, output_every=span).ticks(_const(dt_raw)))
    assert len(ticks) == max(1, math.ceil(span / dt_raw))
    assert all(t.dt <= dt_raw + 1e-12 for t in ticks)
    assert all(t.dt == pytest.approx(ticks[0].dt, rel=1e-9) for t in ticks)
    assert ticks[-1].t1 == pytest.approx(span)


def test_fill_span_never_returns_a_step_above_the_one_asked_for():
    """The ulp case: span / n can round above dt_raw when span / dt_raw is just above an integer."""
    for span, dt_raw in ((0.30000000000000004, 0.1), (1.0000000000000002, 0.5), (7.0, 7.0 / 3.0)):
        dt = fill_span(span, dt_raw)
        assert 0.0 < dt <= dt_raw
    assert fill_span(math.inf, 3.0) == 3.0


def test_a_span_of_two_steps_is_the_worst_case_for_requantisation():
    it = iter([100.0, 60.0, 40.0, 30.0, 25.0] + [25.0] * 100)
    ticks = list(MultiRateScheduler(end_time=100.0, output_every=100.0).ticks(lambda: next(it)))
    assert ticks[-1].t1 == pytest.approx(100.0)
    jumps = [abs(b.dt - a.dt) / a.dt for a, b in zip(ticks, ticks[1:], strict=False)]
    assert max(jumps, default=0.0) <= 0.5 + 1e-12


def test_steps_never_cross_a_sync_point_and_land_on_every_one():
    sched = MultiRateScheduler(end_time=1000.0, output_every=250.0, events=[137.0, 610.0],
                               processes=[SlowProcess("slow", 400.0, lambda t, e: None)])  # fmt: skip
    ticks = list(sched.ticks(_const(97.0)))
    landed = {round(t.t1, 9) for t in ticks}
    for s in sched.sync_times:
        assert not any(t.t0 < s - EPS_T and t.t1 > s + EPS_T for t in ticks), s
        assert round(s, 9) in landed, s
    assert ticks[-1].t1 == pytest.approx(1000.0)


def test_output_ticks_land_on_the_cadence_and_count_the_frames():
    sched = MultiRateScheduler(end_time=900.0, output_every=300.0)
    outs = [t.t1 for t in sched.ticks(_const(37.0)) if t.is_output]
    assert outs == pytest.approx([300.0, 600.0, 900.0]) and len(outs) == sched.n_frames - 1


@pytest.mark.parametrize("dt", [7.0, 60.0, 121.0, 1e9])
def test_slow_activations_are_exact_multiples_whatever_the_fast_step(dt):
    fired = []
    proc = SlowProcess("res", 900.0, lambda t, e: fired.append((t, e)))
    for tick in MultiRateScheduler(end_time=3600.0, output_every=1800.0, processes=[proc]).ticks(_const(dt)):
        for p, elapsed in tick.due:
            p.advance(tick.t1, elapsed)
    assert [t for t, _ in fired] == pytest.approx([900.0, 1800.0, 2700.0, 3600.0])
    assert [e for _, e in fired] == pytest.approx([900.0] * 4)


def test_a_partial_final_interval_invents_no_activation():
    proc = SlowProcess("res", 400.0, lambda t, e: None)
    sched = MultiRateScheduler(end_time=1000.0, output_every=500.0, processes=[proc])
    fired = [(tick.t1, tick.due[0][1]) for tick in sched.ticks(_const(60.0)) if tick.due]
    assert [t for t, _ in fired] == pytest.approx([400.0, 800.0])
    assert [e for _, e in fired] == pytest.approx([400.0, 400.0])


def test_two_processes_at_different_rates_stay_independent():
    sched = MultiRateScheduler(end_time=1200.0, output_every=600.0,
                               processes=[SlowProcess("fast", 300.0, lambda t, e: None),
                                          SlowProcess("slow", 600.0, lambda t, e: None)])  # fmt: skip
    seen = {"fast": [], "slow": []}
    for tick in sched.ticks(_const(55.0)):
        for p, _ in tick.due:
            seen[p.name].append(tick.t1)
    assert seen["fast"] == pytest.approx([300.0, 600.0, 900.0, 1200.0])
    assert seen["slow"] == pytest.approx([600.0, 1200.0])


def test_no_slow_processes_means_the_sync_set_is_outputs_events_and_end():
    sched = MultiRateScheduler(end_time=600.0, output_every=200.0, events=[150.0])
    assert sched.sync_times == [200.0, 400.0, 600.0, 150.0, 600.0]


def test_bad_inputs_fail_loudly():
    with pytest.raises(RuntimeError, match="non-positive timestep"):
        list(MultiRateScheduler(end_time=100.0, output_every=50.0).ticks(_const(0.0)))
    with pytest.raises(ValueError, match="interval must be > 0"):
        SlowProcess("bad", 0.0, lambda t, e: None)
    with pytest.raises(ValueError, match="end_time"):
        MultiRateScheduler(end_time=0.0, output_every=1.0)
    with pytest.raises(ValueError, match="output_every"):
        MultiRateScheduler(end_time=1.0, output_every=0.0)


def test_activations_of_a_slow_process():
    p = SlowProcess("p", 250.0, lambda t, e: None)
    assert p.activations(1000.0) == pytest.approx([250.0, 500.0, 750.0, 1000.0])
    assert p.activations(240.0) == []


def test_get_scheme_dispatches_by_name():
    """solver/core/test_schemes.py:11-30: the two scheme modules, and a ValueError otherwise."""
    from rbsim import get_scheme
    from rbsim.schemes import hllc, local_inertial

    assert get_scheme("local_inertial") is local_inertial and get_scheme("hllc_fv") is hllc
    for mod in (local_inertial, hllc):
        assert callable(mod.compute_dt) and callable(mod.step)
    with pytest.raises(ValueError, match="unknown scheme"):
        get_scheme("nope")


def test_fill_span_properties_over_random_spans():
    """For any span and CFL step: 0 < dt <= dt_raw, a whole number of steps tiles the span, and
    that number is the fewest that respect dt_raw (one more only where span / n rounds up)."""
    hypothesis = pytest.importorskip("hypothesis")
    st = hypothesis.strategies

    @hypothesis.settings(max_examples=400, deadline=None)
    @hypothesis.given(st.floats(1e-3, 1e5), st.floats(1e-4, 1e4))
    def check(span, dt_raw):
        dt = fill_span(span, dt_raw)
        assert 0.0 < dt <= dt_raw
        n = round(span / dt)
        assert abs(n * dt - span) <= 1e-9 * span
        fewest = max(1, math.ceil(span / dt_raw))
        assert n in (fewest, fewest + 1)

    check()
