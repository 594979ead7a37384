"""The reference's sync-point gates (validation/test_clamp_ripple.py) on the CPU oracle.

The scheduler under test is this package's ``rbsim.scheduler.MultiRateScheduler``.
It is the host clock the scheme API runs on, and the device clock replays its step
sequence. It drives the oracle's local-inertial step over the uniform one-row reach
of tests/morph_gates.py with the bump removed, so the reach should stay flat and
steady. The scheduler fills each span to a sync point with equal steps. If it
instead took full steps plus a short remainder, the abrupt shorten-then-restore
would excite a cell-to-cell standing mode in the depth. The mass balance cannot see
that mode, but the second difference of the depth along the reach can. The
thresholds are the reference's: 5 mm of curvature, a mean step-to-step change in dt
below 1 %, and no step longer than the scheme's own CFL step.

``test_the_curvature_gate_catches_a_remainder_step`` plants that defect on the CPU
in a test-local span fill. It shows that the curvature and dt-jump gates fail on it.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from functools import lru_cache

import numpy as np
import pytest

from backends import OracleBackend
from morph_gates import MASS_GATE, Reach
from rbsim.scheduler import EPS_T, MultiRateScheduler

CURVATURE_MM = 5.0
DT_JUMP = 0.01
END_S = 2400.0  # 1200 s to reach normal depth, then 1200 s measured
CADENCES = (45.0, 11.25)
LI = "local_inertial"
_EAST_OPEN = {"east": "open", "west": "closed", "north": "closed", "south": "closed"}


@pytest.fixture(scope="module", autouse=True)
def _pow_mode():
    import oracle

    yield
    oracle.set_pow_mode(0)


@dataclass(frozen=True)
class Ripple:
    depth: np.ndarray  # (nx,) final depth, float64
    dts: np.ndarray  # every step taken, in order
    raw_ratio: float  # largest dt / (the scheme's own CFL dt) over the run
    mass_rel_error: float
    interior: slice

    @property
    def curvature_mm(self) -> float:
        """max |second difference of depth| over the interior, in mm."""
        return 1000.0 * float(np.abs(np.diff(self.depth[self.interior], 2)).max())

    def mean_dt_jump(self, after_s: float = 2000.0) -> float:
        """Mean relative change of dt between adjacent steps once the reach is steady."""
        tail = self.dts[np.cumsum(self.dts) > after_s]
        return float((np.abs(np.diff(tail)) / tail[:-1]).mean()) if tail.size > 1 else 0.0


def _remainder_ticks(end_s: float, cadence: float, dt_fn):
    """The defect, for the planted-mistake test only: full steps, then a short remainder."""
    t = 0.0
    while t < end_s - EPS_T:
        sync = min(end_s, cadence * (math.floor((t + EPS_T) / cadence) + 1))
        dt = min(float(dt_fn()), sync - t)
        yield t, dt
        t += dt


def _scheduler_ticks(end_s: float, cadence: float | None, dt_fn):
    sched = MultiRateScheduler(end_time=end_s, output_every=end_s if cadence is None else cadence)
    for tick in sched.ticks(dt_fn):
        yield tick.t0, tick.dt


@lru_cache(maxsize=None)
def drive(cadence: float | None, planted: bool = False) -> Ripple:
    be = OracleBackend()
    fx = Reach(bump_m=0.0)
    st = be.make(fx.bed(), fx.dx, depth=fx.normal_depth, manning=fx.manning)
    be.set_bc(st, _EAST_OPEN)
    q_in = fx.unit_q * fx.dx
    inj = be.injector([((0, 0), [(0.0, q_in), (1.0e9, q_in)])], st)
    led = be.ledger(st)
    raws: list[float] = []

    def dt_fn() -> float:
        raws.append(be.compute_dt(st, LI, 0.7, 5.0))
        return raws[-1]

    ticks = _remainder_ticks(END_S, cadence, dt_fn) if planted else _scheduler_ticks(END_S, cadence, dt_fn)
    dts, worst = [], 0.0
    for t0, dt in ticks:
        worst = max(worst, dt / raws[-1])
        led.add_inflow(inj.apply(st, t0, dt))
        be.step(st, LI, dt)
        dts.append(dt)
    led.record(st, END_S)
    return Ripple(be.h(st)[0].astype(np.float64), np.asarray(dts), worst, led.max_rel_error, fx.interior)


@pytest.mark.parametrize("cadence", CADENCES)
def test_a_frequent_sync_cadence_does_not_ripple_the_reach(cadence):
    """validation/test_clamp_ripple.py:235."""
    r = drive(cadence)
    assert r.mass_rel_error < MASS_GATE
    assert r.curvature_mm < CURVATURE_MM, r.curvature_mm


def test_the_answer_does_not_depend_on_how_often_the_clock_is_interrupted():
    """validation/test_clamp_ripple.py:260: every cadence lands within 5 mm of the uninterrupted run."""
    control = drive(None)
    assert control.curvature_mm < CURVATURE_MM
    for c in CADENCES:
        r = drive(c)
        delta = 1000.0 * float(np.abs(r.depth[r.interior] - control.depth[control.interior]).max())
        assert delta < CURVATURE_MM, (c, delta)


@pytest.mark.parametrize("cadence", CADENCES)
def test_no_step_is_a_small_fraction_of_its_neighbour(cadence):
    """validation/test_clamp_ripple.py:291."""
    assert drive(cadence).mean_dt_jump() < DT_JUMP


def test_the_step_never_exceeds_the_cfl_limit_against_a_real_scheme():
    """validation/test_clamp_ripple.py:314: dt <= the state-derived dt on every step."""
    assert drive(11.25).raw_ratio <= 1.0 + 1e-12


def test_the_curvature_gate_catches_a_remainder_step():
    """A remainder-step span fill (the defect) trips both gates at a 45 s cadence."""
    bad = drive(45.0, planted=True)
    assert bad.mass_rel_error < MASS_GATE  # the mass balance cannot see it
    assert bad.curvature_mm > CURVATURE_MM, bad.curvature_mm
    assert bad.mean_dt_jump() > DT_JUMP
