"""The reference's edge gates, re-expressed against a backend.

These restate ``validation/test_fixed_stage.py`` (the prescribed-stage ghost: inert
at equilibrium, a source that fills a dry domain from each edge, a sink that drains
into the limiter regime with exact banking, tracking a time-varying level) and
``validation/test_hllc_boundaries.py`` (each open edge drains its own way, a full
drain to empty under the mass gate, a closed wall that reflects a moving slab, and a
steady channel at its Manning normal depth), and the local-inertial half of
``validation/test_channel_flow.py`` (an open edge that never over-drains, a channel
near normal depth). The thresholds are the reference tests'. The drivers are this
build's own.

``EDGE_GATES`` maps a name to a gate that takes a backend from tests/backends.py.
"""

from __future__ import annotations

import math

import numpy as np

from backends import as_f64

MASS_GATE = 1.0e-6
H_DRY = 1.0e-3
HLLC = "hllc_fv"
EDGES = ("north", "south", "east", "west")


def _only(edge: str, kind: str) -> dict[str, str]:
    return {e: (kind if e == edge else "closed") for e in EDGES}


def _toward(edge: str, ny: int, nx: int, high: float) -> np.ndarray:
    """A bed falling linearly from ``high`` on the far side to 0 at ``edge``."""
    col = np.linspace(0.0, 1.0, nx)[None, :] * np.ones((ny, 1))
    row = np.linspace(0.0, 1.0, ny)[:, None] * np.ones((1, nx))
    frac = {"east": 1.0 - col, "west": col, "south": 1.0 - row, "north": row}[edge]
    return (high * frac).astype(np.float32)


def _run_hllc(be, st, t_end, *, alpha=0.45, dt_max=5.0, records=20):
    """HLLC steps to ``t_end`` (the last one shortened), the ledger recorded ``records`` times."""
    led = be.ledger(st)
    every = t_end / records
    t, mark = 0.0, every
    while t < t_end - 1e-9:
        dt = min(be.compute_dt(st, HLLC, alpha, dt_max), t_end - t)
        be.step(st, HLLC, dt, t=t)
        t += dt
        if t >= mark - 1e-9:
            led.record(st, t)
            mark += every
    led.record(st, t)
    return led


# --- prescribed stage --------------------------------------------------------- #
def gate_stage_equilibrium_is_at_rest(be):
    """validation/test_fixed_stage.py:79 -- a surface already at the stage stays at rest.

    600 s on a wavy bed with the east edge held at the surface: |u, v| < 1e-4 m/s,
    mass closed, and almost nothing banked through the edge either way.
    """
    ny = nx = 24
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    bed = (0.02 * xx + 0.3 * np.sin(0.6 * xx) * np.cos(0.4 * yy)).astype(np.float32)
    surface = float(bed.max()) + 0.4
    st = be.make(bed, 10.0, depth=(surface - as_f64(bed)).astype(np.float32), manning=0.0)
    be.set_bc(st, _only("east", "fixed_stage"), {"east": [(0.0, surface)]})
    led = _run_hllc(be, st, 600.0)
    u, v = be.velocities(st)
    assert max(float(np.abs(u).max()), float(np.abs(v).max())) < 1.0e-4
    assert led.max_rel_error < MASS_GATE
    assert abs(be.loss_volume(st)) < 1e-3 * led.v0


def _stage_fill(be, edge):
    """validation/test_fixed_stage.py:110 -- a stage edge fills a dry domain to its level."""
    ny = nx = 20
    bed = _toward(edge, ny, nx, 1.0)
    level = 0.5
    st = be.make(bed, 10.0, depth=0.0, manning=0.03)
    be.set_bc(st, _only(edge, "fixed_stage"), {edge: [(0.0, level)]})
    led = _run_hllc(be, st, 1800.0, dt_max=2.0)
    h = be.h(st)
    wet = h > 10 * H_DRY
    assert np.isfinite(h).all() and h.min() >= 0.0, edge
    assert led.max_rel_error < MASS_GATE, edge
    assert -be.loss_volume(st) > 0.0, f"{edge}: nothing entered through the stage edge"
    expect = int((bed < level - 0.05).sum())
    assert abs(int(wet.sum()) - expect) <= 0.25 * expect, (edge, int(wet.sum()), expect)
    assert float(np.abs((h + bed)[wet] - level).max()) < 0.05, edge


def gate_stage_fills_from_north(be):
    _stage_fill(be, "north")


def gate_stage_fills_from_south(be):
    _stage_fill(be, "south")


def gate_stage_fills_from_east(be):
    _stage_fill(be, "east")


def gate_stage_fills_from_west(be):
    _stage_fill(be, "west")


def gate_stage_drains_with_exact_banking(be):
    """validation/test_fixed_stage.py:143 -- a low stage drains a ramp into the dry regime.

    More than half the water leaves through the edge, more than 40 % of the cells
    dry out, the mass gate holds, and what is left stands at most 5 cm above the stage.
    """
    ny = nx = 20
    bed = _toward("east", ny, nx, 1.0)
    h0 = np.maximum(0.9 - bed, 0.0).astype(np.float32)
    st = be.make(bed, 10.0, depth=h0, manning=0.03)
    be.set_bc(st, _only("east", "fixed_stage"), {"east": [(0.0, 0.1)]})
    led = _run_hllc(be, st, 3600.0, dt_max=2.0)
    h = be.h(st)
    wet = h > 10 * H_DRY
    assert np.isfinite(h).all() and h.min() >= 0.0
    assert led.max_rel_error < MASS_GATE
    assert be.loss_volume(st) > 0.5 * led.v0
    assert float((h <= H_DRY).mean()) > 0.4
    assert not wet.any() or float((h + bed)[wet].max()) < 0.15


def gate_stage_time_varying_level_is_followed(be):
    """validation/test_fixed_stage.py:179 -- the interior rises and falls with the stage.

    A flat 12 x 30 basin with its west edge at 0.2 -> 0.8 -> 0.2 m over 30 min: the
    mean depth, sampled every 300 s, peaks above 0.45 m and ends below half its peak.
    """
    ny, nx = 12, 30
    curve = [(0.0, 0.2), (900.0, 0.8), (1800.0, 0.2)]
    st = be.make(np.zeros((ny, nx), np.float32), 10.0, depth=0.2, manning=0.03)
    be.set_bc(st, _only("west", "fixed_stage"), {"west": curve})
    led = be.ledger(st)
    means, t = [], 0.0
    while t < 1800.0 - 1e-9:
        dt = min(be.compute_dt(st, HLLC, 0.45, 2.0), 1800.0 - t)
        be.step(st, HLLC, dt, t=t)
        t += dt
        if len(means) < int(t / 300.0):
            led.record(st, t)
            means.append(float(be.h(st).mean()))
    led.record(st, t)
    assert led.max_rel_error < MASS_GATE
    peak = max(means)
    assert peak > 0.45 and means[-1] < 0.5 * peak, means


# --- open edges and walls ------------------------------------------------------ #
def _sloped(ny, nx, dx, edge, slope):
    """A bed falling toward ``edge`` at ``slope``, zero on that edge."""
    i = np.arange(ny)[:, None] * np.ones((1, nx))
    j = np.ones((ny, 1)) * np.arange(nx)[None, :]
    run = {"east": nx - 1 - j, "west": j, "south": ny - 1 - i, "north": i}[edge]
    return (run * slope * dx).astype(np.float32)


def _open_drain(be, edge):
    """validation/test_hllc_boundaries.py:71 -- each open edge drains its own way.

    200 steps from a metre of water on a 0.5 % slope: every cell still wet (this
    isolates the banking sign from the limiter), mass closed, more than half the
    water out through that edge.
    """
    st = be.make(_sloped(24, 24, 10.0, edge, 0.005), 10.0, depth=1.0, manning=0.03)
    be.set_bc(st, _only(edge, "open"))
    led = be.ledger(st)
    t = 0.0
    for _ in range(200):
        dt = be.compute_dt(st, HLLC, 0.45, 5.0)
        be.step(st, HLLC, dt)
        t += dt
    rec = led.record(st, t)
    h = be.h(st)
    assert np.isfinite(h).all() and h.min() > H_DRY, edge
    assert led.max_rel_error < MASS_GATE, edge
    assert rec.outflow_cum > 0.5 * led.v0 and rec.volume < 0.5 * led.v0, edge


def gate_hllc_open_north_drains(be):
    _open_drain(be, "north")


def gate_hllc_open_south_drains(be):
    _open_drain(be, "south")


def gate_hllc_open_east_drains(be):
    _open_drain(be, "east")


def gate_hllc_open_west_drains(be):
    _open_drain(be, "west")


def gate_hllc_drains_to_empty(be):
    """validation/test_hllc_boundaries.py:110 -- a tilted basin empties under the mass gate.

    400 steps on a 2 % slope open to the east, the ledger recorded every 40 steps:
    more than half the cells dry, less than 5 % of the water left, more than 90 % of
    it banked as outflow.
    """
    st = be.make(_sloped(24, 24, 10.0, "east", 0.02), 10.0, depth=0.4, manning=0.025)
    be.set_bc(st, _only("east", "open"))
    led = be.ledger(st)
    t = 0.0
    for k in range(400):
        dt = be.compute_dt(st, HLLC, 0.45, 5.0)
        be.step(st, HLLC, dt)
        t += dt
        if k % 40 == 0:
            led.record(st, t)
    rec = led.record(st, t)
    h = be.h(st)
    assert np.isfinite(h).all() and h.min() >= 0.0
    assert int((h < H_DRY).sum()) > 0.5 * h.size
    assert rec.volume < 0.05 * led.v0 and rec.outflow_cum > 0.9 * led.v0
    assert led.max_rel_error < MASS_GATE


def _throw_slab(be, boundaries):
    """A 1 m slab moving east at 3 m/s in a 4 x 60 channel, 80 HLLC steps."""
    ny, nx, h0, u0 = 4, 60, 1.0, 3.0
    st = be.make(np.zeros((ny, nx), np.float32), 5.0, depth=h0, manning=0.0)
    if boundaries is not None:
        be.set_bc(st, boundaries)
    be.set_hu(st, np.full((ny, nx), h0 * u0, np.float32), np.zeros((ny, nx), np.float32))
    led = be.ledger(st)
    v0 = float(be.h(st).sum())
    min_u, max_h, t = u0, h0, 0.0
    for _ in range(80):
        dt = be.compute_dt(st, HLLC, 0.45, 2.0)
        be.step(st, HLLC, dt)
        t += dt
        u, _ = be.velocities(st)
        min_u = min(min_u, float(np.asarray(u).min()))
        max_h = max(max_h, float(be.h(st).max()))
    led.record(st, t)
    h = be.h(st)
    return v0, float(h.sum()), min_u, max_h, float(h.min()), led.max_rel_error


def gate_hllc_closed_wall_reflects(be):
    """validation/test_hllc_boundaries.py:159 -- a wall piles the slab up and sends it back.

    Closed edges: no depth lost (1e-6), a pile-up above 1.5 m and a reversed flow.
    The same slab with every edge open passes through: no pile-up above 1.2 m, the
    flow keeps more than half its speed, and the banked outflow closes the ledger.
    """
    v0, v, min_u, max_h, h_min, _ = _throw_slab(be, None)
    assert np.isfinite([v, h_min, min_u, max_h]).all() and h_min >= 0.0
    assert abs(v - v0) < 1e-6 * v0
    assert max_h > 1.5 and min_u < 0.0
    _, _, min_u_o, max_h_o, _, mass_o = _throw_slab(be, {e: "open" for e in EDGES})
    assert max_h_o < 1.2 and min_u_o > 1.5 and mass_o < MASS_GATE


def gate_hllc_channel_normal_depth(be):
    """validation/test_hllc_boundaries.py:221 -- a steady channel settles at Manning normal depth.

    A 1 x 120 channel on a 2 % slope, 2 m^3/s into the head cell, the toe open: after
    8000 steps the interior median depth is within 2 % of (q n / sqrt(S))^(3/5), every
    cell is wet, water leaves the toe, and mass closes.
    """
    nx, dx, slope, n, discharge = 120, 10.0, 0.02, 0.03, 2.0
    bed = ((nx - 1 - np.arange(nx)) * dx * slope).reshape(1, nx).astype(np.float32)
    st = be.make(bed, dx, depth=0.0, manning=n)
    be.set_bc(st, _only("east", "open"))
    inj = be.injector([((0, 0), [(0.0, discharge), (1.0e9, discharge)])], st)
    led = be.ledger(st)
    t = 0.0
    for _ in range(8000):
        dt = be.compute_dt(st, HLLC, 0.45, 10.0)
        led.add_inflow(inj.apply(st, t, dt))
        be.step(st, HLLC, dt)
        t += dt
    rec = led.record(st, t)
    h_n = (discharge / dx * n / math.sqrt(slope)) ** 0.6
    h = be.h(st)[0]
    assert np.isfinite(h).all() and h.min() > H_DRY
    assert led.max_rel_error < MASS_GATE and rec.outflow_cum > 0.0
    assert abs(float(np.median(h[10 : nx - 10])) - h_n) < 0.02 * h_n


# --- the local-inertial open edge (validation/test_channel_flow.py) ------------- #
LI = "local_inertial"


def gate_li_open_edge_drains_and_stays_nonnegative(be):
    """validation/test_channel_flow.py:38 -- a 2 % basin open to the east, 2000 steps.

    The capped edge sink cannot over-drain: depth never below -1e-6 m, mass closed,
    more than half the water out through the edge.
    """
    ny, nx, dx = 20, 40, 10.0
    st = be.make(_sloped(ny, nx, dx, "east", 0.02), dx, depth=0.5, manning=0.03)
    be.set_bc(st, _only("east", "open"))
    led = be.ledger(st)
    t = 0.0
    for _ in range(2000):
        dt = be.compute_dt(st, LI, 0.7, 5.0)
        be.step(st, LI, dt)
        t += dt
    rec = led.record(st, t)
    h = be.h(st)
    assert np.isfinite(h).all() and h.min() >= -1e-6
    assert led.max_rel_error < MASS_GATE
    assert rec.outflow_cum > 0.5 * led.v0 and rec.volume < 0.5 * led.v0


def gate_li_channel_normal_depth(be):
    """validation/test_channel_flow.py:70 -- a mild 1 x 80 channel settles near Manning normal depth.

    The local-inertial scheme is diffusive, so the bar is the reference's: the
    interior median within [0.5, 2] x (q n / sqrt(S))^(3/5) after 4000 steps, water
    leaving the toe, mass closed.
    """
    nx, dx, slope, n, discharge = 80, 10.0, 0.001, 0.03, 2.0
    bed = ((nx - 1 - np.arange(nx)) * dx * slope).reshape(1, nx).astype(np.float32)
    st = be.make(bed, dx, depth=0.0, manning=n)
    be.set_bc(st, _only("east", "open"))
    inj = be.injector([((0, 0), [(0.0, discharge), (1.0e9, discharge)])], st)
    led = be.ledger(st)
    t = 0.0
    for _ in range(4000):
        dt = be.compute_dt(st, LI, 0.7, 10.0)
        led.add_inflow(inj.apply(st, t, dt))
        be.step(st, LI, dt)
        t += dt
    rec = led.record(st, t)
    h_n = (discharge / dx * n / math.sqrt(slope)) ** 0.6
    median = float(np.median(be.h(st)[0][5 : nx - 5]))
    assert led.max_rel_error < MASS_GATE and rec.outflow_cum > 0.0
    assert 0.5 * h_n < median < 2.0 * h_n, (median, h_n)


EDGE_GATES = {
    name[len("gate_") :]: fn for name, fn in sorted(globals().items()) if name.startswith("gate_") and callable(fn)
}
