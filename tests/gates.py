"""The reference's physics gates, re-expressed against a backend (oracle or CUDA).

Each gate restates a test of the reference suite with its own thresholds
(file:line of the reference test in the docstring). ``GATES`` maps a name to a
function taking a backend from tests/backends.py; the CPU suite runs them on the
oracle, the GPU suite on the CUDA path.
"""

from __future__ import annotations

import math

import numpy as np

from analytical import ritter, star_depth, stoker, stoker_front
from backends import as_f64, flat

MASS_GATE = 1.0e-6
H_DRY = 1.0e-3
LI, HLLC = "local_inertial", "hllc_fv"


def gate_li_rest_state(be):
    """solver/core/test_local_inertial.py:21 -- uniform depth on a flat bed stays at rest."""
    st = be.make(np.zeros((8, 8), np.float32), 10.0, depth=1.5, manning=0.03)
    m0 = float(be.h(st).sum())
    for _ in range(20):
        be.step(st, LI, 1.0)
    h = be.h(st)
    assert np.allclose(h, 1.5, atol=1e-6) and abs(float(h.sum()) - m0) < 1e-4
    assert np.abs(be.qx(st)).max() < 1e-6 and np.abs(be.qy(st)).max() < 1e-6


def gate_li_flux_sign(be):
    """test_local_inertial.py:35 -- higher water on the left drives +x flow; edges stay closed."""
    st = be.make(np.zeros((1, 2), np.float32), 1.0, depth=np.array([[2.0, 1.0]], np.float32), manning=0.03)
    be.step(st, LI, 0.01)
    qx = be.qx(st)
    assert qx[0, 0] == 0.0 and qx[0, 2] == 0.0 and qx[0, 1] > 0.0


def gate_li_closed_mass(be):
    """test_local_inertial.py:46 -- closed domain, no sources: depth sum invariant (< 1e-6)."""
    rng = np.random.default_rng(0)
    st = be.make(rng.uniform(0, 5, (6, 7)).astype(np.float32), 5.0,
                 depth=rng.uniform(0.5, 3, (6, 7)).astype(np.float32), manning=0.03)  # fmt: skip
    m0 = float(as_f64(be.h(st)).sum())
    for _ in range(10):
        be.step(st, LI, be.compute_dt(st, LI, 0.5, 5.0))
    assert abs(float(as_f64(be.h(st)).sum()) - m0) / m0 < 1e-6


def gate_li_rain_volume(be):
    """test_local_inertial.py:62 -- uniform rain adds rate*area*time (rel < 1e-4)."""
    st = be.make(np.zeros((5, 5), np.float32), 10.0, depth=0.1, manning=0.03)
    rain, dt, n = 36.0 / 1000.0 / 3600.0, 10.0, 30
    h0 = float(as_f64(be.h(st)).sum())
    for _ in range(n):
        be.step(st, LI, dt, rain=rain)
    expected = rain * dt * n * 25
    assert abs((float(as_f64(be.h(st)).sum()) - h0) - expected) / expected < 1e-4


def gate_li_limiter(be):
    """test_local_inertial.py:81 -- steep thin sheet: depths >= -1e-6, mass under the gate."""
    yy = np.arange(24)[:, None] * np.ones((1, 24))
    st = be.make((yy * 5.0).astype(np.float32), 10.0, depth=0.005, manning=0.03)
    led = be.ledger(st)
    t = 0.0
    for _ in range(80):
        dt = be.compute_dt(st, LI, 0.7, 5.0)
        be.step(st, LI, dt)
        t += dt
    led.record(st, t)
    h = be.h(st)
    assert np.isfinite(h).all() and h.min() > -1e-6 and led.max_rel_error < MASS_GATE


def gate_li_manning_ordering(be):
    """test_local_inertial.py:110 -- a rougher n damps a seeded discharge more."""

    def one(n):
        st = be.make(np.zeros((1, 2), np.float32), 1.0, depth=1.0, manning=n)
        be.set_qx(st, np.array([[0.0, 5.0, 0.0]], np.float32))
        be.step(st, LI, 0.01, limit=False)
        return float(be.qx(st)[0, 1])

    q_smooth, q_rough = one(0.02), one(0.20)
    assert 0.0 < q_rough < q_smooth < 5.0


def gate_li_dt_value(be):
    """test_local_inertial.py:132 -- dt = 0.7 * 10 / sqrt(9.81 * 4), deterministic."""
    st = be.make(np.zeros((4, 4), np.float32), 10.0, depth=4.0)
    d1, d2 = be.compute_dt(st, LI, 0.7, 30.0), be.compute_dt(st, LI, 0.7, 30.0)
    assert d1 == d2 and d1 == 0.7 * 10.0 / math.sqrt(9.81 * 4.0)


def _dambreak(be, scheme, h_l, h_r, alpha, nx, dx, t_end, n):
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    depth = np.where(x < 0.0, h_l, h_r).astype(np.float32).reshape(1, nx)
    st = be.make(np.zeros((1, nx), np.float32), dx, depth=depth, manning=n)
    led = be.ledger(st)
    t = 0.0
    while t < t_end - 1e-9:
        dt = min(be.compute_dt(st, scheme, alpha, t_end), t_end - t)
        be.step(st, scheme, dt)
        t += dt
    led.record(st, t)
    return x, as_f64(be.h(st)[0]), led


def _stoker_gate(be, scheme, alpha, nrmse_max, front_max):
    h_l, h_r, nx, dx, t_end = 1.0, 0.3, 800, 0.5, 8.0
    x, h, led = _dambreak(be, scheme, h_l, h_r, alpha, nx, dx, t_end, 0.01)
    assert led.max_rel_error < MASS_GATE and np.isfinite(h).all()
    ref = stoker(x, t_end, h_l, h_r)
    inner = np.abs(x) < 0.9 * nx / 2.0 * dx
    nrmse = math.sqrt(np.mean((h[inner] - ref[inner]) ** 2)) / (h_l - h_r)
    level = 0.5 * (h_r + star_depth(h_l, h_r))
    front = x[h > level].max()
    front_err = abs(front - stoker_front(t_end, h_l, h_r)) / abs(stoker_front(t_end, h_l, h_r))
    assert nrmse < nrmse_max, nrmse
    assert front_err < front_max, front_err
    return nrmse, front_err


def gate_li_stoker(be):
    """validation/test_dam_break.py:94 (LI) -- nRMSE < 0.10, front < 0.15, mass < 1e-6."""
    _stoker_gate(be, LI, 0.7, 0.10, 0.15)


def gate_hllc_stoker(be):
    """validation/test_dam_break.py:94 (HLLC) -- nRMSE < 0.03, front < 0.05, mass < 1e-6."""
    _stoker_gate(be, HLLC, 0.45, 0.03, 0.05)


def _ritter_gate(be, scheme, alpha):
    x, h, led = _dambreak(be, scheme, 1.0, 1e-3, alpha, 800, 0.5, 6.0, 0.02)
    assert led.max_rel_error < MASS_GATE and np.isfinite(h).all()
    inner = np.abs(x) < 0.9 * 200.0
    assert math.sqrt(np.mean((h[inner] - ritter(x, 6.0, 1.0)[inner]) ** 2)) < 0.5


def gate_li_ritter(be):
    """validation/test_dam_break.py:143 (LI) -- dry-bed mass gate, nRMSE ceiling 0.5."""
    _ritter_gate(be, LI, 0.7)


def gate_hllc_ritter(be):
    """validation/test_dam_break.py:143 (HLLC)."""
    _ritter_gate(be, HLLC, 0.45)


def _bumpy(ny, nx, dx):
    yy, xx = np.mgrid[0:ny, 0:nx]
    return (0.5 * np.sin(xx * 0.2) + 0.002 * xx * dx + 0.3 * np.cos(yy * 0.3)).astype(np.float32)


def gate_hllc_lake_at_rest(be):
    """validation/test_hllc_2d.py:36 -- flat surface over a bumpy bed: |u,v| < 1e-4, drift < 1e-3."""
    z = _bumpy(30, 40, 10.0)
    eta0 = float(z.max()) + 2.0
    st = be.make(z, 10.0, depth=np.maximum(eta0 - z, 0.0).astype(np.float32), manning=0.03)
    be.arm_hllc(st)
    for _ in range(200):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
    u, v = be.velocities(st)
    h = be.h(st)
    assert max(np.abs(u).max(), np.abs(v).max()) < 1e-4
    assert np.abs((h + z) - eta0).max() < 1e-3


def gate_hllc_shoreline_lake(be):
    """validation/test_hllc_wetdry.py:49 -- dry islands: peak |u,v| < 5e-5, drift < 1e-4, no leak, mass."""
    n = 50
    yy, xx = np.mgrid[0:n, 0:n].astype(float)
    z = 0.012 * ((xx - 24.5) ** 2 + (yy - 24.5) ** 2)
    z += 2.6 * np.exp(-(((xx - 16) ** 2 + (yy - 27) ** 2) / 22.0))
    z += 3.2 * np.exp(-(((xx - 33) ** 2 + (yy - 21) ** 2) / 26.0))
    z += 2.2 * np.exp(-(((xx - 27) ** 2 + (yy - 34) ** 2) / 18.0))
    z = z.astype(np.float32)
    h0 = np.maximum(3.0 - z, 0.0).astype(np.float32)
    wet0, dry0 = h0 >= H_DRY, h0 < H_DRY
    st = be.make(z, 5.0, depth=h0, manning=0.03)
    be.arm_hllc(st)
    v0 = float(be.h(st).sum())
    peak = 0.0
    for _ in range(100):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
        u, v = be.velocities(st)
        peak = max(peak, float(np.abs(u).max()), float(np.abs(v).max()))
    h = be.h(st)
    assert peak < 5e-5, peak
    assert np.abs((h + z)[wet0] - 3.0).max() < 1e-4 and h[dry0].max() < H_DRY
    assert abs(float(h.sum()) - v0) < 1e-6 * v0


def gate_hllc_puddle(be):
    """validation/test_hllc_wetdry.py:111 -- a bowl with a dry rim stays put."""
    n = 40
    yy, xx = np.mgrid[0:n, 0:n]
    z = (0.04 * ((xx - n / 2.0) ** 2 + (yy - n / 2.0) ** 2)).astype(np.float32)
    h0 = np.maximum(4.0 - z, 0.0).astype(np.float32)
    wet0, dry0 = h0 >= H_DRY, h0 < H_DRY
    st = be.make(z, 5.0, depth=h0, manning=0.03)
    be.arm_hllc(st)
    v0 = float(be.h(st).sum())
    for _ in range(300):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
    h = be.h(st)
    u, v = be.velocities(st)
    assert max(np.abs(u).max(), np.abs(v).max()) < 1e-4
    assert np.abs((h + z)[wet0] - 4.0).max() < 1e-3 and h[dry0].max() < H_DRY
    assert abs(float(h.sum()) - v0) < 1e-4 * v0


def gate_hllc_dry_front(be):
    """validation/test_hllc_wetdry.py:153 -- Ritter front band and fan nRMSE < 0.05."""
    nx, dx, t_end = 800, 0.5, 6.0
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    st = be.make(np.zeros((1, nx), np.float32), dx, depth=np.where(x < 0, 1.0, 0.0).astype(np.float32).reshape(1, nx),
                 manning=0.0)  # fmt: skip
    be.arm_hllc(st)
    m0 = float(be.h(st).sum()) * dx
    t = 0.0
    while t < t_end - 1e-9:
        dt = min(be.compute_dt(st, HLLC, 0.45, t_end), t_end - t)
        be.step(st, HLLC, dt)
        t += dt
    h = as_f64(be.h(st)[0])
    assert h.min() >= 0.0 and abs(h.sum() * dx - m0) / m0 < 1e-5
    front_ana = 2.0 * math.sqrt(9.81) * t_end
    front = float(x[h > H_DRY].max())
    assert 0.75 * front_ana <= front <= front_ana + 2.0 * dx
    ref = ritter(x, t_end, 1.0)
    fan = ref > 0.05
    assert math.sqrt(np.mean((h[fan] - ref[fan]) ** 2)) < 0.05


def gate_hllc_friction_monotone(be):
    """validation/test_hllc_wetdry.py:199 -- a moving slab decays monotonically; n = 0 keeps speed."""

    def run(n):
        st = be.make(np.zeros((4, 40), np.float32), 10.0, depth=0.5, manning=n)
        be.set_bc(st, {e: "open" for e in ("north", "south", "east", "west")})
        be.set_hu(st, np.full((4, 40), 1.0, np.float32), np.zeros((4, 40), np.float32))
        us = []
        for _ in range(25):
            be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
            u, _ = be.velocities(st)
            us.append(float(np.mean(u[1:3, 10:30])))
        return us

    us = run(0.05)
    assert all(a > b for a, b in zip(us, us[1:], strict=False)) and 0.0 < us[-1] < 1.0
    assert us[-1] < 0.5 * 2.0
    us0 = run(0.0)
    assert abs(us0[-1] - 2.0) < 0.02


def _accumulate(be, st, rain, dt, steps, scheme=LI):
    for _ in range(steps):
        be.step(st, scheme, dt, rain=rain, limit=False)
    return float(as_f64(be.h(st)).mean())


def gate_sources_sub_ulp_rain(be):
    """solver/core/test_sources.py:45 -- sub-ulp rain is lost plain and kept compensated (ratio > 100)."""
    rain, dt, steps = 4.0e-8, 1.0, 2000
    expected = rain * dt * steps
    plain = flat(24, 1.0, be)
    got_plain = _accumulate(be, plain, rain, dt, steps) - 1.0
    comp = flat(24, 1.0, be)
    be.arm_comp(comp)
    got_comp = _accumulate(be, comp, rain, dt, steps) - 1.0
    assert abs(got_plain) < 1e-9 and abs(got_comp - expected) < 2e-3 * expected
    assert abs(got_plain - expected) / max(abs(got_comp - expected), 1e-30) > 100.0


def gate_sources_canary(be):
    """test_sources.py:73 -- the Kahan residue is actually written (fast-math canary)."""
    st = flat(24, 1.0, be)
    be.arm_comp(st)
    be.step(st, LI, 1.0, rain=4.0e-8, limit=False)
    assert np.any(be.hcomp(st) != 0.0)


def gate_sources_storm_drift(be):
    """test_sources.py:89 -- realistic storm: compensated drift 20x smaller; ledger residual too (:109)."""
    rain, dt, steps = 15.0 / 1000.0 / 3600.0, 20.0, 1500
    expected = rain * dt * steps
    errs, rels = [], []
    for comp in (False, True):
        st = flat(24, 0.3, be)
        if comp:
            be.arm_comp(st)
        led = be.ledger(st)
        for k in range(steps):
            be.step(st, LI, dt, rain=rain, limit=False)
            led.add_rain_step(rain, dt, be.n_cells(st))
            if (k + 1) % 300 == 0:
                led.record(st, (k + 1) * dt)
        errs.append(abs((float(as_f64(be.h(st)).mean()) - 0.3) - expected))
        rels.append(led.max_rel_error)
    assert errs[0] / max(errs[1], 1e-30) > 20.0
    assert rels[0] / max(rels[1], 1e-30) > 20.0


def gate_sources_rain_field_both_schemes(be):
    """test_sources.py:134 -- the compensated rain field on both schemes (ratio > 100)."""
    for scheme in (LI, HLLC):
        got = []
        for comp in (False, True):
            st = flat(24, 1.0, be)
            be.set_rain(st, np.full((24, 24), 4.0e-8, np.float32))
            if comp:
                be.arm_comp(st)
            for _ in range(1500):
                be.step(st, scheme, 1.0, rain_scale=1.0)
            got.append(float(as_f64(be.h(st)).mean()) - 1.0)
        expected = 4.0e-8 * 1500
        assert abs(got[0]) < 1e-9 and abs(got[1] - expected) < 5e-3 * expected


def gate_mass_closed_box(be):
    """solver/core/test_massbalance.py:23 -- sloshing closed box, no sources."""
    rng = np.random.default_rng(1)
    st = be.make(rng.uniform(0, 3, (12, 10)).astype(np.float32), 8.0,
                 depth=rng.uniform(1, 4, (12, 10)).astype(np.float32), manning=0.03)  # fmt: skip
    led = be.ledger(st)
    t = 0.0
    for _ in range(50):
        dt = be.compute_dt(st, LI, 0.5, 5.0)
        be.step(st, LI, dt)
        t += dt
    led.record(st, t)
    assert led.max_rel_error < MASS_GATE


def gate_mass_rain_and_infiltration(be):
    """test_massbalance.py:46, :137 -- rain + partial infiltration balances to the gate."""
    st = be.make(np.zeros((16, 16), np.float32), 10.0, depth=0.5)
    be.set_infil(st, np.full((16, 16), 5.0 / 1000.0 / 3600.0, np.float32))
    led = be.ledger(st)
    rain = 50.0 / 1000.0 / 3600.0
    t = 0.0
    for _ in range(60):
        dt = be.compute_dt(st, LI, 0.5, 5.0)
        be.step(st, LI, dt, rain=rain)
        led.add_rain_step(rain, dt, be.n_cells(st))
        t += dt
    rec = led.record(st, t)
    assert led.max_rel_error < MASS_GATE and rec.outflow_cum > 0.0


def gate_mass_infiltration_capped(be):
    """test_massbalance.py:68 -- one huge infiltration step drains to exactly 0 and banks it."""
    st = be.make(np.zeros((4, 4), np.float32), 10.0, depth=0.01)
    be.set_infil(st, np.full((4, 4), 1.0, np.float32))
    led = be.ledger(st)
    be.step(st, LI, 1.0)
    rec = led.record(st, 1.0)
    h = be.h(st)
    assert h.min() >= 0.0 and float(h.max()) < 1e-7
    removed = be.loss_volume(st)
    assert abs(removed - 0.01 * 100.0 * 16) < 1e-5 * 0.01 * 100.0 * 16
    assert abs(rec.outflow_cum - removed) <= 1e-6 * removed


def gate_mass_rain_field_volume(be):
    """test_massbalance.py:156 -- a ramp rain field adds sum(rate) * area * time."""
    st = be.make(np.zeros((8, 8), np.float32), 10.0, depth=0.1)
    rate = ((np.arange(64, dtype=np.float32).reshape(8, 8) + 1.0) * 2.0 / 1000.0 / 3600.0).astype(np.float32)
    be.set_rain(st, rate)
    led = be.ledger(st)
    for _ in range(40):
        be.step(st, LI, 5.0, rain_scale=1.0)
        led.add_inflow(float(rate.astype(np.float64).sum()) * 5.0 * 100.0)
    led.record(st, 200.0)
    assert led.max_rel_error < MASS_GATE


def gate_mass_drain_to_empty(be):
    """test_massbalance.py:172 -- open edge + infiltration empty the domain; the gate still holds."""
    ny, nx, dx = 16, 24, 10.0
    xx = np.broadcast_to(np.arange(nx), (ny, nx))
    st = be.make(((nx - 1 - xx) * dx * 0.02).astype(np.float32), dx, depth=0.5, manning=0.03)
    be.set_bc(st, {"east": "open", "west": "closed", "north": "closed", "south": "closed"})
    be.set_infil(st, np.full((ny, nx), 2.0e-4, np.float32))
    led = be.ledger(st)
    v0 = led.v0
    t = 0.0
    for _ in range(4000):
        dt = be.compute_dt(st, LI, 0.7, 5.0)
        be.step(st, LI, dt)
        t += dt
        if float(be.h(st).max()) < 1e-9:
            break
    rec = led.record(st, t)
    assert float(be.h(st).max()) < 1e-6 and rec.volume < 1e-9 * v0
    assert led.max_rel_error < MASS_GATE


def gate_open_edges_each_drain(be):
    """solver/core/test_boundaries.py:41 -- each open edge drains its way, never negative."""
    for edge in ("north", "south", "east", "west"):
        n, dx = 24, 10.0
        i = np.arange(n)[:, None] * np.ones((1, n))
        j = np.ones((n, 1)) * np.arange(n)[None, :]
        s = 0.02 * dx
        z = {"east": (n - 1 - j) * s, "west": j * s, "south": (n - 1 - i) * s, "north": i * s}[edge]
        st = be.make(z.astype(np.float32), dx, depth=0.5, manning=0.03)
        be.set_bc(st, {e: ("open" if e == edge else "closed") for e in ("north", "south", "east", "west")})
        led = be.ledger(st)
        v0 = led.v0
        t = 0.0
        for _ in range(1500):
            dt = be.compute_dt(st, LI, 0.7, 5.0)
            be.step(st, LI, dt)
            t += dt
        rec = led.record(st, t)
        h = be.h(st)
        assert np.isfinite(h).all() and h.min() >= -1e-6 and led.max_rel_error < MASS_GATE, edge
        assert rec.outflow_cum > 0.5 * v0 and rec.volume < 0.5 * v0, edge


def gate_inflow_closed_basin(be):
    """solver/processes/test_inflow.py:76, :93 -- injected volume and a balanced closed basin."""
    st = be.make(np.zeros((5, 5), np.float32), 10.0)
    inj = be.injector([((2, 2), [(0.0, 3.0), (100.0, 3.0)])], st)
    total, t = 0.0, 0.0
    for _ in range(10):
        total += inj.apply(st, t, 10.0)
        t += 10.0
    assert abs(total - 300.0) < 1e-4 * 300.0 and abs(float(be.h(st)[2, 2]) * 100.0 - 300.0) < 1e-4 * 300.0
    st = be.make(np.zeros((12, 12), np.float32), 10.0, depth=0.05)
    inj = be.injector([((6, 6), [(0.0, 0.0), (200.0, 4.0), (600.0, 0.0)])], st)
    led = be.ledger(st)
    t = 0.0
    for _ in range(120):
        dt = be.compute_dt(st, LI, 0.5, 5.0)
        led.add_inflow(inj.apply(st, t, dt))
        be.step(st, LI, dt)
        t += dt
    rec = led.record(st, t)
    assert led.max_rel_error < MASS_GATE and rec.inflow_cum > 0.0


# --- sub-grid channels ------------------------------------------------------- #
_EAST_OPEN = {"east": "open", "west": "closed", "north": "closed", "south": "closed"}


def _slope_bed(ny, nx, dx, slope, base=5.0):
    xx = np.broadcast_to(np.arange(nx), (ny, nx))
    return ((nx - 1 - xx) * dx * slope + base).astype(np.float32)


def normal_depth(discharge, width, slope, manning):
    """Manning normal depth of a rectangular section, R = A/P (bisection on Q(h))."""

    def q_of(h):
        area = width * h
        return area * (area / (width + 2.0 * h)) ** (2.0 / 3.0) * math.sqrt(slope) / manning

    lo, hi = 1e-6, 100.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if q_of(mid) < discharge:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _run_steady(be, st, inflows, steps, dt_max):
    inj = be.injector(inflows, st)
    led = be.ledger(st)
    t = 0.0
    for _ in range(steps):
        dt = be.compute_dt(st, LI, 0.7, dt_max)
        led.add_inflow(inj.apply(st, t, dt))
        be.step(st, LI, dt)
        t += dt
    led.record(st, t)
    return led


def gate_channels_zero_width_is_m1_bitwise(be):
    """solver/core/test_channels.py:162 -- w = 0 channels reproduce the plain scheme bit for bit."""
    ny, nx, dx = 8, 24, 40.0
    bed = _slope_bed(ny, nx, dx, 0.004)
    plain = be.make(bed, dx, depth=0.05, manning=0.03)
    armed = be.make(bed, dx, depth=0.05, manning=0.03)
    be.arm_channels(armed, np.zeros((ny, nx), np.float32), np.zeros((ny, nx), np.float32))
    for _ in range(60):
        dt_p = be.compute_dt(plain, LI, 0.7, 5.0)
        dt_a = be.compute_dt(armed, LI, 0.7, 5.0)
        assert dt_p == dt_a
        be.step(plain, LI, dt_p, rain=1e-5)
        be.step(armed, LI, dt_a, rain=1e-5)
    np.testing.assert_array_equal(be.h(armed), be.h(plain))
    np.testing.assert_array_equal(be.qx(armed), be.qx(plain))
    np.testing.assert_array_equal(be.qy(armed), be.qy(plain))


def gate_channels_dt_sees_the_water_column(be):
    """test_channels.py:187 -- in-bank the CFL depth is h dx / w, not h."""
    ny, nx, dx = 4, 8, 200.0
    w, d, h0 = 20.0, 3.0, 0.05
    bed = np.full((ny, nx), 10.0, np.float32)
    plain = be.make(bed, dx, depth=h0, manning=0.035)
    armed = be.make(bed, dx, depth=h0, manning=0.035)
    be.arm_channels(armed, np.full((ny, nx), w, np.float32), np.full((ny, nx), d, np.float32))
    dt_plain = be.compute_dt(plain, LI, 0.7, 1e6)
    dt_armed = be.compute_dt(armed, LI, 0.7, 1e6)
    assert abs(dt_plain / (0.7 * dx / math.sqrt(9.81 * h0)) - 1.0) < 1e-5
    assert abs(dt_armed / (0.7 * dx / math.sqrt(9.81 * h0 * dx / w)) - 1.0) < 1e-5
    assert dt_armed < dt_plain / 3.0


def gate_channels_default_roughness_is_the_floodplain(be):
    """test_channels.py:146 -- arming without a roughness field uses the cell's n."""
    bed = np.full((6, 10), 10.0, np.float32)
    st = be.make(bed, 50.0, depth=0.0, manning=0.035)
    be.arm_channels(st, np.full((6, 10), 8.0, np.float32), np.full((6, 10), 1.5, np.float32))
    np.testing.assert_array_equal(be.channel_n(st), np.full((6, 10), np.float32(0.035)))


def gate_channels_closed_box_mass(be):
    """test_channels.py:203 -- a closed channelled bowl conserves volume (rel < 1e-6)."""
    ny, nx, dx = 10, 20, 50.0
    yy, xx = np.mgrid[0:ny, 0:nx]
    bed = (20.0 + 0.02 * ((yy - ny / 2) ** 2 + (xx - nx / 2) ** 2)).astype(np.float32)
    st = be.make(bed, dx, depth=0.2, manning=0.03)
    w = np.zeros((ny, nx), np.float32)
    d = np.zeros((ny, nx), np.float32)
    w[ny // 2, :] = 15.0
    d[ny // 2, :] = 2.0
    be.arm_channels(st, w, d)
    v0 = float(as_f64(be.h(st)).sum())
    for _ in range(300):
        be.step(st, LI, be.compute_dt(st, LI, 0.7, 5.0))
    h = be.h(st)
    assert np.isfinite(h).all() and h.min() >= -1e-9
    assert abs(float(as_f64(h).sum()) - v0) / v0 < 1e-6


def gate_subgrid_channel_normal_depth(be):
    """validation/test_subgrid_channel.py:100 -- a 20 m channel in 50 m cells settles at the
    Manning normal depth of its own section (within 5 %), mass within the gate."""
    nx, dx = 100, 50.0
    slope, n_ch, width, bankfull, discharge = 0.001, 0.03, 20.0, 4.0, 30.0
    st = be.make(_slope_bed(1, nx, dx, slope), dx, depth=0.0, manning=0.05)
    be.arm_channels(st, np.full((1, nx), width, np.float32), np.full((1, nx), bankfull, np.float32),
                    np.full((1, nx), n_ch, np.float32))  # fmt: skip
    be.set_bc(st, _EAST_OPEN)
    led = _run_steady(be, st, [((0, 0), [(0.0, discharge), (1.0e9, discharge)])], 3000, 10.0)
    column = be.h(st)[0] * dx / width
    median = float(np.median(column[10 : nx - 10]))
    h_n = normal_depth(discharge, width, slope, n_ch)
    assert np.isfinite(column).all() and led.max_rel_error < MASS_GATE
    assert median < bankfull
    assert abs(median / h_n - 1.0) < 0.05, (median, h_n)


def gate_subgrid_channel_overbank_spill(be):
    """validation/test_subgrid_channel.py:140 -- past bank full water reaches the floodplain;
    the closed-domain ledger holds."""
    ny, nx, dx = 7, 30, 50.0
    st = be.make(_slope_bed(ny, nx, dx, 0.0005), dx, depth=0.0, manning=0.05)
    row = ny // 2
    w = np.zeros((ny, nx), np.float32)
    d = np.zeros((ny, nx), np.float32)
    w[row, :] = 20.0
    d[row, :] = 1.0
    be.arm_channels(st, w, d, np.full((ny, nx), 0.03, np.float32))
    led = _run_steady(be, st, [((row, 2), [(0.0, 60.0), (1.0e9, 60.0)])], 1200, 5.0)
    h = be.h(st)
    h_bf = 20.0 * 1.0 / dx
    floodplain = np.delete(h, row, axis=0)
    assert np.isfinite(h).all() and h.min() >= -1e-9
    assert h[row].max() > h_bf and (floodplain > 1e-3).sum() > 0
    assert led.max_rel_error < MASS_GATE


def gate_subgrid_channel_matches_resolved_reach(be):
    """validation/test_subgrid_channel.py:177 -- a 100 m-cell sub-grid reach against the same
    channel resolved at 10 m: each near its own analytical section (10 %), the two depths
    within 12 % and the stored volumes within 20 %."""
    length_m, slope, n_ch, width, bankfull, discharge = 2000.0, 0.0008, 0.035, 40.0, 2.0, 40.0
    dxf = 10.0
    nyf, nxf = 10, int(length_m / dxf)
    bed_f = _slope_bed(nyf, nxf, dxf, slope)
    bed_f[3:7, :] -= bankfull
    fine = be.make(bed_f, dxf, depth=0.0, manning=n_ch)
    be.set_bc(fine, _EAST_OPEN)
    per_cell = discharge / 4.0
    led_f = _run_steady(be, fine, [((r, 0), [(0.0, per_cell), (1.0e9, per_cell)]) for r in range(3, 7)], 6000, 5.0)
    dxc = 100.0
    nxc = int(length_m / dxc)
    coarse = be.make(_slope_bed(1, nxc, dxc, slope), dxc, depth=0.0, manning=n_ch)
    be.arm_channels(coarse, np.full((1, nxc), width, np.float32), np.full((1, nxc), bankfull, np.float32),
                    np.full((1, nxc), n_ch, np.float32))  # fmt: skip
    be.set_bc(coarse, _EAST_OPEN)
    led_c = _run_steady(be, coarse, [((0, 0), [(0.0, discharge), (1.0e9, discharge)])], 2000, 10.0)

    def interior(a):
        k = len(a)
        return a[k // 5 : -k // 5]

    fine_depth = float(np.median(interior(be.h(fine)[3:7].mean(axis=0))))
    coarse_depth = float(np.median(interior(be.h(coarse)[0] * dxc / width)))
    fine_volume = float(as_f64(be.h(fine)).sum()) * dxf * dxf
    coarse_volume = float(as_f64(be.h(coarse)).sum()) * dxc * dxc
    h_wide = (discharge / width * n_ch / math.sqrt(slope)) ** 0.6
    h_section = normal_depth(discharge, width, slope, n_ch)
    assert led_f.max_rel_error < MASS_GATE and led_c.max_rel_error < MASS_GATE
    assert abs(fine_depth / h_wide - 1.0) < 0.10, (fine_depth, h_wide)
    assert abs(coarse_depth / h_section - 1.0) < 0.10, (coarse_depth, h_section)
    assert abs(coarse_depth / fine_depth - 1.0) < 0.12
    assert abs(coarse_volume / fine_volume - 1.0) < 0.20


# --- reservoirs (solver/processes/test_reservoir.py) ------------------------- #
_RNY, _RNX, _RDX, _DAM_ROW, _CREST = 12, 8, 10.0, 6, 5.0


def _basin():
    z = np.zeros((_RNY, _RNX), np.float32)
    z[: _DAM_ROW + 1] = 2.0
    z[_DAM_ROW + 1 :] = np.linspace(2.0, 0.0, _RNY - _DAM_ROW - 1, dtype=np.float32)[:, None]
    return z


def _dam(**kw):
    base = dict(name="d", kind="dam", cells=[(_DAM_ROW, j) for j in range(_RNX)], crest_m=_CREST,
                release_rule="fixed", release_m3_s=1.0, pool=(0, 0, 5, _RNX - 1), outlet=(8, 2, 10, 5),
                interval_s=300.0)  # fmt: skip
    base.update(kw)
    return base


def _barriers(bed, dam):
    out = bed.copy()
    for i, j in dam["cells"]:
        out[i, j] = max(float(out[i, j]), float(dam["crest_m"]))
    return out


def _pool_depth(surface):
    bed = _basin()
    h = np.zeros((_RNY, _RNX), np.float32)
    h[:_DAM_ROW] = np.maximum(surface - bed[:_DAM_ROW], 0.0)
    return h


def _vol(h):
    return float(np.asarray(h, np.float64).sum()) * _RDX * _RDX


def _run_pool(be, bed, h0, steps=300):
    st = be.make(bed, _RDX, depth=h0, manning=0.03)
    be.arm_hllc(st)
    for _ in range(steps):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
    return be.h(st)


def gate_reservoir_barrier_impounds(be):
    """test_reservoir.py:108 -- the dam keeps > 90 % of the pool; without it most escapes."""
    h0 = _pool_depth(4.5)
    kept = _run_pool(be, _barriers(_basin(), _dam()), h0)
    spilt = _run_pool(be, _basin(), h0)
    v0 = _vol(h0)
    assert _vol(kept[:_DAM_ROW]) > 0.9 * v0
    assert _vol(spilt[:_DAM_ROW]) < 0.5 * _vol(kept[:_DAM_ROW])
    assert np.isfinite(kept).all() and kept.min() >= 0.0


def gate_reservoir_pool_above_crest_overtops(be):
    """test_reservoir.py:128 -- overtopping is ordinary solver physics."""
    bed = _barriers(_basin(), _dam())
    over = _run_pool(be, bed, _pool_depth(_CREST + 0.5))
    under = _run_pool(be, bed, _pool_depth(_CREST - 0.5))
    below_over, below_under = _vol(over[_DAM_ROW + 1 :]), _vol(under[_DAM_ROW + 1 :])
    assert below_over > 100.0 and below_over > 10.0 * max(below_under, 1e-9)


def gate_reservoir_transfer_is_mass_exact(be):
    """test_reservoir.py:141 -- pool loss == released volume; the domain total moves only by
    the banked rounding."""
    dam = _dam()
    st = be.make(_barriers(_basin(), dam), _RDX, depth=_pool_depth(4.5), manning=0.03)
    op = be.reservoir(st, dam)
    before = be.h(st)
    v_before, pool_before = _vol(before), _vol(before[0:6, :])
    rec = op.advance(300.0, 300.0)
    after = be.h(st)
    v_after, pool_after = _vol(after), _vol(after[0:6, :])
    banked = be.loss_volume(st)
    assert abs(rec.volume_m3 / 300.0 - 1.0) < 1e-6
    assert abs((pool_before - pool_after) / rec.volume_m3 - 1.0) < 1e-9
    assert abs((v_before - v_after) - banked) <= 1e-9 * v_before
    assert abs(v_before - v_after) < 1e-6 * v_before


def gate_reservoir_release_capped_by_pool(be):
    """test_reservoir.py:177 -- a rule that outruns its reservoir delivers what it holds."""
    dam = _dam(release_m3_s=10_000.0)
    h0 = _pool_depth(2.02)
    st = be.make(_barriers(_basin(), dam), _RDX, depth=h0, manning=0.03)
    rec = be.reservoir(st, dam).advance(300.0, 300.0)
    stored = _vol(h0)
    assert rec.volume_m3 <= stored + 1e-9 and abs(rec.volume_m3 / stored - 1.0) < 1e-6
    assert float(be.h(st)[: _DAM_ROW + 1].min()) >= 0.0


def gate_reservoir_dry_pool_is_a_no_op(be):
    """test_reservoir.py:191."""
    dam = _dam()
    st = be.make(_barriers(_basin(), dam), _RDX, depth=0.0, manning=0.03)
    rec = be.reservoir(st, dam).advance(300.0, 300.0)
    assert rec.stage is None and rec.discharge_m3_s == 0.0 and rec.volume_m3 == 0.0


def gate_reservoir_target_stage_draws_down(be):
    """test_reservoir.py:199 -- the closed-loop rule draws the pool toward its target and eases off."""
    dam = _dam(release_rule="target_stage", target_stage_m=3.0, release_max_m3_s=8.0)
    st = be.make(_barriers(_basin(), dam), _RDX, depth=_pool_depth(4.8), manning=0.03)
    op = be.reservoir(st, dam)
    recs = [op.advance(300.0 * k, 300.0) for k in range(1, 25)]
    stages = [r.stage for r in recs]
    qs = [r.discharge_m3_s for r in recs]
    assert stages[0] > stages[-1] and qs[0] > qs[-1]
    assert max(qs) <= dam["release_max_m3_s"] + 1e-9
    assert stages[-1] >= dam["target_stage_m"] - 0.05 and stages[-1] < 4.8


def gate_reservoir_gauge_is_the_deepest_cell(be):
    """test_reservoir.py:313 -- a film high on a wall of the pool box does not read as the stage."""
    bed = _basin().copy()
    bed[0, 0] = 8.0
    bed[3, 3] = 1.0
    depth = np.zeros_like(bed)
    depth[0, 0] = 0.05
    st = be.make(bed, _RDX, depth=depth, manning=0.03)
    op = be.reservoir(st, _dam())
    assert op.pool_stage() is None


GATES = {name[len("gate_"):]: fn for name, fn in sorted(globals().items()) if name.startswith("gate_")}
