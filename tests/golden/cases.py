"""Small seeded scenarios that pin the solver path, shared by every runner.

Each case is a plain dict of numpy inputs plus a stepping recipe. The same case is
run (a) through the reference's own kernel source by ``make_golden.py`` to make the
committed fixtures, (b) through the CPU oracle by ``tests/test_oracle_golden.py``,
and (c) through the CUDA path by the GPU parity tests. Sizes are small on purpose:
the reference run goes through a per-thread Python interpreter.

Every optional physics branch of the reference step is reached by at least one
case: the donor limiter, closed/open/fixed_stage edges, compensated and plain
uniform rain, compensated and plain rain fields, infiltration, inflow point sources
(compensated), bedload accumulation with Exner activations and bounds, wet/dry
fronts, dry cells, one-row domains, sub-grid channels (in and over bank,
with and without bedload) and reservoir releases (fixed and target-stage rules).
"""

from __future__ import annotations

import numpy as np

EDGES = ("north", "south", "east", "west")


def _bc(**kw):
    return {e: kw.get(e, "closed") for e in EDGES}


def _bumps(ny, nx, dx, rng, n_bumps, amp, sigma):
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    z = np.zeros((ny, nx))
    for _ in range(n_bumps):
        a = rng.uniform(*amp)
        s = rng.uniform(*sigma)
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        z += a * np.exp(-(((yy - cy) ** 2 + (xx - cx) ** 2) * dx * dx) / (2 * s * s))
    return z


def case_li_closed_random():
    rng = np.random.default_rng(0)
    bed = rng.uniform(0.0, 5.0, size=(6, 7)).astype(np.float32)
    depth = rng.uniform(0.5, 3.0, size=(6, 7)).astype(np.float32)
    return dict(scheme="local_inertial", bed=bed, dx=5.0, depth=depth, manning=0.03,
                steps=10, alpha=0.5, dt_max=5.0)  # fmt: skip


def case_li_steep_sheet():
    ny = nx = 12
    yy = np.arange(ny)[:, None] * np.ones((1, nx))
    bed = (yy * 5.0).astype(np.float32)
    return dict(scheme="local_inertial", bed=bed, dx=10.0, depth=0.005, manning=0.03,
                steps=25, alpha=0.7, dt_max=5.0)  # fmt: skip


def case_li_rain_open_infil():
    rng = np.random.default_rng(1)
    ny, nx, dx = 10, 12, 10.0
    xx = np.broadcast_to(np.arange(nx), (ny, nx))
    bed = (1e-2 * (nx - 1 - xx) * dx + _bumps(ny, nx, dx, rng, 4, (0.1, 0.6), (10, 30))).astype(np.float32)
    infil = rng.uniform(0.0, 20.0, size=(ny, nx)) / 1000.0 / 3600.0
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.05, manning=0.03,
                boundaries=_bc(east="open", south="open"), infil=infil.astype(np.float32),
                compensated=True, rain=50.0 / 1000.0 / 3600.0, steps=20, alpha=0.7, dt_max=5.0)  # fmt: skip


def case_li_rain_field_plain():
    rng = np.random.default_rng(2)
    ny, nx, dx = 9, 8, 10.0
    bed = rng.uniform(0.0, 0.3, size=(ny, nx)).astype(np.float32)
    rain = ((np.arange(ny * nx).reshape(ny, nx) + 1.0) * 2.0 / 1000.0 / 3600.0).astype(np.float32)
    manning = rng.uniform(0.02, 0.06, size=(ny, nx)).astype(np.float32)
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.1, manning=manning, rain_field=rain,
                rain_scale=1.0, boundaries=_bc(west="open"), steps=15, alpha=0.7, dt_max=5.0)  # fmt: skip


def case_li_rain_field_comp():
    rng = np.random.default_rng(3)
    ny, nx, dx = 8, 9, 20.0
    bed = rng.uniform(0.0, 0.5, size=(ny, nx)).astype(np.float32)
    rain = rng.uniform(1e-6, 2e-5, size=(ny, nx)).astype(np.float32)
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.2, manning=0.035, rain_field=rain,
                compensated=True, rain_scale=1.0, boundaries=_bc(north="open", west="open"),
                steps=12, alpha=0.7, dt_max=10.0)  # fmt: skip


def case_li_inflow():
    ny = nx = 10
    bed = np.zeros((ny, nx), np.float32)
    inflows = [((3, 3), [(0.0, 0.0), (30.0, 4.0), (90.0, 0.0)]), ((6, 7), [(0.0, 1.5), (200.0, 1.5)])]
    return dict(scheme="local_inertial", bed=bed, dx=10.0, depth=0.05, manning=0.03, inflows=inflows,
                steps=20, alpha=0.5, dt_max=5.0)  # fmt: skip


def case_li_sediment():
    ny, nx, dx = 8, 14, 5.0
    xx = np.broadcast_to(np.arange(nx), (ny, nx)).astype(np.float64)
    yy = np.arange(ny)[:, None] * np.ones((1, nx))
    bed = (0.01 * (nx - 1 - xx) * dx + 0.05 * np.cos(yy * 0.7) + 0.03 * np.sin(xx * 1.3)).astype(np.float32)
    qx0 = np.zeros((ny, nx + 1), np.float32)
    qx0[:, 1:nx] = 0.8
    d50 = np.full((ny, nx), 0.002, np.float32)
    d50[2:4, 5:9] = 0.004
    lo = np.full((ny, nx), -np.inf, np.float32)
    hi = np.full((ny, nx), np.inf, np.float32)
    lo[:, 3:6] = -0.002  # an alluvium floor
    lo[4, 10] = hi[4, 10] = 0.0  # a frozen structure cell
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.5, manning=0.03, qx0=qx0,
                boundaries=_bc(east="open"), sediment=dict(d50=d50, porosity=0.4, every=10, dz_lo=lo, dz_hi=hi),
                steps=25, alpha=0.7, dt_max=2.0)  # fmt: skip


def _channel_valley(ny, nx, dx, rng):
    """A down-valley slope with a V cross-section, a sub-grid channel along the
    valley floor (two rows, one gap), and per-cell channel roughness."""
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    mid = (ny - 1) / 2.0
    bed = (2e-3 * (nx - 1 - xx) * dx + 0.02 * np.abs(yy - mid) * dx + 0.05 * np.sin(0.9 * xx)).astype(np.float32)
    w = np.zeros((ny, nx), np.float32)
    d = np.zeros((ny, nx), np.float32)
    rows = [int(np.floor(mid)), int(np.ceil(mid))]
    w[rows, :] = rng.uniform(8.0, 20.0, size=(2, nx)).astype(np.float32)
    d[rows, :] = rng.uniform(0.8, 2.5, size=(2, nx)).astype(np.float32)
    w[rows[0], nx // 3] = d[rows[0], nx // 3] = 0.0  # a gap: the narrower side controls the face
    cn = rng.uniform(0.02, 0.04, size=(ny, nx)).astype(np.float32)
    return bed, w, d, cn


def case_li_channels():
    rng = np.random.default_rng(11)
    ny, nx, dx = 10, 16, 40.0
    bed, w, d, cn = _channel_valley(ny, nx, dx, rng)
    depth = np.full((ny, nx), 0.02, np.float32)
    depth[:, :4] = 0.9  # spills over bank full upstream, in-bank downstream
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=depth, manning=0.045,
                channels=dict(width=w, depth=d, manning=cn), compensated=True, rain=30.0 / 3.6e6,
                boundaries=_bc(east="open"), steps=30, alpha=0.7, dt_max=8.0)  # fmt: skip


def case_li_channels_sediment():
    rng = np.random.default_rng(12)
    ny, nx, dx = 8, 14, 20.0
    bed, w, d, cn = _channel_valley(ny, nx, dx, rng)
    bed = bed + (0.01 * dx * np.arange(nx)[::-1]).astype(np.float32)  # steeper: transport above critical
    d50 = np.full((ny, nx), 0.002, np.float32)
    lo = np.full((ny, nx), -np.inf, np.float32)
    hi = np.full((ny, nx), np.inf, np.float32)
    lo[:, 2:5] = -0.003
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.4, manning=0.04,
                channels=dict(width=w, depth=d, manning=cn), boundaries=_bc(east="open"),
                sediment=dict(d50=d50, porosity=0.4, every=8, dz_lo=lo, dz_hi=hi),
                steps=24, alpha=0.7, dt_max=2.0)  # fmt: skip


def _reservoir_basin(ny, nx, dam_row, crest):
    """A flat reservoir floor behind a dam row, a valley falling away below it; the
    dam cells already raised to the crest (what apply_barriers does)."""
    z = np.zeros((ny, nx), np.float32)
    z[: dam_row + 1] = 2.0
    z[dam_row + 1 :] = np.linspace(2.0, 0.0, ny - dam_row - 1, dtype=np.float32)[:, None]
    z[dam_row, :] = np.maximum(z[dam_row, :], crest)
    return z


def _reservoir_case(scheme, rule, steps, every, alpha):
    ny, nx, dam_row, crest = 12, 8, 6, 5.0
    bed = _reservoir_basin(ny, nx, dam_row, crest)
    depth = np.zeros((ny, nx), np.float32)
    depth[:dam_row] = np.maximum(4.6 - bed[:dam_row], 0.0)
    dam = dict(name="d", kind="dam", cells=[(dam_row, j) for j in range(nx)], crest_m=crest, pool=(0, 0, 5, nx - 1),
               outlet=(8, 2, 10, 5), interval_s=60.0, **rule)  # fmt: skip
    return dict(scheme=scheme, bed=bed, dx=10.0, depth=depth, manning=0.03, reservoir=dict(structure=dam, every=every),
                boundaries=_bc(south="open"), steps=steps, alpha=alpha, dt_max=3.0)  # fmt: skip


def case_li_reservoir_fixed():
    return _reservoir_case("local_inertial", dict(release_rule="fixed", release_m3_s=3.0), 30, 6, 0.7)


def case_hllc_reservoir_target_stage():
    rule = dict(release_rule="target_stage", target_stage_m=3.0, release_max_m3_s=40.0)
    return _reservoir_case("hllc_fv", rule, 24, 4, 0.45)


def case_li_dambreak_row():
    nx, dx = 40, 0.5
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    depth = np.where(x < 0.0, 1.0, 0.3).astype(np.float32).reshape(1, nx)
    return dict(scheme="local_inertial", bed=np.zeros((1, nx), np.float32), dx=dx, depth=depth,
                manning=0.01, steps=15, alpha=0.7, dt_max=8.0)  # fmt: skip


def _hllc_bumpy(ny, nx, dx):
    yy, xx = np.mgrid[0:ny, 0:nx]
    return (0.5 * np.sin(xx * 0.2) + 0.002 * xx * dx + 0.3 * np.cos(yy * 0.3)).astype(np.float32)


def case_hllc_bumpy_moving():
    ny, nx, dx = 10, 12, 10.0
    yy, xx = np.mgrid[0:ny, 0:nx]
    depth = (0.5 + 0.3 * np.sin(xx * 0.5 + yy * 0.3)).astype(np.float32)
    return dict(scheme="hllc_fv", bed=_hllc_bumpy(ny, nx, dx), dx=dx, depth=depth, manning=0.03,
                rain=1e-5, steps=12, alpha=0.45, dt_max=5.0)  # fmt: skip


def case_hllc_open_comp_infil():
    rng = np.random.default_rng(4)
    ny, nx, dx = 10, 11, 10.0
    bed = rng.uniform(0.0, 0.4, size=(ny, nx)).astype(np.float32)
    depth = rng.uniform(0.2, 0.8, size=(ny, nx)).astype(np.float32)
    hu0 = rng.uniform(-0.3, 0.3, size=(ny, nx)).astype(np.float32)
    hv0 = rng.uniform(-0.3, 0.3, size=(ny, nx)).astype(np.float32)
    infil = rng.uniform(0.0, 3e-5, size=(ny, nx)).astype(np.float32)
    return dict(scheme="hllc_fv", bed=bed, dx=dx, depth=depth, manning=0.035, hu0=hu0, hv0=hv0,
                boundaries=_bc(west="open", north="open"), infil=infil, compensated=True,
                rain=20.0 / 1000.0 / 3600.0, steps=10, alpha=0.45, dt_max=5.0)  # fmt: skip


def case_hllc_stage():
    ny, nx, dx = 8, 10, 10.0
    xx = np.broadcast_to(np.arange(nx), (ny, nx))
    bed = (0.01 * xx * dx * 0.1).astype(np.float32)
    return dict(scheme="hllc_fv", bed=bed, dx=dx, depth=0.5, manning=0.03,
                boundaries=_bc(east="fixed_stage", west="open"),
                stage_curves={"east": [(0.0, 0.6), (20.0, 0.9), (60.0, 0.9)]},
                steps=10, alpha=0.45, dt_max=5.0)  # fmt: skip


def case_hllc_shoreline():
    ny = nx = 14
    dx = 5.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(float)
    z = 0.05 * ((xx - 6.5) ** 2 + (yy - 6.5) ** 2)
    z += 2.6 * np.exp(-(((xx - 4) ** 2 + (yy - 7) ** 2) / 4.0))
    z += 3.2 * np.exp(-(((xx - 9) ** 2 + (yy - 5) ** 2) / 5.0))
    z = z.astype(np.float32)
    h0 = np.maximum(3.0 - z, 0.0).astype(np.float32)
    return dict(scheme="hllc_fv", bed=z, dx=dx, depth=h0, manning=0.03, steps=10, alpha=0.45, dt_max=5.0)


def case_hllc_rain_field_plain():
    rng = np.random.default_rng(5)
    ny, nx, dx = 8, 8, 10.0
    bed = rng.uniform(0.0, 0.2, size=(ny, nx)).astype(np.float32)
    rain = rng.uniform(0.0, 3e-5, size=(ny, nx)).astype(np.float32)
    infil = rng.uniform(0.0, 1e-5, size=(ny, nx)).astype(np.float32)
    return dict(scheme="hllc_fv", bed=bed, dx=dx, depth=0.3, manning=0.03, rain_field=rain, rain_scale=1.0,
                infil=infil, boundaries=_bc(south="open"), steps=8, alpha=0.45, dt_max=5.0)  # fmt: skip


def case_hllc_dambreak_row():
    nx, dx = 40, 0.5
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    depth = np.where(x < 0.0, 1.0, 0.3).astype(np.float32).reshape(1, nx)
    return dict(scheme="hllc_fv", bed=np.zeros((1, nx), np.float32), dx=dx, depth=depth, manning=0.01,
                steps=15, alpha=0.45, dt_max=8.0)  # fmt: skip


def case_hllc_dry_front_row():
    nx, dx = 30, 0.5
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    depth = np.where(x < 0.0, 1.0, 0.0).astype(np.float32).reshape(1, nx)
    return dict(scheme="hllc_fv", bed=np.zeros((1, nx), np.float32), dx=dx, depth=depth, manning=0.0,
                boundaries=_bc(east="open", west="open"), steps=15, alpha=0.45, dt_max=6.0)  # fmt: skip


CASES = {
    name[len("case_"):]: fn
    for name, fn in sorted(globals().items())
    if name.startswith("case_") and callable(fn)
}


# --- combinations of branches ------------------------------------------------- #
# The cases above reach each branch on its own. These two run many at once, as the
# reach (configuration 3) and a storm over an HLLC basin do, and pin the oracle
# against the reference kernels on those combinations. They sit outside CASES, which
# the GPU runners also iterate: the CUDA path is checked against the oracle on the
# reach combination at full width (tests/test_gpu_parity.py, 200 steps of an
# 8192-wide band with inflows, infiltration, a Manning field, bedload and Exner).


def combined_li_reach():
    """A small valley reach: cross-slope, lognormal Manning, infiltration field, two
    triangular inflow hydrographs, the east edge open, bedload on a floored bed with a
    frozen cell, Exner every 8 steps."""
    rng = np.random.default_rng(21)
    ny, nx, dx = 10, 24, 5.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    bed = (4e-3 * (nx - 1 - xx) * dx + 0.04 * np.abs(yy - 4.5) * dx + 0.05 * np.sin(0.9 * xx)).astype(np.float32)
    manning = np.exp(np.log(0.035) + 0.3 * rng.standard_normal((ny, nx))).astype(np.float32)
    infil = (rng.uniform(0.0, 20.0, (ny, nx)) / 1000.0 / 3600.0).astype(np.float32)
    inflows = [((4, 0), [(0.0, 0.0), (40.0, 6.0), (120.0, 0.5)]), ((5, 1), [(0.0, 1.0), (400.0, 1.0)])]
    lo = np.full((ny, nx), -0.003, np.float32)
    hi = np.full((ny, nx), np.inf, np.float32)
    lo[5, 12] = hi[5, 12] = 0.0
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=0.2, manning=manning, infil=infil,
                inflows=inflows, boundaries=_bc(east="open"),
                sediment=dict(d50=0.002, porosity=0.4, every=8, dz_lo=lo, dz_hi=hi),
                steps=32, alpha=0.7, dt_max=3.0)  # fmt: skip


def combined_hllc_storm():
    """A bumpy basin with moving water: compensated rain field, infiltration, open south
    and west edges and a rising fixed stage on the east edge."""
    rng = np.random.default_rng(22)
    ny, nx, dx = 12, 13, 8.0
    bed = (_bumps(ny, nx, dx, rng, 5, (0.2, 1.0), (8.0, 30.0)) + 0.01 * np.arange(nx) * dx).astype(np.float32)
    depth = np.maximum(1.2 - bed, 0.0).astype(np.float32)
    hu0 = (rng.uniform(-0.2, 0.2, (ny, nx)) * (depth > 0)).astype(np.float32)
    hv0 = (rng.uniform(-0.2, 0.2, (ny, nx)) * (depth > 0)).astype(np.float32)
    rain = rng.uniform(0.0, 4e-5, (ny, nx)).astype(np.float32)
    infil = rng.uniform(0.0, 1e-5, (ny, nx)).astype(np.float32)
    return dict(scheme="hllc_fv", bed=bed, dx=dx, depth=depth, manning=0.03, hu0=hu0, hv0=hv0,
                rain_field=rain, rain_scale=1.0, infil=infil, compensated=True,
                boundaries=_bc(south="open", west="open", east="fixed_stage"),
                stage_curves={"east": [(0.0, 1.3), (15.0, 1.6), (90.0, 1.6)]},
                steps=14, alpha=0.45, dt_max=4.0)  # fmt: skip


COMBINED_CASES = {"li_reach_combined": combined_li_reach, "hllc_storm_combined": combined_hllc_storm}


def run_case(case: dict, api) -> dict:
    """Step ``case`` through ``api`` and return the recorded outputs.

    ``api`` adapts one implementation (reference, oracle or CUDA) to a fixed set of
    calls: ``make_state(case)``, ``compute_dt(st, alpha, dt_max)``,
    ``step(st, dt, rain, rain_scale, t)``, ``injector(case, st)`` returning an object
    with ``apply(st, t, dt)``, ``morphology(case, st)`` returning an object with
    ``advance(t, elapsed)``, and ``outputs(st, case)`` returning a dict of arrays.
    """
    st = api.make_state(case)
    inj = api.injector(case, st) if case.get("inflows") else None
    morph = api.morphology(case, st) if case.get("sediment") else None
    every = case["sediment"]["every"] if morph else 0
    res = api.reservoir(case, st) if case.get("reservoir") else None
    res_every = case["reservoir"]["every"] if res else 0
    t = 0.0
    dts, vols, releases = [], [], []
    last_act = last_rel = 0.0
    for k in range(case["steps"]):
        dt = api.compute_dt(st, case["alpha"], case["dt_max"])
        dts.append(dt)
        if inj is not None:
            vols.append(inj.apply(st, t, dt))
        api.step(st, dt, case.get("rain", 0.0), case.get("rain_scale", 1.0), t)
        t += dt
        if res is not None and (k + 1) % res_every == 0:
            rec = res.advance(t, t - last_rel)
            last_rel = t
            releases.append([rec.time, np.nan if rec.stage is None else rec.stage, rec.discharge_m3_s, rec.volume_m3])
        if morph is not None and (k + 1) % every == 0:
            morph.advance(t, t - last_act)
            last_act = t
    out = api.outputs(st, case)
    out["dts"] = np.asarray(dts, np.float64)
    if inj is not None:
        out["inflow_volumes"] = np.asarray(vols, np.float64)
    if res is not None:
        out["releases"] = np.asarray(releases, np.float64)
    return out
