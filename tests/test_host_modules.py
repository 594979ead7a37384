"""Host-side modules of the package: scheduler, Zarr store, status.json, config.

The scheduler is pinned tick for tick to fixtures recorded from the reference's own
``MultiRateScheduler`` (tests/golden/scheduler_ticks.json, made by
tests/golden/make_golden.py) for the same stub dt sequences.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from make_golden import SCHEDULER_CASES, _dt_fn
from rbsim.scheduler import MultiRateScheduler, SlowProcess, fill_span

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "scheduler_ticks.json")


@pytest.mark.parametrize("name", sorted(SCHEDULER_CASES))
def test_scheduler_replays_reference_ticks_exactly(name):
    want = json.load(open(GOLDEN))[name]
    end, every, events, procs, recipe = SCHEDULER_CASES[name]
    sp = [SlowProcess(name=n, interval=iv, advance=lambda t, e: None) for n, iv in procs]
    sched = MultiRateScheduler(end_time=end, output_every=every, events=events, processes=sp)
    assert sched.n_frames == want["n_frames"]
    assert sched.sync_times == want["sync"]
    got = [[t.index, t.t0, t.dt, t.t1, t.is_output, [[p.name, el] for p, el in t.due]]
           for t in sched.ticks(_dt_fn(recipe))]  # fmt: skip
    assert got == want["ticks"]


def test_fill_span_invariants():
    for span in (1.0, 7.3, 599.999999, 1e4, 3.0):
        for dt_raw in (0.1, 0.7, 2.0, 7.3, 1e5):
            dt = fill_span(span, dt_raw)
            assert dt <= dt_raw
            n = round(span / dt)
            assert abs(n * dt - span) < 1e-9 * max(span, 1.0)
    assert fill_span(float("inf"), 3.0) == 3.0


def test_scheduler_rejects_bad_inputs():
    with pytest.raises(ValueError):
        MultiRateScheduler(end_time=0.0, output_every=1.0)
    with pytest.raises(ValueError):
        MultiRateScheduler(end_time=10.0, output_every=0.0)
    with pytest.raises(ValueError):
        SlowProcess("p", 0.0, lambda t, e: None)
    sched = MultiRateScheduler(end_time=10.0, output_every=5.0)
    with pytest.raises(RuntimeError, match="non-positive timestep"):
        next(iter(sched.ticks(lambda: 0.0)))


def test_zarr_store_layout_and_roundtrip(tmp_path):
    from rbsim.grid import Grid
    from rbsim.io.zarr_writer import ZarrWriter, read_array, read_attrs

    g = Grid(3, 4, 10.0)
    w = ZarrWriter(tmp_path / "r.zarr", g, 3, {"scheme": "local_inertial", "dx": 10.0}, bed_change=True)
    bed = np.arange(12, dtype=np.float32).reshape(3, 4)
    w.write_bed(bed)
    rng = np.random.default_rng(0)
    frames = [rng.random((4, 3, 4)).astype(np.float32) for _ in range(2)]
    for k, f in enumerate(frames):
        w.append(10.0 * k, f[0], f[1], f[2], f[3].astype(np.float64))
    with pytest.raises(ValueError, match="bed_change"):
        w.append(20.0, frames[0][0], frames[0][1], frames[0][2])
    w.finalize({"mass_gate": 1e-6, "series": [{"t": 1.0}]})
    store = tmp_path / "r.zarr"
    meta = json.loads((store / "depth" / "zarr.json").read_text())
    assert meta["zarr_format"] == 3 and meta["dimension_names"] == ["time", "y", "x"]
    assert meta["chunk_grid"]["configuration"]["chunk_shape"] == [1, 3, 4]
    assert (store / "depth" / "c" / "1" / "0" / "0").exists()
    depth = read_array(store, "depth")
    np.testing.assert_array_equal(depth[:2], np.stack([f[0] for f in frames]))
    np.testing.assert_array_equal(depth[2], 0.0)
    np.testing.assert_array_equal(read_array(store, "bed"), bed)
    np.testing.assert_array_equal(read_array(store, "time"), [0.0, 10.0, 0.0])
    attrs = read_attrs(store)
    assert attrs["n_frames"] == 2 and attrs["n_frames_allocated"] == 3 and attrs["mass_gate"] == 1e-6


def test_status_writer_states(tmp_path):
    from rbsim.io.status import StatusWriter

    s = StatusWriter(tmp_path / "status.json", end_time=100.0)
    s.write("starting")
    s.write("running", sim_time=25.0, message="t=25s")
    rec = json.loads((tmp_path / "status.json").read_text())
    assert rec["state"] == "running" and rec["progress"] == 0.25 and rec["message"] == "t=25s"
    s.write("done", sim_time=50.0)
    assert json.loads((tmp_path / "status.json").read_text())["progress"] == 1.0
    with pytest.raises(ValueError):
        s.write("paused")
    assert sorted(q.name for q in tmp_path.iterdir()) == ["status.json"]


def test_status_writer_drops_an_update_that_cannot_land(tmp_path, monkeypatch):
    """solver/io/status.py:96-117: a rename a reader keeps blocking drops that one update."""
    import rbsim.io.status as status_mod

    s = status_mod.StatusWriter(tmp_path / "status.json", end_time=10.0)
    assert s.write("starting") is True
    assert s.document("starting")["eta_s"] is None

    def blocked(src, dst):
        raise PermissionError("held by a reader")

    monkeypatch.setattr(status_mod, "RENAME_DEADLINE_S", 0.01)
    monkeypatch.setattr(status_mod.os, "replace", blocked)
    assert s.write("running", sim_time=5.0) is False and s.dropped == 1
    monkeypatch.undo()
    assert json.loads((tmp_path / "status.json").read_text())["state"] == "starting"
    assert sorted(q.name for q in tmp_path.iterdir()) == ["status.json"]


def test_exact_sum_is_exact():
    import math
    import random

    from rbsim.massbalance import ExactSum

    rng = random.Random(7)
    for trial in range(20):
        xs = [rng.uniform(-1, 1) * 10.0 ** rng.randint(-20, 20) for _ in range(500)]
        acc = ExactSum()
        for x in xs:
            acc.add(x)
        assert acc.value == math.fsum(xs)
    acc = ExactSum()
    acc.add(1e16)
    for _ in range(1000):
        acc.add(1.0)  # each add alone is below half an ulp of the total
    acc.add(-1e16)
    assert acc.value == 1000.0


class _FakeGrid:
    cell_area = 4.0


class _FakeState:
    """Duck-typed stand-in for State: the ledger reads only these on the host."""

    def __init__(self, volume, loss):
        self.grid = _FakeGrid()
        self.volume, self.loss = volume, loss

    def volume_sum(self):
        return self.volume

    def loss_volume(self, area):
        return self.loss * area


def test_mass_ledger_residual_and_causal_peak():
    """solver/core/massbalance.py:109-135: residual = in - out - (V - V0), relative to a causal peak."""
    from rbsim.massbalance import MASS_GATE, MassLedger

    st = _FakeState(volume=100.0, loss=0.0)
    led = MassLedger.from_state(st)
    assert led.series[0].residual == 0.0 and led.v0 == 400.0
    led.add_rain_step(1e-3, 10.0, 25)  # 1e-3 m/s * 10 s * 4 m^2 * 25 cells = 1 m^3
    st.volume = 100.25
    rec = led.record(st, 10.0)
    assert rec.inflow_cum == pytest.approx(1.0) and rec.residual == pytest.approx(0.0, abs=1e-12)
    # drain to empty through a sink: the scale stays the peak volume, not the empty domain
    st.volume, st.loss = 0.0, 100.25 + 1e-6
    rec = led.record(st, 20.0)
    assert rec.outflow_cum == pytest.approx(401.0 + 4e-6)
    assert rec.rel_error == pytest.approx(abs(rec.residual) / 401.0)
    assert led.max_rel_error == rec.rel_error and rec.rel_error < MASS_GATE
    attrs = led.as_attrs()
    assert attrs["mass_gate"] == MASS_GATE and len(attrs["mass_balance_series"]) == 3
    assert set(attrs["mass_balance_series"][0]) == {"time", "volume", "inflow_cum", "outflow_cum", "residual",
                                                    "rel_error"}


def test_config_loader(tmp_path):
    from rbsim.config import ConfigError, load_config

    (tmp_path / "n.r32").write_bytes(np.full((4, 5), 0.04, "<f4").tobytes())
    toml = tmp_path / "s.toml"
    toml.write_text(
        '[meta]\nname = "t"\nscheme = "local_inertial"\n[grid]\ndx = 10.0\nshape = [4, 5]\n'
        '[run]\nend_time = 600.0\noutput_every = 60.0\ncfl = 0.7\n'
        '[rainfall]\ntype = "uniform"\nrate_mm_hr = 36.0\nduration_s = 300.0\n'
        '[parameters]\nmanning_n = "n.r32"\ninfiltration = 2.0\n'
        '[sediment]\nd50 = 0.002\nporosity = 0.4\ninterval_s = 120.0\n'
        '[[inflow]]\ncell = [1, 2]\nhydrograph = [[0.0, 1.0], [600.0, 2.0]]\n'
        '[boundaries]\ndefault = "closed"\neast = "open"\n'
    )
    sc = load_config(toml)
    assert sc.rain_m_s == pytest.approx(1e-5) and sc.boundaries["east"] == "open"
    assert sc.manning.shape == (4, 5) and sc.has_sediment and sc.inflows[0].cell == (1, 2)
    bad = tmp_path / "b.toml"
    bad.write_text('[meta]\nscheme = "hllc_fv"\n[sediment]\nd50 = 0.002\n')
    with pytest.raises(ConfigError, match="local-inertial-only"):
        load_config(bad)
    bad.write_text('[meta]\nscheme = "local_inertial"\n[boundaries]\neast = { type = "fixed_stage", level = 1.0 }\n')
    with pytest.raises(ConfigError, match="hllc_fv"):
        load_config(bad)
    bad.write_text("[channels]\nwidth = 3.0\n")  # a width without a bank-full depth
    with pytest.raises(ConfigError, match="bank-full depth"):
        load_config(bad)
    bad.write_text('[meta]\nscheme = "hllc_fv"\n[channels]\nwidth = 3.0\ndepth = 1.0\n')
    with pytest.raises(ConfigError, match="local_inertial"):
        load_config(bad)
    bad.write_text('[channels]\nwidth = 3.0\ndepth = 1.5\nmanning = 0.03\n'
                   '[[structures]]\nname = "d"\ncells = [[1, 1], [1, 2]]\ncrest_m = 5.0\n'
                   'release_rule = "fixed"\nrelease_m3_s = 2.0\npool = [0, 0, 0, 4]\noutlet = [3, 2]\n')
    sc = load_config(bad)
    assert sc.has_channels and sc.channel_depth == 1.5 and sc.channel_manning == 0.03
    (dam,) = sc.structures
    assert dam.outlet == (3, 2, 3, 2) and dam.cells == [(1, 1), (1, 2)] and dam.discharge_at(4.0) == 2.0
    bad.write_text('[[structures]]\nname = "d"\ncells = [[1, 1]]\ncrest_m = 5.0\nrelease_rule = "fixed"\n'
                   'release_m3_s = 2.0\npool = [0, 0, 2, 4]\noutlet = [1, 2]\n')
    with pytest.raises(ConfigError, match="overlaps the pool"):
        load_config(bad)


def test_main_writes_error_status_on_bad_config(tmp_path):
    """solver/test_run.py:142: a config the loader refuses is reported through status.json
    (state "error", the loader's message) and re-raised, so a polling viewer does not wait forever."""
    from rbsim.config import ConfigError
    from rbsim.run import main

    cfg = tmp_path / "bad.toml"
    cfg.write_text("[rainfall]\ntype = 'storm_cells'\n", encoding="utf-8")
    status = tmp_path / "status.json"
    with pytest.raises(ConfigError):
        main(["--config", str(cfg), "--out", str(tmp_path / "out.zarr"), "--status", str(status)])
    rec = json.loads(status.read_text(encoding="utf-8"))
    assert rec["state"] == "error" and "storm_cells" in rec["message"]
    with pytest.raises(ConfigError, match="not found"):
        main(["--config", str(tmp_path / "missing.toml"), "--status", str(status)])
    assert json.loads(status.read_text(encoding="utf-8"))["state"] == "error"


def test_a_config_that_cannot_be_read_is_a_config_error(tmp_path):
    """solver/io/test_config.py:316, and a file that is not TOML."""
    from rbsim.config import ConfigError, load_config

    with pytest.raises(ConfigError, match="not found"):
        load_config(tmp_path / "nope.toml")
    broken = tmp_path / "broken.toml"
    broken.write_text("[grid\ndx = ", encoding="utf-8")
    with pytest.raises(ConfigError, match="not valid TOML"):
        load_config(broken)


_RUN = ('[meta]\nname = "r"\nscheme = "local_inertial"\n[grid]\ndx = 10.0\n'
        '[run]\nend_time = 1200.0\noutput_every = 300.0\ndt_max = 20.0\ncfl = 0.6\n'
        '[rainfall]\ntype = "uniform"\nrate_mm_hr = 40.0\nduration_s = 600.0\n'
        '[parameters]\nmanning_n = 0.03\ninfiltration = 1.0\n')  # fmt: skip


@pytest.mark.parametrize(("mutation", "repl", "needle"), [
    ("output_every = 300.0", "output_every = 0.0", "output_every"),
    ("end_time = 1200.0", "end_time = -5.0", "end_time"),
    ("dt_max = 20.0", "dt_max = 0.0", "dt_max"),
    ("cfl = 0.6", "cfl = 0.0", "cfl"),
    ("end_time = 1200.0", "end_time = 1000.0", "multiple of output_every"),
    ("manning_n = 0.03", "manning_n = -0.01", "manning_n"),
    ("infiltration = 1.0", "infiltration = -1.0", "infiltration"),
    ("rate_mm_hr = 40.0", "rate_mm_hr = -1.0", "rainfall rate"),
])  # fmt: skip
def test_bad_run_params_rejected(tmp_path, mutation, repl, needle):
    """solver/io/test_config.py:337."""
    from rbsim.config import ConfigError, load_config

    assert mutation in _RUN
    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN.replace(mutation, repl))
    with pytest.raises(ConfigError, match=needle):
        load_config(cfg)


def test_high_cfl_warns_but_loads(tmp_path):
    """solver/io/test_config.py:343."""
    from rbsim.config import load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN.replace("cfl = 0.6", "cfl = 5.0"))
    with pytest.warns(UserWarning, match="stability limit"):
        assert load_config(cfg).alpha == 5.0


def test_scenario_validates_direct_construction():
    """solver/io/test_config.py:349 and solver/test_run.py:205, :220: the in-code path is checked too."""
    from rbsim.config import Scenario

    with pytest.raises(ValueError, match="output_every"):
        Scenario(output_every=0.0)
    with pytest.raises(ValueError, match="multiple of output_every"):
        Scenario(end_time=3500.0, output_every=300.0)
    stage = {"north": "fixed_stage", "south": "closed", "east": "closed", "west": "closed"}
    with pytest.raises(ValueError, match="hllc_fv"):
        Scenario(scheme="local_inertial", boundaries=stage, stage_curves={"north": [(0.0, 1.0)]})
    with pytest.raises(ValueError, match="no stage curve"):
        Scenario(scheme="hllc_fv", boundaries=stage)
    with pytest.raises(ValueError, match="unknown boundary"):
        Scenario(boundaries={"north": "leaky"})
    Scenario(scheme="hllc_fv", boundaries=stage, stage_curves={"north": [(0.0, 1.0)]}, end_time=600.0,
             output_every=300.0)  # fmt: skip


_HLLC_RUN = _RUN.replace('scheme = "local_inertial"', 'scheme = "hllc_fv"') + '[boundaries]\ndefault = "closed"\n'


@pytest.mark.parametrize(("table", "needle"), [
    ('{ type = "fixed_stage" }', "exactly one of"),
    ('{ type = "fixed_stage", level = 1.0, stage = [[0.0, 1.0]] }', "exactly one of"),
    ('{ type = "fixed_stage", level = "high" }', "must be a number"),
    ('{ type = "fixed_stage", stage = [] }', "non-empty"),
    ('{ type = "fixed_stage", stage = [[10.0, 1.0], [0.0, 2.0]] }', "non-decreasing"),
    ('{ type = "tidal" }', "unknown boundary type"),
    ("42", "must be 'closed'"),
    ('"fixed_stage"', "fixed_stage table"),
])  # fmt: skip
def test_fixed_stage_malformed(tmp_path, table, needle):
    """solver/io/test_config.py:423, :429."""
    from rbsim.config import ConfigError, load_config

    cfg = tmp_path / "s.toml"
    cfg.write_text(_HLLC_RUN + f"east = {table}\n")
    with pytest.raises(ConfigError, match=needle):
        load_config(cfg)


def test_fixed_stage_level_and_curve(tmp_path):
    """solver/io/test_config.py:380, :390: a level is a one-point curve; curve knots are sync events."""
    from rbsim.config import load_config

    cfg = tmp_path / "s.toml"
    cfg.write_text(_HLLC_RUN + 'east = { type = "fixed_stage", level = 10.35 }\n'
                   'west = { type = "fixed_stage", stage = [[0.0, 9.7], [3600.0, 10.35], [7200.0, 9.7]] }\n')  # fmt: skip
    sc = load_config(cfg)
    assert sc.boundaries["east"] == sc.boundaries["west"] == "fixed_stage"
    assert sc.stage_curves["east"] == [(0.0, 10.35)]
    assert sc.stage_curves["west"] == [(0.0, 9.7), (3600.0, 10.35), (7200.0, 9.7)]
    assert sc.stage_events == [0.0, 3600.0, 7200.0]


@pytest.mark.parametrize(("mutation", "repl", "needle"), [
    ('type = "uniform"\nrate_mm_hr = 40.0', 'type = "field"', "requires a 'field' path"),
    ("manning_n = 0.03", "manning_n = true", "manning_n"),
    ('scheme = "local_inertial"', 'scheme = "quantum_flux"', "known scheme"),
    ("infiltration = 1.0", 'infiltration = "absent.r32"', "not found"),
])  # fmt: skip
def test_config_refusals(tmp_path, mutation, repl, needle):
    """solver/io/test_config.py:156, :218, :310: a missing rain field path, a boolean roughness, an
    unknown scheme, and a field file that is not there."""
    from rbsim.config import ConfigError, load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN.replace(mutation, repl).replace("[grid]\n", "[grid]\nshape = [4, 5]\n"))
    with pytest.raises(ConfigError, match=needle):
        load_config(cfg)


def test_inflow_hydrograph_parsed_and_bad_shapes_rejected(tmp_path):
    """solver/io/test_config.py:162, :173."""
    from rbsim.config import ConfigError, load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN + "[[inflow]]\ncell = [10, 20]\nhydrograph = [[0.0, 0.0], [600.0, 5.0]]\n")
    (inf,) = load_config(cfg).inflows
    assert inf.cell == (10, 20) and inf.breakpoints == [0.0, 600.0]
    assert inf.discharge_at(300.0) == pytest.approx(2.5) and inf.discharge_at(1e9) == 0.0
    cfg.write_text(_RUN + "[[inflow]]\ncell = [10]\nhydrograph = [[0.0, 0.0]]\n")
    with pytest.raises(ConfigError, match="cell"):
        load_config(cfg)
    cfg.write_text(_RUN + "[[inflow]]\ncell = [1, 2]\nhydrograph = [[0.0]]\n")
    with pytest.raises(ConfigError, match="hydrograph"):
        load_config(cfg)


def test_sediment_table(tmp_path):
    """solver/io/test_config.py:545-630: defaults, refusals, and the typo guard."""
    from rbsim.config import ConfigError, load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN + '[sediment]\nd50 = 0.008\nporosity = 0.35\nlaw = "mpm"\ninterval_s = 600.0\n'
                   "alluvium_thickness = 2.0\n")  # fmt: skip
    sc = load_config(cfg)
    assert sc.has_sediment and sc.sediment_d50 == 0.008 and sc.sediment_porosity == 0.35
    assert sc.sediment_interval_s == 600.0 and sc.alluvium_thickness == 2.0
    cfg.write_text(_RUN + "[sediment]\nd50 = 0.01\n")
    sc = load_config(cfg)
    assert sc.sediment_porosity == 0.4 and sc.sediment_interval_s == 900.0 and sc.alluvium_thickness is None
    cfg.write_text(_RUN)
    assert not load_config(cfg).has_sediment
    for bad, needle in (("porosity = 0.4", "needs a grain size"), ("d50 = 0.0", "needs a grain size"),
                        ("d50 = 0.008\nporosity = 0.0", r"porosity must be in \(0, 1\)"),
                        ("d50 = 0.008\nporosity = 1.0", r"porosity must be in \(0, 1\)"),
                        ("d50 = 0.008\ninterval_s = 0.0", "interval_s must be > 0"),
                        ("d50 = 0.008\nalluvium_thickness = -1.0", "alluvium_thickness must be >= 0"),
                        ('d50 = 0.008\nlaw = "engelund_hansen"', "not a transport law"),
                        ('d50 = 0.008\nporosity = "wet"', r"\[sediment\] porosity must be a number")):  # fmt: skip
        cfg.write_text(_RUN + f"[sediment]\n{bad}\n")
        with pytest.raises(ConfigError, match=needle):
            load_config(cfg)
    cfg.write_text(_RUN + "[sediment]\nd_50 = 0.008\n")
    with pytest.warns(UserWarning, match="unknown key 'd_50'"):
        with pytest.raises(ConfigError, match="needs a grain size"):
            load_config(cfg)
    cfg.write_text(_RUN.replace('scheme = "local_inertial"', 'scheme = "hllc_fv"') + "[sediment]\nd50 = 0.008\n")
    with pytest.raises(ConfigError, match="requires scheme='local_inertial'"):
        load_config(cfg)


_DAM_TOML = ('[[structures]]\nname = "upper_dam"\ntype = "dam"\ncells = [[6, 4], [7, 4]]\ncrest_m = 145.0\n'
             'release_rule = "target_stage"\ntarget_stage_m = 143.0\nrelease_max_m3_s = 40.0\npool = [2, 0, 5, 9]\n'
             'outlet = [8, 4]\ninterval_s = 600.0\n')  # fmt: skip


def test_structures_parse(tmp_path):
    """solver/io/test_config.py:241-275: a dam with a target-stage rule, a one-cell levee, a fixed rule."""
    from rbsim.config import load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN + _DAM_TOML)
    (s,) = load_config(cfg).structures
    assert (s.name, s.kind, s.cells) == ("upper_dam", "dam", [(6, 4), (7, 4)])
    assert (s.crest_m, s.target_stage_m, s.release_max_m3_s, s.interval_s) == (145.0, 143.0, 40.0, 600.0)
    assert s.pool == (2, 0, 5, 9) and s.outlet == (8, 4, 8, 4)
    assert s.discharge_at(None) == 0.0 and s.discharge_at(142.0) == 0.0
    assert s.discharge_at(144.0) == pytest.approx(20.0) and s.discharge_at(150.0) == 40.0
    cfg.write_text(_RUN + '[[structures]]\ntype = "levee"\ncell = [3, 3]\ncrest_m = 12.0\n')
    (s,) = load_config(cfg).structures
    assert s.kind == "levee" and s.release_rule == "none" and s.cells == [(3, 3)]
    cfg.write_text(_RUN + '[[structures]]\ntype = "dam"\ncell = [5, 5]\ncrest_m = 20.0\nrelease_rule = "fixed"\n'
                   'release_m3_s = 7.5\npool = [0, 0, 4, 9]\noutlet = [6, 5]\n')  # fmt: skip
    (s,) = load_config(cfg).structures
    assert s.discharge_at(19.0) == 7.5 and s.discharge_at(1.0) == 7.5 and s.discharge_at(None) == 0.0


@pytest.mark.parametrize(("body", "needle"), [
    ('type = "weir"\ncell = [1, 1]\ncrest_m = 5.0', "type must be one of"),
    ('type = "dam"\ncrest_m = 5.0', "at least one barrier cell"),
    ('type = "dam"\ncell = [1, 1]', "crest_m' is required"),
    ('type = "dam"\ncell = [1, 1]\ncrest_m = 5.0\nrelease_rule = "spill"', "release_rule"),
    ('type = "levee"\ncell = [1, 1]\ncrest_m = 5.0\nrelease_rule = "fixed"\nrelease_m3_s = 1.0\npool = [0, 0, 0, 1]\n'
     "outlet = [3, 3]", "levee is barrier geometry only"),
    ('type = "dam"\ncell = [1, 1]\ncrest_m = 5.0\nrelease_rule = "fixed"\nrelease_m3_s = 1.0',
     "needs both a 'pool' box and an 'outlet'"),
    ('type = "dam"\ncell = [1, 1]\ncrest_m = 5.0\nrelease_rule = "fixed"\nrelease_m3_s = 1.0\npool = [0, 0, 3, 3]\n'
     "outlet = [1, 1]", "overlaps the pool"),
    ('type = "dam"\ncell = [1, 1]\ncrest_m = 5.0\nrelease_rule = "target_stage"\ntarget_stage_m = 6.0\n'
     "release_max_m3_s = 2.0\npool = [0, 0, 0, 1]\noutlet = [3, 3]", "must be below crest_m"),
])  # fmt: skip
def test_structure_validation(tmp_path, body, needle):
    """solver/io/test_config.py:305."""
    from rbsim.config import ConfigError, load_config

    cfg = tmp_path / "r.toml"
    cfg.write_text(_RUN + "[[structures]]\n" + body + "\n")
    with pytest.raises(ConfigError, match=needle):
        load_config(cfg)


def _fake_run(calls):
    """Stands in for run_simulation (which needs the device): writes a small result store
    of a filling basin, as a run would, and returns a ledger-shaped record."""
    from types import SimpleNamespace

    from rbsim.grid import Grid
    from rbsim.io.zarr_writer import ZarrWriter

    def run(sc, bed, out, **kw):
        calls.append((sc.name, str(out), kw))
        grid = Grid(ny=6, nx=9, dx=10.0)
        w = ZarrWriter(out, grid, 3, {"scheme": sc.scheme, "dx": 10.0, "coarsen": 1})
        z = np.linspace(0.0, 1.0, 54, dtype=np.float32).reshape(6, 9)
        w.write_bed(z)
        for i in range(3):
            d = np.full((6, 9), 0.1 * i, np.float32)
            w.append(300.0 * i, d, d * 0, d * 0)
        w.finalize({})
        return SimpleNamespace(max_rel_error=3.0e-9)

    return run


def test_main_runs_exports_frames_and_reports_done(tmp_path, monkeypatch):
    """solver/run.py:530-580: status.json beside the store by default, the viewer frames
    exported after the run (unless --no-frames), state "done" with the mass error."""
    import rbsim.run as run_mod

    calls = []
    monkeypatch.setattr(run_mod, "run_simulation", _fake_run(calls))
    cfg = tmp_path / "s.toml"
    cfg.write_text(_RUN)
    out = tmp_path / "res" / "r.zarr"
    assert run_mod.main(["--config", str(cfg), "--out", str(out)]) == 0
    rec = json.loads((out.parent / "status.json").read_text())
    assert rec["state"] == "done" and rec["progress"] == 1.0 and "mass_max_rel_err=3.00e-09" in rec["message"]
    assert (out.parent / "frames" / "manifest.json").is_file()
    assert calls[0][0] == "r" and calls[0][2]["use_device_clock"] is True
    out2 = tmp_path / "other" / "r.zarr"
    assert run_mod.main(["--config", str(cfg), "--out", str(out2), "--no-frames", "--host-loop",
                         "--status", str(tmp_path / "st.json")]) == 0  # fmt: skip
    assert not (out2.parent / "frames").exists() and calls[1][2]["use_device_clock"] is False
    assert json.loads((tmp_path / "st.json").read_text())["state"] == "done"


def test_main_reports_a_failed_run_with_its_exception_type(tmp_path, monkeypatch):
    import rbsim.run as run_mod

    def boom(*a, **kw):
        raise RuntimeError("the device clock made no progress")

    monkeypatch.setattr(run_mod, "run_simulation", boom)
    cfg = tmp_path / "s.toml"
    cfg.write_text(_RUN)
    with pytest.raises(RuntimeError):
        run_mod.main(["--config", str(cfg), "--out", str(tmp_path / "r.zarr")])
    rec = json.loads((tmp_path / "status.json").read_text())
    assert rec["state"] == "error" and rec["message"] == "RuntimeError: the device clock made no progress"
