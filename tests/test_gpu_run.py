"""run_simulation end to end: the device-clock path equals the host loop, bit for bit.

Scenarios reach every source the clock samples on the device: uniform rain with
an end time, point inflows with hydrograph knots, infiltration, open edges,
morphology activations (LI), and a fixed_stage curve (HLLC). The stores written by
the two paths must be identical frame by frame, and the mass ledger must close.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _li_scenario():
    from rbsim.config import Scenario
    from rbsim.processes.inflow import Inflow

    ny, nx, dx = 48, 64, 20.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    bed = (5e-3 * (nx - 1 - xx) * dx + 0.3 * np.cos(yy * 0.25)).astype(np.float32)
    return Scenario(
        name="li_mix", scheme="local_inertial", dx=dx, end_time=1200.0, output_every=200.0, alpha=0.7,
        dt_max=20.0, initial_depth=0.05, rain_mm_hr=40.0, rain_duration=500.0, manning=0.03,
        infiltration_mm_hr=3.0, boundaries={"north": "closed", "south": "closed", "east": "open", "west": "closed"},
        inflows=[Inflow((10, 2), [(0.0, 0.0), (300.0, 8.0), (900.0, 0.0)]), Inflow((30, 3), [(0.0, 2.0), (1200.0, 2.0)])],
        sediment_d50=0.002, sediment_porosity=0.4, sediment_interval_s=300.0, bed=bed,
    )  # fmt: skip


def _hllc_scenario():
    from rbsim.config import Scenario

    ny, nx, dx = 40, 56, 5.0
    xx = np.broadcast_to(np.arange(nx), (ny, nx)).astype(np.float64)
    bed = (2e-3 * xx * dx).astype(np.float32)
    return Scenario(
        name="hllc_stage", scheme="hllc_fv", dx=dx, end_time=120.0, output_every=30.0, alpha=0.45, dt_max=10.0,
        initial_depth=0.4, manning=0.03, boundaries={"north": "closed", "south": "closed", "east": "fixed_stage",
                                                     "west": "open"},
        stage_curves={"east": [(0.0, 0.9), (60.0, 1.2), (200.0, 1.2)]}, bed=bed,
    )  # fmt: skip


def _dam(**kw):
    from rbsim.config import Structure

    base = dict(name="d", kind="dam", cells=[(6, j) for j in range(8)], crest_m=5.0, release_rule="fixed",
                release_m3_s=2.0, pool=(0, 0, 5, 7), outlet=(8, 2, 10, 5), interval_s=300.0)  # fmt: skip
    base.update(kw)
    return Structure(**base)


def _basin():
    z = np.zeros((12, 8), np.float32)
    z[:7] = 2.0
    z[7:] = np.linspace(2.0, 0.0, 5, dtype=np.float32)[:, None]
    return z


def _hllc_reservoir_scenario(**kw):
    """The reference's reservoir run (solver/processes/test_reservoir.py:227-238)."""
    from rbsim.config import Scenario

    base = dict(name="reservoir_run", scheme="hllc_fv", dx=10.0, end_time=1200.0, output_every=600.0, dt_max=5.0,
                alpha=0.45, initial_depth=1.0, structures=[_dam()], bed=_basin())  # fmt: skip
    base.update(kw)
    return Scenario(**base)


def _li_channel_reservoir_scenario():
    """Sub-grid channel along a valley, a dam across it with a target-stage rule, rain and an open toe."""
    from rbsim.config import Scenario, Structure

    ny, nx, dx = 20, 40, 25.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    bed = (2e-3 * (nx - 1 - xx) * dx + 0.02 * np.abs(yy - 9.5) * dx).astype(np.float32)
    w = np.zeros((ny, nx), np.float32)
    w[9:11, :] = 10.0
    dam = Structure(name="weir", cells=[(i, 20) for i in range(ny)], crest_m=float(bed[9, 20]) + 1.5,
                    release_rule="target_stage", target_stage_m=float(bed[9, 20]) + 0.5, release_max_m3_s=6.0,
                    pool=(5, 12, 14, 19), outlet=(8, 24, 11, 25), interval_s=120.0)  # fmt: skip
    return Scenario(
        name="li_channel_reservoir", scheme="local_inertial", dx=dx, end_time=900.0, output_every=300.0, alpha=0.7,
        dt_max=10.0, initial_depth=0.3, rain_mm_hr=20.0, rain_duration=600.0, manning=0.04,
        boundaries={"north": "closed", "south": "closed", "east": "open", "west": "closed"},
        channel_width=w, channel_depth=np.where(w > 0, 1.2, 0.0).astype(np.float32), channel_manning=0.03,
        structures=[dam], bed=bed,
    )  # fmt: skip


@pytest.mark.parametrize("make", [_li_scenario, _hllc_scenario, _hllc_reservoir_scenario,
                                  _li_channel_reservoir_scenario])
def test_device_clock_run_equals_host_loop(make, tmp_path):
    from rbsim.io.zarr_writer import read_array, read_attrs
    from rbsim.run import run_simulation

    stores = {}
    for mode, dev in (("host", False), ("device", True)):
        out = tmp_path / f"{mode}.zarr"
        ledger = run_simulation(make(), None, out, verbose=False, use_device_clock=dev, graph_steps=8)
        assert ledger.max_rel_error < 1e-6, (mode, ledger.max_rel_error)
        stores[mode] = out
    for name in ("time", "depth", "u", "v", "bed"):
        np.testing.assert_array_equal(read_array(stores["device"], name), read_array(stores["host"], name),
                                      err_msg=name)  # fmt: skip
    a_dev, a_host = read_attrs(stores["device"]), read_attrs(stores["host"])
    assert a_dev["n_frames"] == a_host["n_frames"]
    if "morphology" in a_host:
        np.testing.assert_array_equal(read_array(stores["device"], "bed_change"),
                                      read_array(stores["host"], "bed_change"))  # fmt: skip
        assert len(a_dev["morphology"]) == len(a_host["morphology"]) == 4
        assert a_dev["sediment_max_rel_error"] < 1e-11
    for rd, rh in zip(a_dev["mass_balance_series"], a_host["mass_balance_series"], strict=True):
        assert rd["volume"] == pytest.approx(rh["volume"], rel=1e-14)
        assert rd["inflow_cum"] == pytest.approx(rh["inflow_cum"], rel=1e-12)
    if "reservoir_releases" in a_host:
        assert a_dev["reservoir_releases"] == a_host["reservoir_releases"]


def test_reservoir_releases_land_on_the_slow_clock(tmp_path):
    """solver/processes/test_reservoir.py:241, :259, :283 -- releases at exact multiples of the
    interval, independent of dt_max; the dam is in the stored bed; a rule changes the run."""
    from rbsim.io.zarr_writer import read_array, read_attrs
    from rbsim.run import run_simulation

    ledger = run_simulation(_hllc_reservoir_scenario(), None, tmp_path / "res.zarr", verbose=False)
    assert ledger.max_rel_error < 1e-6
    series = read_attrs(tmp_path / "res.zarr")["reservoir_releases"]["d"]
    assert [r["time"] for r in series] == pytest.approx([300.0, 600.0, 900.0, 1200.0])
    assert all(r["volume_m3"] > 0.0 for r in series)
    assert float(read_array(tmp_path / "res.zarr", "bed")[6, 0]) == pytest.approx(5.0)

    times = []
    for tag, dt_max in (("coarse", 5.0), ("fine", 1.0)):
        sc = _hllc_reservoir_scenario(structures=[_dam(interval_s=400.0)], dt_max=dt_max)
        run_simulation(sc, None, tmp_path / f"{tag}.zarr", verbose=False)
        times.append([r["time"] for r in read_attrs(tmp_path / f"{tag}.zarr")["reservoir_releases"]["d"]])
    assert times[0] == pytest.approx([400.0, 800.0, 1200.0]) and times[0] == pytest.approx(times[1])

    off = _hllc_reservoir_scenario(structures=[_dam(release_rule="none", pool=None, outlet=None)])
    on = _hllc_reservoir_scenario(structures=[_dam(release_m3_s=4.0)])
    run_simulation(off, None, tmp_path / "off.zarr", verbose=False)
    run_simulation(on, None, tmp_path / "on.zarr", verbose=False)
    a = read_array(tmp_path / "off.zarr", "depth")[-1]
    b = read_array(tmp_path / "on.zarr", "depth")[-1]
    assert float(a[:6].astype(np.float64).sum()) > float(b[:6].astype(np.float64).sum())


def test_channel_run_writes_its_geometry(tmp_path):
    from rbsim.io.zarr_writer import read_array, read_attrs
    from rbsim.run import run_simulation

    sc = _li_channel_reservoir_scenario()
    run_simulation(sc, None, tmp_path / "ch.zarr", verbose=False)
    attrs = read_attrs(tmp_path / "ch.zarr")
    assert attrs["channels"]["channel_cells"] == 80
    np.testing.assert_array_equal(read_array(tmp_path / "ch.zarr", "channel_width"), sc.channel_width)
