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


@pytest.mark.parametrize("make", [_li_scenario, _hllc_scenario])
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
