"""The device-resident clock replays the host run loop bit for bit.

Host loop: ``MultiRateScheduler.ticks(compute_dt)`` + ``step`` per tick, rain gated
on ``t < rain_duration - EPS_T`` and banked with ``add_rain_step`` (the shape of
solver/run.py:369-388). Device loop: ``DeviceClock`` with the scheduler's sync
times, CUDA-graph replays, stopping at each output time. Same step count, same
simulated times, identical fields at every output and the same banked rain.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _li_state(n=96, seed=3):
    import rbsim

    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    z = 2e-3 * xx * 10.0 + 0.5 * np.sin(yy * 0.2) * np.cos(xx * 0.15)
    st = rbsim.State.from_bed(z.astype(np.float32), 10.0, depth=rng.uniform(0, 0.2, (n, n)).astype(np.float32),
                              manning=0.03)  # fmt: skip
    st.arm_source_compensation()
    st.set_infiltration(np.full((n, n), 2e-6, np.float32))
    st.set_open_boundaries({"east": "open", "south": "open"})
    return st


def _li_channel_state(n=96, seed=4):
    """The LI state above plus a sub-grid channel along the valley rows."""
    from rbsim.channels import arm_channels

    st = _li_state(n, seed)
    rng = np.random.default_rng(seed + 100)
    w = np.zeros((n, n), np.float32)
    d = np.zeros((n, n), np.float32)
    w[n // 2 - 1 : n // 2 + 1, :] = rng.uniform(2.0, 8.0, (2, n)).astype(np.float32)
    d[n // 2 - 1 : n // 2 + 1, :] = rng.uniform(0.5, 1.5, (2, n)).astype(np.float32)
    arm_channels(st, w, d, np.full((n, n), 0.025, np.float32))
    return st


def _hllc_state(n=80):
    import rbsim
    from rbsim.schemes import hllc

    depth = np.ones((n, n), np.float32)
    depth[:, : n // 2] = 3.0
    st = rbsim.State.from_bed(np.zeros((n, n), np.float32), 1.0, depth=depth, manning=0.02)
    hllc.arm_hllc(st)
    return st


def _host_run(st, scheme_name, end, every, rain, rain_dur, alpha, dt_max):
    import rbsim
    from rbsim.scheduler import EPS_T, MultiRateScheduler

    scheme = rbsim.get_scheme(scheme_name)
    sched = MultiRateScheduler(end_time=end, output_every=every, events=[rain_dur])
    frames, rain_vol, nsteps = [], 0.0, 0
    area, ncell = st.grid.cell_area, st.grid.n_cells
    for tick in sched.ticks(lambda: scheme.compute_dt(st, alpha=alpha, dt_max=dt_max)):
        r = rain if tick.t0 < rain_dur - EPS_T else 0.0
        scheme.step(st, dt=tick.dt, rain=r, t=tick.t0)
        if r > 0.0:
            rain_vol += r * tick.dt * area * ncell
        nsteps += 1
        if tick.is_output:
            frames.append((tick.t1, nsteps, st.h.cpu().numpy().copy()))
    return frames, rain_vol, sched.sync_times


@pytest.mark.parametrize("scheme_name", ["local_inertial", "local_inertial+channels", "hllc_fv"])
@pytest.mark.parametrize("graph_steps", [1, 7, 32])
def test_device_clock_matches_host_scheduler(scheme_name, graph_steps):
    from rbsim.device_clock import DeviceClock

    if scheme_name.startswith("local_inertial"):
        end, every, rain, rain_dur, alpha, dt_max = 600.0, 120.0, 30.0 / 3.6e6, 250.0, 0.7, 30.0
        make = _li_channel_state if scheme_name.endswith("channels") else _li_state
        scheme_name = "local_inertial"
    else:
        end, every, rain, rain_dur, alpha, dt_max = 6.0, 1.5, 1e-4, 2.0, 0.45, 30.0
        make = _hllc_state
    host = make()
    frames, rain_vol, sync = _host_run(host, scheme_name, end, every, rain, rain_dur, alpha, dt_max)

    dev = make()
    clk = DeviceClock(dev, scheme_name, alpha=alpha, dt_max=dt_max, sync_times=sync, rain_rate=rain,
                      rain_until=rain_dur, graph_steps=graph_steps)  # fmt: skip
    for t_out, nsteps, h in frames:
        clk.run_until(t_out)
        assert abs(clk.t - t_out) < 1e-6
        assert clk.steps == nsteps
        np.testing.assert_array_equal(dev.h.cpu().numpy(), h)
    assert clk.rain_volume == pytest.approx(rain_vol, rel=1e-13, abs=0.0)
    np.testing.assert_array_equal(dev.h.cpu().numpy(), host.h.cpu().numpy())
    if dev.loss_cum is not None:
        assert dev.loss_cum.total() == pytest.approx(host.loss_cum.total(), rel=1e-12)
    clk.close()


def test_device_clock_span_budget_is_exact():
    from rbsim.device_clock import DeviceClock

    st = _hllc_state(64)
    clk = DeviceClock(st, "hllc_fv", alpha=0.45, dt_max=30.0, sync_times=[1000.0], graph_steps=16)
    assert clk.run_until(1000.0, max_steps=37) == 37
    assert clk.run_until(1000.0, max_steps=5) == 5
    assert clk.steps == 42
