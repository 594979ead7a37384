"""Failure detection on the CUDA path, without any GPU fault.

A non-finite depth (a NaN or infinity planted in the input state on the host) is
ordinary float arithmetic on the device; the step kernels flag it in the
workspace error word, and every host entry that reads the device back (the
scheme's check, the device clock, the ensemble) turns the flag into
``DeviceError``. Argument errors come back as Python exceptions before anything
is launched.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _li_state(poison=None):
    import rbsim

    n = 64
    depth = np.full((n, n), 0.5, np.float32)
    if poison is not None:
        depth[10, 20] = poison
    return rbsim.State.from_bed(np.zeros((n, n), np.float32), 10.0, depth=depth, manning=0.03)


def _hllc_state():
    import rbsim
    from rbsim.schemes import hllc

    n = 48
    depth = np.where(np.arange(n)[None, :] < n // 2, 2.0, 1.0).astype(np.float32) * np.ones((n, 1), np.float32)
    st = rbsim.State.from_bed(np.zeros((n, n), np.float32), 1.0, depth=depth, manning=0.02)
    hllc.arm_hllc(st)
    return st


@pytest.mark.parametrize("poison", [float("nan"), float("inf")])
def test_non_finite_depth_is_flagged_by_the_li_step(poison):
    from rbsim import _lib
    from rbsim.schemes import local_inertial as li

    st = _li_state(poison)
    li.step(st, dt=0.5)
    with pytest.raises(_lib.DeviceError):
        st.check_device_errors()
    st.check_device_errors()  # reading clears the word
    clean = _li_state()
    li.step(clean, dt=0.5)
    clean.check_device_errors()


def test_an_overflowing_rain_source_is_flagged_by_the_hllc_step():
    """HLLC clamps every stage's depth with the reference's max(h, 0), which turns a
    NaN into 0 and resets its momentum, so a planted NaN never survives a step. What
    can reach the stored state is a source added after the clamp: a rain rate whose
    depth over the step overflows float32."""
    from rbsim import _lib
    from rbsim.schemes import hllc

    st = _hllc_state()
    hllc.step(st, dt=10.0, rain=3.0e38)
    with pytest.raises(_lib.DeviceError):
        st.check_device_errors()


@pytest.mark.parametrize("poison", [float("nan"), float("inf")])
def test_the_device_clock_stops_and_raises_on_a_non_finite_state(poison):
    from rbsim import _lib
    from rbsim.device_clock import DeviceClock

    st = _li_state(poison)
    clk = DeviceClock(st, "local_inertial", alpha=0.5, dt_max=1.0, sync_times=[100.0], graph_steps=4)
    with pytest.raises((_lib.DeviceError, RuntimeError)):
        clk.run_until(100.0, max_steps=8)
    clk.close()


def test_an_ensemble_member_with_a_non_finite_state_raises():
    from rbsim import _lib
    from rbsim.ensemble import Ensemble

    members = [_li_state(), _li_state(float("nan"))]
    ens = Ensemble(members, ["local_inertial"] * 2, alpha=0.5, dt_max=1.0, sync_times=[[50.0]] * 2, graph_steps=4)
    with pytest.raises((_lib.DeviceError, RuntimeError)):
        ens.run_until(50.0, max_replays=8)


def test_argument_errors_raise_before_any_launch():
    from rbsim.schemes import hllc
    from rbsim.schemes import local_inertial as li

    st = _li_state()
    with pytest.raises((ValueError, RuntimeError)):
        li.step(st, dt=0.0)
    with pytest.raises((ValueError, RuntimeError)):
        li.step(st, dt=float("nan"))
    hs = _hllc_state()
    with pytest.raises((ValueError, RuntimeError)):
        hllc.step(hs, dt=-1.0)
    st.check_device_errors()
    hs.check_device_errors()
