"""The headline configuration at full size, checked against physics.

The 2048 x 2048 HLLC dam break (h = 10 m | 1 m, flat frictionless bed, closed walls,
alpha 0.45) run to its 30 s horizon on the device clock: every row is the 1-D Stoker
problem, so each row must sit on the analytical wet-bed solution (the reference's
gate, validation/test_dam_break.py:94: nRMSE < 0.03, front error < 0.05), all rows
must be identical (the problem is uniform in y), the walls have not been reached,
and the volume is unchanged to float64 round-off of the float32 field. These are
size-independent properties; bitwise parity with the CPU oracle at this size is in
test_gpu_parity.py (12 steps).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_headline_dam_break_matches_stoker_at_full_size():
    import rbsim
    from analytical import star_depth, stoker, stoker_front
    from rbsim.device_clock import DeviceClock
    from rbsim.schemes import hllc

    n, dx, h_l, h_r, t_end = 2048, 1.0, 10.0, 1.0, 30.0
    depth = np.full((n, n), h_r, np.float32)
    depth[:, : n // 2] = h_l
    st = rbsim.State.from_bed(np.zeros((n, n), np.float32), dx, depth=depth, manning=0.0)
    hllc.arm_hllc(st)
    v0 = st.volume_sum()
    clk = DeviceClock(st, "hllc_fv", alpha=0.45, dt_max=30.0, sync_times=[t_end], graph_steps=64)
    steps = clk.run_until(t_end)
    assert abs(clk.t - t_end) < 1e-6 and steps > 500
    h = st.h.cpu().numpy().astype(np.float64)
    assert np.isfinite(h).all()
    # uniform in y: every row the same profile (closed north/south walls reflect nothing)
    assert np.abs(h - h[n // 2]).max() < 1e-4
    x = (np.arange(n) + 0.5 - n / 2.0) * dx
    row = h[n // 2]
    ref = stoker(x, t_end, h_l, h_r)
    inner = np.abs(x) < 0.9 * n / 2.0 * dx
    nrmse = math.sqrt(np.mean((row[inner] - ref[inner]) ** 2)) / (h_l - h_r)
    level = 0.5 * (h_r + star_depth(h_l, h_r))
    front = x[row > level].max()
    front_err = abs(front - stoker_front(t_end, h_l, h_r)) / abs(stoker_front(t_end, h_l, h_r))
    assert nrmse < 0.03, nrmse
    assert front_err < 0.05, front_err
    # the waves are still inside: undisturbed depth at both walls
    assert abs(row[0] - h_l) < 1e-5 and abs(row[-1] - h_r) < 1e-5
    assert abs(st.volume_sum() - v0) / v0 < 1e-6
    clk.close()
