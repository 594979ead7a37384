"""Ensembles: every member of a batch equals the same domain run alone, bit for bit.

Members mix schemes and sizes (ragged, one-row, tile-multiple), carry their own
rain and horizons, and are stepped by the persistent (domain, tile) kernels for
every tile variant; each member's final fields must match a DeviceClock run of
that member alone.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SPECS = [  # (scheme, ny, nx, dx, horizon, rain m/s)
    ("local_inertial", 96, 130, 10.0, 400.0, 2e-5),
    ("hllc_fv", 64, 64, 1.0, 3.0, 0.0),
    ("local_inertial", 1, 300, 5.0, 200.0, 0.0),
    ("hllc_fv", 45, 77, 2.0, 5.0, 1e-4),
    ("local_inertial", 256, 256, 20.0, 900.0, 1e-5),
]


def _member(scheme, ny, nx, dx, seed):
    import rbsim
    from rbsim.schemes import hllc

    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    z = (1e-3 * xx * dx + 0.2 * np.sin(yy * 0.3) * np.cos(xx * 0.2)).astype(np.float32)
    depth = rng.uniform(0.05, 0.6, (ny, nx)).astype(np.float32)
    if scheme == "hllc_fv":
        depth[:, : nx // 2] += 1.0
    st = rbsim.State.from_bed(z, dx, depth=depth, manning=0.03)
    if scheme == "hllc_fv":
        hllc.arm_hllc(st)
    else:
        st.arm_source_compensation()
        st.set_open_boundaries({"east": "open"})
    return st


@pytest.mark.parametrize("variants", [(0, 0), (1, 1), (2, 0), (3, 1), (3, 2)])
def test_members_equal_solo_runs(variants):
    from rbsim.device_clock import DeviceClock
    from rbsim.ensemble import Ensemble

    alpha = {"local_inertial": 0.7, "hllc_fv": 0.45}
    solo = []
    for k, (sch, ny, nx, dx, hz, rain) in enumerate(SPECS):
        st = _member(sch, ny, nx, dx, seed=k)
        clk = DeviceClock(st, sch, alpha=alpha[sch], dt_max=30.0, sync_times=[hz], rain_rate=rain,
                          rain_until=hz, graph_steps=16)  # fmt: skip
        clk.run_until(hz)
        solo.append((st.h.cpu().numpy(), clk.steps, st.loss_cum.total() if st.loss_cum is not None else 0.0))
        clk.close()

    members = [_member(sch, ny, nx, dx, seed=k) for k, (sch, ny, nx, dx, _, _) in enumerate(SPECS)]
    ens = Ensemble(members, [s[0] for s in SPECS], alpha=[alpha[s[0]] for s in SPECS], dt_max=30.0,
                   sync_times=[[s[4]] for s in SPECS], rain_rate=[s[5] for s in SPECS],
                   rain_until=[s[4] for s in SPECS], li_variant=variants[0], hllc_variant=variants[1],
                   graph_steps=8)  # fmt: skip
    ens.run_until([s[4] for s in SPECS])
    for k, (st, (h, steps, loss)) in enumerate(zip(members, solo, strict=True)):
        assert ens.clock[k].steps == steps, k
        np.testing.assert_array_equal(st.h.cpu().numpy(), h, err_msg=f"member {k}")
        if loss:
            assert st.loss_cum.total() == pytest.approx(loss, rel=1e-12)


LARGE_SPECS = [  # at least 1024 tiles of 32 x 32: stepped by the single-domain kernels
    ("local_inertial", 1024, 1100, 10.0, 300.0, 2e-5),
    ("hllc_fv", 1024, 1056, 1.0, 1.0, 0.0),
    ("local_inertial", 96, 130, 10.0, 400.0, 2e-5),
    ("hllc_fv", 45, 77, 2.0, 5.0, 1e-4),
]


def test_large_members_on_the_single_domain_kernels_equal_solo_runs():
    """Members of 1024 tiles or more run the single-domain kernels inside the ensemble's
    step (launched per member), the others the persistent kernels; every member still
    equals its run alone, bit for bit."""
    from rbsim.device_clock import DeviceClock
    from rbsim.ensemble import Ensemble

    alpha = {"local_inertial": 0.7, "hllc_fv": 0.45}
    solo = []
    for k, (sch, ny, nx, dx, hz, rain) in enumerate(LARGE_SPECS):
        st = _member(sch, ny, nx, dx, seed=60 + k)
        clk = DeviceClock(st, sch, alpha=alpha[sch], dt_max=30.0, sync_times=[hz], rain_rate=rain,
                          rain_until=hz, graph_steps=16)  # fmt: skip
        clk.run_until(hz)
        solo.append((st.h.cpu().numpy(), clk.steps, st.loss_cum.total() if st.loss_cum is not None else 0.0))
        clk.close()
        del st
    members = [_member(sch, ny, nx, dx, seed=60 + k) for k, (sch, ny, nx, dx, _, _) in enumerate(LARGE_SPECS)]
    ens = Ensemble(members, [s[0] for s in LARGE_SPECS], alpha=[alpha[s[0]] for s in LARGE_SPECS], dt_max=30.0,
                   sync_times=[[s[4]] for s in LARGE_SPECS], rain_rate=[s[5] for s in LARGE_SPECS],
                   rain_until=[s[4] for s in LARGE_SPECS], li_variant=3, hllc_variant=2,
                   graph_steps=8)  # fmt: skip
    ens.run_until([s[4] for s in LARGE_SPECS])
    for k, (st, (h, steps, loss)) in enumerate(zip(members, solo, strict=True)):
        assert ens.clock[k].steps == steps, k
        np.testing.assert_array_equal(st.h.cpu().numpy(), h, err_msg=f"member {k}")
        if loss:
            assert st.loss_cum.total() == pytest.approx(loss, rel=1e-12)


def test_autotune_picks_a_candidate_and_keeps_results_exact():
    from rbsim.device_clock import DeviceClock
    from rbsim.ensemble import Ensemble, autotune

    specs = [("local_inertial", 200, 333, 10.0), ("local_inertial", 128, 128, 10.0)]
    members = [_member(s, ny, nx, dx, seed=40 + k) for k, (s, ny, nx, dx) in enumerate(specs)]

    def make(li_v, hl_v, t0):
        e = Ensemble(members, [s[0] for s in specs], alpha=0.7, dt_max=30.0, sync_times=[[1e6]] * 2,
                     li_variant=li_v, hllc_variant=hl_v, graph_steps=4, t0=0.0 if t0 is None else t0)  # fmt: skip
        e.set_targets(1e6)
        return e

    best, timings, t_reached = autotune(make, probe_replays=1, candidates=[(0, 0), (1, 0), (2, 0)])
    assert best in timings and len(timings) == 3 and t_reached[0] > 0.0
    steps = [members[0].cur]  # 3 candidates x (1 + 1) replays x 4 steps = 24 steps each
    solo = _member("local_inertial", 200, 333, 10.0, seed=40)
    clk = DeviceClock(solo, "local_inertial", alpha=0.7, dt_max=30.0, sync_times=[1e6], graph_steps=24)
    clk.run_until(1e6, max_steps=24)
    np.testing.assert_array_equal(members[0].h.cpu().numpy(), solo.h.cpu().numpy())
    assert steps is not None
