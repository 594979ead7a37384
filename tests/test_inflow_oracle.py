"""Point inflows: the reference's compensation gates on the oracle, and the host API.

The gates (solver/processes/test_inflow.py:129-220) run on the oracle's point-source
add. The CUDA injection (``rb_inject_points``) equals it bit for bit on the golden
inflow cases. The host part of ``rbsim.processes.inflow`` needs no device: the
hydrograph sampling, and the refusals raised before anything is allocated
(solver/processes/test_inflow.py:50, :57).
"""

from __future__ import annotations

import numpy as np
import pytest

from backends import OracleBackend
from rbsim.grid import Grid
from rbsim.processes.inflow import Inflow, InflowInjector


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


def _accumulate(be, compensated, hydrograph, nsteps, dt, depth=1.0):
    """Inject into the centre of a 3 x 3 grid of 100 m cells with nothing else touching h.

    Returns (|volume the field gained - volume the injector reported|, reported
    volume, the compensation terms).
    """
    st = be.make(np.zeros((3, 3), np.float32), 100.0, depth=depth)
    inj = be.injector([((1, 1), hydrograph)], st, compensated=compensated)
    requested = sum(inj.apply(st, k * dt, dt) for k in range(nsteps))
    got = (float(be.h(st)[1, 1]) - depth) * 100.0 * 100.0
    return abs(got - requested), requested, inj.comp


def test_point_source_add_is_compensated(be):
    """test_inflow.py:129: 0.027 m onto 1 m for 1500 steps; compensated is 100 times closer."""
    flat = [(0.0, 90.0), (1e9, 90.0)]
    uncomp, total, _ = _accumulate(be, False, flat, 1500, 3.0)
    comp, _, _ = _accumulate(be, True, flat, 1500, 3.0)
    assert total == pytest.approx(405_000.0, rel=1e-6)
    assert uncomp / comp > 100.0, (uncomp, comp)


def test_sub_ulp_point_source_lands_nothing_uncompensated(be):
    """test_inflow.py:143: 4e-8 m onto 1 m is under half an ulp: plain adds land nothing."""
    q = 4.0e-8 * 100.0 * 100.0 / 10.0
    flat = [(0.0, q), (1e9, q)]
    uncomp, total, _ = _accumulate(be, False, flat, 2000, 10.0)
    comp, _, _ = _accumulate(be, True, flat, 2000, 10.0)
    assert uncomp == pytest.approx(total, rel=1e-9)
    assert uncomp / comp > 100.0


def test_compensation_term_is_nonzero_fast_math_canary(be):
    """test_inflow.py:161: the compensation is not folded away."""
    _, _, comp = _accumulate(be, True, [(0.0, 90.0), (1e9, 90.0)], 1, 3.0)
    assert comp is not None and np.any(comp != 0.0)


def test_uncompensated_arm_reproduces_the_plain_add(be):
    """test_inflow.py:176: compensated=False is the plain float32 running sum, bit for bit."""
    st = be.make(np.zeros((3, 3), np.float32), 100.0, depth=1.0)
    inj = be.injector([((1, 1), [(0.0, 90.0), (1e9, 90.0)])], st, compensated=False)
    assert inj.comp is None
    expect = np.float32(1.0)
    for k in range(200):
        vol = inj.apply(st, k * 3.0, 3.0)
        expect = np.float32(expect + np.float32(vol / 1.0e4))
    assert np.float32(be.h(st)[1, 1]) == expect


def test_receded_hydrograph_keeps_carrying_its_debt(be):
    """test_inflow.py:196: after the hydrograph falls to zero the debt is still repaid, and stays small."""
    hydro = [(0.0, 0.0), (300.0, 90.0), (900.0, 90.0), (1200.0, 0.0), (6000.0, 0.0)]
    uncomp, _, _ = _accumulate(be, False, hydro, 2000, 3.0)
    comp, _, debt = _accumulate(be, True, hydro, 2000, 3.0)
    assert uncomp / comp > 20.0, (uncomp, comp)
    assert debt is not None and np.all(np.abs(debt) < 1.0e-5)


def test_discharge_is_linear_between_knots_and_zero_outside():
    """config.py:111-121: the hydrograph the injector samples at each step's midpoint."""
    inf = Inflow((0, 0), [(0.0, 0.0), (100.0, 10.0), (100.0, 4.0), (300.0, 0.0)])
    assert inf.discharge_at(-1.0) == 0.0 and inf.discharge_at(300.5) == 0.0
    assert inf.discharge_at(50.0) == 5.0
    assert inf.discharge_at(100.0) == 10.0  # the first segment that holds t wins
    assert inf.discharge_at(200.0) == 2.0
    assert inf.breakpoints == [0.0, 100.0, 100.0, 300.0]
    assert Inflow((0, 0), []).discharge_at(0.0) == 0.0


def test_out_of_bounds_cell_rejected():
    """test_inflow.py:50."""
    with pytest.raises(ValueError, match="outside"):
        InflowInjector([Inflow((9, 0), [(0.0, 1.0)])], Grid(ny=4, nx=4, dx=10.0), "cpu")


def test_duplicate_cell_rejected():
    """test_inflow.py:57: two sources on one cell would race."""
    with pytest.raises(ValueError, match="duplicate"):
        InflowInjector([Inflow((2, 2), [(0.0, 1.0), (100.0, 1.0)]), Inflow((2, 2), [(0.0, 2.0), (100.0, 2.0)])],
                       Grid(ny=4, nx=4, dx=10.0), "cpu")  # fmt: skip


def test_an_injector_without_sources_adds_nothing():
    inj = InflowInjector([], Grid(ny=4, nx=4, dx=10.0), "cpu")
    assert inj.breakpoints() == [] and inj.apply(None, 0.0, 1.0) == 0.0
