"""Areal rain sources and the sinks beside them: the reference's remaining tests on the oracle.

These restate solver/core/test_sources.py:109, :180, :202 and :225, and
solver/core/test_massbalance.py:41 and :81 (uniform rain balancing to the gate, the
uncapped infiltration rate). The rest of
that file is in tests/gates.py (sub-ulp rain, the compensation canary, storm drift,
the field on both schemes). Those gates run on the CUDA path too, and the CUDA rain
paths equal the oracle bit for bit on the golden rain cases.
"""

from __future__ import annotations

import numpy as np
import pytest

from backends import OracleBackend

LI, HLLC = "local_inertial", "hllc_fv"


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


def _flat(be, depth):
    return be.make(np.zeros((8, 8), np.float32), 100.0, depth=depth, manning=0.03)


def test_mass_ledger_residual_improves_under_compensation(be):
    """test_sources.py:109: the ledger's residual is the accumulation error compensation removes."""
    rain, dt, steps = 15.0 / 1000.0 / 3600.0, 20.0, 1500

    def run(compensate):
        st = _flat(be, 0.3)
        if compensate:
            be.arm_comp(st)
        led = be.ledger(st)
        for k in range(steps):
            be.step(st, LI, dt, rain=rain, limit=False)
            led.add_rain_step(rain, dt, be.n_cells(st))
            if (k + 1) % 300 == 0:
                led.record(st, (k + 1) * dt)
        return led.max_rel_error

    assert run(False) / max(run(True), 1e-30) > 20.0


@pytest.mark.parametrize("scheme", [LI, HLLC])
def test_rain_field_is_read_per_cell(be, scheme):
    """test_sources.py:180: sub-ulp rain on the west half banks compensation there and nowhere else."""
    st = _flat(be, 1.0)
    field = np.zeros((8, 8), np.float32)
    field[:, :4] = 4.0e-8
    be.set_rain(st, field)
    be.arm_comp(st)
    be.step(st, scheme, 1.0, rain_scale=1.0)
    comp = be.hcomp(st)
    assert np.all(comp[:, :4] != 0.0) and np.all(comp[:, 4:] == 0.0)


def test_unarmed_state_keeps_the_original_kernels(be):
    """test_sources.py:202: no compensation array unless something arms it; the plain add loses sub-ulp rain."""
    st = _flat(be, 1.0)
    assert st.h_comp is None
    be.step(st, LI, 1.0, rain=4.0e-8, limit=False)
    assert st.h_comp is None and (be.h(st) == np.float32(1.0)).all()


def test_arming_is_idempotent_and_preserves_the_running_debt(be):
    """test_sources.py:225."""
    st = _flat(be, 1.0)
    be.arm_comp(st)
    be.step(st, LI, 1.0, rain=4.0e-8, limit=False)
    before = be.hcomp(st)
    assert np.any(before != 0.0)
    be.arm_comp(st)
    assert np.array_equal(be.hcomp(st), before)


def test_uniform_rain_balances_to_gate(be):
    """solver/core/test_massbalance.py:41: 40 steps of 50 mm/h on a closed basin close the ledger."""
    st = be.make(np.zeros((16, 16), np.float32), 10.0, depth=0.2, manning=0.03)
    led = be.ledger(st)
    rain, t = 50.0 / 1000.0 / 3600.0, 0.0
    for _ in range(40):
        dt = be.compute_dt(st, LI, 0.5, 5.0)
        be.step(st, LI, dt, rain=rain)
        led.add_rain_step(rain, dt, be.n_cells(st))
        t += dt
    rec = led.record(st, t)
    assert led.max_rel_error < 1e-6 and rec.volume > led.v0


def test_uncapped_infiltration_removes_exactly_its_rate(be):
    """solver/core/test_massbalance.py:81: 20 steps of 2 s at 5e-5 m/s on 0.3 m of water
    bank rate x time x area, to 1e-3 (the mass gate cannot see a mis-scaled rate)."""
    rate = 5.0e-5
    st = be.make(np.zeros((5, 5), np.float32), 10.0, depth=0.3)
    be.set_infil(st, np.full((5, 5), rate, np.float32))
    for _ in range(20):
        be.step(st, LI, 2.0)
    want = rate * 2.0 * 20 * be.cell_area(st) * be.n_cells(st)
    assert abs(be.loss_volume(st) - want) < 1e-3 * want
