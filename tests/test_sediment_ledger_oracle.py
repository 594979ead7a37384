"""The sediment ledger's gates (solver/core/test_massbalance.py:248-387) on oracle-driven beds.

``rbsim.massbalance.SedimentLedger`` is the product gauge. Here it reads the
float64 bed-change fields of an oracle state through torch views that share their
memory. The oracle's local-inertial step fills the bedload integral and its Exner
update moves the bed. So the gauge's arithmetic and the reference's balance
(``residual = -(net bed change + banked)`` against the gross volume moved, gate
1e-11) are checked together on the CPU. The bounds come from this package's
``bed_change_bounds``.
"""

from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from backends import OracleBackend
from rbsim.massbalance import SEDIMENT_GATE, SedimentLedger
from rbsim.processes.morphology import bed_change_bounds

LI = "local_inertial"


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


class _View:
    """What SedimentLedger reads from a state, over an oracle state's own arrays."""

    def __init__(self, st):
        self.grid = SimpleNamespace(cell_area=st.dx * st.dx)
        sed = st.sediment
        self.sediment = None if sed is None else SimpleNamespace(
            dz_cum=torch.from_numpy(sed.dz_cum), dz_unapplied=torch.from_numpy(sed.dz_unapplied),
            porosity=sed.porosity,
        )  # fmt: skip


def _sloping_reach(be, nx=30, dx=2.0, slope=0.01, thickness=None):
    """A wet one-row reach closed at both ends, steep enough to move 2 mm grains."""
    j = np.arange(nx, dtype=np.float64)
    bed = (2.0 + (nx - 1 - j) * dx * slope).reshape(1, nx).astype(np.float32)
    st = be.make(bed, dx, depth=0.5, manning=0.03)
    be.arm_sediment(st, 0.002, 0.4)
    lo, hi = bed_change_bounds((1, nx), alluvium_thickness=thickness)
    return st, be.morphology(st, 5.0, lo, hi)


def _drive(be, st, morph, *, end=60.0, interval=5.0):
    """Steps landing exactly on every 5 s activation; the ledger recorded after each one."""
    led = SedimentLedger.from_state(_View(st))
    t, acts = 0.0, 0
    while t < end - 1e-9:
        edge = min((acts + 1) * interval, end)
        dt = min(be.compute_dt(st, LI, 0.7, 1.0), edge - t)
        be.step(st, LI, dt)
        t += dt
        if t >= (acts + 1) * interval - 1e-9:
            morph.advance(t, interval)
            acts += 1
            led.record(_View(st), t)
    assert acts == int(round(end / interval))
    return led


def test_a_closed_bedload_domain_nets_to_zero_far_inside_the_gate(be):
    """test_massbalance.py:248: no bound fires, nothing is banked, the net is float64 round-off."""
    st, morph = _sloping_reach(be)
    led = _drive(be, st, morph)
    last = led.series[-1]
    assert (st.sediment.dz_unapplied == 0.0).all() and last.banked_volume == 0.0
    assert last.gross_volume > 1e-3
    assert led.max_rel_error < 1e-13


def test_the_boundary_faces_carry_no_bedload(be):
    """test_massbalance.py:269: the edge face rows of the transport integral stay exactly zero.

    Read between activations, while the interior faces carry a non-zero integral, so
    the check is not vacuous.
    """
    st, _ = _sloping_reach(be)
    for _ in range(20):
        be.step(st, LI, be.compute_dt(st, LI, 0.7, 1.0))
    qx, qy = st.sediment.qs_int_x, st.sediment.qs_int_y
    assert (qx[:, 0] == 0.0).all() and (qx[:, -1] == 0.0).all()
    assert (qy[0, :] == 0.0).all() and (qy[-1, :] == 0.0).all()
    assert np.abs(qx[:, 1:-1]).max() > 0.0


def test_a_bound_supplies_the_domain_and_the_ledger_says_how_much(be):
    """test_massbalance.py:291: an alluvium floor is a source, and banked is exactly its size."""
    st, morph = _sloping_reach(be, thickness=1.0e-5)
    led = _drive(be, st, morph)
    last = led.series[-1]
    assert (st.sediment.dz_unapplied != 0.0).any()
    assert last.banked_volume < 0.0 and last.bed_volume > 0.0
    assert led.max_rel_error < SEDIMENT_GATE
    assert last.bed_volume == pytest.approx(-last.banked_volume, rel=1e-12)


def test_the_gross_volume_tells_a_balanced_bed_from_a_still_one(be):
    """test_massbalance.py:315: still water moves nothing; only gross tells it from a balanced bed."""
    st = be.make(np.full((1, 12), 5.0, np.float32), 2.0, depth=0.5, manning=0.03)
    be.arm_sediment(st, 0.002, 0.4)
    lo, hi = bed_change_bounds((1, 12))
    still = _drive(be, st, be.morphology(st, 5.0, lo, hi), end=20.0)
    assert still.series[-1].gross_volume == 0.0 and still.series[-1].residual == 0.0
    assert still.max_rel_error == 0.0
    moving, morph = _sloping_reach(be)
    assert _drive(be, moving, morph).series[-1].gross_volume > 0.0


def test_a_cell_that_lifts_off_its_floor_keeps_the_balance(be):
    """test_massbalance.py:345: erode onto the floor and bank the refusal, then deposit back.

    The second activation stays inside the bounds, so it banks nothing and must
    leave the cumulative bank as it was.
    """
    nx, dx, floor, p = 3, 2.0, 1.0e-4, 0.4
    st = be.make(np.full((1, nx), 5.0, np.float32), dx, depth=0.5)
    be.arm_sediment(st, 0.002, p)
    lo, hi = bed_change_bounds((1, nx), alluvium_thickness=floor)
    morph = be.morphology(st, 5.0, lo, hi)
    led = SedimentLedger.from_state(_View(st))
    a = 5.0 * floor * (1.0 - p) * dx  # cell 0 wants to erode five times its alluvium

    def activate(face_load, t):
        st.sediment.qs_int_x[...] = 0.0
        st.sediment.qs_int_x[0, 1:-1] = face_load
        morph.advance(t, 5.0)
        return led.record(_View(st), t)

    first = activate([a, 0.0], 5.0)
    banked = st.sediment.dz_unapplied.copy()
    assert st.sediment.dz_cum[0, 0] == pytest.approx(-floor, rel=1e-6)
    assert banked[0, 0] < 0.0 and first.banked_volume < 0.0 and first.rel_error < SEDIMENT_GATE
    second = activate([-a, 0.0], 10.0)
    assert st.sediment.dz_cum[0, 0] > -floor
    assert (st.sediment.dz_unapplied == banked).all()
    assert second.banked_volume == pytest.approx(first.banked_volume, rel=1e-12)
    assert led.max_rel_error < SEDIMENT_GATE


def test_an_unarmed_state_has_nothing_to_balance(be):
    """test_massbalance.py:380."""
    st = be.make(np.zeros((3, 4), np.float32), 5.0)
    with pytest.raises(ValueError, match="arm_sediment"):
        SedimentLedger.from_state(_View(st))


def test_the_sediment_series_is_serializable_for_the_store(be):
    """test_massbalance.py:387: the .zattrs keys, one record per activation plus t = 0, JSON-clean."""
    st, morph = _sloping_reach(be)
    attrs = _drive(be, st, morph).as_attrs()
    assert attrs["sediment_gate"] == SEDIMENT_GATE
    assert attrs["sediment_max_rel_error"] < SEDIMENT_GATE
    series = attrs["sediment_balance_series"]
    assert len(series) == 13 and series[0]["gross_volume"] == 0.0
    assert set(series[0]) == {"time", "bed_volume", "banked_volume", "gross_volume", "residual", "rel_error"}
    json.dumps(attrs)
