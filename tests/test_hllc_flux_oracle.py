"""Riemann-solver properties of the HLLC step, on the oracle.

These restate validation/test_hllc1d.py:86, :92 and :101. The reference states them
for its 1-D flux function. Here they are checked through the 2-D step, on a strip
with open edges that is uniform across, so the transverse fluxes cancel:
* two dry states exchange nothing, and an all-dry domain stays dry without NaNs;
* consistency: a uniform state, which the solver sees as F(U, U) on every face, does
  not change at all;
* the transverse momentum hv is carried from the upwind side of the contact.
"""

from __future__ import annotations

import numpy as np
import pytest

from backends import OracleBackend

HLLC = "hllc_fv"
OPEN = {e: "open" for e in ("north", "south", "east", "west")}


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


def _strip(be, h, u, v, ny=3, nx=40):
    st = be.make(np.zeros((ny, nx), np.float32), 1.0, depth=np.asarray(h, np.float32) * np.ones((ny, nx), np.float32),
                 manning=0.0)  # fmt: skip
    be.set_bc(st, OPEN)
    hh = be.h(st)
    be.set_hu(st, (hh * u).astype(np.float32), (hh * v).astype(np.float32))
    return st


def test_dry_over_dry_exchanges_nothing(be):
    st = _strip(be, 0.0, 0.0, 0.0)
    for _ in range(5):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 2.0))
    assert (be.h(st) == 0.0).all() and (be.hu(st) == 0.0).all() and (be.hv(st) == 0.0).all()


def test_a_uniform_state_does_not_change(be):
    """F(U, U) is the physical flux on every face, so every divergence is exactly zero."""
    st = _strip(be, 2.0, 1.5, -0.7)
    h0, hu0, hv0 = be.h(st).copy(), be.hu(st).copy(), be.hv(st).copy()
    for _ in range(20):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
    assert (be.h(st) == h0).all() and (be.hu(st) == hu0).all() and (be.hv(st) == hv0).all()


@pytest.mark.parametrize("u", [0.5, -0.5])
def test_transverse_momentum_is_carried_from_the_upwind_side(be, u):
    """hv = 0.2 west of the middle, 0 east of it, in a uniform flow: it moves with the flow,
    and the upwind side keeps its value exactly; the depth does not change."""
    nx = 40
    v = np.where(np.arange(nx) < nx // 2, 0.2, 0.0)
    st = _strip(be, 1.0, u, v)
    for _ in range(10):
        be.step(st, HLLC, be.compute_dt(st, HLLC, 0.45, 5.0))
    row = be.hv(st)[1]
    assert (be.h(st) == 1.0).all()
    if u > 0:
        assert (row[: nx // 2] == np.float32(0.2)).all() and row[nx // 2] > 0.05
    else:
        assert (row[nx // 2 :] == 0.0).all() and row[nx // 2 - 1] < 0.15
