"""The reference's HLLC edge gates (tests/edge_gates.py) on the CPU oracle.

The prescribed-stage ghost, open edges, walls and a steady channel, run through the
oracle's HLLC step with its fixed-stage and open-edge banking. The stage curve is
also checked in both of its implementations: the oracle's and the one that
``rbsim.schemes.hllc`` samples on the host for each CUDA step.
"""

from __future__ import annotations

import pytest

from backends import OracleBackend
from edge_gates import EDGE_GATES


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


@pytest.mark.parametrize("name", sorted(EDGE_GATES))
def test_edge_gate(name, be):
    EDGE_GATES[name](be)


@pytest.mark.parametrize("which", ["oracle", "rbsim"])
def test_stage_curve_is_piecewise_linear_and_held_outside(which):
    """validation/test_fixed_stage.py:217: linear between knots, held (not zeroed) outside."""
    if which == "oracle":
        from oracle import stage_at
    else:
        from rbsim.schemes.hllc import stage_at
    curve = [(0.0, 9.7), (3600.0, 10.35), (7200.0, 9.7)]
    assert stage_at(curve, -100.0) == 9.7
    assert stage_at(curve, 1800.0) == pytest.approx(10.025)
    assert stage_at(curve, 3600.0) == pytest.approx(10.35)
    assert stage_at(curve, 1e9) == 9.7
    assert stage_at([(0.0, 4.2)], 555.0) == 4.2
    with pytest.raises(ValueError):
        stage_at([], 0.0)
