"""The reference's morphology gates (tests/morph_gates.py) on the CPU oracle.

The bed-wave celerity, the Shields-threshold pair, interval independence and the
flat reach, run through the oracle's local-inertial step with its fused bedload
integral, its Exner update, the point inflow and the open east edge.
"""

from __future__ import annotations

import pytest

from backends import OracleBackend
from morph_gates import MORPH_GATES, Reach, reach_sizing_problems
from rbsim.sediment import SHIELDS_CRITICAL, shields_from_flow


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


def test_reach_is_sized_for_the_transport_law():
    """validation/test_bed_wave.py:63: the design point meets every constraint it was derived under."""
    fx = Reach()
    assert reach_sizing_problems(fx) == []
    assert fx.activations * fx.interval_s == pytest.approx(fx.morph_s)
    # at the 900 s cadence of the slow clock the bed wave would cross more than a cell per activation
    assert fx.celerity * 900.0 / fx.dx > 1.0


def test_every_arm_transports_inside_the_laws_range():
    """validation/test_morphology_gates.py:170: each arm's flow is more than 20 grains deep,
    unlike a 1 mm overland sheet on 2 mm grains, which reads over ten times theta_c."""
    base = Reach()
    for fx in (base, base.regrained(0.90), base.regrained(1.20)):
        assert fx.normal_depth / fx.d50 > 20.0
    assert float(shields_from_flow(0.5e-3, 1e-3, 0.03, 0.002)) > 10.0 * SHIELDS_CRITICAL
    assert base.regrained(0.90).shields == pytest.approx(0.90 * SHIELDS_CRITICAL, rel=1e-12)


@pytest.mark.parametrize("name", sorted(MORPH_GATES))
def test_morph_gate(name, be):
    MORPH_GATES[name](be)
