"""The reference's morphology gates (tests/morph_gates.py) on the CUDA path, through rbsim.

The gates run through the scheme API, ``InflowInjector`` and ``MorphologyProcess``
in the exact arithmetic. Then the full bed-wave run is compared with the same run on
the oracle, bit for bit. That run is about 13 000 local-inertial steps with the
bedload integral and 103 Exner activations.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from backends import GpuBackend, OracleBackend  # noqa: E402
from morph_gates import MORPH_GATES, Reach, run_reach  # noqa: E402


@pytest.fixture(scope="module")
def be():
    return GpuBackend()


@pytest.mark.parametrize("name", sorted(MORPH_GATES))
def test_morph_gate(name, be):
    MORPH_GATES[name](be)


def test_bed_wave_run_matches_the_oracle_bit_for_bit(be):
    import oracle

    fx = Reach()
    got = run_reach(be, fx)
    try:
        want = run_reach(OracleBackend(), fx)
    finally:
        oracle.set_pow_mode(0)
    assert (got.steps, got.activations) == (want.steps, want.activations)
    assert got.t == want.t
    for key in ("bed", "depth", "face_q", "dz_cum"):
        np.testing.assert_array_equal(getattr(got, key), getattr(want, key), err_msg=key)
    assert got.mass_rel_error < 1e-6
