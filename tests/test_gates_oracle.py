"""The reference's physics gates (tests/gates.py) on the CPU oracle.

The oracle is the checker of the CUDA path; these show it also clears every gate
the reference's own suite holds its solver to (dam breaks against Stoker / Ritter,
lake-at-rest, shorelines, Kahan ratio gates, mass closure, open edges, inflow).
"""

from __future__ import annotations

import pytest

from backends import OracleBackend
from gates import GATES


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


@pytest.mark.parametrize("name", sorted(GATES))
def test_gate(name, be):
    GATES[name](be)
