"""The reference's physics gates (tests/gates.py) on the CUDA path, through rbsim."""

from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from backends import GpuBackend  # noqa: E402
from gates import GATES  # noqa: E402


@pytest.fixture(scope="module")
def be():
    return GpuBackend()


@pytest.mark.parametrize("name", sorted(GATES))
def test_gate(name, be):
    GATES[name](be)
