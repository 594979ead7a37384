"""Shared pytest setup: the ``gpu`` marker, import paths, and the oracle build."""

from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "river-basin-sim_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests", "golden")):  # fmt: skip
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built librbsim.so")
    config.addinivalue_line("markers", "slow: long CPU-only test")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    import oracle

    oracle.build()
    yield
