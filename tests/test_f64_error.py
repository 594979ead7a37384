"""The float32 path's error against the float64 build of the same kernels, on every
golden case: the depth stays within 1e-4 m of float64 (the bound the solver path is
specified against) and the relative depth and discharge errors stay at float32
round-off carried through the dynamics. The CUDA path equals the float32 oracle bit
for bit (test_gpu_parity.py), so these figures are the CUDA path's too;
test_gpu_f64_error.py measures them on the device directly. CPU only."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from cases import CASES, run_case
from f64_error import check, error_vs_f64
from test_oracle_golden import OracleAPI


@pytest.fixture(autouse=True)
def _pow_mode():
    oracle.set_pow_mode(1)
    yield
    oracle.set_pow_mode(0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_float32_oracle_error_against_float64(name):
    case = CASES[name]()
    got = run_case(case, OracleAPI(np.float32))
    err = error_vs_f64(CASES[name](), got)
    # float32 round-off carried through 8-30 steps: ~1e-7 relative on most cases; the
    # thin sheet on a steep slope (li_steep_sheet, 6 cm deep) reaches 1.1e-5 of its depth
    # at its worst cell and 1.6e-5 in the L2 norm
    check(err, rel=2e-5)
    assert err["max_rel_depth"] <= 2e-5, err
    assert err["max_rel_discharge"] <= 1e-5, err
