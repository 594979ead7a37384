"""The CUDA path's error against the float64 build of the same kernels.

Each case runs on the device through the public scheme API; the float64 oracle
(``librbo_f64.so``) then runs the same inputs with the device's own timestep
sequence, and the difference of the final states is the error of the float32
result (tests/f64_error.py). Cases: every golden case, the 512 x 512 rain-on-grid
configuration shape (60 steps), the 2048 x 2048 dam break (12 steps) and a
1024 x 8192 band of the 8192 x 8192 valley reach (8 steps, infiltration, inflows,
bedload). Bound: depth within 1e-4 m of float64 (the solver path's specified
bound); relative depth, discharge and volume differences at float32 round-off.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

import oracle  # noqa: E402
from cases import CASES, run_case  # noqa: E402
from f64_error import error_vs_f64  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    oracle.set_pow_mode(1)
    yield
    oracle.set_pow_mode(0)


def _check(case, rel_depth=2e-5):
    from gpu_api import GpuAPI

    got = run_case(dict(case), GpuAPI())
    err = error_vs_f64(case, got)
    assert err["max_abs_depth_m"] <= 1e-4, err
    assert err["max_rel_depth"] <= rel_depth, err
    assert err["max_rel_discharge"] <= 1e-5, err
    assert err["rel_volume"] <= 1e-6, err
    return err


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_against_float64(name):
    _check(CASES[name]())


def test_li_512_rain_on_grid_against_float64():
    from test_gpu_parity import _synthetic_li

    case = _synthetic_li(512, 512, seed=1)
    case["steps"] = 60
    _check(case)


def test_hllc_dambreak_2048_against_float64():
    n = 2048
    depth = np.ones((n, n), np.float32)
    depth[:, : n // 2] = 10.0
    _check(dict(scheme="hllc_fv", bed=np.zeros((n, n), np.float32), dx=1.0, depth=depth, manning=0.0, steps=12,
                alpha=0.45, dt_max=30.0))  # fmt: skip


def test_valley_reach_band_against_float64():
    """Rows n/2 - 512 .. n/2 + 511 of the reach (the meandering channel and all eight
    inflow cells lie inside), with an Exner activation every 4 steps."""
    from bench_workloads import reach_inputs

    n, rows = 8192, 1024
    z, manning, infil, inflows, depth = reach_inputs(n, 5.0)
    r0 = n // 2 - rows // 2
    band = slice(r0, r0 + rows)
    srcs = [((inf.cell[0] - r0, inf.cell[1]), inf.hydrograph) for inf in inflows]
    assert all(0 <= c[0] < rows for c, _ in srcs)
    case = dict(scheme="local_inertial", bed=z[band].copy(), dx=5.0, depth=depth[band].copy(),
                manning=manning[band].copy(), infil=infil[band].copy(), inflows=srcs, boundaries={"east": "open"},
                sediment=dict(d50=np.full((rows, n), 0.002, np.float32), porosity=0.4, every=4,
                              dz_lo=np.full((rows, n), -np.inf, np.float32),
                              dz_hi=np.full((rows, n), np.inf, np.float32)),
                steps=8, alpha=0.7, dt_max=30.0)  # fmt: skip
    _check(case)
