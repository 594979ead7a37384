"""The CUDA path's error against the float64 build of the same kernels.

Each case runs on the device through the public scheme API; the float64 oracle
(``librbo_f64.so``) then runs the same inputs with the device's own timestep
sequence, and the difference of the final states is the error of the float32
result (tests/f64_error.py). Cases: every golden case, the 512 x 512 rain-on-grid
configuration shape (60 steps), the 2048 x 2048 dam break (12 steps) and a
1024 x 8192 band of the 8192 x 8192 valley reach (8 steps, infiltration, inflows,
bedload). Bound (tests/f64_error.py ``check``): depth within 1e-4 m of float64
(1e-3 m where a random initial depth puts cells at the dry threshold), 2e-5
relative in the L2 norm for depth (in RMS over the discharge scale for discharge:
float32 round-off on a 6 cm sheet reaches 1.6e-5), at most 0.1 % of cells off by more
than 1e-5 of the largest depth, volume within 1e-6.
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


def _check(case, max_depth_m=1e-4):
    from f64_error import check
    from gpu_api import GpuAPI

    got = run_case(dict(case), GpuAPI())
    err = error_vs_f64(case, got)
    check(err, max_depth_m=max_depth_m, rel=2e-5)
    return err


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_against_float64(name):
    _check(CASES[name]())


def test_li_512_rain_on_grid_against_float64():
    """A random initial depth of 0-0.3 m puts many cells at the 1 mm dry threshold, where
    float32 and float64 can take different branches: a few cells then differ by a few
    tenths of a millimetre (2.5e-4 m measured) while the field agrees to round-off."""
    from test_gpu_parity import _synthetic_li

    case = _synthetic_li(512, 512, seed=1)
    case["steps"] = 60
    _check(case, max_depth_m=1e-3)


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
