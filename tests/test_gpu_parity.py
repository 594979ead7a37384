"""CUDA path vs the CPU oracle: bit-for-bit on seeded inputs.

The kernels and the oracle share one arithmetic contract (one IEEE rounding per
operation in the reference's expression order, no fused multiply-add, the
deterministic powers of include/rb_detmath.h), so with the oracle in
``pow_mode=1`` every state field must match exactly -- depth, discharge,
momenta, Kahan residues, transport integrals, float64 bed change -- after many
steps. The only quantity compared with a tolerance is the float64 loss ledger,
whose per-tile partial sums are added in a different order from the oracle's
per-cell field (relative 1e-12).

The oracle itself is pinned bit-for-bit to the reference's own kernels
(tests/test_oracle_golden.py), and within 1e-5 relative in this power mode.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

import oracle  # noqa: E402
from cases import CASES, run_case  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    from rbsim import _lib

    _lib.lib()
    oracle.set_pow_mode(1)
    yield
    oracle.set_pow_mode(0)


def _oracle_outputs(case):
    from test_oracle_golden import OracleAPI

    out = run_case(case, OracleAPI())
    if "loss_cum" in out:
        out["loss_total"] = np.float64(out.pop("loss_cum").sum())
    return out


def _compare(got, want, name):
    assert sorted(got) == sorted(want), (sorted(got), sorted(want))
    for key in want:
        if key == "loss_total":
            np.testing.assert_allclose(got[key], want[key], rtol=1e-12, atol=1e-300, err_msg=f"{name}:{key}")
        else:
            np.testing.assert_array_equal(got[key], want[key], err_msg=f"{name}:{key}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_match_oracle_bitwise(name):
    from gpu_api import GpuAPI

    case = CASES[name]()
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), name)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_track_reference_fixtures(name):
    """The CUDA path against the reference-kernel fixtures, at the solver tolerance."""
    from gpu_api import GpuAPI

    want = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    got = run_case(CASES[name](), GpuAPI())
    for key, ref in want.items():
        if key in ("h_comp", "qs_comp_x", "qs_comp_y"):
            continue
        if key == "loss_cum":
            np.testing.assert_allclose(got["loss_total"], ref.sum(), rtol=1e-5, atol=1e-9)
            continue
        np.testing.assert_allclose(got[key], ref, rtol=1e-5, atol=1e-6, err_msg=f"{name}:{key}")


def _synthetic_li(ny, nx, seed):
    rng = np.random.default_rng(seed)
    dx = 10.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    z = 1e-3 * xx * dx
    for _ in range(12):
        a, s = rng.uniform(0.5, 5.0), rng.uniform(50.0, 300.0)
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        z += a * np.exp(-(((yy - cy) ** 2 + (xx - cx) ** 2) * dx * dx) / (2 * s * s))
    return dict(
        scheme="local_inertial", bed=z.astype(np.float32), dx=dx, depth=rng.uniform(0.0, 0.3, (ny, nx)).astype(
            np.float32), manning=0.03, compensated=True, rain=50.0 / 1000.0 / 3600.0,
        infil=rng.uniform(0, 1e-5, (ny, nx)).astype(np.float32),
        boundaries={"north": "open", "south": "open", "east": "open", "west": "open"},
        steps=40, alpha=0.7, dt_max=30.0,
    )  # fmt: skip


def _synthetic_hllc(ny, nx, seed):
    rng = np.random.default_rng(seed)
    dx = 1.0
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    z = np.zeros((ny, nx))
    for _ in range(10):
        a, s = rng.uniform(0.5, 3.5), rng.uniform(10.0, 80.0)
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        z += a * np.exp(-(((yy - cy) ** 2 + (xx - cx) ** 2)) / (2 * s * s))
    depth = np.where(xx < nx / 2, 10.0, 1.0) - 0.5 * z
    return dict(scheme="hllc_fv", bed=z.astype(np.float32), dx=dx, depth=np.maximum(depth, 0).astype(np.float32),
                manning=0.02, steps=25, alpha=0.45, dt_max=30.0)  # fmt: skip


@pytest.mark.parametrize("shape", [(256, 256), (333, 517), (1, 700), (700, 1), (37, 3)])
def test_li_seeded_grids_match_oracle_bitwise(shape):
    """Ragged sizes (not multiples of the tile), one-row / one-column domains."""
    from gpu_api import GpuAPI

    case = _synthetic_li(*shape, seed=11)
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), f"li{shape}")


@pytest.mark.parametrize("shape", [(256, 256), (301, 419), (1, 600), (5, 2)])
def test_hllc_seeded_grids_match_oracle_bitwise(shape):
    from gpu_api import GpuAPI

    case = _synthetic_hllc(*shape, seed=12)
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), f"hllc{shape}")


def test_li_open_edges_without_infiltration_match_oracle_bitwise():
    """Open edges bank their outflow in the float64 ledger; without infiltration an
    interior tile banks nothing, and its block sum is skipped. 300 x 420 has 80 interior
    tiles of 32 x 32 between edge tiles that bank, and the banked total must still be
    the oracle's."""
    from gpu_api import GpuAPI

    case = _synthetic_li(300, 420, seed=21)
    del case["infil"]
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), "li(300, 420) without infiltration")


def test_li_config_scale_512_matches_oracle_bitwise():
    """The 512 x 512 rain-on-grid configuration shape, 60 steps."""
    from gpu_api import GpuAPI

    case = _synthetic_li(512, 512, seed=1)
    case["steps"] = 60
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), "li512")


def test_hllc_dambreak_2048_matches_oracle_bitwise():
    """The 2048 x 2048 dam-break configuration (flat bed, h 10 | 1 m), 12 steps."""
    from gpu_api import GpuAPI

    n = 2048
    depth = np.ones((n, n), np.float32)
    depth[:, : n // 2] = 10.0
    case = dict(scheme="hllc_fv", bed=np.zeros((n, n), np.float32), dx=1.0, depth=depth, manning=0.0,
                steps=12, alpha=0.45, dt_max=30.0)  # fmt: skip
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), "hllc2048")


def test_hllc_lake_at_rest_with_islands_matches_oracle_bitwise():
    """The lake-at-rest configuration's generator on a 256 x 256 crop (dx 1 m, four
    Gaussian bumps of amplitude U(0.5, 3.5) m and sigma U(10, 80) m, seed 2,
    h = max(2 - z, 0), n 0.03) run to the configuration's 600 s horizon: 5881 steps,
    bit for bit against the float32 oracle. The deep-water speed at the horizon
    (~5e-4 m/s) and the shoreline films' (~6.5e-3 m/s) are the scheme's own residual
    at wet/dry fronts on slopes this steep: the float64 oracle shows the same speeds
    (test_lake_at_rest_f64.py)."""
    from gpu_api import GpuAPI
    from test_lake_at_rest_f64 import lake_crop

    z = lake_crop()
    case = dict(scheme="hllc_fv", bed=z, dx=1.0, depth=np.maximum(2.0 - z, 0.0).astype(np.float32), manning=0.03,
                steps=5881, alpha=0.45, dt_max=30.0)  # fmt: skip
    got = run_case(case, GpuAPI())
    assert got["dts"].sum() >= 600.0 - 1e-6 > got["dts"][:-1].sum()
    _compare(got, _oracle_outputs(case), "hllc_lake256_600s")
    deep = got["h"] > 0.1
    speed = np.maximum(np.abs(got["hu"]), np.abs(got["hv"]))[deep] / got["h"][deep]
    assert speed.max() < 1e-3, speed.max()


@pytest.mark.parametrize("name", ["hllc_bumpy_moving", "li_rain_open_infil", "li_sediment"])
def test_reruns_are_bitwise_identical(name):
    from gpu_api import GpuAPI

    a = run_case(CASES[name](), GpuAPI())
    b = run_case(CASES[name](), GpuAPI())
    for key in a:
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def _hllc_variants():
    import ctypes

    from rbsim import _lib

    n = ctypes.c_int32(0)
    _lib.check(_lib.lib().rb_hllc_kernel_variants(ctypes.byref(n)))
    return n.value


@pytest.mark.parametrize("shape", [(301, 419), (300, 420), (5, 2), (1, 600)])
def test_every_hllc_kernel_variant_matches_oracle_bitwise(shape):
    """The stage kernel's variants (tile shape, block size, faces per thread, load batching,
    tensor-memory staging) are a speed choice only: each reproduces the oracle exactly, on
    ragged grids with open and fixed_stage edges and on degenerate shapes. 300 x 420 has
    16-byte rows, so the TMA-staged variant copies its interior tiles with tensor copies
    (the other shapes take its plain-load fallback)."""
    from gpu_api import GpuAPI
    from rbsim import _lib

    case = _synthetic_hllc(*shape, seed=13)
    case["boundaries"] = {"north": "closed", "south": "open", "east": "fixed_stage", "west": "open"}
    case["stage_curves"] = {"east": [(0.0, 4.0), (10.0, 6.0)]}
    case["steps"] = 12
    want = _oracle_outputs(case)
    L = _lib.lib()
    try:
        for v in range(_hllc_variants()):
            _lib.check(L.rb_hllc_set_kernel_variant(v))
            _compare(run_case(case, GpuAPI()), want, f"hllc{shape} variant {v}")
    finally:
        _lib.check(L.rb_hllc_set_kernel_variant(6))  # the library's default


def test_persistent_tma_variant_walks_more_tiles_than_resident_blocks():
    """Variant 8 launches one block per resident slot (296 on a 148-SM B200) and walks
    the tiles, copying the halo of each block's next interior tile while it computes
    the current one. 1000 x 1028 has 1056 tiles of 32 x 32, about 3.6 a block, ragged
    on both axes: the barrier phases alternate, edge tiles take plain loads between
    copied ones, and the result is the oracle's bits."""
    from gpu_api import GpuAPI
    from rbsim import _lib

    case = _synthetic_hllc(1000, 1028, seed=17)
    case["boundaries"] = {"north": "open", "south": "closed", "east": "open", "west": "fixed_stage"}
    case["stage_curves"] = {"west": [(0.0, 9.0), (10.0, 11.0)]}
    case["steps"] = 6
    want = _oracle_outputs(case)
    L = _lib.lib()
    try:
        _lib.check(L.rb_hllc_set_kernel_variant(8))
        _compare(run_case(case, GpuAPI()), want, "hllc(1000, 1028) variant 8")
    finally:
        _lib.check(L.rb_hllc_set_kernel_variant(6))


@pytest.mark.parametrize("shape", [(333, 517), (1, 700), (37, 3)])
def test_every_li_kernel_variant_matches_oracle_bitwise(shape):
    """The local-inertial step's tile variants are a speed choice only."""
    import ctypes

    from gpu_api import GpuAPI
    from rbsim import _lib

    case = _synthetic_li(*shape, seed=14)
    case["steps"] = 15
    want = _oracle_outputs(case)
    L = _lib.lib()
    n = ctypes.c_int32(0)
    _lib.check(L.rb_li_kernel_variants(ctypes.byref(n)))
    try:
        for v in range(n.value):
            _lib.check(L.rb_li_set_kernel_variant(v))
            _compare(run_case(case, GpuAPI()), want, f"li{shape} variant {v}")
    finally:
        _lib.check(L.rb_li_set_kernel_variant(1))  # the library's default


def test_li_reach_8192_matches_oracle_bitwise():
    """The full-size 8192 x 8192 reach configuration (67 M cells: V valley with a
    meandering channel, lognormal roughness, infiltration, eight inflow cells, an open
    downstream edge, bedload with an Exner activation), two steps, bit for bit."""
    from bench_workloads import reach_inputs
    from gpu_api import GpuAPI

    z, manning, infil, inflows, depth = reach_inputs(8192, 5.0)
    n = z.shape[0]
    case = dict(scheme="local_inertial", bed=z, dx=5.0, depth=depth, manning=manning, infil=infil,
                inflows=[(inf.cell, inf.hydrograph) for inf in inflows], boundaries={"east": "open"},
                sediment=dict(d50=np.full((n, n), 0.002, np.float32), porosity=0.4, every=2,
                              dz_lo=np.full((n, n), -np.inf, np.float32), dz_hi=np.full((n, n), np.inf, np.float32)),
                steps=2, alpha=0.7, dt_max=30.0)  # fmt: skip
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), "reach8192")


def test_li_reach_band_long_run_matches_oracle_bitwise():
    """A 512 x 8192 band of the 8192 x 8192 reach (the meandering channel and all eight
    inflow cells, infiltration, lognormal roughness, bedload, the open downstream edge)
    for 200 steps with an Exner activation every 50: the long-run complement of the
    two full-size steps above, bit for bit against the oracle."""
    from bench_workloads import reach_band_spec, reach_inputs
    from gpu_api import GpuAPI

    z, manning, infil, inflows, depth = reach_inputs(8192, 5.0)
    spec = reach_band_spec(z, manning, infil, inflows, depth, rows=512)
    rows, n = spec["bed"].shape
    case = dict(scheme="local_inertial", bed=spec["bed"], dx=5.0, depth=spec["depth"], manning=spec["manning"],
                infil=spec["infil"], inflows=spec["inflows"], boundaries={"east": "open"},
                sediment=dict(d50=np.full((rows, n), 0.002, np.float32), porosity=0.4, every=50,
                              dz_lo=np.full((rows, n), -np.inf, np.float32),
                              dz_hi=np.full((rows, n), np.inf, np.float32)),
                steps=200, alpha=0.7, dt_max=30.0)  # fmt: skip
    _compare(run_case(case, GpuAPI()), _oracle_outputs(case), "reach_band_200")
