"""Is the lake-at-rest residual on steep emergent bumps round-off or the scheme?

The HLLC lake-at-rest configuration (2048^2, dx 1 m, surface 2 m over Gaussian bumps
of amplitude 0.5-3.5 m and sigma 10-80 m that pierce it) keeps ~1e-4 m/s in deep
water and mm/s in the shoreline films, above the reference's gates for gentler beds
(solver/core/test_hllc_wetdry.py:105, test_hllc_2d.py:54). This test settles where
that comes from by running the same scheme in float64 (the oracle's double build) on
a 256^2 crop of the generator: with every bump submerged the float64 scheme is at rest
to 1e-8 m/s (well balanced; float32 round-off alone gives ~3e-5 m/s), but with
emergent bumps float64 shows the same deep-water and shoreline speeds as float32, so
the residual is the scheme's own behaviour at wet/dry fronts on slopes this steep,
not float32 round-off growth. CPU only (the oracle is the checker here)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

STEPS = 400


def lake_crop(n=256, seed=2):
    """The lake-at-rest generator on an n x n crop: four bumps, h = max(2 - z, 0)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float32)
    z = np.zeros((n, n), np.float32)
    for _ in range(4):
        a, s = rng.uniform(0.5, 3.5), rng.uniform(10.0, 80.0)
        cy, cx = rng.uniform(0, n), rng.uniform(0, n)
        z += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    return z.astype(np.float32)


def _speeds(bed, dtype):
    st = oracle.State.from_bed(bed, 1.0, depth=np.maximum(2.0 - bed, 0.0).astype(np.float32), manning=0.03,
                               dtype=dtype)  # fmt: skip
    st.arm_hllc()
    for _ in range(STEPS):
        oracle.hllc_step(st, oracle.hllc_compute_dt(st, 0.45, 30.0))
    h = st.h.astype(np.float64)
    wet = h >= oracle.H_DRY
    safe = np.where(wet, h, 1.0)
    speed = np.maximum(np.abs(np.where(wet, st.hu / safe, 0.0)), np.abs(np.where(wet, st.hv / safe, 0.0)))
    return float(speed[h > 0.1].max()), float(speed.max())


@pytest.fixture(scope="module", autouse=True)
def _pow_mode():
    oracle.set_pow_mode(1)
    yield
    oracle.set_pow_mode(0)


def test_submerged_bumps_are_at_rest_in_float64():
    z = lake_crop()
    z = (z * (1.8 / z.max())).astype(np.float32)  # every bump under the 2 m surface
    deep64, _ = _speeds(z, np.float64)
    deep32, _ = _speeds(z, np.float32)
    assert deep64 < 1e-6, deep64  # well balanced: float64 round-off only
    assert deep32 < 1e-4, deep32  # float32 round-off


def test_emergent_bumps_residual_is_the_schemes_not_float32():
    z = lake_crop()
    deep64, film64 = _speeds(z, np.float64)
    deep32, film32 = _speeds(z, np.float32)
    assert deep64 > 5e-5 and film64 > 1e-3, (deep64, film64)  # present in float64 too
    assert deep32 == pytest.approx(deep64, rel=0.25)
    assert film32 == pytest.approx(film64, rel=0.05)
