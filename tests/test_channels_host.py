"""Host side of the sub-grid channels (rbsim.channels): the storage curve and validation.

Restates the algebraic and structural tests of the reference's
solver/core/test_channels.py (:42, :64, :97, :127, :136) against the host
functions; the kernel side (zero-width seam, column CFL, mass) is in tests/gates.py.
"""

from __future__ import annotations

import numpy as np
import pytest

from rbsim.channels import ChannelError, column_depth, eta_from_h, h_from_eta, validate_geometry
from rbsim.grid import Grid


def test_storage_curve_is_continuous_monotone_and_invertible():
    dx, w, d, z = 100.0, 20.0, 3.0, 12.0
    h_bf = w * d / dx
    assert eta_from_h(h_bf, z, w, d, dx) == pytest.approx(z, abs=1e-12)
    assert eta_from_h(h_bf - 1e-9, z, w, d, dx) == pytest.approx(z, abs=1e-6)
    assert eta_from_h(h_bf + 1e-9, z, w, d, dx) == pytest.approx(z, abs=1e-6)
    assert eta_from_h(h_bf / 2, z, w, d, dx) == pytest.approx(z - d / 2)
    assert eta_from_h(h_bf + 0.4, z, w, d, dx) == pytest.approx(z + 0.4)
    h = np.linspace(0.0, 5.0, 501)
    eta = eta_from_h(h, z, w, d, dx)
    assert np.all(np.diff(eta) > 0.0)
    np.testing.assert_allclose(h_from_eta(eta, z, w, d, dx), h, atol=1e-12)
    assert eta_from_h(0.0, z, w, d, dx) == pytest.approx(z - d)


def test_no_channel_is_exactly_the_plain_relation():
    h = np.linspace(0.0, 3.0, 64)
    z = np.full_like(h, 7.25)
    zero = np.zeros_like(h)
    np.testing.assert_array_equal(eta_from_h(h, z, zero, zero, 30.0), z + h)
    np.testing.assert_array_equal(column_depth(h, zero, zero, 30.0), h)


def test_column_depth_in_and_over_bank():
    dx, w, d = 200.0, 20.0, 3.0
    assert column_depth(0.05, w, d, dx) == pytest.approx(0.05 * dx / w)
    h_bf = w * d / dx
    assert column_depth(h_bf + 0.5, w, d, dx) == pytest.approx(d + 0.5)


def test_geometry_that_cannot_mean_anything_is_refused():
    grid = Grid(ny=3, nx=4, dx=50.0)
    ok_w = np.full((3, 4), 10.0, np.float32)
    ok_d = np.full((3, 4), 2.0, np.float32)
    ok_n = np.full((3, 4), 0.03, np.float32)
    wide = ok_w.copy()
    wide[1, 1] = 60.0
    with pytest.raises(ChannelError, match="wider than the cell"):
        validate_geometry(wide, ok_d, ok_n, grid)
    half = ok_d.copy()
    half[0, 0] = 0.0
    with pytest.raises(ChannelError, match="width without a bank-full depth"):
        validate_geometry(ok_w, half, ok_n, grid)
    neg = ok_w.copy()
    neg[2, 3] = -1.0
    with pytest.raises(ChannelError, match=">= 0"):
        validate_geometry(neg, ok_d, ok_n, grid)
    with pytest.raises(ChannelError, match="shape"):
        validate_geometry(np.zeros((2, 2), np.float32), ok_d, ok_n, grid)
    bad_n = ok_n.copy()
    bad_n[0, 0] = 0.0
    with pytest.raises(ChannelError, match="manning > 0"):
        validate_geometry(ok_w, ok_d, bad_n, grid)
    nan = ok_w.copy()
    nan[0, 1] = np.nan
    with pytest.raises(ChannelError, match="non-finite"):
        validate_geometry(nan, ok_d, ok_n, grid)
    assert issubclass(ChannelError, ValueError)


def test_a_hairline_channel_warns_because_it_will_crawl():
    grid = Grid(ny=2, nx=2, dx=200.0)
    with pytest.warns(UserWarning, match="timestep"):
        validate_geometry(np.full((2, 2), 0.01, np.float32), np.full((2, 2), 1.0, np.float32),
                          np.full((2, 2), 0.03, np.float32), grid)  # fmt: skip


def test_no_channel_normalises_to_zero_in_both_fields():
    grid = Grid(ny=2, nx=2, dx=50.0)
    w = np.array([[0.0, 10.0], [0.0, 0.0]], np.float32)
    d = np.array([[0.0, 2.0], [0.0, 0.0]], np.float32)
    w_out, d_out, _ = validate_geometry(w, d, np.full((2, 2), 0.03, np.float32), grid)
    assert w_out[0, 0] == 0.0 and d_out[0, 0] == 0.0
    assert w_out[0, 1] == 10.0 and d_out[0, 1] == 2.0


def test_kernel_storage_curve_matches_the_host_reference():
    """solver/core/test_channels.py:71: the oracle's compute_eta_channels kernel and the host
    storage curve agree (in-bank and overbank cells, channel and plain cells)."""
    import ctypes

    import oracle

    ny, nx, dx = 4, 16, 100.0
    rng = np.random.default_rng(7)
    h = rng.uniform(0.0, 2.0, (ny, nx)).astype(np.float32)
    z = rng.uniform(5.0, 15.0, (ny, nx)).astype(np.float32)
    w = np.where(rng.random((ny, nx)) < 0.5, 0.0, rng.uniform(5.0, 40.0, (ny, nx))).astype(np.float32)
    d = np.where(w > 0, rng.uniform(0.5, 4.0, (ny, nx)), 0.0).astype(np.float32)
    eta = np.zeros((ny, nx), np.float32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    oracle.lib().rbo_compute_eta_channels_f32(ny, nx, p(h), p(z), p(w), p(d), ctypes.c_float(dx), p(eta))
    np.testing.assert_allclose(eta, eta_from_h(h, z, w, d, dx), rtol=1e-5, atol=1e-5)
    plain = w == 0
    assert plain.any() and (~plain).any()
    np.testing.assert_array_equal(eta[plain], (z + h)[plain])
