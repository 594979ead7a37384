"""The bedload law, its face integral and Exner: the reference's kernel tests on the oracle.

These restate solver/core/test_sediment.py:174-740 against the oracle's
``rbo_accumulate_qs``, ``rbo_accumulate_qs_channels``, ``rbo_exner_update`` and
``rbo_rebuild_bed``, and against
this package's host references (``rbsim.sediment``). The CUDA step fuses the same
face integral into the local-inertial tile and runs the same Exner update in
``rb_exner_apply``. It equals the oracle bit for bit on the golden sediment cases and
on the long bed-wave run. The checks are: MPM by hand; a bit-exact zero below
threshold and on dry faces; the integral equal to transport times elapsed time, with
its compensation kept; the x and y kernels transposes of each other; Exner's
divergence, bounds and banking; and the bed rebuilt from the pristine bed. Also a
channel face carries its conveyance fraction, the channel kernel collapses onto the
plain one at zero width, clearing keeps the compensation debt, and a zero grain size
does not immobilise a cell.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from rbsim.grid import GRAVITY, H_DRY
from rbsim.sediment import (
    MPM_COEFFICIENT,
    SHIELDS_CRITICAL,
    SUBMERGED_SG,
    bed_celerity,
    capacity_from_flow,
    morphological_courant,
    shields_from_flow,
)


@pytest.fixture(scope="module", autouse=True)
def _pow_mode():
    oracle.set_pow_mode(1)
    yield
    oracle.set_pow_mode(0)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def accumulate(qx, qy, eta, z, n, d50, dt, acc):
    """One ``rbo_accumulate_qs`` call; ``acc`` holds (qs_x, comp_x, qs_y, comp_y), updated in place."""
    ny, nx = z.shape
    qx, qy, eta, z, n, d50 = (_f32(a) for a in (qx, qy, eta, z, n, d50))
    oracle.lib().rbo_accumulate_qs_f32(ny, nx, _p(qx), _p(qy), _p(eta), _p(z), _p(n), _p(d50), ctypes.c_float(dt),
                                       *(_p(a) for a in acc))  # fmt: skip


def new_acc(ny, nx):
    z = np.zeros
    return (z((ny, nx + 1), np.float32), z((ny, nx + 1), np.float32), z((ny + 1, nx), np.float32),
            z((ny + 1, nx), np.float32))  # fmt: skip


def exner(qs_x, qs_y, *, dx=50.0, porosity=0.4, lo=None, hi=None, dz=None, banked=None):
    ny, nx = qs_y.shape[0] - 1, qs_x.shape[1] - 1
    dz = np.zeros((ny, nx)) if dz is None else dz
    banked = np.zeros((ny, nx)) if banked is None else banked
    lo = _f32(np.full((ny, nx), -np.inf) if lo is None else lo)
    hi = _f32(np.full((ny, nx), np.inf) if hi is None else hi)
    qs_x, qs_y = _f32(qs_x), _f32(qs_y)
    oracle.lib().rbo_exner_update_f32(ny, nx, _p(qs_x), _p(qs_y), _p(lo), _p(hi), ctypes.c_float(dx),
                                      ctypes.c_float(1.0 / (1.0 - porosity)), _p(dz), _p(banked))  # fmt: skip
    return dz, banked


def _rows_of_faces(depths, q, n=0.03, d50=0.008):
    """One row per depth, two cells, one interior x-face carrying ``q`` at that depth."""
    k = len(depths)
    z = np.full((k, 2), 10.0, np.float32)
    eta = (z + np.asarray(depths, np.float32)[:, None]).astype(np.float32)
    qx = np.full((k, 3), q, np.float32)
    acc = new_acc(k, 2)
    accumulate(qx, np.zeros((k + 1, 2)), eta, z, np.full((k, 2), n), np.full((k, 2), d50), 1.0, acc)
    return acc[0][:, 1]


def test_capacity_is_hand_computable():
    """test_sediment.py:174."""
    q, h, n, d50 = 2.0, 1.0, 0.03, 0.008
    theta = GRAVITY * n**2 * q**2 / h ** (7.0 / 3.0) / (SUBMERGED_SG * GRAVITY * d50)
    assert theta == pytest.approx(0.27273, rel=1e-4)
    qs = MPM_COEFFICIENT * (theta - SHIELDS_CRITICAL) ** 1.5 * np.sqrt(SUBMERGED_SG * GRAVITY * d50**3)
    assert qs == pytest.approx(2.4699e-3, rel=1e-4)
    assert capacity_from_flow(q, h, n, d50) == pytest.approx(qs, rel=1e-9)
    assert float(shields_from_flow(q, h, n, d50)) == pytest.approx(theta, rel=1e-12)


def test_below_threshold_the_capacity_is_bit_exact_zero():
    """test_sediment.py:188: either side of the depth that puts theta at theta_c."""
    q, n, d50 = 1.0, 0.03, 0.008
    h_c = (GRAVITY * n**2 * q**2 / (SUBMERGED_SG * GRAVITY * d50 * SHIELDS_CRITICAL)) ** (3 / 7)
    got = _rows_of_faces([h_c * 1.05, h_c * 2.0, 5.0, h_c * 0.95, h_c * 0.5], q, n, d50)
    assert (got[:3] == 0.0).all() and (got[3:] > 0.0).all()


def test_a_dry_face_transports_nothing():
    """test_sediment.py:217: below H_DRY the face carries no bedload."""
    got = _rows_of_faces([0.0, 0.5 * H_DRY, 2.0 * H_DRY], 0.5)
    assert got[0] == 0.0 and got[1] == 0.0 and got[2] > 0.0


def test_the_face_integral_is_transport_times_elapsed_time():
    """test_sediment.py:253: a steady flow for 25 steps of 4 s integrates to q_s dt N."""
    ny, nx, dt, steps = 3, 5, 4.0, 25
    depth, q, n, d50 = 1.2, 2.5, 0.03, 0.008
    z = np.full((ny, nx), 10.0, np.float32)
    acc = new_acc(ny, nx)
    for _ in range(steps):
        accumulate(np.full((ny, nx + 1), q), np.zeros((ny + 1, nx)), z + depth, z, np.full((ny, nx), n),
                   np.full((ny, nx), d50), dt, acc)  # fmt: skip
    got = acc[0]
    assert np.allclose(got[:, 1:nx], capacity_from_flow(q, depth, n, d50) * dt * steps, rtol=1e-5)
    assert (got[:, 0] == 0.0).all() and (got[:, nx] == 0.0).all()


def test_the_transport_integral_is_compensated_not_merely_added():
    """test_sediment.py:282: increments under half an ulp of the integral still land.

    Seeded at 4 m^2, each 1 us step adds about 2.5e-9 against an ulp of 4.8e-7, so a
    plain add would leave the integral at 4.0 forever.
    """
    ny, nx, q, depth = 1, 2, 2.0, 1.0
    z = np.full((ny, nx), 10.0, np.float32)
    acc = new_acc(ny, nx)
    acc[0][:, 1] = 4.0
    step_qs = float(capacity_from_flow(q, depth, 0.03, 0.008)) * 1e-6
    assert step_qs < 0.5 * float(np.spacing(np.float32(4.0)))
    for _ in range(2000):
        accumulate(np.full((ny, nx + 1), q), np.zeros((ny + 1, nx)), z + depth, z, np.full((ny, nx), 0.03),
                   np.full((ny, nx), 0.008), 1e-6, acc)  # fmt: skip
    total = float(acc[0][0, 1]) - 4.0 - float(acc[1][0, 1])
    assert acc[0][0, 1] > 4.0 and acc[1][0, 1] != 0.0
    assert total == pytest.approx(2000 * step_qs, rel=1e-3)


def test_the_two_directions_are_transposes_of_each_other():
    """test_sediment.py:328: the y kernel on the transposed problem is the x kernel, bit for bit."""
    ny, nx, dt = 3, 6, 2.5
    rng = np.random.default_rng(19)
    z = (20.0 - 0.1 * np.arange(nx)[None, :] * np.ones((ny, 1))).astype(np.float32)
    eta = (z + rng.uniform(0.3, 1.5, (ny, nx))).astype(np.float32)
    qx = rng.uniform(-2.5, 2.5, (ny, nx + 1)).astype(np.float32)
    n = rng.uniform(0.025, 0.05, (ny, nx)).astype(np.float32)
    d50 = rng.uniform(2e-3, 2e-2, (ny, nx)).astype(np.float32)
    ax = new_acc(ny, nx)
    accumulate(qx, np.zeros((ny + 1, nx)), eta, z, n, d50, dt, ax)
    ay = new_acc(nx, ny)
    accumulate(np.zeros((nx, ny + 1)), qx.T, eta.T, z.T, n.T, d50.T, dt, ay)
    assert (ay[2] == ax[0].T).all() and (ay[0] == 0.0).all()
    dz_x, _ = exner(ax[0], np.zeros((ny + 1, nx)))
    dz_y, _ = exner(np.zeros((nx, ny + 1)), ay[2])
    assert (dz_y == dz_x.T).all() and np.abs(dz_x).max() > 0.0


def test_still_water_writes_no_transport_at_all():
    """test_sediment.py:374."""
    z = np.full((4, 4), 10.0, np.float32)
    acc = new_acc(4, 4)
    accumulate(np.zeros((4, 5)), np.zeros((5, 4)), z + 2.0, z, np.full((4, 4), 0.03), np.full((4, 4), 0.008), 10.0,
               acc)  # fmt: skip
    assert all((a == 0.0).all() for a in acc)


def test_uniform_transport_moves_no_bed():
    """test_sediment.py:509."""
    dz, banked = exner(np.full((4, 5), 3.7e-3), np.full((5, 4), -1.1e-3))
    assert (dz == 0.0).all() and (banked == 0.0).all()


def test_exner_matches_the_hand_computed_divergence():
    """test_sediment.py:517: a net export of 2 mm^2 per face drops every cell by gain / dx / (1 - p)."""
    ny, nx, dx, p, gain = 3, 5, 50.0, 0.4, 2.0e-3
    qs_x = gain * np.arange(nx + 1)[None, :] * np.ones((ny, 1))
    dz, _ = exner(qs_x, np.zeros((ny + 1, nx)), dx=dx, porosity=p)
    assert np.allclose(dz, -gain / dx / (1.0 - p), rtol=1e-6)


def test_a_bound_banks_exactly_what_it_refuses():
    """test_sediment.py:528: a frozen cell banks the whole change, a floor the part below it."""
    ny, nx, dx, p, gain = 1, 3, 50.0, 0.4, 2.0e-3
    qs_x = gain * np.arange(nx + 1)[None, :] * np.ones((ny, 1))
    want = -gain / dx / (1.0 - p)
    frozen = np.zeros((ny, nx), np.float32)
    dz, banked = exner(qs_x, np.zeros((ny + 1, nx)), dx=dx, porosity=p, lo=frozen, hi=frozen)
    assert (dz == 0.0).all() and np.allclose(banked, want, rtol=1e-6)
    floor = np.full((ny, nx), 0.5 * want, np.float32)
    dz, banked = exner(qs_x, np.zeros((ny + 1, nx)), dx=dx, porosity=p, lo=floor)
    assert (dz == floor.astype(np.float64)).all()
    assert np.allclose(banked, want - floor.astype(np.float64), rtol=1e-5)
    assert np.allclose(dz + banked, want, rtol=1e-6)  # nothing lost: applied + banked = wanted


def test_the_bed_is_rebuilt_from_the_pristine_bed_not_incremented():
    """test_sediment.py:551: 1 um activations at z = 175 m survive only when rebuilt from z0."""
    z0 = np.full((2, 2), 175.0, np.float32)
    z = z0.copy()
    dz = np.zeros((2, 2))
    for k in range(100):
        dz[:] = 1.0e-6 * (k + 1)
        oracle.lib().rbo_rebuild_bed_f32(2, 2, _p(z0), _p(dz), _p(z))
    assert np.abs((z.astype(np.float64) - 175.0) - 1.0e-4).max() <= float(np.spacing(np.float32(175.0)))
    naive = np.float32(175.0)
    for _ in range(100):
        naive = np.float32(naive + np.float32(1.0e-6))
    assert naive == np.float32(175.0)


def test_bed_celerity_matches_a_finite_difference_of_the_law():
    """test_sediment.py:584 (the wide section; sub-grid channel celerity is outside this path)."""
    q, h, n, d50, p, eps = 2.0, 1.0, 0.03, 0.008, 0.4, 1e-6
    fd = (capacity_from_flow(q, h - eps, n, d50) - capacity_from_flow(q, h + eps, n, d50)) / (2 * eps)
    assert float(bed_celerity(q, h, n, d50, p)) == pytest.approx(float(fd) / (1 - p), rel=1e-5)


def test_the_morphological_courant_number_is_the_ratio_it_claims():
    """test_sediment.py:617."""
    assert morphological_courant(1e-4, 900.0, 50.0) == pytest.approx(1.8e-3)
    assert morphological_courant(0.0, 900.0, 50.0) == 0.0


def test_no_shear_means_no_celerity():
    """test_sediment.py:622."""
    assert float(bed_celerity(0.0, 1.0, 0.03, 0.008, 0.4)) == 0.0
    assert float(shields_from_flow(1.0, 20.0, 0.03, 0.008)) < SHIELDS_CRITICAL
    assert float(bed_celerity(1.0, 20.0, 0.03, 0.008, 0.4)) == 0.0


def accumulate_channels(qx_ch, qx_fp, eta, z, n, d50, w, d, cn, dx, dt, acc):
    """One ``rbo_accumulate_qs_channels`` call over x-faces (the y components are zero)."""
    ny, nx = z.shape
    zy = np.zeros((ny + 1, nx), np.float32)
    args = [_f32(a) for a in (qx_ch, qx_fp)] + [zy, zy.copy()] + [_f32(a) for a in (eta, z, n, d50, w, d, cn)]
    oracle.lib().rbo_accumulate_qs_channels_f32(ny, nx, *(_p(a) for a in args), ctypes.c_float(dx),
                                                ctypes.c_float(dt), *(_p(a) for a in acc))  # fmt: skip


def test_a_channel_face_carries_its_conveyance_fraction():
    """test_sediment.py:402: with the floodplain dry, the cell-width flux is the channel's
    capacity (from its own depth and radius A/P) scaled by w / dx."""
    ny, nx, dx = 1, 4, 200.0
    w, bank, n_ch, d50, h_ch, q_ch = 20.0, 1.0, 0.028, 0.008, 0.5, 1.8
    z = np.full((ny, nx), 10.0, np.float32)
    acc = new_acc(ny, nx)
    accumulate_channels(np.full((ny, nx + 1), q_ch), np.zeros((ny, nx + 1)), z - bank + h_ch, z,
                        np.full((ny, nx), 0.05), np.full((ny, nx), d50), np.full((ny, nx), w),
                        np.full((ny, nx), bank), np.full((ny, nx), n_ch), dx, 1.0, acc)  # fmt: skip
    qs_channel = float(capacity_from_flow(q_ch, h_ch, n_ch, d50, radius=w * h_ch / (w + 2.0 * h_ch)))
    assert qs_channel > 0.0
    assert float(acc[0][0, 1]) * dx == pytest.approx(qs_channel * w, rel=1e-4)
    assert float(capacity_from_flow(q_ch, h_ch * w / dx, n_ch, d50)) > 10.0 * qs_channel


def test_the_channel_kernel_collapses_onto_the_plain_one_at_zero_width():
    """test_sediment.py:446: w = d = 0 is the no-channel case, bit for bit."""
    ny, nx, dx, dt = 3, 6, 50.0, 3.0
    rng = np.random.default_rng(3)
    z = (10.0 - 0.05 * np.arange(nx)[None, :] * np.ones((ny, 1))).astype(np.float32)
    eta = (z + rng.uniform(0.3, 1.5, (ny, nx))).astype(np.float32)
    qx = rng.uniform(-2.0, 2.0, (ny, nx + 1)).astype(np.float32)
    n, d50, zero = np.full((ny, nx), 0.033), np.full((ny, nx), 0.006), np.zeros((ny, nx))
    plain, chan = new_acc(ny, nx), new_acc(ny, nx)
    accumulate(qx, np.zeros((ny + 1, nx)), eta, z, n, d50, dt, plain)
    accumulate_channels(np.zeros((ny, nx + 1)), qx, eta, z, n, d50, zero, zero, zero, dx, dt, chan)
    assert (plain[0] == chan[0]).all() and (plain[1] == chan[1]).all() and np.abs(plain[0]).max() > 0.0


def test_clearing_keeps_the_compensation_debt():
    """test_sediment.py:479: an activation consumes the integral; the bits it never held stay owed."""
    st = oracle.State.from_bed(np.full((2, 3), 5.0, np.float32), 10.0, depth=0.5)
    st.arm_sediment(0.002, 0.4)
    sed = st.sediment
    sed.qs_int_x[...] = 4.0
    sed.qs_comp_x[...] = 1.25e-9
    lo, hi = np.full((2, 3), -np.inf, np.float32), np.full((2, 3), np.inf, np.float32)
    oracle.exner_activate(st, lo, hi)
    assert (sed.qs_int_x == 0.0).all() and (sed.qs_comp_x == np.float32(1.25e-9)).all()


def test_a_zero_grain_size_does_not_make_a_cell_immobile():
    """test_sediment.py:727: d50 is face-averaged, so a lone zero cell's faces still transport
    and its bed moves (immobility is what a zero alluvium bound is for)."""
    ny, nx = 1, 3
    d50 = np.array([[0.004, 0.0, 0.004]], np.float32)
    acc = new_acc(ny, nx)
    accumulate(np.array([[0.0, 2.0, 2.6, 0.0]]), np.zeros((ny + 1, nx)), np.ones((ny, nx)), np.zeros((ny, nx)),
               np.full((ny, nx), 0.03), d50, 60.0, acc)  # fmt: skip
    assert (acc[0][0, 1:3] != 0.0).all()
    dz, _ = exner(acc[0], acc[2], dx=5.0)
    assert dz[0, 1] != 0.0


def _armed_reach():
    """A wet 4 x 6 reach with a bedload integral of an uneven flow, armed at bed z0."""
    ny, nx = 4, 6
    rng = np.random.default_rng(8)
    st = oracle.State.from_bed((100.0 + 0.02 * rng.standard_normal((ny, nx))).astype(np.float32), 10.0, depth=0.6)
    st.arm_sediment(0.004, 0.4)
    acc = new_acc(ny, nx)
    accumulate(rng.uniform(0.5, 3.0, (ny, nx + 1)), rng.uniform(-1.0, 1.0, (ny + 1, nx)), st.z + st.h, st.z,
               np.full((ny, nx), 0.03), np.full((ny, nx), 0.004), 30.0, acc)  # fmt: skip
    sed = st.sediment
    sed.qs_int_x[...], sed.qs_comp_x[...], sed.qs_int_y[...], sed.qs_comp_y[...] = acc
    return st


def test_an_activation_rebuilds_the_bed_from_z0_and_leaves_the_water():
    """solver/processes/test_morphology.py:164, :194: z = float32(z0 + dz_cum), the integral
    cleared, depth untouched, eta refreshed from the new bed."""
    st = _armed_reach()
    h0, z0 = st.h.copy(), st.sediment.z0.copy()
    free = np.full(z0.shape, -np.inf, np.float32), np.full(z0.shape, np.inf, np.float32)
    oracle.exner_activate(st, *free)
    sed = st.sediment
    assert np.abs(sed.dz_cum).max() > 0.0
    assert (st.z == (z0.astype(np.float64) + sed.dz_cum).astype(np.float32)).all()
    assert (sed.qs_int_x == 0.0).all() and (sed.qs_int_y == 0.0).all()
    assert (st.h == h0).all() and (st.eta == (st.h + st.z)).all()


def test_a_frozen_cell_banks_exactly_what_the_free_bed_moved_there():
    """solver/processes/test_morphology.py:257: the same integral applied with and without a
    frozen cell; the frozen run keeps that cell's bed and banks the free run's change there."""
    free_st, frozen_st = _armed_reach(), _armed_reach()
    shape = free_st.z.shape
    lo, hi = np.full(shape, -np.inf, np.float32), np.full(shape, np.inf, np.float32)
    oracle.exner_activate(free_st, lo, hi)
    lo_f, hi_f = lo.copy(), hi.copy()
    lo_f[2, 3] = hi_f[2, 3] = 0.0
    oracle.exner_activate(frozen_st, lo_f, hi_f)
    want = free_st.sediment.dz_cum[2, 3]
    assert want != 0.0
    assert frozen_st.sediment.dz_cum[2, 3] == 0.0 and frozen_st.z[2, 3] == frozen_st.sediment.z0[2, 3]
    assert frozen_st.sediment.dz_unapplied[2, 3] == want
    others = np.ones(shape, bool)
    others[2, 3] = False
    assert (frozen_st.sediment.dz_cum[others] == free_st.sediment.dz_cum[others]).all()
