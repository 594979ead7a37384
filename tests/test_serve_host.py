"""Host logic of the solve server, without a device: the request stream, frame times,
the memory each request reserves for admission, and latency bookkeeping."""

from __future__ import annotations

import math

import numpy as np
import pytest

from rbsim.serve import Request, Result, output_times, poisson_stream, request_bytes


def test_the_request_stream_has_the_configured_mix():
    """Poisson arrivals; sides log-uniform in [256, 4096]; about 70 % local-inertial and
    30 % HLLC; morphology only on local-inertial requests (10 % of all); seeded."""
    reqs = poisson_stream(rate=10.0, n=4000, seed=3)
    arrivals = np.array([r.arrival for r in reqs])
    assert (np.diff(arrivals) > 0).all() and arrivals[0] > 0
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert abs(gaps.mean() - 0.1) < 0.01  # exponential gaps of mean 1 / rate
    sides = np.array([r.side for r in reqs])
    assert sides.min() >= 256 and sides.max() <= 4096
    assert abs(np.log(sides).mean() - 0.5 * (math.log(256) + math.log(4096))) < 0.05
    li = np.array([r.scheme == "local_inertial" for r in reqs])
    assert abs(li.mean() - 0.7) < 0.03
    exner = np.array([r.exner for r in reqs])
    assert not exner[~li].any() and abs(exner.mean() - 0.1) < 0.02
    assert all(r.dx == (10.0 if r.scheme == "local_inertial" else 2.0) for r in reqs)
    assert all(600.0 <= r.horizon <= 7200.0 for r in reqs)
    again = poisson_stream(rate=10.0, n=4000, seed=3)
    assert [(r.arrival, r.side, r.scheme, r.seed) for r in again] == [(r.arrival, r.side, r.scheme, r.seed)
                                                                       for r in reqs]  # fmt: skip


def test_frame_times_are_the_multiples_of_the_cadence_and_the_horizon():
    req = Request(rid=0, arrival=0.0, scheme="local_inertial", side=256, horizon=1000.0, seed=1, output_every=300.0)
    assert output_times(req) == [300.0, 600.0, 900.0, 1000.0]
    req.output_every = 250.0
    assert output_times(req) == [250.0, 500.0, 750.0, 1000.0]
    req.output_every = 0.0
    assert output_times(req) == []


def test_request_memory_counts_the_resident_fields():
    li = Request(rid=0, arrival=0.0, scheme="local_inertial", side=1000, horizon=600.0, seed=1)
    hllc = Request(rid=1, arrival=0.0, scheme="hllc_fv", side=1000, horizon=600.0, seed=1)
    morph = Request(rid=2, arrival=0.0, scheme="local_inertial", side=1000, horizon=600.0, seed=1, exner=True)
    cells = 1000 * 1000
    assert request_bytes(li) == 36 * cells + (1 << 20)  # h/qx/qy double-buffered, z, n, rain residue
    assert request_bytes(hllc) == 44 * cells + (1 << 20)  # h/hu/hv double-buffered, z, n, stage-1 state
    assert request_bytes(morph) - request_bytes(li) == 40 * cells  # d50, z0, dz_cum, dz_unapplied, transport
    big = Request(rid=3, arrival=0.0, scheme="local_inertial", side=2000, horizon=600.0, seed=1)
    assert request_bytes(big) - (1 << 20) == pytest.approx(4 * (request_bytes(li) - (1 << 20)))


def test_latency_is_from_arrival_to_finish():
    r = Result(rid=0, arrival=2.0, admitted=2.5, finished=9.0, steps=100, t=600.0)
    assert r.latency == 7.0
