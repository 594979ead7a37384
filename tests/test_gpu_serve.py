"""Serving: continuous batching returns, for every request, what solving it alone returns.

A Poisson stream of small mixed requests (LI / HLLC, some with Exner) arrives while
earlier ones are still running; the server admits them between graph replays,
retires finished ones and rebuilds the batch. Each request's final depth must be
bit-identical to the same request served alone. A tight HBM budget forces queueing
behind the budget (requests wait for memory to free up) without changing results.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _stream():
    from rbsim.serve import poisson_stream

    reqs = poisson_stream(rate=40.0, n=10, seed=7, side_lo=48, side_hi=192, horizon_lo=60.0, horizon_hi=400.0)
    reqs[1].exner = True  # make sure a morphology request is in the mix
    reqs[1].scheme = "local_inertial"
    reqs[1].morph_interval = 50.0
    return reqs


@pytest.mark.parametrize("room", ["ample", "tight"])
def test_results_are_the_same_alone_and_in_the_mix(room):
    from rbsim.serve import Server, request_bytes, solve_alone

    reqs = _stream()
    # tight: room for the largest request and a little more, so later arrivals queue
    budget = 150e9 if room == "ample" else 1.1 * max(request_bytes(r) for r in reqs)
    srv = Server(hbm_budget=budget, graph_steps=4, keep_depth=True)
    results = srv.run(reqs)
    assert [r.rid for r in results] == [r.rid for r in reqs]
    assert srv.stats["solves"] == len(reqs) and srv.stats["p99_s"] >= srv.stats["p50_s"] > 0.0
    if budget < 1e9:
        assert srv.stats["ensemble_rebuilds"] >= 3
    for req, res in zip(reqs, results, strict=True):
        assert abs(res.t - req.horizon) < 1e-6
        alone = solve_alone(req, graph_steps=4)
        assert alone.steps == res.steps, req.rid
        np.testing.assert_array_equal(res.depth, alone.depth, err_msg=f"request {req.rid}")


def test_frames_stream_and_are_the_same_alone_and_in_the_mix(tmp_path):
    """Each request with output_every > 0 gets its own result store: frame 0, one frame at
    every multiple of output_every and at the horizon, written while the batch steps on.
    Every frame (time, depth, u, v, bed change) is bit-identical to the request served alone."""
    from rbsim.io.zarr_writer import read_array, read_attrs
    from rbsim.serve import Server, output_times, solve_alone

    reqs = _stream()
    for k, r in enumerate(reqs):
        r.output_every = 0.0 if k == 2 else 50.0  # one request streams nothing
    srv = Server(hbm_budget=150e9, graph_steps=4, out_dir=str(tmp_path / "mix"))
    srv.run(reqs)
    want_frames = sum(1 + len(output_times(r)) for r in reqs if r.output_every > 0)
    assert srv.stats["frames"] == want_frames
    assert not (tmp_path / "mix" / "req_2.zarr").exists()
    for req in reqs:
        if req.output_every <= 0:
            continue
        solve_alone(req, graph_steps=4, out_dir=str(tmp_path / "alone"))
        mix, alone = tmp_path / "mix" / f"req_{req.rid}.zarr", tmp_path / "alone" / f"req_{req.rid}.zarr"
        n = 1 + len(output_times(req))
        assert read_attrs(mix)["n_frames"] == read_attrs(alone)["n_frames"] == n
        times = read_array(mix, "time")
        np.testing.assert_allclose(times, [0.0, *output_times(req)], rtol=0, atol=1e-6)
        names = ["time", "depth", "u", "v", "bed"] + (["bed_change"] if req.exner else [])
        for name in names:
            np.testing.assert_array_equal(read_array(mix, name), read_array(alone, name),
                                          err_msg=f"request {req.rid}: {name}")  # fmt: skip
        assert np.isfinite(read_array(mix, "depth")).all()


def test_the_reference_shaped_loop_gives_the_servers_frames(tmp_path):
    """solve_per_step (compute_dt + step per tick through the scheme API, the shape of the
    reference's run loop) and the server's device clock take the same steps: every frame
    of an LI request with Exner and of an HLLC request is bit-identical."""
    from rbsim.io.zarr_writer import read_array
    from rbsim.serve import solve_alone, solve_per_step

    reqs = _stream()
    picks = [reqs[1]] + [r for r in reqs if r.scheme == "hllc_fv"][:1]
    assert picks[0].exner and len(picks) == 2
    for req in picks:
        req.output_every = 60.0
        res = solve_alone(req, graph_steps=4, out_dir=str(tmp_path / "server"))
        steps = solve_per_step(req, out_dir=str(tmp_path / "loop"))
        assert steps == res.steps
        a, b = tmp_path / "server" / f"req_{req.rid}.zarr", tmp_path / "loop" / f"req_{req.rid}.zarr"
        for name in ["time", "depth", "u", "v", "bed"] + (["bed_change"] if req.exner else []):
            np.testing.assert_array_equal(read_array(b, name), read_array(a, name), err_msg=f"{req.rid}: {name}")
