"""Randomized properties of the oracle (the checker the CUDA path is held to bit for bit).

On random closed basins (random bed, depth with dry cells, Manning), both schemes
keep depths finite and non-negative through wetting and drying, and conserve the
stored volume to the mass gate. Non-negative means what the reference's gates mean:
HLLC's positivity net makes depths exactly >= 0, while the local-inertial donor
limiter is exact in mass but rounds in float32, so a depth may sit a few ulp below
zero (solver/core/test_local_inertial.py:81 allows -1e-6 m). The oracle's OpenMP loops write disjoint cells, so its
results do not depend on the thread count, which is checked in a child process with one
thread.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
st_ = hypothesis.strategies

from backends import OracleBackend  # noqa: E402

MASS_GATE = 1.0e-6


@pytest.fixture(scope="module")
def be():
    import oracle

    b = OracleBackend()
    yield b
    oracle.set_pow_mode(0)


def _basin(seed, ny, nx):
    rng = np.random.default_rng(seed)
    bed = rng.uniform(0.0, 1.0, (ny, nx)).astype(np.float32)
    depth = np.maximum(rng.uniform(-0.3, 0.8, (ny, nx)), 0.0).astype(np.float32)  # some cells dry
    n = rng.uniform(0.0, 0.06, (ny, nx)).astype(np.float32)
    return bed, depth, n


@pytest.mark.parametrize("scheme, alpha, floor", [("local_inertial", 0.7, -1e-6), ("hllc_fv", 0.45, 0.0)])
def test_closed_random_basins_stay_non_negative_and_conserve(be, scheme, alpha, floor):
    @hypothesis.settings(max_examples=40, deadline=None)
    @hypothesis.given(st_.integers(0, 2**31 - 1), st_.integers(1, 12), st_.integers(1, 12), st_.integers(1, 25))
    def check(seed, ny, nx, steps):
        bed, depth, n = _basin(seed, ny, nx)
        s = be.make(bed, 5.0, depth=depth, manning=n)
        v0 = float(be.h(s).astype(np.float64).sum())
        for _ in range(steps):
            be.step(s, scheme, be.compute_dt(s, scheme, alpha, 5.0))
        h = be.h(s)
        assert np.isfinite(h).all() and h.min() >= floor
        if v0 > 0.0:
            assert abs(float(h.astype(np.float64).sum()) - v0) <= MASS_GATE * v0

    check()


def test_the_oracle_does_not_depend_on_its_thread_count():
    """A golden case stepped with one OpenMP thread equals the same case stepped here."""
    code = (
        "import json, sys\n"
        "sys.path[:0] = sys.argv[1:]\n"
        "import numpy as np, oracle\n"
        "from cases import CASES, run_case\n"
        "from test_oracle_golden import OracleAPI\n"
        "oracle.set_pow_mode(1)\n"
        "out = {}\n"
        "for name in ('li_sediment', 'hllc_open_comp_infil', 'li_channels'):\n"
        "    r = run_case(CASES[name](), OracleAPI())\n"
        "    out[name] = {k: np.asarray(v).tobytes().hex() for k, v in r.items()}\n"
        "print(json.dumps(out))\n"
    )
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    paths = [here, os.path.join(here, "golden"), os.path.join(root, "oracle"), os.path.join(root, "river-basin-sim_b200")]
    runs = []
    for threads in ("1", "4"):
        env = {**os.environ, "OMP_NUM_THREADS": threads}
        out = subprocess.run([sys.executable, "-c", code, *paths], capture_output=True, text=True, env=env,
                             timeout=600, cwd=root)  # fmt: skip
        assert out.returncode == 0, out.stderr[-2000:]
        runs.append(json.loads(out.stdout.strip().splitlines()[-1]))
    assert runs[0] == runs[1]
