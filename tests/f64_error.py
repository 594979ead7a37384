"""Error of a float32 result against the float64 build of the same kernels.

The oracle's double build (``librbo_f64.so``: the reference's kernels restated with
every field and every operation in float64) is run on the same inputs and driven
with the float32 run's own timestep sequence, so the two differ only by the
precision of the arithmetic. ``errors`` reports, for the final state: the largest
absolute depth difference in metres, the depth and discharge differences relative
to the largest float64 depth and to the discharge scale (the larger of the largest
float64 unit discharge and the gravity-wave discharge h_max * sqrt(g h_max), so that
still water, whose float64 discharge is zero, gets a meaningful denominator), and
the relative difference of the stored volume.
"""

from __future__ import annotations

import numpy as np

from cases import run_case
from test_oracle_golden import OracleAPI


class ReplayDt:
    """An OracleAPI that takes its timesteps from a recorded sequence."""

    def __init__(self, api, dts):
        self.api, self.dts, self.k = api, list(dts), 0

    def __getattr__(self, name):
        return getattr(self.api, name)

    def compute_dt(self, st, alpha, dt_max):
        dt = self.dts[self.k]
        self.k += 1
        return float(dt)


def reference_f64(case, dts) -> dict:
    return run_case(case, ReplayDt(OracleAPI(np.float64), dts))


def _rel(a, b) -> float:
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a.astype(np.float64) - b))) / scale if scale > 0.0 else 0.0


def errors(got32: dict, ref64: dict) -> dict:
    h32, h64 = got32["h"].astype(np.float64), ref64["h"]
    q = ("hu", "hv") if "hu" in ref64 else ("qx", "qy")
    vol64 = float(h64.sum())
    h_max = float(np.max(np.abs(h64)))
    q_scale = max([float(np.max(np.abs(ref64[k]))) for k in q] + [h_max * np.sqrt(9.81 * h_max)])
    dq = max(float(np.max(np.abs(got32[k].astype(np.float64) - ref64[k]))) for k in q)
    return {
        "max_abs_depth_m": float(np.max(np.abs(h32 - h64))),
        "max_rel_depth": _rel(h32, h64),
        "max_abs_discharge_m2_s": dq,
        "max_rel_discharge": dq / q_scale if q_scale > 0.0 else 0.0,
        "rel_volume": abs(float(h32.sum()) - vol64) / vol64 if vol64 > 0.0 else 0.0,
    }


def error_vs_f64(case, got32) -> dict:
    """``errors`` of a float32 run's outputs (with its ``dts``) against the float64 run."""
    return errors(got32, reference_f64(case, got32["dts"]))
