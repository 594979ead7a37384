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


def _rel_l2(a, b) -> float:
    d = np.linalg.norm((a.astype(np.float64) - b.astype(np.float64)).ravel())
    n = np.linalg.norm(b.astype(np.float64).ravel())
    return float(d / n) if n > 0.0 else float(d)


def errors(got32: dict, ref64: dict) -> dict:
    """Differences of a run's final state from a reference run's. Besides the largest
    differences, the relative L2 norms and the share of cells whose depth differs by
    more than 1e-5 of the largest depth (+ 1 um): two arithmetics can take different
    sides of a wet / dry threshold (H_DRY = 1 mm) in a few cells, which moves those
    cells' depth by up to a few tenths of a millimetre while the rest agree to
    round-off."""
    h32, h64 = got32["h"].astype(np.float64), ref64["h"].astype(np.float64)
    q = ("hu", "hv") if "hu" in ref64 else ("qx", "qy")
    vol64 = float(h64.sum())
    h_max = float(np.max(np.abs(h64)))
    q_scale = max([float(np.max(np.abs(ref64[k]))) for k in q] + [h_max * np.sqrt(9.81 * h_max)])
    dq = max(float(np.max(np.abs(got32[k].astype(np.float64) - ref64[k]))) for k in q)
    dh = np.abs(h32 - h64)
    return {
        "max_abs_depth_m": float(np.max(dh)),
        "max_rel_depth": _rel(h32, h64),
        "rel_l2_depth": _rel_l2(h32, h64),
        "share_of_cells_off": float(np.mean(dh > 1e-5 * h_max + 1e-6)),
        "max_abs_discharge_m2_s": dq,
        "max_rel_discharge": dq / q_scale if q_scale > 0.0 else 0.0,
        # root-mean-square over the discharge scale (still water has no L2 norm to divide by)
        "rms_rel_discharge": max(float(np.sqrt(np.mean((got32[k].astype(np.float64) - ref64[k]) ** 2))) for k in q)
        / q_scale if q_scale > 0.0 else 0.0,
        "rel_volume": abs(float(h32.sum()) - vol64) / vol64 if vol64 > 0.0 else 0.0,
    }


def check(err: dict, *, max_depth_m: float = 1e-4, rel: float = 1e-5) -> None:
    """The bar a float32 result is held to against a reference run of the same case:
    depth within ``max_depth_m`` everywhere; ``rel`` relative in the L2 norm for depth
    and in root-mean-square over the discharge scale for discharge; at most 0.1 % of
    cells off by more than 1e-5 of the largest depth; stored volume within 1e-6."""
    assert err["max_abs_depth_m"] <= max_depth_m, err
    assert err["rel_l2_depth"] <= rel, err
    assert err["rms_rel_discharge"] <= rel, err
    assert err["share_of_cells_off"] <= 1e-3, err
    assert err["rel_volume"] <= 1e-6, err


def error_vs_f64(case, got32) -> dict:
    """``errors`` of a float32 run's outputs (with its ``dts``) against the float64 run."""
    return errors(got32, reference_f64(case, got32["dts"]))
