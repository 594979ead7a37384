"""Well-balanced HLLC finite-volume scheme on the B200 -- solver/core/hllc.py.

Same calls as the reference module (``arm_hllc`` :123, ``compute_dt`` :972,
``step`` :1272); each SSP-RK2 step is two kernel launches in librbsim.so.
"""

from __future__ import annotations

import ctypes

from .. import _lib
from ..state import EDGES, State


def stage_at(curve, t: float) -> float:
    """Prescribed surface at ``t`` (boundaries.py:199-220): linear, held at the ends."""
    if not curve:
        raise ValueError("empty stage curve")
    if t <= curve[0][0]:
        return float(curve[0][1])
    if t >= curve[-1][0]:
        return float(curve[-1][1])
    for (t0, s0), (t1, s1) in zip(curve, curve[1:], strict=False):
        if t0 <= t <= t1:
            if t1 == t0:
                return float(s1)
            return float(s0 + (s1 - s0) * (t - t0) / (t1 - t0))
    return float(curve[-1][1])


def arm_hllc(state: State) -> None:
    """Allocate the cell momenta (at rest) and the stage workspace (idempotent)."""
    state.arm_hllc_fields()


def compute_dt(state: State, alpha: float = 0.45, dt_max: float = 30.0) -> float:
    """``dt = alpha dx / max(|u|,|v| + sqrt(g h))`` (:972-990). Synchronising."""
    arm_hllc(state)
    out = ctypes.c_double(0.0)
    _lib.check(_lib.lib().rb_hllc_compute_dt(ctypes.byref(state.hllc_fields()), state.cur, float(alpha),
                                             float(dt_max), state.workspace.data_ptr(), state.stream,
                                             ctypes.byref(out)))  # fmt: skip
    return float(out.value)


def step(state: State, dt: float, rain: float = 0.0, rain_scale: float = 1.0, t: float = 0.0) -> None:
    """One SSP-RK2 step with friction and sources (:1272-1373).

    A fixed_stage edge's surface is evaluated once, at ``t + dt/2``, on the host
    (:1308-1312) and held across both stages.
    """
    arm_hllc(state)
    stages = [0.0, 0.0, 0.0, 0.0]
    for k, e in enumerate(EDGES):
        if e in state.stage_curves:
            stages[k] = stage_at(state.stage_curves[e], t + 0.5 * float(dt))
    args = _lib.StepArgs(float(dt), float(rain), float(rain_scale), 0, 0, (ctypes.c_double * 4)(*stages))
    _lib.check(_lib.lib().rb_hllc_step(ctypes.byref(state.hllc_fields()), state.cur, ctypes.byref(args),
                                       state.workspace.data_ptr(), state.stream))  # fmt: skip
    state.flip()
