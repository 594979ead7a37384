"""Local-inertial scheme (Bates et al. 2010) on the B200 -- solver/core/local_inertial.py.

Same two calls as the reference module (local_inertial.py:515, :547), same
argument meaning; the work is one fused kernel launch per step in librbsim.so.
"""

from __future__ import annotations

import ctypes

from .. import _lib
from ..state import State


def compute_dt(state: State, alpha: float = 0.7, dt_max: float = 30.0) -> float:
    """``dt = alpha dx / sqrt(g h_max)``, ``dt_max`` when ``h_max <= H_DRY`` (:515-544).

    With sub-grid channels armed, ``h_max`` is the deepest water column
    (channels.column_depth), which is what the wave speed sees.

    Synchronising: the max-depth reduction runs on the device and its one float
    is read back, as the reference reads ``h_max`` back every step.
    """
    out = ctypes.c_double(0.0)
    _lib.check(_lib.lib().rb_li_compute_dt(ctypes.byref(state.li_fields()), state.cur, float(alpha),
                                           float(dt_max), state.workspace.data_ptr(), state.stream,
                                           ctypes.byref(out)))  # fmt: skip
    return float(out.value)


def step(state: State, dt: float, rain: float = 0.0, limit: bool = True, rain_scale: float = 1.0,
         t: float = 0.0) -> None:  # noqa: ARG001 -- scheme-interface parity, as in the reference
    """Advance one step of ``dt`` seconds (:547-727), fused into a single launch.

    ``rain`` is the uniform rate (m/s), ``rain_scale`` gates ``state.rain`` (the
    field), ``limit`` the donor limiter. Optional physics (compensation, rain
    field, infiltration, open edges, morphology, sub-grid channels) runs when
    armed on the state.
    """
    args = _lib.StepArgs(float(dt), float(rain), float(rain_scale), 1 if limit else 0, 0)
    _lib.check(_lib.lib().rb_li_step(ctypes.byref(state.li_fields()), state.cur, ctypes.byref(args),
                                     state.workspace.data_ptr(), state.stream))  # fmt: skip
    state.flip()
