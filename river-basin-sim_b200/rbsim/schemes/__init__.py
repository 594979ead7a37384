"""Scheme dispatch -- the seam of solver/core/schemes.py:41-52.

``get_scheme(name)`` returns a module with ``compute_dt(state, alpha, dt_max)`` and
``step(state, dt, rain, rain_scale, t)``; the run loop never branches on scheme.
"""

from __future__ import annotations

from types import ModuleType

from . import hllc, local_inertial

KNOWN_SCHEMES = ("local_inertial", "hllc_fv")


def get_scheme(name: str) -> ModuleType:
    if name == "local_inertial":
        return local_inertial
    if name == "hllc_fv":
        return hllc
    raise ValueError(f"unknown scheme '{name}'; known schemes: {list(KNOWN_SCHEMES)}")
