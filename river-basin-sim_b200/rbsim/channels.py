"""Sub-grid channels: geometry, validation and the storage curve (solver/core/channels.py).

A cell may carry a channel narrower than the cell: width ``w`` (0 < w <= dx),
bank-full depth ``d`` below the floodplain bed, and its own Manning roughness. The
state variable stays the cell-mean depth ``h``; the channel enters through the
storage curve ``h -> eta`` and through a second (channel) component on every
face, which the local-inertial kernel carries next to the floodplain component
and recombines into the total ``qx`` / ``qy`` that continuity reads. Arming is
what switches ``librbsim``'s LI step onto its channel instantiation; an unarmed
state never touches any of it.

Public names, argument meaning and errors follow the reference module:
``ChannelError`` (a ``ValueError``), ``validate_geometry``, ``arm_channels`` (with
``manning=None`` defaulting to the floodplain roughness), ``ChannelState``
(``summary`` / ``as_attrs``), and the host references ``eta_from_h`` /
``h_from_eta`` (channels.py:140-179).
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass

import numpy as np
import torch

from .grid import Grid

# channels.py:50-52: a channel narrower than dx / 1000 is almost always a data
# artefact, and it collapses the timestep (the column is h * dx / w).
WIDTH_WARN_RATIO = 1000.0


class ChannelError(ValueError):
    """Sub-grid channel geometry is inconsistent with the grid or with itself."""


def eta_from_h(h, z, w, d, dx: float) -> np.ndarray:
    """Host-side storage curve in float64 (channels.py:140-157)."""
    h, z, w, d = (np.asarray(v, dtype=np.float64) for v in (h, z, w, d))
    has = (w > 0.0) & (d > 0.0)
    h_bf = np.where(has, w * d / dx, 0.0)
    in_channel = has & (h <= h_bf)
    return np.where(has, np.where(in_channel, z - d + h * dx / np.where(has, w, 1.0), z + (h - h_bf)), z + h)


def h_from_eta(eta, z, w, d, dx: float) -> np.ndarray:
    """Inverse storage curve: the cell-mean depth holding a surface (channels.py:160-179)."""
    eta, z, w, d = (np.asarray(v, dtype=np.float64) for v in (eta, z, w, d))
    has = (w > 0.0) & (d > 0.0)
    h_bf = np.where(has, w * d / dx, 0.0)
    below = has & (eta <= z)
    return np.clip(np.where(has, np.where(below, (eta - (z - d)) * w / dx, h_bf + (eta - z)), eta - z), 0.0, None)


def column_depth(h, w, d, dx: float) -> np.ndarray:
    """Host copy of the water column the timestep sees (channels.py:73-83), float64."""
    h, w, d = (np.asarray(v, dtype=np.float64) for v in (h, w, d))
    has = (w > 0.0) & (d > 0.0)
    h_bf = np.where(has, w * d / dx, 0.0)
    return np.where(has, np.where(h <= h_bf, h * dx / np.where(has, w, 1.0), d + (h - h_bf)), h)


@dataclass
class ChannelState:
    """Device channel geometry plus the split face discharges (channels.py:182-211).

    ``qx_ch`` / ``qy_ch`` are discharge per unit channel width, ``qx_fp`` /
    ``qy_fp`` per unit floodplain width; the attributes name the current buffer
    of each double-buffered pair (the step reads it and writes the other).
    """

    w: torch.Tensor
    d: torch.Tensor
    n: torch.Tensor
    width_max: float
    depth_max: float
    channel_cells: int
    _state: object = None
    _pairs: dict | None = None

    def _cur(self, key):
        return self._pairs[key].bufs[self._state.cur]

    qx_ch = property(lambda s: s._cur("qx_ch"))
    qx_fp = property(lambda s: s._cur("qx_fp"))
    qy_ch = property(lambda s: s._cur("qy_ch"))
    qy_fp = property(lambda s: s._cur("qy_fp"))

    def summary(self) -> str:
        return (f"{self.channel_cells} channel cells, width <= {self.width_max:.1f} m, "
                f"bank-full depth <= {self.depth_max:.2f} m")  # fmt: skip

    def as_attrs(self) -> dict:
        return {"channel_cells": self.channel_cells, "width_max_m": self.width_max, "depth_max_m": self.depth_max}


def validate_geometry(width, depth, manning, grid: Grid) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Check and normalise channel fields against the grid (channels.py:214-262).

    Refuses a channel wider than its cell, negative or non-finite geometry, a
    width without a depth (or the reverse) and a channel cell without roughness;
    normalises "no channel" to w = d = 0 in both fields; warns about a hairline
    channel that will collapse the timestep.
    """
    ny, nx = grid.shape
    for name, arr in (("width", width), ("depth", depth), ("manning", manning)):
        if np.shape(arr) != (ny, nx):
            raise ChannelError(f"channel {name} shape {np.shape(arr)} != grid {(ny, nx)}")
    w = np.ascontiguousarray(width, dtype=np.float32).copy()
    d = np.ascontiguousarray(depth, dtype=np.float32).copy()
    n = np.ascontiguousarray(manning, dtype=np.float32).copy()
    if not np.isfinite(w).all() or not np.isfinite(d).all():
        raise ChannelError("channel width/depth fields contain non-finite values")
    if (w < 0).any() or (d < 0).any():
        raise ChannelError("channel width and depth must be >= 0 everywhere")
    too_wide = w > grid.dx
    if too_wide.any():
        raise ChannelError(
            f"{int(too_wide.sum())} cells have a channel wider than the cell (max {float(w[too_wide].max()):.1f} m "
            f"> dx {grid.dx:.1f} m); a sub-grid channel must fit inside its cell -- resolve the river or coarsen less"
        )
    has = (w > 0) & (d > 0)
    half = (w > 0) != (d > 0)
    if half.any():
        raise ChannelError(
            f"{int(half.sum())} cells give a channel width without a bank-full depth (or the reverse); a channel "
            "needs both, and 'no channel' is width = depth = 0"
        )
    if has.any() and (n[has] <= 0).any():
        raise ChannelError("channel cells need manning > 0")
    w[~has] = 0.0
    d[~has] = 0.0
    if has.any():
        w_min = float(w[has].min())
        if w_min < grid.dx / WIDTH_WARN_RATIO:
            warnings.warn(
                f"narrowest sub-grid channel is {w_min:g} m in a {grid.dx:g} m cell "
                f"(1:{grid.dx / max(w_min, 1e-12):.0f}); the water column -- and so the timestep -- is set by "
                "dx/w, so this will run very slowly",
                stacklevel=2,
            )
    return w, d, n


def arm_channels(state, width, depth, manning=None) -> ChannelState:
    """Attach validated channel geometry and its face components to ``state``
    (channels.py:265-312). ``manning=None`` uses the floodplain roughness."""
    fp_n = state.n.cpu().numpy()
    w, d, n = validate_geometry(np.asarray(width, dtype=np.float32), np.asarray(depth, dtype=np.float32),
                                fp_n if manning is None else np.asarray(manning, dtype=np.float32),
                                state.grid)  # fmt: skip
    return state.arm_channel_fields(w, d, n)
