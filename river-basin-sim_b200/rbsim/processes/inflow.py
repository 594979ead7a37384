"""Inflow hydrographs as point sources (solver/processes/inflow.py, config.py:100-122).

The discharge is sampled at the step midpoint on the host in float64, converted to
a float32 depth per entry, uploaded, and Kahan-added on the device by one launch
(``rb_inject_points``). The returned volume is the float32 *request* times the
cell area -- the ledger's independent witness, exactly as in the reference.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib
from ..grid import Grid


@dataclass
class Inflow:
    """``cell`` (row, col) receives a piecewise-linear ``hydrograph`` [(t_s, Q_m3_s)]."""

    cell: tuple[int, int]
    hydrograph: list[tuple[float, float]]

    @property
    def breakpoints(self) -> list[float]:
        return [t for t, _ in self.hydrograph]

    def discharge_at(self, t: float) -> float:
        """Linear between knots, zero outside the curve."""
        hg = self.hydrograph
        if not hg or t < hg[0][0] or t > hg[-1][0]:
            return 0.0
        for (t0, q0), (t1, q1) in zip(hg, hg[1:], strict=False):
            if t0 <= t <= t1:
                if t1 == t0:
                    return q1
                return q0 + (q1 - q0) * (t - t0) / (t1 - t0)
        return hg[-1][1]


class InflowInjector:
    """Applies a set of hydrographs each step; duplicate or outside cells are refused."""

    def __init__(self, inflows, grid: Grid, device="cuda", compensated: bool = True):
        self.inflows = list(inflows)
        self.grid = grid
        self.device = torch.device(device)
        self.cell_area = grid.cell_area
        self.compensated = compensated
        ny, nx = grid.shape
        rows, cols, seen = [], [], set()
        for inf in self.inflows:
            i, j = inf.cell
            if not (0 <= i < ny and 0 <= j < nx):
                raise ValueError(f"inflow cell {inf.cell} is outside the {ny}x{nx} grid")
            if tuple(inf.cell) in seen:
                raise ValueError(
                    f"duplicate inflow cell {inf.cell}; merge their hydrographs into one [[inflow]] entry "
                    "(concurrent same-cell sources would race)"
                )
            seen.add(tuple(inf.cell))
            rows.append(i)
            cols.append(j)
        k = len(self.inflows)
        self._rows = torch.tensor(rows, dtype=torch.int32, device=self.device)
        self._cols = torch.tensor(cols, dtype=torch.int32, device=self.device)
        self._add = torch.zeros(k, dtype=torch.float32, device=self.device)
        self._add_host = torch.zeros(k, dtype=torch.float32).pin_memory() if k else None
        self._comp = torch.zeros(k, dtype=torch.float32, device=self.device) if compensated else None

    def compensation_numpy(self):
        return None if self._comp is None else self._comp.cpu().numpy()

    def breakpoints(self) -> list[float]:
        return sorted({t for inf in self.inflows for t in inf.breakpoints})

    def apply(self, state, t: float, dt: float) -> float:
        """Inject the midpoint discharge over [t, t+dt]; return the requested volume (m^3)."""
        if not self.inflows:
            return 0.0
        t_mid = t + 0.5 * dt
        vols = np.array([inf.discharge_at(t_mid) * dt for inf in self.inflows], dtype=np.float64)
        add_depth = (vols / self.cell_area).astype(np.float32)
        self._add_host.numpy()[:] = add_depth
        self._add.copy_(self._add_host, non_blocking=True)
        _lib.check(_lib.lib().rb_inject_points(
            state.h.data_ptr(), state.grid.ny, state.grid.nx, len(self.inflows), self._rows.data_ptr(),
            self._cols.data_ptr(), self._add.data_ptr(), None if self._comp is None else self._comp.data_ptr(),
            state.stream,
        ))  # fmt: skip
        return float(add_depth.astype(np.float64).sum()) * self.cell_area
