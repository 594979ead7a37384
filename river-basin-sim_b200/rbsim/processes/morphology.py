"""Exner on the slow clock (solver/processes/morphology.py:75-379).

``advance`` applies one interval's accumulated bedload to the float64 cumulative
bed change, rebuilds ``z = float32(z0 + dz_cum)`` and clears the transport
integral (keeping its Kahan residue) in one ``rb_exner_apply`` call, then
reports the activation record.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib
from ..scheduler import EPS_T, SlowProcess
from ..sediment import SedimentError, courant_summary
from ..state import State


def bed_change_bounds(shape, *, alluvium_thickness=None, frozen_cells=()):
    """Per-cell (dz_lo, dz_hi) on the cumulative change; unbounded by default."""
    ny, nx = shape
    lo = np.full((ny, nx), -np.inf, dtype=np.float32)
    hi = np.full((ny, nx), np.inf, dtype=np.float32)
    if alluvium_thickness is not None:
        thickness = np.asarray(alluvium_thickness, dtype=np.float32)
        if thickness.ndim and thickness.shape != (ny, nx):
            raise SedimentError(f"alluvium thickness shape {thickness.shape} != grid {(ny, nx)}")
        if (thickness < 0).any():
            raise SedimentError("alluvium thickness must be >= 0 m (0 = bedrock, not a hole)")
        lo = np.broadcast_to(-thickness, (ny, nx)).astype(np.float32).copy()
    for i, j in frozen_cells:
        if not (0 <= i < ny and 0 <= j < nx):
            raise SedimentError(f"frozen cell {(i, j)} is outside the {ny}x{nx} grid")
        lo[i, j] = 0.0
        hi[i, j] = 0.0
    return lo, hi


@dataclass
class BedChangeRecord:
    time: float
    interval_s: float
    applied_m3: float
    cumulative_m3: float
    banked_m3: float
    dz_min_m: float
    dz_max_m: float
    celerity_m_s: float
    courant: float
    courant_moving: float
    courant_in_regime: float
    over_courant_share: float
    courant_cells: int
    live_cells: int

    def as_dict(self) -> dict:
        return dict(self.__dict__)


class MorphologyProcess:
    def __init__(self, state: State, interval_s: float, *, dz_lo=None, dz_hi=None, name: str = "morphology"):
        sed = state.sediment
        if sed is None:
            raise SedimentError("morphology needs a state armed with arm_sediment()")
        if interval_s <= 0:
            raise SedimentError(f"morphology interval_s must be > 0, got {interval_s}")
        self.state, self.sediment, self.interval_s, self.name = state, sed, float(interval_s), name
        self.records: list[BedChangeRecord] = []
        shape = state.grid.shape
        if (dz_lo is None) != (dz_hi is None):
            raise SedimentError("give both dz_lo and dz_hi, or neither")
        if dz_lo is None:
            dz_lo, dz_hi = bed_change_bounds(shape)
        lo = np.ascontiguousarray(dz_lo, dtype=np.float32)
        hi = np.ascontiguousarray(dz_hi, dtype=np.float32)
        if lo.shape != shape or hi.shape != shape:
            raise SedimentError(f"bed-change bounds {lo.shape}/{hi.shape} != grid {shape}")
        if (lo > hi).any():
            raise SedimentError("bed-change bounds cross: dz_lo must be <= dz_hi everywhere")
        self.dz_lo = torch.from_numpy(lo).to(state.device)
        self.dz_hi = torch.from_numpy(hi).to(state.device)
        frozen = (lo == 0.0) & (hi == 0.0)
        self.frozen_cells = int(frozen.sum())
        self.floored_cells = int((np.isfinite(lo) & ~frozen).sum())
        self._peak = dict(courant=0.0, moving=0.0, regime=0.0, share=0.0, cells=0, live=0)

    def as_slow_process(self) -> SlowProcess:
        return SlowProcess(name=self.name, interval=self.interval_s, advance=self.advance)

    def advance(self, t: float, dt_slow: float) -> BedChangeRecord:
        if dt_slow > self.interval_s * (1.0 + 1e-6) + EPS_T:
            raise SedimentError(
                f"morphology was handed {dt_slow} s to apply but is configured for {self.interval_s} s: "
                "several intervals collapsed into one bed update coarsen the operator splitting, "
                "and no balance would show it"
            )
        st, sed, g = self.state, self.sediment, self.state.grid
        prev_dz = sed.dz_cum.clone()
        _lib.check(_lib.lib().rb_exner_apply(
            g.ny, g.nx, g.dx, sed.qs_int_x.data_ptr(), sed.qs_int_y.data_ptr(), self.dz_lo.data_ptr(),
            self.dz_hi.data_ptr(), ctypes.c_float(sed.inv_one_minus_p), sed.dz_cum.data_ptr(),
            sed.dz_unapplied.data_ptr(), sed.z0.data_ptr(), st.z.data_ptr(), st.stream,
        ))  # fmt: skip
        solid = g.cell_area * (1.0 - sed.porosity)
        dz = sed.dz_cum.cpu().numpy()
        before = float(prev_dz.sum().item())
        cumulative = float(dz.sum())
        cs = courant_summary(st, dz - prev_dz.cpu().numpy(), dt_slow)
        pk = self._peak
        pk["courant"] = max(pk["courant"], cs.courant)
        pk["moving"] = max(pk["moving"], cs.courant_moving)
        pk["regime"] = max(pk["regime"], cs.courant_in_regime)
        pk["share"] = max(pk["share"], cs.over_courant_share)
        pk["cells"] = max(pk["cells"], cs.courant_cells)
        pk["live"] = max(pk["live"], cs.live_cells)
        rec = BedChangeRecord(
            time=float(t), interval_s=float(dt_slow), applied_m3=(cumulative - before) * solid,
            cumulative_m3=cumulative * solid, banked_m3=float(sed.dz_unapplied.sum().item()) * solid,
            dz_min_m=float(dz.min()), dz_max_m=float(dz.max()), celerity_m_s=cs.celerity_m_s, courant=cs.courant,
            courant_moving=cs.courant_moving, courant_in_regime=cs.courant_in_regime,
            over_courant_share=cs.over_courant_share, courant_cells=cs.courant_cells, live_cells=cs.live_cells,
        )  # fmt: skip
        self.records.append(rec)
        return rec

    @property
    def peak_courant(self) -> float:
        return self._peak["courant"]

    @property
    def series(self) -> list[dict]:
        return [r.as_dict() for r in self.records]

    def summary(self) -> str:
        bounds = []
        if self.frozen_cells:
            bounds.append(f"{self.frozen_cells} frozen cells")
        if self.floored_cells:
            bounds.append(f"{self.floored_cells} cells on an alluvium floor")
        limits = f", {' + '.join(bounds)}" if bounds else ", unbounded"
        return f"{self.sediment.summary()}, every {self.interval_s:g} s{limits}"

    def as_attrs(self) -> dict:
        return {**self.sediment.as_attrs(), "interval_s": self.interval_s, "frozen_cells": self.frozen_cells,
                "floored_cells": self.floored_cells}  # fmt: skip
