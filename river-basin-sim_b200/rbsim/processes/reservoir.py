"""Reservoir operations on the slow clock (solver/processes/reservoir.py).

A dam is geometry plus a rule. ``apply_barriers`` raises the bed to the crest at
the structure's cells once, before stepping, so impoundment and overtopping are
ordinary shallow-water physics. ``ReservoirOperator`` is the release rule: at each
activation it reads the pool stage at the deepest pool cell, asks the rule for a
discharge, and moves ``Q * dt_slow`` from the pool box to the outlet box in one
operator-split transfer that is mass-exact:

* the withdrawal kernel (``rb_reservoir_withdraw``) takes ``h * scale`` from each
  pool cell and records the exact float64 depth each cell gave up; the host sums
  those (numpy, as the reference does) to learn what actually left;
* the request is capped by what the pool holds (``scale <= 1``);
* the delivery kernel (``rb_reservoir_deliver``) spreads the removed depth over the
  outlet box and banks the float32 rounding shortfall in the loss ledger.

Names, arguments, records and errors follow the reference: ``ReleaseRecord``,
``ReservoirOperator(structure, state)`` with ``as_slow_process``, ``pool_stage``,
``advance(t, dt_slow)``, ``series``; ``build_operators``; ``apply_barriers``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib
from ..config import Structure
from ..grid import H_DRY
from ..scheduler import SlowProcess


def apply_barriers(bed: np.ndarray, structures: list[Structure]) -> np.ndarray:
    """Raise the bed to each structure's crest at its cells; never lowers it (reservoir.py:62-85)."""
    if not structures:
        return bed
    out = np.array(bed, dtype=np.float32, copy=True)
    ny, nx = out.shape
    for s in structures:
        for i, j in s.cells:
            if not (0 <= i < ny and 0 <= j < nx):
                raise ValueError(f"structure '{s.name}': cell {(i, j)} is outside the {ny}x{nx} grid")
            out[i, j] = max(float(out[i, j]), float(s.crest_m))
    return out


@dataclass
class ReleaseRecord:
    """One slow-clock activation of a release rule (reservoir.py:128-146)."""

    time: float
    stage: float | None
    discharge_m3_s: float
    volume_m3: float

    def as_dict(self) -> dict:
        return {"time": self.time, "stage": self.stage, "discharge_m3_s": self.discharge_m3_s,
                "volume_m3": self.volume_m3}  # fmt: skip


class ReservoirOperator:
    """Applies one structure's release rule on the slow clock (reservoir.py:149-263)."""

    def __init__(self, structure: Structure, state):
        if structure.release_rule == "none":
            raise ValueError(f"structure '{structure.name}' has no release rule to operate")
        self.structure = structure
        self.state = state
        self.records: list[ReleaseRecord] = []
        ny, nx = state.grid.shape
        r0, c0, r1, c1 = structure.pool
        if not (0 <= r0 <= r1 < ny and 0 <= c0 <= c1 < nx):
            raise ValueError(f"structure '{structure.name}': pool {structure.pool} is outside the {ny}x{nx} grid")
        o0, p0, o1, p1 = structure.outlet
        if not (0 <= o0 <= o1 < ny and 0 <= p0 <= p1 < nx):
            raise ValueError(
                f"structure '{structure.name}': outlet {structure.outlet} is outside the {ny}x{nx} grid"
            )
        self._pool = (r0, c0, r1, c1)
        self._pool_shape = (r1 - r0 + 1, c1 - c0 + 1)
        self._outlet = (o0, p0, o1, p1)
        self._outlet_cells = (o1 - o0 + 1) * (p1 - p0 + 1)
        self._taken = torch.zeros(self._pool_shape, dtype=torch.float64, device=state.device)
        # the stage gauge: the lowest-bed cell of the pool box (first in row-major order on ties)
        pool_z = state.z[r0 : r1 + 1, c0 : c1 + 1].cpu().numpy()
        a, b = np.unravel_index(int(np.argmin(pool_z)), pool_z.shape)
        self._gauge = (r0 + int(a), c0 + int(b))
        state.arm_loss_accumulator()

    def as_slow_process(self) -> SlowProcess:
        return SlowProcess(name=f"reservoir:{self.structure.name}", interval=self.structure.interval_s,
                           advance=self.advance)  # fmt: skip

    def pool_stage(self) -> float | None:
        """``z + h`` at the gauge (the deepest pool cell), ``None`` when it is dry (:194-213)."""
        gi, gj = self._gauge
        h = float(self.state.h[gi, gj].item())
        if h <= H_DRY:
            return None
        return float(self.state.z[gi, gj].item()) + h

    def advance(self, t: float, dt_slow: float) -> ReleaseRecord:
        """Move one slow interval's release from the pool to the outlet (:215-231)."""
        stage = self.pool_stage()
        q = self.structure.discharge_at(stage)
        volume = 0.0
        if q > 0.0:
            volume = self._transfer(q * float(dt_slow))
        rec = ReleaseRecord(time=float(t), stage=stage, discharge_m3_s=q, volume_m3=volume)
        self.records.append(rec)
        return rec

    def _transfer(self, requested_m3: float) -> float:
        """Move up to ``requested_m3`` from the pool to the outlet; return what moved (:234-263)."""
        st = self.state
        area = st.grid.cell_area
        ny, nx = st.grid.shape
        r0, c0, r1, c1 = self._pool
        pool_h = st.h[r0 : r1 + 1, c0 : c1 + 1].cpu().numpy().astype(np.float64)
        stored = float(pool_h.sum()) * area
        if stored <= 0.0:
            return 0.0
        scale = min(1.0, requested_m3 / stored)
        L = _lib.lib()
        _lib.check(L.rb_reservoir_withdraw(st.h.data_ptr(), ny, nx, r0, c0, r1, c1, float(np.float32(scale)),
                                           self._taken.data_ptr(), st.stream))  # fmt: skip
        removed_m3 = float(self._taken.cpu().numpy().sum()) * area
        if removed_m3 <= 0.0:
            return 0.0
        o0, p0, o1, p1 = self._outlet
        _lib.check(L.rb_reservoir_deliver(st.h.data_ptr(), ny, nx, o0, p0, o1, p1,
                                          removed_m3 / area / self._outlet_cells, st.workspace.data_ptr(),
                                          st.stream))  # fmt: skip
        return removed_m3

    @property
    def series(self) -> list[dict]:
        return [r.as_dict() for r in self.records]


def build_operators(structures: list[Structure], state) -> list[ReservoirOperator]:
    """An operator for every structure that carries a release rule (reservoir.py:266-268)."""
    return [ReservoirOperator(s, state) for s in structures if s.release_rule != "none"]
