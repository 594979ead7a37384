"""Water and bed-material balance gauges (the ledgers of solver/core/massbalance.py:36-306).

Each gauge compares what entered and left the domain with what the domain now
holds and reports a relative residual at every accounting point; a residual
above the gate is a defect in the solver, not a warning.

* **What the domain holds comes from the device, in float64.** Stored water is a
  fixed-order float64 reduction of the depth in librbsim (the same bits on every
  rerun); the banked sinks (infiltration, open and fixed_stage edges) are the
  per-tile float64 totals the step kernels keep. Bed material is three float64
  reductions of the morphology fields taken in one device round trip.
* **What the host adds is summed exactly.** A host-side source volume extends an
  expansion of non-overlapping float64 terms (Shewchuk's grow-expansion, "Adaptive
  Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates", 1997),
  so no add loses a bit and the reported total is the correctly rounded sum.
  Sources the device clock integrates arrive as per-span deltas of its own
  compensated float64 totals.
* **The scale of the residual is causal.** Water divides by the largest of the
  cumulative source volume, the stored volume and the largest stored volume seen
  so far, so a domain that drains to empty keeps the scale it had. Bed material
  divides by the banked volume or the largest gross volume the bed has moved so
  far: the net bed change of a domain closed to bedload is zero by construction,
  so only the gross movement gives the residual a meaning.

The gates, the residual definitions and the ``.zattrs`` keys are those of the
reference, so its readers and gate tests apply unchanged.
"""

from __future__ import annotations

import math
from typing import NamedTuple

import torch

from .state import State

MASS_GATE = 1.0e-6
SEDIMENT_GATE = 1.0e-11
_TINY = 1e-12  # the scale below which a residual is not divided by anything smaller


class ExactSum:
    """A float64 running sum with no rounding error: the exact total is held as
    non-overlapping float64 terms, ``value`` rounds it once."""

    __slots__ = ("_terms",)

    def __init__(self) -> None:
        self._terms: list[float] = []

    def add(self, x: float) -> None:
        x = float(x)
        kept = []
        for t in self._terms:
            big, small = (x, t) if abs(x) >= abs(t) else (t, x)
            s = big + small
            err = small - (s - big)  # exact: |big| >= |small|
            if err != 0.0:
                kept.append(err)
            x = s
        kept.append(x)
        self._terms = kept

    @property
    def value(self) -> float:
        return math.fsum(self._terms)


class MassRecord(NamedTuple):
    time: float
    volume: float
    inflow_cum: float
    outflow_cum: float
    residual: float
    rel_error: float


class SedimentRecord(NamedTuple):
    time: float
    bed_volume: float  # net solid volume gained by the bed since t = 0 (m^3, signed)
    banked_volume: float  # solid volume the per-cell bounds refused to apply
    gross_volume: float  # solid volume moved, sum |dz|: the scale of the residual
    residual: float
    rel_error: float


class _Gauge:
    """Series bookkeeping shared by both ledgers: ``tag`` names the ``.zattrs`` keys."""

    tag = ""
    gate = 0.0

    def __init__(self) -> None:
        self.series: list = []
        self._peak = 0.0

    def _close(self, rec_type, time: float, *terms: float, residual: float, scale: float):
        rec = rec_type(float(time), *terms, residual, abs(residual) / max(scale, _TINY))
        self.series.append(rec)
        return rec

    @property
    def max_rel_error(self) -> float:
        return max((r.rel_error for r in self.series), default=0.0)

    def as_attrs(self) -> dict:
        return {
            f"{self.tag}_gate": self.gate,
            f"{self.tag}_max_rel_error": self.max_rel_error,
            f"{self.tag}_balance_series": [r._asdict() for r in self.series],
        }


class MassLedger(_Gauge):
    """Water balance of one run: ``residual = inflow - outflow - (V - V0)``.

    Build it with ``from_state`` (which takes the t = 0 baseline), report sources
    with ``add_inflow`` / ``add_rain_step`` and host-side sinks with ``add_outflow``
    as they act, and call ``record`` at each output time.
    """

    tag = "mass"
    gate = MASS_GATE

    def __init__(self, cell_area: float, v0: float):
        super().__init__()
        self.cell_area = float(cell_area)
        self.v0 = float(v0)
        self._sources = ExactSum()
        self._sinks = ExactSum()

    @classmethod
    def from_state(cls, state: State) -> MassLedger:
        area = state.grid.cell_area
        ledger = cls(area, state.volume_sum() * area)
        ledger.record(state, 0.0)
        return ledger

    def add_inflow(self, volume: float) -> None:
        self._sources.add(volume)

    def add_outflow(self, volume: float) -> None:
        self._sinks.add(volume)

    def add_rain_step(self, rain_m_s: float, dt: float, n_cells: int) -> None:
        """Areal rain at ``rain_m_s`` over ``n_cells`` cells for ``dt`` seconds."""
        self.add_inflow(rain_m_s * dt * self.cell_area * n_cells)

    def record(self, state: State, time: float) -> MassRecord:
        stored = state.volume_sum() * self.cell_area
        came_in = self._sources.value
        went_out = self._sinks.value + state.loss_volume(self.cell_area)
        residual = came_in - went_out - (stored - self.v0)
        self._peak = max(self._peak, stored)
        scale = max(abs(came_in), abs(stored), self._peak)
        return self._close(MassRecord, time, stored, came_in, went_out, residual=residual, scale=scale)


class SedimentLedger(_Gauge):
    """Solid-volume balance of a morphology run: ``residual = -(bed + banked)``.

    The transport kernels never move bedload across the domain edge, so whatever
    the bed gained in one cell it lost in another, and a cell whose bounds refused
    a change banked it instead. The balance is over the float64 cumulative change
    ``dz_cum``, not over the float32 bed rendered from it.
    """

    tag = "sediment"
    gate = SEDIMENT_GATE

    def __init__(self, cell_area: float, solid_fraction: float):
        super().__init__()
        self.cell_area = float(cell_area)
        self.solid_fraction = float(solid_fraction)

    @classmethod
    def from_state(cls, state: State) -> SedimentLedger:
        sed = state.sediment
        if sed is None:
            raise ValueError("SedimentLedger needs a state armed with arm_sediment(): an unarmed run has a "
                             "static bed and nothing to balance")  # fmt: skip
        ledger = cls(state.grid.cell_area, 1.0 - sed.porosity)
        ledger.record(state, 0.0)
        return ledger

    def record(self, state: State, time: float) -> SedimentRecord:
        sed = state.sediment
        sums = torch.stack((sed.dz_cum.sum(), sed.dz_unapplied.sum(), sed.dz_cum.abs().sum()))
        solid = self.cell_area * self.solid_fraction  # m^3 of solid per metre of bed change in one cell
        net, banked, gross = (v * solid for v in sums.double().tolist())
        self._peak = max(self._peak, gross)
        return self._close(SedimentRecord, time, net, banked, gross, residual=-(net + banked),
                           scale=max(abs(banked), self._peak))  # fmt: skip
