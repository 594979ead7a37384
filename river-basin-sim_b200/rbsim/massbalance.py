"""Float64 mass and sediment ledgers (solver/core/massbalance.py:36-306).

The stored volume and the banked losses are float64 reductions on the device
(fixed reduction order, so a rerun reproduces them bit for bit); the source
accumulators are host float64 Kahan sums, as in the reference.
"""

from __future__ import annotations

from dataclasses import dataclass, field

from .state import State

MASS_GATE = 1.0e-6
SEDIMENT_GATE = 1.0e-11


@dataclass
class _Kahan:
    total: float = 0.0
    comp: float = 0.0

    def add(self, x: float) -> None:
        y = x - self.comp
        t = self.total + y
        self.comp = (t - self.total) - y
        self.total = t


@dataclass
class MassRecord:
    time: float
    volume: float
    inflow_cum: float
    outflow_cum: float
    residual: float
    rel_error: float


@dataclass
class MassLedger:
    cell_area: float
    v0: float
    _inflow: _Kahan = field(default_factory=_Kahan)
    _outflow: _Kahan = field(default_factory=_Kahan)
    series: list[MassRecord] = field(default_factory=list)
    _peak_v: float = 0.0

    @classmethod
    def from_state(cls, state: State) -> MassLedger:
        area = state.grid.cell_area
        ledger = cls(cell_area=area, v0=state.volume_sum() * area)
        ledger.record(state, 0.0)
        return ledger

    def add_inflow(self, volume: float) -> None:
        self._inflow.add(volume)

    def add_outflow(self, volume: float) -> None:
        self._outflow.add(volume)

    def add_rain_step(self, rain_m_s: float, dt: float, n_cells: int) -> None:
        self.add_inflow(rain_m_s * dt * self.cell_area * n_cells)

    def record(self, state: State, time: float) -> MassRecord:
        """residual = inflow - outflow - (V - V0), relative to a causal peak floor."""
        v = state.volume_sum() * self.cell_area
        inflow = self._inflow.total
        outflow = self._outflow.total + state.loss_volume(self.cell_area)
        residual = inflow - outflow - (v - self.v0)
        self._peak_v = max(self._peak_v, v)
        denom = max(abs(inflow), abs(v), self._peak_v, 1e-12)
        rec = MassRecord(time, v, inflow, outflow, residual, abs(residual) / denom)
        self.series.append(rec)
        return rec

    @property
    def max_rel_error(self) -> float:
        return max((r.rel_error for r in self.series), default=0.0)

    def as_attrs(self) -> dict:
        return {
            "mass_gate": MASS_GATE,
            "mass_max_rel_error": self.max_rel_error,
            "mass_balance_series": [dict(r.__dict__) for r in self.series],
        }


@dataclass
class SedimentRecord:
    time: float
    bed_volume: float
    banked_volume: float
    gross_volume: float
    residual: float
    rel_error: float


@dataclass
class SedimentLedger:
    """Solid-volume balance: the domain is closed to bedload, so bed + banked == 0."""

    cell_area: float
    solid_fraction: float
    series: list[SedimentRecord] = field(default_factory=list)
    _peak_gross: float = 0.0

    @classmethod
    def from_state(cls, state: State) -> SedimentLedger:
        sed = state.sediment
        if sed is None:
            raise ValueError("SedimentLedger needs a state armed with arm_sediment()")
        ledger = cls(cell_area=state.grid.cell_area, solid_fraction=1.0 - sed.porosity)
        ledger.record(state, 0.0)
        return ledger

    def record(self, state: State, time: float) -> SedimentRecord:
        sed = state.sediment
        solid = self.cell_area * self.solid_fraction
        bed = float(sed.dz_cum.sum().item()) * solid
        banked = float(sed.dz_unapplied.sum().item()) * solid
        gross = float(sed.dz_cum.abs().sum().item()) * solid
        residual = -(bed + banked)
        self._peak_gross = max(self._peak_gross, gross)
        denom = max(abs(banked), self._peak_gross, 1e-12)
        rec = SedimentRecord(float(time), bed, banked, gross, residual, abs(residual) / denom)
        self.series.append(rec)
        return rec

    @property
    def max_rel_error(self) -> float:
        return max((r.rel_error for r in self.series), default=0.0)

    def as_attrs(self) -> dict:
        return {
            "sediment_gate": SEDIMENT_GATE,
            "sediment_max_rel_error": self.max_rel_error,
            "sediment_balance_series": [dict(r.__dict__) for r in self.series],
        }
