"""Morphology arming and host-side transport diagnostics (solver/core/sediment.py).

The fast-step bedload integral is fused into the local-inertial step kernel
(librbsim.so, li_step.cu) and the Exner activation is ``rb_exner_apply``; this
module holds what the reference keeps on the host: validation and arming
(:619-709) and the numpy diagnostics a run reports at each activation
(shields / capacity / celerity, :719-801; Courant summary, :811-1042, without the
sub-grid channel branches, which are outside this build's path).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .grid import GRAVITY, H_DRY
from .state import SedimentState, State

SUBMERGED_SG = 1.65
SHIELDS_CRITICAL = 0.047
MPM_COEFFICIENT = 8.0
MPM_EXPONENT = 1.5
MORPH_COURANT_GATE = 1.0
MORPH_REGIME_FLOOR = 35.0


class SedimentError(ValueError):
    """Sediment inputs are inconsistent with the grid or with themselves."""


def validate_grain_size(d50, grid) -> np.ndarray:
    ny, nx = grid.shape
    if np.isscalar(d50):
        arr = np.full((ny, nx), float(d50), dtype=np.float32)
    else:
        arr = np.ascontiguousarray(d50, dtype=np.float32).copy()
        if arr.shape != (ny, nx):
            raise SedimentError(f"d50 shape {arr.shape} != grid {(ny, nx)}")
    if not np.isfinite(arr).all():
        raise SedimentError("d50 field contains non-finite values")
    if (arr < 0).any():
        raise SedimentError("d50 must be >= 0 everywhere (0 = an inert cell)")
    return arr


def arm_sediment(state: State, d50, porosity: float) -> SedimentState:
    """Attach the accumulators; ``z0`` is the bed now (call after barriers). Not idempotent."""
    if state.sediment is not None:
        raise SedimentError(
            "state is already armed for morphology; re-arming would recapture z0 from "
            "a moved bed and discard the cumulative change that moved it"
        )
    if not 0.0 < porosity < 1.0:
        raise SedimentError(f"porosity must be in (0, 1), got {porosity}")
    g, dev = state.grid, state.device
    grain = validate_grain_size(d50, g)
    z32 = lambda shape: torch.zeros(shape, dtype=torch.float32, device=dev)  # noqa: E731
    sed = SedimentState(
        d50=torch.from_numpy(grain).to(dev), porosity=float(porosity), z0=state.z.clone(),
        dz_cum=torch.zeros(g.shape, dtype=torch.float64, device=dev),
        dz_unapplied=torch.zeros(g.shape, dtype=torch.float64, device=dev),
        qs_int_x=z32(g.qx_shape), qs_comp_x=z32(g.qx_shape), qs_int_y=z32(g.qy_shape), qs_comp_y=z32(g.qy_shape),
        d50_min=float(grain.min()), d50_max=float(grain.max()), zero_d50_cells=int((grain == 0).sum()),
    )  # fmt: skip
    state.sediment = sed
    state._invalidate()
    return sed


def _f64(*vals):
    return tuple(np.asarray(v, dtype=np.float64) for v in vals)


def shields_from_flow(q, h, n, d50, radius=None) -> np.ndarray:
    """Shields number from Manning shear, tau/rho = g n^2 q^2 / (h^2 R^(1/3))."""
    q, h, n, d50 = _f64(q, h, n, d50)
    r = h if radius is None else np.asarray(radius, dtype=np.float64)
    return GRAVITY * n**2 * q**2 / (h**2 * np.cbrt(r)) / (SUBMERGED_SG * GRAVITY * d50)


def capacity_from_flow(q, h, n, d50, radius=None) -> np.ndarray:
    """Meyer-Peter-Mueller capacity magnitude (m^2/s)."""
    theta = shields_from_flow(q, h, n, d50, radius)
    d50 = np.asarray(d50, dtype=np.float64)
    excess = np.maximum(theta - SHIELDS_CRITICAL, 0.0)
    return MPM_COEFFICIENT * excess**MPM_EXPONENT * np.sqrt(SUBMERGED_SG * GRAVITY * d50**3)


def bed_celerity(q, h, n, d50, porosity: float) -> np.ndarray:
    """Linearised Exner bed-wave speed for a wide section: c_b = (1/(1-p)) dq_s/dz.

    With theta ~ h^(-7/3) at fixed q, dq_s/dz = 1.5 * 8 * (7/3) (theta/h)
    sqrt(theta - theta_c) sqrt(s' g d50^3).
    """
    q, h, n, d50 = _f64(q, h, n, d50)
    theta = shields_from_flow(q, h, n, d50)
    excess = np.maximum(theta - SHIELDS_CRITICAL, 0.0)
    dqs_dz = (MPM_COEFFICIENT * MPM_EXPONENT * (7.0 / 3.0) * (theta / h) * np.sqrt(excess)
              * np.sqrt(SUBMERGED_SG * GRAVITY * d50**3))  # fmt: skip
    return dqs_dz / (1.0 - float(porosity))


def morphological_courant(celerity: float, interval_s: float, dx: float) -> float:
    return float(celerity) * float(interval_s) / float(dx)


def celerity_field(state: State) -> np.ndarray:
    """Per-cell bed-wave celerity from the cell-centred discharge the state carries now."""
    sed = state.sediment
    if sed is None:
        raise SedimentError("celerity_field requires arm_sediment(); nothing is armed")
    h = state.h.double().cpu().numpy()
    n = state.n.double().cpu().numpy()
    d50 = sed.d50.double().cpu().numpy()
    qx = state.qx.double().cpu().numpy()
    qy = state.qy.double().cpu().numpy()
    q = np.hypot(0.5 * (qx[:, :-1] + qx[:, 1:]), 0.5 * (qy[:-1, :] + qy[1:, :]))
    grain_ok = d50 > 0.0
    wet = (h >= H_DRY) & grain_ok & (q > 0.0)
    d50_safe = np.where(grain_ok, d50, 1.0)
    return np.where(wet, bed_celerity(np.where(wet, q, 0.0), np.where(wet, h, 1.0), n, d50_safe, sed.porosity), 0.0)


@dataclass(frozen=True)
class CourantSummary:
    celerity_m_s: float
    courant: float
    courant_moving: float
    courant_in_regime: float
    over_courant_share: float
    courant_cells: int
    live_cells: int

    def as_dict(self) -> dict:
        return dict(self.__dict__)


def courant_summary(state: State, dz: np.ndarray, interval_s: float) -> CourantSummary:
    """The morphological Courant number of one activation, reduced four ways."""
    g = state.grid
    cel = celerity_field(state)
    celerity = float(cel.max()) if cel.size else 0.0
    courant = morphological_courant(celerity, interval_s, g.dx)
    cour = cel * float(interval_s) / float(g.dx)
    absdz = np.abs(np.asarray(dz, dtype=np.float64))
    gross = float(absdz.sum())
    live = cel > 0.0
    moving = absdz > 0.0
    h = state.h.double().cpu().numpy()
    d50 = state.sediment.d50.double().cpu().numpy()
    regime = np.where(d50 > 0.0, h / np.where(d50 > 0.0, d50, 1.0), 0.0) >= MORPH_REGIME_FLOOR
    over = cour > MORPH_COURANT_GATE
    return CourantSummary(
        celerity_m_s=celerity, courant=courant,
        courant_moving=float(cour[moving].max()) if moving.any() else 0.0,
        courant_in_regime=float(cour[regime].max()) if regime.any() else 0.0,
        over_courant_share=float(absdz[over].sum()) / gross if gross > 0.0 else 0.0,
        courant_cells=int(over.sum()), live_cells=int(live.sum()),
    )  # fmt: skip
