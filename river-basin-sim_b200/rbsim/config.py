"""Scenario configuration for the solver path (the subset of solver/io/config.py it reads).

Reads the same TOML tables and keys as the reference (``[meta] [grid] [run]
[rainfall] [parameters] [sediment] [[inflow]] [boundaries]``, HANDOFF.md's schema);
terrain comes from ``[grid] dem`` (a raw little-endian float32 ``.r32`` with
``shape = [ny, nx]``) or is handed to ``run_simulation`` as an array, since tile
mosaics, coarsening, datums, sub-grid channels and structures are outside this
build's path. Unsupported tables raise ``ConfigError`` rather than being ignored.
"""

from __future__ import annotations

import tomllib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .processes.inflow import Inflow
from .schemes import KNOWN_SCHEMES

EDGES = ("north", "south", "east", "west")
_UNSUPPORTED = ("channels", "structures")


class ConfigError(ValueError):
    """A scenario config is malformed or asks for something outside the solver path."""


@dataclass
class Scenario:
    name: str = "scenario"
    scheme: str = "local_inertial"
    dx: float | None = None
    end_time: float = 3600.0
    output_every: float = 600.0
    alpha: float = 0.7
    dt_max: float = 30.0
    initial_depth: float = 0.0
    rain_type: str = "uniform"
    rain_mm_hr: float = 0.0
    rain_duration: float = 0.0
    rain_field: np.ndarray | None = None  # mm/hr
    manning: float | np.ndarray = 0.035
    infiltration_mm_hr: float | np.ndarray = 0.0
    boundaries: dict = field(default_factory=lambda: {e: "closed" for e in EDGES})
    stage_curves: dict = field(default_factory=dict)
    inflows: list = field(default_factory=list)
    sediment_d50: float | np.ndarray | None = None
    sediment_porosity: float = 0.4
    sediment_interval_s: float = 900.0
    alluvium_thickness: float | np.ndarray | None = None
    bed: np.ndarray | None = None

    @property
    def rain_m_s(self) -> float:
        return float(self.rain_mm_hr) / 1000.0 / 3600.0

    @property
    def has_sediment(self) -> bool:
        return self.sediment_d50 is not None

    @property
    def stage_events(self) -> list[float]:
        return sorted({t for c in self.stage_curves.values() for t, _ in c})


def _field(value, base: Path, shape, name):
    if isinstance(value, (int, float)):
        return float(value)
    if isinstance(value, str):
        if shape is None:
            raise ConfigError(f"{name}: a field file needs [grid] shape")
        arr = np.fromfile(base / value, dtype="<f4")
        if arr.size != shape[0] * shape[1]:
            raise ConfigError(f"{name}: {value} has {arr.size} values, grid is {shape}")
        return arr.reshape(shape)
    raise ConfigError(f"{name}: expected a number or a .r32 path, got {value!r}")


def load_config(path) -> Scenario:
    path = Path(path)
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    base = path.parent
    for t in _UNSUPPORTED:
        if t in doc:
            raise ConfigError(f"[{t}] is outside this build's solver path")
    meta, grid, run = doc.get("meta", {}), doc.get("grid", {}), doc.get("run", {})
    sc = Scenario(name=meta.get("name", path.stem), scheme=meta.get("scheme", "local_inertial"))
    if sc.scheme not in KNOWN_SCHEMES:
        raise ConfigError(f"unknown scheme {sc.scheme!r}; known: {list(KNOWN_SCHEMES)}")
    shape = tuple(grid["shape"]) if "shape" in grid else None
    sc.dx = float(grid["dx"]) if "dx" in grid else None
    if "dem" in grid:
        sc.bed = _field(grid["dem"], base, shape, "[grid] dem")
    sc.end_time = float(run.get("end_time", sc.end_time))
    sc.output_every = float(run.get("output_every", sc.output_every))
    sc.alpha = float(run.get("cfl", 0.7 if sc.scheme == "local_inertial" else 0.45))
    sc.dt_max = float(run.get("dt_max", sc.dt_max))
    sc.initial_depth = float(run.get("initial_depth", 0.0))
    rain = doc.get("rainfall", {})
    sc.rain_type = rain.get("type", "uniform")
    if sc.rain_type not in ("uniform", "field"):
        raise ConfigError(f"rainfall type {sc.rain_type!r} is not supported (uniform | field)")
    sc.rain_duration = float(rain.get("duration_s", 0.0))
    if sc.rain_type == "uniform":
        sc.rain_mm_hr = float(rain.get("rate_mm_hr", 0.0))
    else:
        sc.rain_field = _field(rain["field"], base, shape, "[rainfall] field")
    par = doc.get("parameters", {})
    sc.manning = _field(par.get("manning_n", 0.035), base, shape, "manning_n")
    sc.infiltration_mm_hr = _field(par.get("infiltration", 0.0), base, shape, "infiltration")
    bc = doc.get("boundaries", {})
    default = bc.get("default", "closed")
    for e in EDGES:
        v = bc.get(e, default)
        if isinstance(v, dict):
            if v.get("type") != "fixed_stage":
                raise ConfigError(f"[boundaries] {e}: a table must be type = 'fixed_stage'")
            if sc.scheme != "hllc_fv":
                raise ConfigError("fixed_stage boundaries need scheme = 'hllc_fv'")
            curve = v.get("stage", [[0.0, v["level"]]] if "level" in v else None)
            if not curve:
                raise ConfigError(f"[boundaries] {e}: fixed_stage needs level or stage")
            sc.stage_curves[e] = [(float(t), float(s)) for t, s in curve]
            sc.boundaries[e] = "fixed_stage"
        elif v in ("closed", "open"):
            sc.boundaries[e] = v
        else:
            raise ConfigError(f"[boundaries] {e}: unknown kind {v!r}")
    for entry in doc.get("inflow", []):
        sc.inflows.append(Inflow(cell=tuple(entry["cell"]), hydrograph=[tuple(map(float, p))
                                                                         for p in entry["hydrograph"]]))  # fmt: skip
    sed = doc.get("sediment")
    if sed is not None:
        if sc.scheme != "local_inertial":
            raise ConfigError("[sediment] is local-inertial-only (with scheme = 'hllc_fv' it is refused)")
        if sed.get("law", "mpm") != "mpm":
            raise ConfigError("only the Meyer-Peter-Mueller law ('mpm') is implemented")
        sc.sediment_d50 = _field(sed["d50"], base, shape, "[sediment] d50")
        sc.sediment_porosity = float(sed.get("porosity", 0.4))
        sc.sediment_interval_s = float(sed.get("interval_s", 900.0))
        if "alluvium_thickness" in sed:
            sc.alluvium_thickness = _field(sed["alluvium_thickness"], base, shape, "alluvium_thickness")
    return sc
