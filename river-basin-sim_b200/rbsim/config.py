"""Scenario configuration for the solver path (the subset of solver/io/config.py it reads).

Reads the same TOML tables and keys as the reference (``[meta] [grid] [run]
[rainfall] [parameters] [sediment] [channels] [[inflow]] [[structures]]
[boundaries]``, HANDOFF.md's schema); terrain comes from ``[grid] dem`` (a raw
little-endian float32 ``.r32`` with ``shape = [ny, nx]``) or is handed to
``run_simulation`` as an array, since tile mosaics, coarsening and datums are
outside this build's path.
"""

from __future__ import annotations

import tomllib
import warnings
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .processes.inflow import Inflow
from .schemes import KNOWN_SCHEMES

EDGES = ("north", "south", "east", "west")
_UNSUPPORTED: tuple[str, ...] = ()
_STRUCTURE_KINDS = {"dam", "levee"}
_RELEASE_RULES = {"none", "fixed", "target_stage"}
_DEFAULT_RELEASE_INTERVAL_S = 900.0
_SEDIMENT_KEYS = {"d50", "porosity", "law", "interval_s", "alluvium_thickness"}


class ConfigError(ValueError):
    """A scenario config is malformed or asks for something outside the solver path."""


@dataclass
class Structure:
    """A dam or levee with an optional release rule (solver/io/config.py:147-241).

    ``cells`` + ``crest_m`` raise the bed to the crest (processes.reservoir.apply_barriers);
    a ``dam`` may carry a release rule evaluated on the slow clock every ``interval_s``,
    moving water from the inclusive ``pool`` box to the inclusive ``outlet`` box.
    """

    name: str = "dam"
    kind: str = "dam"
    cells: list = field(default_factory=list)
    crest_m: float = 0.0
    release_rule: str = "none"
    release_m3_s: float = 0.0
    target_stage_m: float | None = None
    release_max_m3_s: float = 0.0
    pool: tuple | None = None
    outlet: tuple | None = None
    interval_s: float = _DEFAULT_RELEASE_INTERVAL_S

    def __post_init__(self) -> None:
        n = self.name
        if self.kind not in _STRUCTURE_KINDS:
            raise ValueError(f"structure '{n}': type must be one of {sorted(_STRUCTURE_KINDS)}")
        if not self.cells:
            raise ValueError(f"structure '{n}': needs at least one barrier cell")
        if self.release_rule not in _RELEASE_RULES:
            raise ValueError(f"structure '{n}': release_rule must be one of {sorted(_RELEASE_RULES)}")
        if self.kind == "levee" and self.release_rule != "none":
            raise ValueError(f"structure '{n}': a levee is barrier geometry only; use type='dam' for a release rule")
        if self.interval_s <= 0:
            raise ValueError(f"structure '{n}': interval_s must be > 0")
        if self.release_rule == "none":
            return
        if self.pool is None or self.outlet is None:
            raise ValueError(f"structure '{n}': release_rule='{self.release_rule}' needs both a 'pool' box and an "
                             "'outlet' cell (where the released water is delivered)")  # fmt: skip
        r0, c0, r1, c1 = self.pool
        if r1 < r0 or c1 < c0:
            raise ValueError(f"structure '{n}': pool must be [row0, col0, row1, col1]")
        o0, p0, o1, p1 = self.outlet
        if o1 < o0 or p1 < p0:
            raise ValueError(f"structure '{n}': outlet must be [row, col] or [row0, col0, row1, col1]")
        if not (o1 < r0 or o0 > r1 or p1 < c0 or p0 > c1):
            raise ValueError(f"structure '{n}': the outlet {self.outlet} overlaps the pool {self.pool}; the release "
                             "would just shuffle water within the reservoir")  # fmt: skip
        if self.release_rule == "fixed" and self.release_m3_s <= 0:
            raise ValueError(f"structure '{n}': release_rule='fixed' needs release_m3_s > 0")
        if self.release_rule == "target_stage":
            if self.target_stage_m is None:
                raise ValueError(f"structure '{n}': release_rule='target_stage' needs target_stage_m")
            if self.release_max_m3_s <= 0:
                raise ValueError(f"structure '{n}': release_rule='target_stage' needs release_max_m3_s > 0 (the cap "
                                 "the proportional rule scales toward)")  # fmt: skip
            if self.target_stage_m >= self.crest_m:
                raise ValueError(f"structure '{n}': target_stage_m ({self.target_stage_m}) must be below crest_m "
                                 f"({self.crest_m}) -- the rule ramps between the two")  # fmt: skip

    def discharge_at(self, stage: float | None) -> float:
        """Release the rule asks for at a pool stage (config.py:228-241): ``fixed`` is
        constant; ``target_stage`` ramps from 0 at the target to the cap at the crest."""
        if self.release_rule == "none" or stage is None:
            return 0.0
        if self.release_rule == "fixed":
            return float(self.release_m3_s)
        span = self.crest_m - float(self.target_stage_m)
        frac = (stage - float(self.target_stage_m)) / span
        return float(self.release_max_m3_s) * min(max(frac, 0.0), 1.0)


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
    channel_width: float | np.ndarray = 0.0  # m; a scenario has channels iff a width is given
    channel_depth: float | np.ndarray = 0.0  # bank-full depth below the floodplain bed, m
    channel_manning: float | np.ndarray | None = None  # None: the floodplain roughness
    structures: list = field(default_factory=list)
    bed: np.ndarray | None = None

    def __post_init__(self) -> None:
        self.validate()

    def validate(self) -> None:
        """Refuse run parameters no run can honour (config.py:357-498); ``load_config``
        calls it again once every table is read, so both construction paths are checked.

        Raises ValueError (``load_config`` re-raises it as ConfigError) and warns above
        the CFL number the local-inertial scheme is stable at.
        """
        for name, v in (("end_time", self.end_time), ("output_every", self.output_every), ("dt_max", self.dt_max),
                        ("cfl", self.alpha)):  # fmt: skip
            if not v > 0:
                raise ValueError(f"{name} must be > 0, got {v}")
        frames = self.end_time / self.output_every
        if abs(frames - round(frames)) > 1e-6:
            raise ValueError(f"end_time ({self.end_time}) must be a whole multiple of output_every "
                             f"({self.output_every}): frames land on its multiples, so the state at end_time "
                             "would never be written")  # fmt: skip
        for name, v in (("manning_n", self.manning), ("infiltration", self.infiltration_mm_hr),
                        ("rainfall rate", self.rain_mm_hr), ("rainfall duration", self.rain_duration)):  # fmt: skip
            if np.any(np.asarray(v) < 0):
                raise ValueError(f"{name} must be >= 0")
        unknown = sorted(f"{e}={v!r}" for e, v in self.boundaries.items() if v not in ("closed", "open", "fixed_stage"))
        if unknown:
            raise ValueError(f"unknown boundary type(s): {', '.join(unknown)}; use closed, open or fixed_stage")
        staged = [e for e, v in self.boundaries.items() if v == "fixed_stage"]
        if staged and self.scheme != "hllc_fv":
            raise ValueError(f"fixed_stage edges ({', '.join(staged)}) need scheme = 'hllc_fv': the local-inertial "
                             "scheme has no boundary face to impose a water level on")  # fmt: skip
        missing = [e for e in staged if not self.stage_curves.get(e)]
        if missing:
            raise ValueError(f"fixed_stage edge(s) {', '.join(missing)} have no stage curve")
        if self.alpha > 0.9:
            warnings.warn(f"cfl={self.alpha} is above the ~0.7 stability limit of the local-inertial scheme; the run "
                          "may go unstable", stacklevel=3)  # fmt: skip

    @property
    def rain_m_s(self) -> float:
        return float(self.rain_mm_hr) / 1000.0 / 3600.0

    @property
    def has_sediment(self) -> bool:
        return self.sediment_d50 is not None

    @property
    def has_channels(self) -> bool:
        return not np.isscalar(self.channel_width) or float(self.channel_width) > 0.0

    @property
    def stage_events(self) -> list[float]:
        return sorted({t for c in self.stage_curves.values() for t, _ in c})


def _field(value, base: Path, shape, name):
    if isinstance(value, (int, float)) and not isinstance(value, bool):  # TOML true is not a roughness
        return float(value)
    if isinstance(value, str):
        if shape is None:
            raise ConfigError(f"{name}: a field file needs [grid] shape")
        if not (base / value).is_file():
            raise ConfigError(f"{name}: field file {value} not found next to the config")
        arr = np.fromfile(base / value, dtype="<f4")
        if arr.size != shape[0] * shape[1]:
            raise ConfigError(f"{name}: {value} has {arr.size} values, grid is {shape}")
        return arr.reshape(shape)
    raise ConfigError(f"{name}: expected a number or a .r32 path, got {value!r}")


def _number(value, what: str) -> float:
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise ConfigError(f"{what} must be a number, got {value!r}")
    return float(value)


def _stage_edge(edge: str, table, scheme: str) -> list[tuple[float, float]]:
    """One ``[boundaries]`` table: ``{ type = "fixed_stage", level = L }`` or ``stage = [[t, L], ...]``
    (config.py:600-667). Returns the stage curve, knot times non-decreasing."""
    kind = table.get("type")
    if kind != "fixed_stage":
        raise ConfigError(f"[boundaries] {edge}: unknown boundary type {kind!r}; a table edge is "
                          "{ type = 'fixed_stage', level = ... } or { type = 'fixed_stage', stage = [[t, level], ...] }")
    if ("level" in table) == ("stage" in table):
        raise ConfigError(f"[boundaries] {edge}: a fixed_stage edge takes exactly one of 'level' or 'stage'")
    if scheme != "hllc_fv":
        raise ConfigError(f"[boundaries] {edge}: fixed_stage needs scheme = 'hllc_fv'")
    if "level" in table:
        return [(0.0, _number(table["level"], f"[boundaries] {edge} level"))]
    knots = table["stage"]
    if not isinstance(knots, list) or not knots:
        raise ConfigError(f"[boundaries] {edge}: stage must be a non-empty list of [time_s, level_m] pairs")
    curve = []
    for k in knots:
        if not (isinstance(k, list) and len(k) == 2):
            raise ConfigError(f"[boundaries] {edge}: each stage knot must be [time_s, level_m], got {k!r}")
        curve.append((_number(k[0], f"[boundaries] {edge} stage time"), _number(k[1], f"[boundaries] {edge} stage")))
    if any(b[0] < a[0] for a, b in zip(curve, curve[1:], strict=False)):
        raise ConfigError(f"[boundaries] {edge}: stage knot times must be non-decreasing")
    return curve


def load_config(path) -> Scenario:
    path = Path(path)
    try:
        with open(path, "rb") as f:
            doc = tomllib.load(f)
    except FileNotFoundError as e:  # both refusals are ConfigError, as config.py:791-797 raises them
        raise ConfigError(f"scenario config not found: {path}") from e
    except tomllib.TOMLDecodeError as e:
        raise ConfigError(f"{path} is not valid TOML: {e}") from e
    base = path.parent
    for t in _UNSUPPORTED:
        if t in doc:
            raise ConfigError(f"[{t}] is outside this build's solver path")
    meta, grid, run = doc.get("meta", {}), doc.get("grid", {}), doc.get("run", {})
    sc = Scenario(name=meta.get("name", path.stem), scheme=meta.get("scheme", "local_inertial"))
    if sc.scheme not in KNOWN_SCHEMES:
        raise ConfigError(f"unknown scheme {sc.scheme!r}; known schemes: {list(KNOWN_SCHEMES)}")
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
        sc.rain_mm_hr = _number(rain.get("rate_mm_hr", 0.0), "[rainfall] rate_mm_hr")
    elif "field" not in rain:
        raise ConfigError("[rainfall] type = 'field' requires a 'field' path (a .r32 grid of mm/hr)")
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
            sc.stage_curves[e] = _stage_edge(e, v, sc.scheme)
            sc.boundaries[e] = "fixed_stage"
        elif v in ("closed", "open"):
            sc.boundaries[e] = v
        elif v == "fixed_stage":
            raise ConfigError(f"[boundaries] {e}: a fixed_stage edge needs its level, so write it as a fixed_stage "
                              "table: { type = 'fixed_stage', level = ... }")  # fmt: skip
        else:
            raise ConfigError(f"[boundaries] {e}: must be 'closed', 'open' or a fixed_stage table, got {v!r}")
    for k, entry in enumerate(doc.get("inflow", [])):
        cell = entry.get("cell")
        if not (isinstance(cell, list) and len(cell) == 2):
            raise ConfigError(f"[[inflow]] #{k}: cell must be [row, col], got {cell!r}")
        try:
            hydrograph = [(float(t), float(q)) for t, q in entry["hydrograph"]]
        except (KeyError, TypeError, ValueError) as err:
            raise ConfigError(f"[[inflow]] #{k}: hydrograph must be a list of [time_s, discharge_m3_s]") from err
        sc.inflows.append(Inflow(cell=(int(cell[0]), int(cell[1])), hydrograph=hydrograph))
    sed = doc.get("sediment")
    if sed is not None:  # config.py:444-490, 905-940: the table's presence arms morphology
        for key in sed:
            if key not in _SEDIMENT_KEYS:
                warnings.warn(f"[sediment] unknown key '{key}' ignored", stacklevel=2)
        if sc.scheme != "local_inertial":
            raise ConfigError("[sediment] requires scheme='local_inertial': morphology is local-inertial-only "
                              f"(with scheme = '{sc.scheme}' it is refused)")  # fmt: skip
        if sed.get("law", "mpm") != "mpm":
            raise ConfigError(f"[sediment] law={sed['law']!r} is not a transport law this solver has; only 'mpm' "
                              "(Meyer-Peter-Mueller) is implemented")  # fmt: skip
        d50 = _field(sed["d50"], base, shape, "[sediment] d50") if "d50" in sed else 0.0
        if np.isscalar(d50) and not d50 > 0.0:
            raise ConfigError("[sediment] needs a grain size: set d50 (metres, or a .r32 field); the table itself "
                              "arms morphology, so no d50 means 'off'")  # fmt: skip
        sc.sediment_d50 = d50
        sc.sediment_porosity = _number(sed.get("porosity", 0.4), "[sediment] porosity")
        if not 0.0 < sc.sediment_porosity < 1.0:
            raise ConfigError(f"[sediment] porosity must be in (0, 1), got {sc.sediment_porosity}")
        sc.sediment_interval_s = _number(sed.get("interval_s", 900.0), "[sediment] interval_s")
        if not sc.sediment_interval_s > 0.0:
            raise ConfigError(f"[sediment] interval_s must be > 0, got {sc.sediment_interval_s}")
        if "alluvium_thickness" in sed:
            sc.alluvium_thickness = _field(sed["alluvium_thickness"], base, shape, "alluvium_thickness")
            if np.any(np.asarray(sc.alluvium_thickness) < 0):
                raise ConfigError("[sediment] alluvium_thickness must be >= 0 m (0 is bedrock)")
    chan = doc.get("channels")
    if chan is not None:  # config.py:873-885, validated as :421-441
        sc.channel_width = _field(chan.get("width", 0.0), base, shape, "[channels] width")
        sc.channel_depth = _field(chan.get("depth", 0.0), base, shape, "[channels] depth")
        if "manning" in chan:
            sc.channel_manning = _field(chan["manning"], base, shape, "[channels] manning")
        if sc.has_channels and sc.scheme != "local_inertial":
            raise ConfigError(f"[channels] requires scheme='local_inertial'; the '{sc.scheme}' scheme has no "
                              "sub-grid channel model")  # fmt: skip
        if np.isscalar(sc.channel_width) and sc.channel_width < 0:
            raise ConfigError(f"[channels] width must be >= 0, got {sc.channel_width}")
        if sc.has_channels and np.isscalar(sc.channel_depth) and sc.channel_depth <= 0:
            raise ConfigError("[channels] a width without a bank-full depth is not a channel; set [channels] depth")
        if sc.channel_manning is not None and np.isscalar(sc.channel_manning) and sc.channel_manning <= 0:
            raise ConfigError(f"[channels] manning must be > 0, got {sc.channel_manning}")
    for k, entry in enumerate(doc.get("structures", [])):  # config.py:676-730
        name = str(entry.get("name", f"structure{k}"))
        if "crest_m" not in entry:
            raise ConfigError(f"[[structures]] #{k} ('{name}'): 'crest_m' is required")
        pool = entry.get("pool")
        if pool is not None:
            if not (isinstance(pool, list) and len(pool) == 4):
                raise ConfigError(f"[[structures]] #{k} ('{name}'): 'pool' must be [row0, col0, row1, col1]")
            pool = tuple(int(v) for v in pool)
        outlet = entry.get("outlet")
        if outlet is not None:
            if not (isinstance(outlet, list) and len(outlet) in (2, 4)):
                raise ConfigError(f"[[structures]] #{k} ('{name}'): 'outlet' must be [row, col] or "
                                  "[row0, col0, row1, col1]")  # fmt: skip
            vals = tuple(int(v) for v in outlet)
            outlet = (vals[0], vals[1], vals[0], vals[1]) if len(vals) == 2 else vals
        try:
            sc.structures.append(Structure(
                name=name, kind=str(entry.get("type", "dam")),
                cells=[(int(c[0]), int(c[1])) for c in entry.get("cells", [entry["cell"]] if "cell" in entry else [])],
                crest_m=float(entry["crest_m"]), release_rule=str(entry.get("release_rule", "none")),
                release_m3_s=float(entry.get("release_m3_s", 0.0)),
                target_stage_m=float(entry["target_stage_m"]) if "target_stage_m" in entry else None,
                release_max_m3_s=float(entry.get("release_max_m3_s", 0.0)), pool=pool, outlet=outlet,
                interval_s=float(entry.get("interval_s", _DEFAULT_RELEASE_INTERVAL_S)),
            ))  # fmt: skip
        except (TypeError, ValueError, IndexError) as e:
            raise ConfigError(f"[[structures]] #{k} ('{name}'): {e}") from e
    try:
        sc.validate()
    except ValueError as e:
        raise ConfigError(str(e)) from e
    return sc
