"""CPU oracle for the river-basin solver hot path -- Python side.

TEST INFRASTRUCTURE: the checker the CUDA path is compared against. Only ``tests/``,
``__graft_entry__.smoke`` and the CPU-baseline and float64-error legs of ``bench.py``
use it; the product package never imports it.

The kernels live in ``rbo.c`` (built into ``_build/librbo_{f32,f64}.so`` by the
``Makefile`` beside it); this module holds the state arrays, binds the C entry
points with ctypes, and restates the host-side Python of the reference path:

* ``State`` / ``from_bed`` / arming      -- solver/core/state.py:38-256
* LI ``compute_dt`` / ``step``           -- solver/core/local_inertial.py:515-727
* HLLC ``compute_dt`` / ``step``         -- solver/core/hllc.py:972-1373
* ``stage_at``                           -- solver/core/boundaries.py:199-220
* ``Inflow.discharge_at``                -- solver/io/config.py:111-122
* ``InflowInjector.apply``               -- solver/processes/inflow.py:116-200
* ``arm_channels`` / storage curve       -- solver/core/channels.py:140-312
* ``arm_sediment`` / Exner activation    -- solver/core/sediment.py:658-709,
                                            solver/processes/morphology.py:223-321
* ``ReservoirOperator``                  -- solver/processes/reservoir.py:149-263
* ``MassLedger``                         -- solver/core/massbalance.py:39-158

``pow_mode`` selects how the four fractional powers are evaluated: 0 = libm
``powf`` (what the reference's CPU build calls), 1 = the deterministic functions
of ``include/rb_detmath.h`` that the CUDA kernels use (bit-identical to them).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

GRAVITY = 9.81
H_DRY = 1.0e-3
EDGES = ("north", "south", "east", "west")
BC_CODE = {"closed": 0, "open": 1, "fixed_stage": 2}
EPS_T = 1e-6


def build() -> None:
    """Compile the oracle libraries with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_LIBS: dict[str, ctypes.CDLL] = {}


def lib(dtype=np.float32) -> ctypes.CDLL:
    key = "f32" if np.dtype(dtype) == np.float32 else "f64"
    if key not in _LIBS:
        path = os.path.join(_BUILD, f"librbo_{key}.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        _LIBS[key] = L
    return _LIBS[key]


def set_pow_mode(mode: int) -> None:
    lib(np.float32).rbo_set_pow_mode_f32(ctypes.c_int(mode))


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _li_struct(R):
    P = ctypes.c_void_p
    return type(
        "rbo_li_state",
        (ctypes.Structure,),
        {
            "_fields_": [
                ("ny", ctypes.c_int32), ("nx", ctypes.c_int32), ("dx", ctypes.c_double),
                ("h", P), ("z", P), ("n", P), ("qx", P), ("qy", P), ("eta", P), ("beta", P),
                ("h_comp", P), ("rain", P), ("infil", P), ("loss_cum", P),
                ("bc", ctypes.c_int32 * 4),
                ("d50", P), ("qs_int_x", P), ("qs_comp_x", P), ("qs_int_y", P), ("qs_comp_y", P),
                ("chan_w", P), ("chan_d", P), ("chan_n", P),
                ("qx_ch", P), ("qx_fp", P), ("qy_ch", P), ("qy_fp", P),
            ]
        },
    )  # fmt: skip


def _hllc_struct():
    P = ctypes.c_void_p
    return type(
        "rbo_hllc_state",
        (ctypes.Structure,),
        {
            "_fields_": [
                ("ny", ctypes.c_int32), ("nx", ctypes.c_int32), ("dx", ctypes.c_double),
                ("h", P), ("hu", P), ("hv", P), ("z", P), ("n", P), ("eta", P), ("beta", P),
                ("h_comp", P), ("rain", P), ("infil", P), ("loss_cum", P),
                ("bc", ctypes.c_int32 * 4), ("stage", ctypes.c_double * 4),
                ("uvel", P), ("vvel", P),
                ("fx_h", P), ("fx_mn_l", P), ("fx_mn_r", P), ("fx_mt", P),
                ("fy_h", P), ("fy_mn_l", P), ("fy_mn_r", P), ("fy_mt", P),
                ("dh", P), ("dhu", P), ("dhv", P), ("h1", P), ("hu1", P), ("hv1", P),
            ]
        },
    )  # fmt: skip


_LI_STRUCT = _li_struct(None)
_HLLC_STRUCT = _hllc_struct()


def stage_at(curve, t: float) -> float:
    """boundaries.py:199-220: piecewise-linear stage, held outside the range."""
    if not curve:
        raise ValueError("empty stage curve")
    if t <= curve[0][0]:
        return float(curve[0][1])
    if t >= curve[-1][0]:
        return float(curve[-1][1])
    for (t0, s0), (t1, s1) in zip(curve, curve[1:], strict=False):
        if t0 <= t <= t1:
            if t1 == t0:
                return float(s1)
            return float(s0 + (s1 - s0) * (t - t0) / (t1 - t0))
    return float(curve[-1][1])


@dataclass
class Sediment:
    d50: np.ndarray
    porosity: float
    z0: np.ndarray
    dz_cum: np.ndarray
    dz_unapplied: np.ndarray
    qs_int_x: np.ndarray
    qs_comp_x: np.ndarray
    qs_int_y: np.ndarray
    qs_comp_y: np.ndarray

    @property
    def inv_one_minus_p(self) -> float:
        return 1.0 / (1.0 - self.porosity)


@dataclass
class Channels:
    """Sub-grid channel geometry and the split face discharges (channels.py:182-208)."""

    w: np.ndarray
    d: np.ndarray
    n: np.ndarray
    qx_ch: np.ndarray
    qx_fp: np.ndarray
    qy_ch: np.ndarray
    qy_fp: np.ndarray


@dataclass
class State:
    """Host arrays of one domain, laid out as the reference State (state.py:38-96)."""

    ny: int
    nx: int
    dx: float
    dtype: type
    h: np.ndarray
    z: np.ndarray
    n: np.ndarray
    qx: np.ndarray
    qy: np.ndarray
    eta: np.ndarray
    beta: np.ndarray
    hu: np.ndarray | None = None
    hv: np.ndarray | None = None
    scratch: dict | None = None
    h_comp: np.ndarray | None = None
    rain: np.ndarray | None = None
    infil: np.ndarray | None = None
    loss_cum: np.ndarray | None = None
    boundaries: dict = field(default_factory=lambda: {e: "closed" for e in EDGES})
    stage_curves: dict = field(default_factory=dict)
    sediment: Sediment | None = None
    channels: Channels | None = None

    # --- construction / arming (state.py:98-226) -------------------------- #
    @classmethod
    def from_bed(cls, bed, dx, *, depth=0.0, manning=0.035, dtype=np.float32) -> State:
        bed = np.ascontiguousarray(bed, dtype=np.float32)
        ny, nx = bed.shape
        h0 = (np.full((ny, nx), float(depth), np.float32) if np.isscalar(depth)
              else np.ascontiguousarray(depth, dtype=np.float32))
        n0 = (np.full((ny, nx), float(manning), np.float32) if np.isscalar(manning)
              else np.ascontiguousarray(manning, dtype=np.float32))  # fmt: skip
        if h0.shape != (ny, nx) or n0.shape != (ny, nx):
            raise ValueError("depth/manning shape does not match the bed")
        eta0 = (h0 + bed).astype(np.float32)
        d = np.dtype(dtype)
        return cls(
            ny=ny, nx=nx, dx=float(dx), dtype=d,
            h=h0.astype(d), z=bed.astype(d), n=n0.astype(d),
            qx=np.zeros((ny, nx + 1), d), qy=np.zeros((ny + 1, nx), d),
            eta=eta0.astype(d), beta=np.zeros((ny, nx), d),
        )  # fmt: skip

    def _ensure_loss_cum(self):
        if self.loss_cum is None:
            self.loss_cum = np.zeros((self.ny, self.nx), np.float64)

    def set_infiltration(self, infil):
        self.infil = np.ascontiguousarray(infil, dtype=np.float32).astype(self.dtype)
        self._ensure_loss_cum()

    def set_rain_field(self, rain):
        self.rain = np.ascontiguousarray(rain, dtype=np.float32).astype(self.dtype)

    def set_open_boundaries(self, boundaries, stage_curves=None):
        self.boundaries = {e: boundaries.get(e, "closed") for e in EDGES}
        self.stage_curves = {
            e: list(c) for e, c in (stage_curves or {}).items() if self.boundaries.get(e) == "fixed_stage"
        }
        missing = [e for e, v in self.boundaries.items() if v == "fixed_stage" and e not in self.stage_curves]
        if missing:
            raise ValueError(f"fixed_stage edges without a stage curve: {sorted(missing)}")
        if any(v == "open" for v in self.boundaries.values()) or self.stage_curves:
            self._ensure_loss_cum()

    def arm_source_compensation(self):
        if self.h_comp is None:
            self.h_comp = np.zeros((self.ny, self.nx), self.dtype)

    def arm_hllc(self):
        if self.hu is not None:
            return
        d, c, fx, fy = self.dtype, (self.ny, self.nx), (self.ny, self.nx + 1), (self.ny + 1, self.nx)
        self.hu = np.zeros(c, d)
        self.hv = np.zeros(c, d)
        self.scratch = {k: np.zeros(c, d) for k in ("uvel", "vvel", "dh", "dhu", "dhv", "h1", "hu1", "hv1")}
        self.scratch.update({k: np.zeros(fx, d) for k in ("fx_h", "fx_mn_l", "fx_mn_r", "fx_mt")})
        self.scratch.update({k: np.zeros(fy, d) for k in ("fy_h", "fy_mn_l", "fy_mn_r", "fy_mt")})

    def arm_sediment(self, d50, porosity):
        """sediment.py:658-709 (the oracle keeps the validation to the essentials)."""
        if self.sediment is not None:
            raise ValueError("state is already armed for morphology")
        if not 0.0 < porosity < 1.0:
            raise ValueError(f"porosity must be in (0, 1), got {porosity}")
        c = (self.ny, self.nx)
        grain = (np.full(c, float(d50), np.float32) if np.isscalar(d50)
                 else np.ascontiguousarray(d50, dtype=np.float32).copy())  # fmt: skip
        d = self.dtype
        self.sediment = Sediment(
            d50=grain.astype(d), porosity=float(porosity), z0=self.z.copy(),
            dz_cum=np.zeros(c, np.float64), dz_unapplied=np.zeros(c, np.float64),
            qs_int_x=np.zeros((self.ny, self.nx + 1), d), qs_comp_x=np.zeros((self.ny, self.nx + 1), d),
            qs_int_y=np.zeros((self.ny + 1, self.nx), d), qs_comp_y=np.zeros((self.ny + 1, self.nx), d),
        )  # fmt: skip
        return self.sediment

    def arm_channels(self, width, depth, manning=None):
        """channels.py:265-312 arm_channels, after the validation of :214-262 (the
        oracle keeps the normalisation "no channel" -> w = d = 0 and the refusals that
        change results; the CUDA path's host code restates the full validation)."""
        c = (self.ny, self.nx)
        w = np.ascontiguousarray(width, dtype=np.float32).copy()
        d = np.ascontiguousarray(depth, dtype=np.float32).copy()
        n = (self.n.astype(np.float32).copy() if manning is None
             else np.ascontiguousarray(manning, dtype=np.float32).copy())  # fmt: skip
        if w.shape != c or d.shape != c or n.shape != c:
            raise ValueError("channel field shape does not match the grid")
        if (w > self.dx).any() or (w < 0).any() or (d < 0).any():
            raise ValueError("channel width must be in [0, dx] and depth >= 0")
        has = (w > 0) & (d > 0)
        if ((w > 0) != (d > 0)).any():
            raise ValueError("a channel needs both a width and a bank-full depth")
        w[~has] = 0.0
        d[~has] = 0.0
        dt = self.dtype
        fx, fy = (self.ny, self.nx + 1), (self.ny + 1, self.nx)
        self.channels = Channels(
            w=w.astype(dt), d=d.astype(dt), n=n.astype(dt),
            qx_ch=np.zeros(fx, dt), qx_fp=np.zeros(fx, dt), qy_ch=np.zeros(fy, dt), qy_fp=np.zeros(fy, dt),
        )  # fmt: skip
        return self.channels

    # --- diagnostics ------------------------------------------------------- #
    @property
    def cell_area(self) -> float:
        return self.dx * self.dx

    def loss_volume(self) -> float:
        if self.loss_cum is None:
            return 0.0
        return float(self.loss_cum.astype(np.float64).sum()) * self.cell_area

    def velocities(self):
        """state.py:232-256 velocities_numpy."""
        h = self.h.astype(np.float32)
        wet = h >= H_DRY
        u = np.zeros_like(h)
        v = np.zeros_like(h)
        if self.hu is not None:
            np.divide(self.hu.astype(np.float32), h, out=u, where=wet)
            np.divide(self.hv.astype(np.float32), h, out=v, where=wet)
        else:
            qx, qy = self.qx.astype(np.float32), self.qy.astype(np.float32)
            np.divide(0.5 * (qx[:, :-1] + qx[:, 1:]), h, out=u, where=wet)
            np.divide(0.5 * (qy[:-1, :] + qy[1:, :]), h, out=v, where=wet)
        return u, v

    def _bc(self):
        return (ctypes.c_int32 * 4)(*[BC_CODE[self.boundaries[e]] for e in EDGES])

    def _suffix(self):
        return "_f32" if self.dtype == np.float32 else "_f64"

    def _real(self):
        return ctypes.c_float if self.dtype == np.float32 else ctypes.c_double


# --------------------------------------------------------------------------- #
# Local-inertial scheme                                                        #
# --------------------------------------------------------------------------- #
def li_compute_dt(st: State, alpha: float = 0.7, dt_max: float = 30.0) -> float:
    L = lib(st.dtype)
    f = getattr(L, "rbo_li_compute_dt" + st._suffix())
    f.restype = ctypes.c_double
    ch = st.channels
    return float(f(st.ny, st.nx, _ptr(st.h), _ptr(ch.w) if ch else None, _ptr(ch.d) if ch else None,
                   ctypes.c_double(st.dx), ctypes.c_double(alpha), ctypes.c_double(dt_max)))  # fmt: skip


def li_step(st: State, dt: float, rain: float = 0.0, limit: bool = True, rain_scale: float = 1.0,
            t: float = 0.0) -> None:  # fmt: skip
    L = lib(st.dtype)
    sed = st.sediment
    ch = st.channels
    chp = [_ptr(getattr(ch, k)) if ch else None for k in ("w", "d", "n", "qx_ch", "qx_fp", "qy_ch", "qy_fp")]
    s = _LI_STRUCT(
        st.ny, st.nx, st.dx, _ptr(st.h), _ptr(st.z), _ptr(st.n), _ptr(st.qx), _ptr(st.qy), _ptr(st.eta),
        _ptr(st.beta), _ptr(st.h_comp), _ptr(st.rain), _ptr(st.infil), _ptr(st.loss_cum), st._bc(),
        _ptr(sed.d50) if sed else None, _ptr(sed.qs_int_x) if sed else None,
        _ptr(sed.qs_comp_x) if sed else None, _ptr(sed.qs_int_y) if sed else None,
        _ptr(sed.qs_comp_y) if sed else None, *chp,
    )  # fmt: skip
    getattr(L, "rbo_li_step" + st._suffix())(
        ctypes.byref(s), ctypes.c_double(dt), ctypes.c_double(rain), ctypes.c_int(int(bool(limit))),
        ctypes.c_double(rain_scale),
    )


# --------------------------------------------------------------------------- #
# HLLC scheme                                                                  #
# --------------------------------------------------------------------------- #
def hllc_compute_dt(st: State, alpha: float = 0.45, dt_max: float = 30.0) -> float:
    st.arm_hllc()
    L = lib(st.dtype)
    f = getattr(L, "rbo_hllc_compute_dt" + st._suffix())
    f.restype = ctypes.c_double
    return float(f(st.ny, st.nx, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), ctypes.c_double(st.dx),
                   ctypes.c_double(alpha), ctypes.c_double(dt_max)))  # fmt: skip


def hllc_step(st: State, dt: float, rain: float = 0.0, rain_scale: float = 1.0, t: float = 0.0) -> None:
    st.arm_hllc()
    L = lib(st.dtype)
    sc = st.scratch
    stages = [0.0, 0.0, 0.0, 0.0]
    for k, e in enumerate(EDGES):
        if e in st.stage_curves:
            stages[k] = stage_at(st.stage_curves[e], t + 0.5 * float(dt))
    s = _HLLC_STRUCT(
        st.ny, st.nx, st.dx, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), _ptr(st.z), _ptr(st.n), _ptr(st.eta),
        _ptr(st.beta), _ptr(st.h_comp), _ptr(st.rain), _ptr(st.infil), _ptr(st.loss_cum), st._bc(),
        (ctypes.c_double * 4)(*stages),
        *[_ptr(sc[k]) for k in ("uvel", "vvel", "fx_h", "fx_mn_l", "fx_mn_r", "fx_mt", "fy_h", "fy_mn_l",
                                "fy_mn_r", "fy_mt", "dh", "dhu", "dhv", "h1", "hu1", "hv1")],
    )  # fmt: skip
    getattr(L, "rbo_hllc_step" + st._suffix())(
        ctypes.byref(s), ctypes.c_double(dt), ctypes.c_double(rain), ctypes.c_double(rain_scale)
    )


SCHEMES = {
    "local_inertial": (li_compute_dt, li_step),
    "hllc_fv": (hllc_compute_dt, hllc_step),
}


# --------------------------------------------------------------------------- #
# Inflow point sources (solver/processes/inflow.py, solver/io/config.py:100-122) #
# --------------------------------------------------------------------------- #
@dataclass
class Inflow:
    cell: tuple
    hydrograph: list

    @property
    def breakpoints(self):
        return [t for t, _ in self.hydrograph]

    def discharge_at(self, t: float) -> float:
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
    def __init__(self, inflows, ny, nx, dx, compensated=True):
        self.inflows = list(inflows)
        self.cell_area = float(dx) * float(dx)
        seen = set()
        for inf in self.inflows:
            i, j = inf.cell
            if not (0 <= i < ny and 0 <= j < nx):
                raise ValueError(f"inflow cell {inf.cell} is outside the {ny}x{nx} grid")
            if inf.cell in seen:
                raise ValueError(f"duplicate inflow cell {inf.cell}")
            seen.add(inf.cell)
        self.rows = np.asarray([c.cell[0] for c in self.inflows], np.int32)
        self.cols = np.asarray([c.cell[1] for c in self.inflows], np.int32)
        self.comp = np.zeros(len(self.inflows), np.float32) if compensated else None

    def breakpoints(self):
        return sorted({t for inf in self.inflows for t in inf.breakpoints})

    def apply(self, st: State, t: float, dt: float) -> float:
        if not self.inflows:
            return 0.0
        t_mid = t + 0.5 * dt
        vols = np.array([inf.discharge_at(t_mid) * dt for inf in self.inflows], dtype=np.float64)
        add_depth = (vols / self.cell_area).astype(np.float32)
        L = lib(st.dtype)
        comp = self.comp
        if st.dtype != np.float32:
            add_depth = add_depth.astype(st.dtype)
            if comp is not None and comp.dtype != st.dtype:
                self.comp = comp = comp.astype(st.dtype)
        getattr(L, "rbo_inject_points" + st._suffix())(
            st.ny, st.nx, _ptr(st.h), _ptr(comp), len(self.inflows), _ptr(self.rows), _ptr(self.cols),
            _ptr(np.ascontiguousarray(add_depth)),
        )
        return float(np.asarray(add_depth, np.float32).astype(np.float64).sum()) * self.cell_area


# --------------------------------------------------------------------------- #
# Morphology activation (morphology.py:223-321)                               #
# --------------------------------------------------------------------------- #
def bed_change_bounds(shape, *, alluvium_thickness=None, frozen_cells=()):
    ny, nx = shape
    lo = np.full((ny, nx), -np.inf, dtype=np.float32)
    hi = np.full((ny, nx), np.inf, dtype=np.float32)
    if alluvium_thickness is not None:
        thickness = np.asarray(alluvium_thickness, dtype=np.float32)
        lo = np.broadcast_to(-thickness, (ny, nx)).astype(np.float32).copy()
    for i, j in frozen_cells:
        lo[i, j] = 0.0
        hi[i, j] = 0.0
    return lo, hi


def exner_activate(st: State, dz_lo: np.ndarray, dz_hi: np.ndarray) -> None:
    """Exner update, bed rebuild from z0, eta refresh, integral clear (keeps comp)."""
    sed = st.sediment
    L = lib(st.dtype)
    sfx = st._suffix()
    lo = np.ascontiguousarray(dz_lo, np.float32)
    hi = np.ascontiguousarray(dz_hi, np.float32)
    getattr(L, "rbo_exner_update" + sfx)(
        st.ny, st.nx, _ptr(sed.qs_int_x), _ptr(sed.qs_int_y), _ptr(lo), _ptr(hi),
        ctypes.c_float(st.dx), ctypes.c_float(sed.inv_one_minus_p), _ptr(sed.dz_cum), _ptr(sed.dz_unapplied),
    )  # fmt: skip
    getattr(L, "rbo_rebuild_bed" + sfx)(st.ny, st.nx, _ptr(sed.z0), _ptr(sed.dz_cum), _ptr(st.z))
    getattr(L, "rbo_compute_eta" + sfx)(st.ny, st.nx, _ptr(st.h), _ptr(st.z), _ptr(st.eta))
    sed.qs_int_x[...] = 0
    sed.qs_int_y[...] = 0


# --------------------------------------------------------------------------- #
# Mass ledger (massbalance.py:39-158)                                         #
# --------------------------------------------------------------------------- #
MASS_GATE = 1.0e-6


class _Kahan:
    def __init__(self):
        self.total = 0.0
        self.comp = 0.0

    def add(self, x):
        y = x - self.comp
        t = self.total + y
        self.comp = (t - self.total) - y
        self.total = t


class ReservoirOperator:
    """solver/processes/reservoir.py:149-263 with config.py:228-241 (the release rule),
    restated in numpy: ``structure`` is a dict of the reference Structure's fields.
    Float32 depth arithmetic and float64 banking as the reference kernels
    ``_withdraw_pool`` (:97-121) and ``_deliver_release`` (:124-144)."""

    def __init__(self, structure: dict, st: State):
        self.s = dict(structure)
        self.st = st
        self.records = []
        r0, c0, r1, c1 = self.s["pool"]
        o0, p0, o1, p1 = self.s["outlet"]
        self.pool = (slice(r0, r1 + 1), slice(c0, c1 + 1))
        self.outlet = (slice(o0, o1 + 1), slice(p0, p1 + 1))
        self.outlet_cells = (o1 - o0 + 1) * (p1 - p0 + 1)
        pool_z = st.z[self.pool].astype(np.float32)
        a, b = np.unravel_index(int(np.argmin(pool_z)), pool_z.shape)
        self.gauge = (r0 + int(a), c0 + int(b))
        st._ensure_loss_cum()

    def discharge_at(self, stage):
        rule = self.s.get("release_rule", "none")
        if rule == "none" or stage is None:
            return 0.0
        if rule == "fixed":
            return float(self.s["release_m3_s"])
        span = self.s["crest_m"] - float(self.s["target_stage_m"])
        frac = (stage - float(self.s["target_stage_m"])) / span
        return float(self.s["release_max_m3_s"]) * min(max(frac, 0.0), 1.0)

    def pool_stage(self):
        h = float(self.st.h[self.gauge])
        if h <= H_DRY:
            return None
        return float(self.st.z[self.gauge]) + h

    def advance(self, t: float, dt_slow: float):
        stage = self.pool_stage()
        q = self.discharge_at(stage)
        volume = self._transfer(q * float(dt_slow)) if q > 0.0 else 0.0
        rec = _Release(float(t), stage, q, volume)
        self.records.append(rec)
        return rec

    def _transfer(self, requested_m3: float) -> float:
        st, area = self.st, self.st.cell_area
        stored = float(st.h[self.pool].astype(np.float64).sum()) * area
        if stored <= 0.0:
            return 0.0
        scale = np.float32(min(1.0, requested_m3 / stored))
        avail = st.h[self.pool].astype(np.float32)
        h_new = (avail - avail * scale).astype(np.float32)
        st.h[self.pool] = h_new
        removed = float((avail.astype(np.float64) - h_new.astype(np.float64)).sum()) * area
        if removed <= 0.0:
            return 0.0
        add = removed / area / self.outlet_cells
        avail = st.h[self.outlet].astype(np.float32)
        h_new = (avail + np.float32(add)).astype(np.float32)
        st.h[self.outlet] = h_new
        st.loss_cum[self.outlet] += add - (h_new.astype(np.float64) - avail.astype(np.float64))
        return removed


@dataclass
class _Release:
    time: float
    stage: float | None
    discharge_m3_s: float
    volume_m3: float


class MassLedger:
    def __init__(self, st: State):
        self.cell_area = st.cell_area
        self.v0 = self._volume(st)
        self._inflow = _Kahan()
        self._outflow = _Kahan()
        self._peak_v = 0.0
        self.series = []
        self.record(st, 0.0)

    def _volume(self, st):
        return float(st.h.astype(np.float64).sum()) * self.cell_area

    def add_inflow(self, v):
        self._inflow.add(v)

    def add_rain_step(self, rain_m_s, dt, n_cells):
        self.add_inflow(rain_m_s * dt * self.cell_area * n_cells)

    def record(self, st, time):
        v = self._volume(st)
        inflow = self._inflow.total
        outflow = self._outflow.total + st.loss_volume()
        residual = inflow - outflow - (v - self.v0)
        self._peak_v = max(self._peak_v, v)
        denom = max(abs(inflow), abs(v), self._peak_v, 1e-12)
        rec = dict(time=time, volume=v, inflow_cum=inflow, outflow_cum=outflow, residual=residual,
                   rel_error=abs(residual) / denom)  # fmt: skip
        self.series.append(rec)
        return rec

    @property
    def max_rel_error(self):
        return max((r["rel_error"] for r in self.series), default=0.0)


def fill_span(span: float, dt_raw: float) -> float:
    """scheduler.py:48-72."""
    if not math.isfinite(span):
        return dt_raw
    if span <= dt_raw:
        return span
    n = math.ceil(span / dt_raw)
    dt = span / n
    if dt > dt_raw:
        dt = span / (n + 1)
    return dt
