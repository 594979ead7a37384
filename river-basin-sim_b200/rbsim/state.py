"""Solver state on the GPU (the contract of solver/core/state.py:38-256).

Fields are float32 CUDA tensors owned by this object (PyTorch is used only as the
device allocator); every kernel that reads or writes them lives in librbsim.so.

Differences from the reference State, all internal to the B200 layout:

* ``h``, ``qx``, ``qy`` (and ``hu``, ``hv`` once HLLC is armed) are double
  buffered, because a fused step's neighbouring tiles read the old values while it
  writes new ones. The attributes always name the *current* buffer; assigning to
  one copies into the current buffer, so ``state.qx = array`` works as in the
  reference.
* The float64 per-cell ``loss_cum`` field is replaced by per-tile float64 ledger
  partials inside the library workspace (``loss_volume`` returns the same
  quantity: everything infiltration and open / fixed_stage edges removed).
  ``loss_cum`` is ``None`` until a sink is armed, as in the reference.
* ``eta`` is computed on demand (``h + z``); the kernels form it in registers.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .grid import H_DRY, Grid

EDGES = _lib.EDGES


def _device(device) -> torch.device:
    d = torch.device(device if device is not None else "cuda")
    if d.type != "cuda":
        raise ValueError(f"the B200 solver runs on CUDA devices only, got {d}")
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device is available; the solver path has no CPU fallback")
    return d


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _f32(a, shape, device) -> torch.Tensor:
    """A float32 device copy of a host or device array (numpy, or a torch tensor:
    a pinned host tensor copies at full bus speed)."""
    if isinstance(a, torch.Tensor):
        if tuple(a.shape) != tuple(shape):
            raise ValueError(f"field shape {tuple(a.shape)} != {shape}")
        out = torch.empty(shape, dtype=torch.float32, device=device)
        out.copy_(a)
        return out
    arr = np.ascontiguousarray(a, dtype=np.float32)
    if arr.shape != shape:
        raise ValueError(f"field shape {arr.shape} != {shape}")
    if not arr.flags.writeable:  # torch.from_numpy wants a writable buffer
        arr = arr.copy()
    return torch.from_numpy(arr).to(device)


def _scalar_or_field(v, shape, device, name) -> torch.Tensor:
    if isinstance(v, torch.Tensor) or not np.isscalar(v):
        sh = tuple(v.shape) if isinstance(v, torch.Tensor) else np.shape(v)
        if tuple(sh) != tuple(shape):
            raise ValueError(f"{name} shape {tuple(sh)} != bed shape {shape}")
        return _f32(v, shape, device)
    return torch.full(shape, float(v), dtype=torch.float32, device=device)


class _Pair:
    """A double-buffered field: ``bufs[cur]`` is current."""

    def __init__(self, t0: torch.Tensor):
        self.bufs = [t0, torch.zeros_like(t0)]
        self.bufs[1].copy_(t0)


class LossLedger:
    """Stands where the reference's float64 ``loss_cum`` field stood.

    The banked depth is held per tile in the library workspace; ``total()`` is the
    float64 sum of everything infiltration and the open / fixed_stage edges removed
    (the reference's ``loss_cum.sum()``), in metres of depth summed over cells.
    """

    def __init__(self, state: "State"):
        self._state = state

    def total(self) -> float:
        return self._state._ledger_total()


@dataclass
class SedimentState:
    """Device morphology accumulators (solver/core/sediment.py:549-616)."""

    d50: torch.Tensor
    porosity: float
    z0: torch.Tensor
    dz_cum: torch.Tensor
    dz_unapplied: torch.Tensor
    qs_int_x: torch.Tensor
    qs_comp_x: torch.Tensor
    qs_int_y: torch.Tensor
    qs_comp_y: torch.Tensor
    d50_min: float
    d50_max: float
    zero_d50_cells: int

    @property
    def inv_one_minus_p(self) -> float:
        return 1.0 / (1.0 - self.porosity)

    def bed_change_numpy(self) -> np.ndarray:
        return self.dz_cum.cpu().numpy()

    def solid_volume(self, cell_area: float) -> float:
        return float(self.dz_cum.sum().item()) * cell_area * (1.0 - self.porosity)

    def banked_volume(self, cell_area: float) -> float:
        return float(self.dz_unapplied.sum().item()) * cell_area * (1.0 - self.porosity)

    def clear_integral(self) -> None:
        self.qs_int_x.zero_()
        self.qs_int_y.zero_()

    def summary(self) -> str:
        grain = (f"d50 = {1000.0 * self.d50_min:.2f}..{1000.0 * self.d50_max:.2f} mm"
                 if self.d50_min != self.d50_max else f"d50 = {1000.0 * self.d50_max:.2f} mm")  # fmt: skip
        zeros = f", {self.zero_d50_cells} cells with no grain size" if self.zero_d50_cells else ""
        return f"{grain}, porosity {self.porosity:.2f}{zeros}"

    def as_attrs(self) -> dict:
        return {"d50_min_m": self.d50_min, "d50_max_m": self.d50_max, "porosity": self.porosity,
                "zero_d50_cells": self.zero_d50_cells}  # fmt: skip


class State:
    """Mutable float32 fields of one simulation on one CUDA device."""

    def __init__(self, grid: Grid, device: torch.device, h, z, n):
        self.grid = grid
        self.device = device
        self._h = _Pair(h)
        self._qx = _Pair(torch.zeros(grid.qx_shape, dtype=torch.float32, device=device))
        self._qy = _Pair(torch.zeros(grid.qy_shape, dtype=torch.float32, device=device))
        self._hu: _Pair | None = None
        self._hv: _Pair | None = None
        self.cur = 0
        self.z = z
        self.n = n
        self.h_comp: torch.Tensor | None = None
        self.infil: torch.Tensor | None = None
        self.rain: torch.Tensor | None = None
        self.sediment: SedimentState | None = None
        self.channels = None  # ChannelState once sub-grid channels are armed (channels.arm_channels)
        self.hllc = None  # set by the HLLC scheme when armed (marker only)
        self.boundaries = {e: "closed" for e in EDGES}
        self.open_edges: frozenset[str] = frozenset()
        self.stage_curves: dict[str, list[tuple[float, float]]] = {}
        self._loss_armed = False
        self._ws: torch.Tensor | None = None
        self._ws_kind = None
        self._fields_cache = None
        self._alloc_workspace("li")

    # --- construction -------------------------------------------------------- #
    @classmethod
    def from_bed(cls, bed, dx, *, depth=0.0, manning=0.035, device="cuda") -> State:
        """state.py:179-226: fields from a bed array; depth / manning scalar or field."""
        dev = _device(device)
        if not isinstance(bed, torch.Tensor):
            bed = np.ascontiguousarray(bed, dtype=np.float32)
        if len(bed.shape) != 2:
            raise ValueError(f"bed must be 2-D, got shape {tuple(bed.shape)}")
        ny, nx = (int(v) for v in bed.shape)
        grid = Grid(ny=ny, nx=nx, dx=float(dx))
        shape = (ny, nx)
        return cls(grid, dev, _scalar_or_field(depth, shape, dev, "depth"), _f32(bed, shape, dev),
                   _scalar_or_field(manning, shape, dev, "manning"))  # fmt: skip

    # --- double-buffered fields ---------------------------------------------- #
    def _get(self, pair):
        return None if pair is None else pair.bufs[self.cur]

    def _set(self, pair, value, shape):
        if pair is None:
            raise ValueError("field is not armed")
        t = pair.bufs[self.cur]
        if isinstance(value, torch.Tensor):
            t.copy_(value.to(device=t.device, dtype=torch.float32).reshape(shape))
        else:
            t.copy_(torch.from_numpy(np.ascontiguousarray(value, dtype=np.float32).reshape(shape)))

    h = property(lambda s: s._get(s._h), lambda s, v: s._set(s._h, v, s.grid.shape))
    qx = property(lambda s: s._get(s._qx), lambda s, v: s._set(s._qx, v, s.grid.qx_shape))
    qy = property(lambda s: s._get(s._qy), lambda s, v: s._set(s._qy, v, s.grid.qy_shape))
    hu = property(lambda s: s._get(s._hu), lambda s, v: s._set(s._hu, v, s.grid.shape))
    hv = property(lambda s: s._get(s._hv), lambda s, v: s._set(s._hv, v, s.grid.shape))

    @property
    def eta(self) -> torch.Tensor:
        return self.h + self.z

    def flip(self) -> None:
        """Make the buffers a step just wrote current."""
        self.cur ^= 1

    # --- arming (state.py:98-171) ----------------------------------------------- #
    def _invalidate(self):
        self._fields_cache = None

    def set_infiltration(self, infil) -> None:
        self.infil = _f32(infil, self.grid.shape, self.device)
        self._loss_armed = True
        self._invalidate()

    def set_rain_field(self, rain) -> None:
        self.rain = _f32(rain, self.grid.shape, self.device)
        self._invalidate()

    def set_open_boundaries(self, boundaries: dict, stage_curves: dict | None = None) -> None:
        self.boundaries = {e: boundaries.get(e, "closed") for e in EDGES}
        for e, v in self.boundaries.items():
            if v not in _lib.BC_CODE:
                raise ValueError(f"edge {e}: unknown boundary kind {v!r}")
        self.open_edges = frozenset(e for e, v in self.boundaries.items() if v == "open")
        self.stage_curves = {
            e: list(c) for e, c in (stage_curves or {}).items() if self.boundaries.get(e) == "fixed_stage"
        }
        missing = [e for e, v in self.boundaries.items() if v == "fixed_stage" and e not in self.stage_curves]
        if missing:
            raise ValueError(f"fixed_stage edges without a stage curve: {sorted(missing)}")
        if self.open_edges or self.stage_curves:
            self._loss_armed = True
        self._invalidate()

    def arm_source_compensation(self) -> None:
        if self.h_comp is None:
            self.h_comp = torch.zeros(self.grid.shape, dtype=torch.float32, device=self.device)
            self._invalidate()

    def arm_channel_fields(self, w: np.ndarray, d: np.ndarray, n: np.ndarray):
        """Device side of channels.arm_channels (geometry already validated there):
        the geometry fields and the four double-buffered face components, zeroed."""
        from .channels import ChannelState

        g, dev = self.grid, self.device
        has = w > 0
        pairs = {
            "qx_ch": _Pair(torch.zeros(g.qx_shape, dtype=torch.float32, device=dev)),
            "qx_fp": _Pair(torch.zeros(g.qx_shape, dtype=torch.float32, device=dev)),
            "qy_ch": _Pair(torch.zeros(g.qy_shape, dtype=torch.float32, device=dev)),
            "qy_fp": _Pair(torch.zeros(g.qy_shape, dtype=torch.float32, device=dev)),
        }
        self.channels = ChannelState(
            w=_f32(w, g.shape, dev), d=_f32(d, g.shape, dev), n=_f32(n, g.shape, dev),
            width_max=float(w.max()), depth_max=float(d.max()), channel_cells=int(has.sum()),
            _state=self, _pairs=pairs,
        )  # fmt: skip
        self._invalidate()
        return self.channels

    def arm_loss_accumulator(self) -> None:
        self._loss_armed = True

    @property
    def loss_cum(self) -> LossLedger | None:
        return LossLedger(self) if self._loss_armed else None

    def arm_hllc_fields(self) -> None:
        """Allocate the cell momenta (zero: fluid at rest) and the HLLC workspace."""
        if self._hu is not None:
            return
        z = torch.zeros(self.grid.shape, dtype=torch.float32, device=self.device)
        self._hu = _Pair(z)
        self._hv = _Pair(z.clone())
        self._alloc_workspace("hllc")
        self.hllc = True
        self._invalidate()

    # --- workspace / ledger ---------------------------------------------------- #
    def _alloc_workspace(self, kind: str) -> None:
        L = _lib.lib()
        ny, nx = self.grid.shape
        nbytes = int(L.rb_li_workspace_bytes(ny, nx) if kind == "li" else L.rb_hllc_workspace_bytes(ny, nx))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        _lib.check(L.rb_workspace_init(ws.data_ptr(), nbytes, self.stream))
        if self._ws is not None:  # keep the ledger and error word already banked
            keep = min(self._ws.numel(), nbytes, int(L.rb_li_workspace_bytes(ny, nx)))
            ws[:keep].copy_(self._ws[:keep])
        self._ws = ws
        self._ws_kind = kind

    @property
    def workspace(self) -> torch.Tensor:
        return self._ws

    @property
    def stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _ledger_total(self) -> float:
        out = ctypes.c_double(0.0)
        _lib.check(_lib.lib().rb_ledger_loss(self._ws.data_ptr(), self.grid.ny, self.grid.nx, self.stream,
                                             ctypes.byref(out)))  # fmt: skip
        return float(out.value)

    def loss_volume(self, cell_area: float) -> float:
        """Cumulative sink volume (m^3): state.py:173-177, from the device ledger."""
        if not self._loss_armed:
            return 0.0
        return self._ledger_total() * cell_area

    def volume_sum(self) -> float:
        """float64 sum of h over the grid (deterministic device reduction)."""
        out = ctypes.c_double(0.0)
        _lib.check(_lib.lib().rb_sum_f64(self.h.data_ptr(), self.grid.n_cells, self._ws.data_ptr(),
                                         self._ws.numel(), self.stream, ctypes.byref(out)))  # fmt: skip
        return float(out.value)

    def check_device_errors(self) -> None:
        """Raise DeviceError if a kernel flagged a non-finite depth since the last check."""
        err = ctypes.c_uint32(0)
        _lib.check(_lib.lib().rb_read_device_error(self._ws.data_ptr(), self.stream, ctypes.byref(err)))
        if err.value & _lib.RB_DEVERR_NONFINITE:
            raise _lib.DeviceError("a step produced a non-finite depth")
        if err.value:
            raise _lib.DeviceError(f"device error bits 0x{err.value:x}")

    # --- C ABI descriptors ------------------------------------------------------ #
    def _bc(self):
        return (ctypes.c_int32 * 4)(*[_lib.BC_CODE[self.boundaries[e]] for e in EDGES])

    def li_fields(self) -> _lib.LiFields:
        if self._fields_cache is None or not isinstance(self._fields_cache, _lib.LiFields):
            g, sed = self.grid, self.sediment
            self._fields_cache = _lib.LiFields(
                g.ny, g.nx, g.dx,
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._h.bufs]),
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._qx.bufs]),
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._qy.bufs]),
                self.z.data_ptr(), self.n.data_ptr(), _ptr(self.h_comp), _ptr(self.rain), _ptr(self.infil),
                self._bc(), _ptr(sed.d50) if sed else None, _ptr(sed.qs_int_x) if sed else None,
                _ptr(sed.qs_comp_x) if sed else None, _ptr(sed.qs_int_y) if sed else None,
                _ptr(sed.qs_comp_y) if sed else None,
            )  # fmt: skip
            ch = self.channels
            if ch is not None:
                f = self._fields_cache
                f.chan_w, f.chan_d, f.chan_n = ch.w.data_ptr(), ch.d.data_ptr(), ch.n.data_ptr()
                for key in ("qx_ch", "qx_fp", "qy_ch", "qy_fp"):
                    setattr(f, key, (ctypes.c_void_p * 2)(*[t.data_ptr() for t in ch._pairs[key].bufs]))
        return self._fields_cache

    def hllc_fields(self) -> _lib.HllcFields:
        if self._fields_cache is None or not isinstance(self._fields_cache, _lib.HllcFields):
            g = self.grid
            self._fields_cache = _lib.HllcFields(
                g.ny, g.nx, g.dx,
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._h.bufs]),
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._hu.bufs]),
                (ctypes.c_void_p * 2)(*[t.data_ptr() for t in self._hv.bufs]),
                self.z.data_ptr(), self.n.data_ptr(), _ptr(self.h_comp), _ptr(self.rain), _ptr(self.infil),
                self._bc(),
            )  # fmt: skip
        return self._fields_cache

    # --- output (state.py:228-256) ---------------------------------------------- #
    def depth_numpy(self) -> np.ndarray:
        return self.h.cpu().numpy()

    def velocities_numpy(self) -> tuple[np.ndarray, np.ndarray]:
        """Cell-centred (u, v), 0 where h < H_DRY; HLLC from hu/hv, LI from face means."""
        h = self.h.cpu().numpy()
        wet = h >= H_DRY
        u = np.zeros_like(h)
        v = np.zeros_like(h)
        if self._hu is not None:
            np.divide(self.hu.cpu().numpy(), h, out=u, where=wet)
            np.divide(self.hv.cpu().numpy(), h, out=v, where=wet)
        else:
            qx = self.qx.cpu().numpy()
            qy = self.qy.cpu().numpy()
            np.divide(0.5 * (qx[:, :-1] + qx[:, 1:]), h, out=u, where=wet)
            np.divide(0.5 * (qy[:-1, :] + qy[1:, :]), h, out=v, where=wet)
        return u.astype(np.float32), v.astype(np.float32)
