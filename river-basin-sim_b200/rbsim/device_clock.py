"""Device-resident stepping: the run loop's clock on the GPU, replayed as CUDA graphs.

The reference run loop (solver/run.py:369-388) reads a float back from the device
every step (``compute_dt``) and clamps it on the host (solver/scheduler.py). Here
the same float64 arithmetic runs in a one-thread plan kernel on the device
(librbsim ``rb_clock_plan``), the step kernels read their dt from it, and a span of
``graph_steps`` steps is captured once into a CUDA graph and replayed. The host only
looks at the clock between replays, and only to ask "has the span's target been
reached?". The result is bit-identical to stepping through ``compute_dt`` /
``step``: same state-derived dt, same fill_span clamp, same rain gating.

Point inflows (an ``InflowInjector``) and fixed_stage curves are sampled on the
device at the step midpoint, as the host loop samples them.

Sync times must include every time a step may not cross (outputs, forcing
breakpoints, slow-process activations, the end time), exactly as they are given
to ``MultiRateScheduler``; ``run_until`` is then called with a sync time as target.

Set-up cost. A span shorter than ``graph_steps`` is enqueued launch by launch, with
no capture at all (the device clock still plans every step; the host only issues
the launches, which overlap the device's work). A captured span graph is kept in a
small process-wide cache keyed by everything its launches bake in -- the field and
workspace pointers, the step count, the inflow flag, the kernel variant and the
arithmetic mode -- so a clock built again over the same buffers (a re-run, the
next request on recycled memory) replays it without capturing or instantiating.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from collections import OrderedDict

from . import _lib, graphs
from .scheduler import EPS_T
from .state import State

_GRAPH_CACHE_SIZE = 8
_graph_cache: OrderedDict = OrderedDict()


def _cached_graph(key, build):
    """The instantiated graph for ``key``, capturing it with ``build()`` on a miss."""
    g = _graph_cache.get(key)
    if g is None:
        g = build()
        _graph_cache[key] = g
        while len(_graph_cache) > _GRAPH_CACHE_SIZE:
            _graph_cache.popitem(last=False)
    else:
        _graph_cache.move_to_end(key)
    return g


def clear_graph_cache() -> None:
    _graph_cache.clear()


class DeviceClock:
    def __init__(self, state: State, scheme: str, *, alpha: float, dt_max: float, sync_times, t0: float = 0.0,
                 rain_rate: float = 0.0, rain_until: float = 0.0, limit: bool = True, graph_steps: int = 32,
                 use_graph: bool = True, injector=None):  # fmt: skip
        if scheme not in ("local_inertial", "hllc_fv"):
            raise ValueError(f"unknown scheme {scheme!r}")
        self.state = state
        self.scheme = scheme
        self.graph_steps = int(graph_steps)
        self.use_graph = use_graph
        self._L = _lib.lib()
        sync = np.sort(np.asarray(list(sync_times), dtype=np.float64))
        self._sync = torch.from_numpy(sync).to(state.device)
        field = state.rain is not None
        rain_sum = float(state.rain.double().sum().item()) if field else 0.0
        self._cfg = _lib.ClockConfig(float(alpha), float(dt_max), float(t0), self._sync.data_ptr(), len(sync),
                                     1 if field else 0, float(rain_rate), float(rain_until), rain_sum,
                                     1 if limit else 0)  # fmt: skip
        self._keep = []  # device tables the clock points at
        self.injector = injector
        if injector is not None and injector.inflows:
            nx = state.grid.nx
            cells = [int(i) * nx + int(j) for i, j in (inf.cell for inf in injector.inflows)]
            offs, kt, kq = [0], [], []
            for inf in injector.inflows:
                kt += [float(t) for t, _ in inf.hydrograph]
                kq += [float(q) for _, q in inf.hydrograph]
                offs.append(len(kt))
            dev = state.device
            tabs = [torch.tensor(cells, dtype=torch.int32, device=dev), torch.tensor(offs, dtype=torch.int32, device=dev),
                    torch.tensor(kt or [0.0], dtype=torch.float64, device=dev),
                    torch.tensor(kq or [0.0], dtype=torch.float64, device=dev)]  # fmt: skip
            self._keep += tabs
            self._cfg.nsrc = len(cells)
            self._cfg.src_cell, self._cfg.knot_off, self._cfg.knot_t, self._cfg.knot_q = [t.data_ptr() for t in tabs]
            self._cfg.src_comp = injector._comp.data_ptr() if injector._comp is not None else None
        curves = state.stage_curves
        if curves:
            from .state import EDGES

            st_t, st_v, off = [], [], [0]
            for e in EDGES:
                for tk, lv in curves.get(e, []):
                    st_t.append(float(tk))
                    st_v.append(float(lv))
                off.append(len(st_t))
            tabs = [torch.tensor(st_t, dtype=torch.float64, device=state.device),
                    torch.tensor(st_v, dtype=torch.float64, device=state.device)]  # fmt: skip
            self._keep += tabs
            for k in range(5):
                self._cfg.stage_off[k] = off[k]
            self._cfg.stage_t, self._cfg.stage_v = tabs[0].data_ptr(), tabs[1].data_ptr()
        if scheme == "hllc_fv":
            state.arm_hllc_fields()
            self._fields = state.hllc_fields()
            _lib.check(self._L.rb_hllc_clock_start(ctypes.byref(self._fields), state.cur, ctypes.byref(self._cfg),
                                                   state.workspace.data_ptr(), state.stream))  # fmt: skip
        else:
            self._fields = state.li_fields()
            _lib.check(self._L.rb_li_clock_start(ctypes.byref(self._fields), state.cur, ctypes.byref(self._cfg),
                                                 state.workspace.data_ptr(), state.stream))  # fmt: skip
        self._graph: torch.cuda.CUDAGraph | None = None
        self.t = float(t0)
        self.steps = 0
        self.rain_volume = 0.0
        self.inflow_volume = 0.0

    # -- enqueue ------------------------------------------------------------------ #
    def _enqueue(self, n: int, stream: int) -> None:
        ws = self.state.workspace.data_ptr()
        src = 1 if self._cfg.nsrc > 0 else 0
        if self.scheme == "hllc_fv":
            _lib.check(self._L.rb_hllc_enqueue_steps(ctypes.byref(self._fields), n, src, ws, stream))
        else:
            _lib.check(self._L.rb_li_enqueue_steps(ctypes.byref(self._fields), n, src, ws, stream))

    def _graph_key(self):
        return (self.state.device.index, self.scheme, bytes(self._fields), self.state.workspace.data_ptr(),
                self.graph_steps, self._cfg.nsrc > 0, _lib.launch_config())  # fmt: skip

    def _replay(self, steps: int | None = None) -> None:
        """Enqueue one span: ``graph_steps`` steps from the (cached) graph, or, for a
        shorter span, ``steps`` steps launched directly."""
        if steps is not None and steps < self.graph_steps or not self.use_graph:
            self._enqueue(self.graph_steps if steps is None else steps, self.state.stream)
            return
        if self._graph is None:
            dev = self.state.device
            self._graph = _cached_graph(self._graph_key(),
                                        lambda: graphs.capture(dev, lambda s: self._enqueue(self.graph_steps, s)))
        self._graph.replay()

    def set_target(self, t_target: float, max_steps: int = 2**31 - 1) -> None:
        _lib.check(self._L.rb_clock_set_target(self.state.workspace.data_ptr(), float(t_target), int(max_steps),
                                               self.state.stream))  # fmt: skip

    def read(self) -> _lib.ClockState:
        out = _lib.ClockState()
        _lib.check(self._L.rb_clock_read(self.state.workspace.data_ptr(), self.state.stream, ctypes.byref(out)))
        self.state.cur = out.cur
        self.t, self.steps, self.rain_volume = out.t, out.steps, out.rain_volume
        self.inflow_volume = out.inflow_volume
        if out.err & _lib.RB_DEVERR_NONFINITE:
            raise _lib.DeviceError(f"a step produced a non-finite depth (t = {out.t})")
        if out.err & _lib.RB_DEVERR_CLOCK:
            raise RuntimeError(f"non-positive timestep at t={out.t}")
        return out

    def run_until(self, t_target: float, max_steps: int = 2**31 - 1) -> int:
        """Step until the state reaches ``t_target`` (a sync time) or ``max_steps`` steps; returns steps taken."""
        start = self.steps
        self.set_target(t_target, max_steps)
        while True:
            before = self.steps
            self._replay(max(max_steps - (self.steps - start), 1))
            st = self.read()
            taken = st.steps - start
            if st.t >= t_target - EPS_T or taken >= max_steps:
                return taken
            if st.steps == before:  # an inactive clock would otherwise spin here forever
                raise RuntimeError(f"device clock made no progress toward t={t_target} (t={st.t}, "
                                   f"steps={st.steps}, err={st.err})")  # fmt: skip

    def reseed(self) -> None:
        """Recompute the next step's CFL reduction from the current state: call after
        anything outside the clocked steps changed h (or hu, hv) between spans."""
        fn = self._L.rb_hllc_clock_reseed if self.scheme == "hllc_fv" else self._L.rb_li_clock_reseed
        _lib.check(fn(ctypes.byref(self._fields), self.state.cur, self.state.workspace.data_ptr(), self.state.stream))

    def enqueue_span(self, max_steps: int) -> None:
        """Enqueue (without waiting) replays covering at most ``max_steps`` more steps."""
        self.set_target(math.inf, max_steps)
        full, rest = divmod(max_steps, self.graph_steps)
        for _ in range(full):
            self._replay()
        if rest:
            self._replay(rest)

    def close(self) -> None:
        self._graph = None
