"""Batched stepping of many independent domains (the ensemble and serving workloads).

Each member is an ordinary ``State`` (local inertial or HLLC) with its own
workspace, rain and horizon; the ensemble gives every member its own device clock
and steps all of them with one persistent kernel per scheme over a (domain, tile)
work-list (librbsim ``rb_ensemble_*``), ``graph_steps`` ensemble steps per CUDA
graph replay. A member of 1024 tiles of 32 x 32 or more fills the GPU by itself and
is stepped by the single-domain kernels, launched for it alone in the same step
(faster than the persistent kernels at that size on B200). A member's arithmetic is that of its single-domain step, so its
result is bit-identical to running it alone; members that reach their target stop
(their tiles return immediately) while the others continue.

``autotune`` picks the tile shapes of the two persistent kernels by timing each
candidate on the run itself (tile shape changes which CTA computes a cell, never
what it computes, so the tuning steps are ordinary steps of the run).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib, graphs
from .state import State

LI_VARIANTS = (0, 1, 2, 3)  # tiles 32x16, 32x8, 64x8, 32x32 (512 threads)
HLLC_VARIANTS = (0, 1, 2)  # tiles 32x16, 32x8 (256 threads, persistent), 32x32 (640 threads, one block per tile)


class Ensemble:
    def __init__(self, states: list[State], schemes: list[str], *, alpha, dt_max, sync_times=None,
                 rain_rate=0.0, rain_until=0.0, limit: bool = True, li_variant: int = 0, hllc_variant: int = 0,
                 graph_steps: int = 16, t0=0.0):  # fmt: skip
        n = len(states)
        if n == 0 or len(schemes) != n:
            raise ValueError("one scheme per state is required")
        self.states, self.schemes = list(states), list(schemes)
        self.graph_steps = int(graph_steps)
        self._L = _lib.lib()
        dev = states[0].device
        self.device = dev
        per = lambda v: list(v) if isinstance(v, (list, tuple, np.ndarray)) else [v] * n  # noqa: E731
        alpha, dt_max, rain_rate, rain_until = per(alpha), per(dt_max), per(rain_rate), per(rain_until)
        t0 = per(t0)
        sync_times = sync_times if sync_times is not None else [[] for _ in range(n)]
        code = {"local_inertial": 0, "hllc_fv": 1}
        self._scheme = (ctypes.c_int32 * n)(*[code[s] for s in schemes])
        ny = (ctypes.c_int32 * n)(*[s.grid.ny for s in states])
        nx = (ctypes.c_int32 * n)(*[s.grid.nx for s in states])
        self.layout = _lib.EnsembleLayout()
        _lib.check(self._L.rb_ensemble_layout_make(n, self._scheme, ny, nx, li_variant, hllc_variant,
                                                   ctypes.byref(self.layout)))  # fmt: skip
        self._ws = torch.zeros(int(self.layout.bytes), dtype=torch.uint8, device=dev)
        li, hl, wss = [], [], []
        self._sync = []
        cfgs = (_lib.ClockConfig * n)()
        for d, (st, sch) in enumerate(zip(states, schemes, strict=True)):
            if sch == "hllc_fv":
                st.arm_hllc_fields()
                hl.append(st.hllc_fields())
            else:
                li.append(st.li_fields())
            wss.append(st.workspace.data_ptr())
            sy = torch.tensor(sorted(sync_times[d]) or [0.0], dtype=torch.float64, device=dev)
            self._sync.append(sy)
            field = st.rain is not None
            cfgs[d] = _lib.ClockConfig(float(alpha[d]), float(dt_max[d]), float(t0[d]), sy.data_ptr(),
                                       len(sync_times[d]),
                                       1 if field else 0, float(rain_rate[d]), float(rain_until[d]),
                                       float(st.rain.double().sum().item()) if field else 0.0,
                                       1 if limit else 0)  # fmt: skip
        self._li = (_lib.LiFields * max(len(li), 1))(*li)
        self._hl = (_lib.HllcFields * max(len(hl), 1))(*hl)
        self._wss = (ctypes.c_void_p * n)(*wss)
        self._cfgs = cfgs
        cur = (ctypes.c_int32 * n)(*[s.cur for s in states])
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(self._L.rb_ensemble_init(ctypes.byref(self.layout), self._ws.data_ptr(), self._scheme, self._li,
                                            self._hl, self._wss, cfgs, cur, stream))  # fmt: skip
        self._graph = None
        self.clock = (_lib.ClockState * n)()

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def set_targets(self, t_target, max_steps=None) -> None:
        n = len(self.states)
        tt = (ctypes.c_double * n)(*[float(x) for x in (t_target if np.ndim(t_target) else [t_target] * n)])
        ms = max_steps if max_steps is not None else 2**31 - 1
        mm = (ctypes.c_int32 * n)(*[int(x) for x in (ms if np.ndim(ms) else [ms] * n)])
        _lib.check(self._L.rb_ensemble_set_targets(ctypes.byref(self.layout), self._ws.data_ptr(), tt, mm,
                                                   self._stream()))  # fmt: skip

    def replay(self) -> None:
        if self._graph is None:
            self._graph = graphs.capture(
                self.device,
                lambda s: _lib.check(self._L.rb_ensemble_enqueue(ctypes.byref(self.layout), self._ws.data_ptr(),
                                                                 self.graph_steps, s)))  # fmt: skip
        self._graph.replay()

    def read(self):
        _lib.check(self._L.rb_ensemble_read(ctypes.byref(self.layout), self._ws.data_ptr(), self.clock,
                                            self._stream()))  # fmt: skip
        for st, c in zip(self.states, self.clock, strict=True):
            st.cur = c.cur
            if c.err & _lib.RB_DEVERR_NONFINITE:
                raise _lib.DeviceError("an ensemble member produced a non-finite depth")
            if c.err & _lib.RB_DEVERR_CLOCK:
                raise RuntimeError(f"non-positive timestep in an ensemble member at t={c.t}")
        return self.clock

    def run_until(self, t_target, max_replays: int = 10**7) -> int:
        """Step every member to its target; returns the number of graph replays."""
        from .scheduler import EPS_T

        self.set_targets(t_target)
        tt = list(t_target) if np.ndim(t_target) else [t_target] * len(self.states)
        before = [c.steps for c in self.read()]
        for k in range(max_replays):
            self.replay()
            clk = self.read()
            if all(c.t >= t - EPS_T for c, t in zip(clk, tt, strict=True)):
                return k + 1
            now = [c.steps for c in clk]
            if now == before:  # no member stepped: the clocks are inactive, stop instead of spinning
                raise RuntimeError("ensemble made no progress toward its targets")
            before = now
        raise RuntimeError("ensemble did not reach its targets")


def autotune(make_ensemble, probe_replays: int = 2, candidates=None):
    """Time each (li_variant, hllc_variant) on the run itself; return (best pair, ms per replay, times).

    ``make_ensemble(li_variant, hllc_variant, t0)`` builds an Ensemble over the same
    member states, already targeted, with each member's clock starting at ``t0[d]``
    (``None`` for the first candidate: the caller's start). Each candidate takes
    1 + ``probe_replays`` replays of real steps, and the next one continues every
    clock where it stopped, so the probing is part of the run: every variant
    computes the same bits, and a clock that restarted at the run's start would
    lay different steps toward its sync times. Build the production ensemble with
    ``t0 = times`` (the simulated time each member reached).
    """
    candidates = candidates or [(a, b) for a in LI_VARIANTS for b in HLLC_VARIANTS]
    timings, t0 = {}, None
    for li_v, hl_v in candidates:
        ens = make_ensemble(li_v, hl_v, t0)
        ens.replay()  # capture + first replay, untimed
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(probe_replays):
            ens.replay()
        stop.record()
        stop.synchronize()
        timings[(li_v, hl_v)] = start.elapsed_time(stop) / probe_replays
        t0 = [c.t for c in ens.read()]
    best = min(timings, key=timings.get)
    return best, timings, t0


def log_uniform_sides(n: int, lo: int, hi: int, seed: int) -> list[int]:
    rng = np.random.default_rng(seed)
    return [int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(n)]
