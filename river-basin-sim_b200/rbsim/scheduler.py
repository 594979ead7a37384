"""The single simulated clock (the sync-point algebra of solver/scheduler.py:48-254).

The fast scheme proposes a state-derived ``dt_raw``; the clock only ever shortens
it, filling the span to the next sync point with ``ceil(span / dt_raw)`` equal
steps (``fill_span``). Sync points are output times, forcing breakpoints,
slow-process activations and the end time. A slow process is handed the exact
elapsed simulated time since it last ran. All arithmetic is host float64, in the
same order as the reference, so a device-side replay (``rbsim.device_clock``)
reproduces the step sequence bit for bit.
"""

from __future__ import annotations

import math
from collections.abc import Callable, Iterable, Iterator, Sequence
from dataclasses import dataclass, field

EPS_T = 1e-6  # simulated-seconds tolerance for "lands on"


def fill_span(span: float, dt_raw: float) -> float:
    """Equal-step fill of ``span`` by steps no longer than ``dt_raw``."""
    if not math.isfinite(span):
        return dt_raw
    if span <= dt_raw:
        return span
    n = math.ceil(span / dt_raw)
    dt = span / n
    # an ulp over dt_raw can happen when span/dt_raw sits just above an integer
    return span / (n + 1) if dt > dt_raw else dt


@dataclass(frozen=True)
class SlowProcess:
    """A process advanced at multiples of ``interval`` by the elapsed simulated time."""

    name: str
    interval: float
    advance: Callable[[float, float], object]

    def __post_init__(self) -> None:
        if self.interval <= 0:
            raise ValueError(f"slow process '{self.name}': interval must be > 0")

    def activations(self, end_time: float) -> list[float]:
        count = int((end_time + EPS_T) // self.interval)
        return [self.interval * k for k in range(1, count + 1)]


@dataclass(frozen=True)
class Tick:
    index: int
    t0: float
    dt: float
    t1: float
    is_output: bool
    due: tuple[tuple[SlowProcess, float], ...] = ()


@dataclass
class MultiRateScheduler:
    end_time: float
    output_every: float
    events: Sequence[float] = ()
    processes: Sequence[SlowProcess] = ()
    _sync: list[float] = field(init=False, repr=False)

    def __post_init__(self) -> None:
        if self.end_time <= 0:
            raise ValueError(f"end_time must be > 0, got {self.end_time}")
        if self.output_every <= 0:
            raise ValueError(f"output_every must be > 0, got {self.output_every}")
        sync = [*self.output_times, *self.events]
        for proc in self.processes:
            sync += proc.activations(self.end_time)
        sync.append(self.end_time)
        self._sync = sync

    @property
    def n_frames(self) -> int:
        return int(round(self.end_time / self.output_every)) + 1

    @property
    def output_times(self) -> list[float]:
        return [self.output_every * k for k in range(1, self.n_frames)]

    @property
    def sync_times(self) -> list[float]:
        return list(self._sync)

    def next_sync(self, t: float) -> float:
        later = [s for s in self._sync if s > t + EPS_T]
        return min(later) if later else math.inf

    def ticks(self, dt_fn: Callable[[], float]) -> Iterator[Tick]:
        """One Tick per fast step until ``end_time``; ``dt_fn`` is the scheme's CFL dt."""
        pending = {p.name: (p, p.activations(self.end_time)) for p in self.processes}
        last_ran = {name: 0.0 for name in pending}
        next_output = self.output_every
        t, index = 0.0, 0
        while t < self.end_time - EPS_T:
            dt_raw = float(dt_fn())
            if dt_raw <= 0.0:
                raise RuntimeError(f"non-positive timestep {dt_raw!r} at t={t}")
            dt = fill_span(self.next_sync(t) - t, dt_raw)
            if dt <= 0.0:
                raise RuntimeError(f"non-positive timestep {dt!r} at t={t}")
            t1 = t + dt
            is_output = t1 >= next_output - EPS_T and next_output <= self.end_time + EPS_T
            if is_output:
                next_output += self.output_every
            due = []
            for name, (proc, times) in pending.items():
                fired = False
                while times and t1 >= times[0] - EPS_T:
                    times.pop(0)
                    fired = True
                if fired:
                    due.append((proc, t1 - last_ran[name]))
                    last_ran[name] = t1
            yield Tick(index=index, t0=t, dt=dt, t1=t1, is_output=is_output, due=tuple(due))
            t = t1
            index += 1


def merge_events(*groups: Iterable[float]) -> list[float]:
    return [float(x) for g in groups for x in g]
