"""The single simulated clock (the sync-point algebra of solver/scheduler.py:48-254).

The fast scheme proposes a state-derived ``dt_raw``; the clock only ever shortens
it, filling the span to the next sync point with ``ceil(span / dt_raw)`` equal
steps (``fill_span``). Sync points are output times, forcing breakpoints,
slow-process activations and the end time. A slow process is handed the exact
elapsed simulated time since it last ran.

The sync points are kept sorted, so the next one is a bisection (the device clock,
``rbsim.device_clock``, walks the same sorted list with a cursor); each slow
process's pending activations are a queue that a step drains. Every comparison and
every float64 operation is the reference's, in its order, so the host loop and the
device replay take the same steps bit for bit.
"""

from __future__ import annotations

import math
from bisect import bisect_right
from collections import deque
from collections.abc import Callable, Iterable, Iterator, Sequence
from dataclasses import dataclass

EPS_T = 1e-6  # simulated-seconds tolerance for "lands on"


def fill_span(span: float, dt_raw: float) -> float:
    """Equal-step fill of ``span`` by steps no longer than ``dt_raw``."""
    if not math.isfinite(span):
        return dt_raw
    if span <= dt_raw:
        return span
    n = math.ceil(span / dt_raw)
    dt = span / n
    # span / n can land an ulp above dt_raw when span / dt_raw sits just above an integer
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


class _Due:
    """One slow process's activations still ahead, and when it last ran."""

    def __init__(self, proc: SlowProcess, end_time: float):
        self.proc = proc
        self.queue = deque(proc.activations(end_time))
        self.last = 0.0

    def fire(self, t1: float) -> float | None:
        """Drain the activations a step ending at ``t1`` reached; the elapsed time if any."""
        if not self.queue or t1 < self.queue[0] - EPS_T:
            return None
        while self.queue and t1 >= self.queue[0] - EPS_T:
            self.queue.popleft()
        elapsed, self.last = t1 - self.last, t1
        return elapsed


class MultiRateScheduler:
    def __init__(self, end_time: float, output_every: float, events: Sequence[float] = (),
                 processes: Sequence[SlowProcess] = ()):  # fmt: skip
        if end_time <= 0:
            raise ValueError(f"end_time must be > 0, got {end_time}")
        if output_every <= 0:
            raise ValueError(f"output_every must be > 0, got {output_every}")
        self.end_time = end_time
        self.output_every = output_every
        self.events = tuple(events)
        self.processes = tuple(processes)
        points = [*self.output_times, *self.events, *(t for p in self.processes for t in p.activations(end_time)),
                  end_time]  # fmt: skip
        self._points = points  # as given: the device clock sorts its own copy
        self._sorted = sorted(points)

    @property
    def n_frames(self) -> int:
        return int(round(self.end_time / self.output_every)) + 1

    @property
    def output_times(self) -> list[float]:
        return [self.output_every * k for k in range(1, self.n_frames)]

    @property
    def sync_times(self) -> list[float]:
        return list(self._points)

    def next_sync(self, t: float) -> float:
        """The first sync point strictly after ``t + EPS_T`` (infinity past the last)."""
        k = bisect_right(self._sorted, t + EPS_T)
        return self._sorted[k] if k < len(self._sorted) else math.inf

    def ticks(self, dt_fn: Callable[[], float]) -> Iterator[Tick]:
        """One Tick per fast step until ``end_time``; ``dt_fn`` is the scheme's CFL dt."""
        dues = [_Due(p, self.end_time) for p in self.processes]
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
            due = tuple((d.proc, e) for d in dues if (e := d.fire(t1)) is not None)
            yield Tick(index=index, t0=t, dt=dt, t1=t1, is_output=is_output, due=due)
            t, index = t1, index + 1


def merge_events(*groups: Iterable[float]) -> list[float]:
    return [float(x) for g in groups for x in g]
