"""Progress channel of a run: ``status.json`` (the contract of solver/io/status.py:36-117).

A viewer that launched the solver as a subprocess polls one small JSON document::

    {"state": "running", "progress": 0.42, "sim_time": 1512.0, "eta_s": 8.3, "message": "..."}

``state`` is one of starting, running, writing, done, error; ``progress`` is
``sim_time / end_time`` clipped to [0, 1] (1 once done); ``eta_s`` extrapolates the
wall time spent so far to the rest of the run, or is null before any simulated time
has passed. The document observes the run and never feeds it.

Every update lands whole: it is written to a temporary file beside the target and
renamed over it, so a poller never sees half a document. Where a reader that holds
the file open blocks the rename (Windows), the rename is retried with growing pauses
until a short deadline; an update that still cannot land is dropped, because the
next one supersedes it and a run must not fail over its progress file.
"""

from __future__ import annotations

import json
import os
import tempfile
import time
from pathlib import Path

VALID_STATES = frozenset({"starting", "running", "writing", "done", "error"})
RENAME_DEADLINE_S = 0.5  # how long one update may keep retrying a blocked rename
_FIRST_PAUSE_S = 0.002


def _clip01(x: float) -> float:
    return 0.0 if x < 0.0 else (1.0 if x > 1.0 else x)


class StatusWriter:
    def __init__(self, path, end_time: float):
        self.path = Path(path)
        self.end_time = float(end_time)
        self._started = time.monotonic()  # wall clock, for eta_s only
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self.dropped = 0  # updates that lost every rename attempt

    def document(self, state: str, sim_time: float = 0.0, message: str = "") -> dict:
        if state not in VALID_STATES:
            raise ValueError(f"invalid status state {state!r}; expected one of {sorted(VALID_STATES)}")
        frac = _clip01(sim_time / self.end_time) if self.end_time > 0.0 else 0.0
        eta = None
        if sim_time > 0.0 and frac > 0.0:
            spent = time.monotonic() - self._started
            eta = max(spent * (1.0 - frac) / frac, 0.0)
        return {"state": state, "progress": 1.0 if state == "done" else frac, "sim_time": float(sim_time),
                "eta_s": eta, "message": message}  # fmt: skip

    def write(self, state: str, *, sim_time: float = 0.0, message: str = "") -> bool:
        """Publish one update; returns False if it was dropped (see the module docstring)."""
        payload = json.dumps(self.document(state, sim_time, message)).encode("utf-8")
        fd, tmp = tempfile.mkstemp(prefix=self.path.name + ".", suffix=".tmp", dir=self.path.parent)
        try:
            with os.fdopen(fd, "wb") as f:
                f.write(payload)
            if self._rename(tmp):
                return True
        except BaseException:
            Path(tmp).unlink(missing_ok=True)
            raise
        Path(tmp).unlink(missing_ok=True)
        self.dropped += 1
        return False

    def _rename(self, tmp: str) -> bool:
        deadline = time.monotonic() + RENAME_DEADLINE_S
        pause = _FIRST_PAUSE_S
        while True:
            try:
                os.replace(tmp, self.path)
                return True
            except PermissionError:
                if time.monotonic() + pause > deadline:
                    return False
                time.sleep(pause)
                pause *= 2.0
