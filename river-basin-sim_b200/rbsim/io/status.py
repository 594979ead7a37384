"""Run-status writer (the status.json channel of solver/io/status.py:36-117).

``{"state", "progress", "sim_time", "eta_s", "message"}`` rewritten atomically
(temp file + os.replace); ``state`` walks starting -> running -> writing -> done
(or error); ``eta_s`` is wall-clock extrapolation and never feeds the solver. A
lost rename race (a reader holding the file on some platforms) is retried with
backoff and, if it keeps losing, that one update is dropped.
"""

from __future__ import annotations

import json
import os
import time
from pathlib import Path

VALID_STATES = {"starting", "running", "writing", "done", "error"}
_RETRIES = 12
_BACKOFF_S = 0.005


class StatusWriter:
    def __init__(self, path, end_time: float):
        self.path = Path(path)
        self.end_time = float(end_time)
        self._t0 = time.monotonic()
        self.path.parent.mkdir(parents=True, exist_ok=True)

    def _eta(self, sim_time: float):
        if sim_time <= 0.0 or self.end_time <= 0.0:
            return None
        elapsed = time.monotonic() - self._t0
        frac = min(sim_time / self.end_time, 1.0)
        if frac <= 0.0:
            return None
        return max(elapsed / frac - elapsed, 0.0)

    def write(self, state: str, *, sim_time: float = 0.0, message: str = "") -> None:
        if state not in VALID_STATES:
            raise ValueError(f"invalid status state {state!r}; expected one of {VALID_STATES}")
        progress = 0.0
        if self.end_time > 0.0:
            progress = min(max(sim_time / self.end_time, 0.0), 1.0)
        if state == "done":
            progress = 1.0
        record = {"state": state, "progress": progress, "sim_time": float(sim_time),
                  "eta_s": self._eta(sim_time), "message": message}  # fmt: skip
        tmp = self.path.with_name(self.path.name + ".tmp")
        tmp.write_text(json.dumps(record), encoding="utf-8")
        delay = _BACKOFF_S
        for attempt in range(_RETRIES):
            try:
                os.replace(tmp, self.path)
                return
            except PermissionError:
                if attempt == _RETRIES - 1:
                    break
                time.sleep(delay)
                delay = min(delay * 2.0, 0.1)
        try:
            tmp.unlink()
        except OSError:
            pass
