"""Which arithmetic the step kernels run with (librbsim ``rb_set_arith_mode``).

* ``"exact"`` (the default): one IEEE rounding per operation in the reference's
  expression order, IEEE division and square root, deterministic powers -- every
  state field bit-identical to the CPU oracle.
* ``"fast"``: the same kernels with contracted multiply-adds and the hardware's
  approximate division, square root and powers (the arithmetic of a GPU build of
  the reference); held to the solver tolerance against the oracle instead of bit
  equality. Compensated additions stay exact.

The choice is process-wide and read at each launch; a CUDA graph keeps the mode it
was captured with, and ensembles always run exact.
"""

from __future__ import annotations

import ctypes
from collections.abc import Iterator
from contextlib import contextmanager

from . import _lib

MODES = {"exact": _lib.RB_ARITH_EXACT, "fast": _lib.RB_ARITH_FAST}


def set_arithmetic(mode: str) -> None:
    if mode not in MODES:
        raise ValueError(f"unknown arithmetic {mode!r}; expected one of {sorted(MODES)}")
    _lib.check(_lib.lib().rb_set_arith_mode(MODES[mode]))


def arithmetic() -> str:
    out = ctypes.c_int32(0)
    _lib.check(_lib.lib().rb_arith_mode(ctypes.byref(out)))
    return {v: k for k, v in MODES.items()}[out.value]


@contextmanager
def using(mode: str) -> Iterator[None]:
    """Run the enclosed steps with ``mode``, then restore the previous one."""
    before = arithmetic()
    set_arithmetic(mode)
    try:
        yield
    finally:
        set_arithmetic(before)
