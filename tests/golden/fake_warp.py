"""A pure-Python stand-in for the parts of NVIDIA Warp the reference solver uses.

Test infrastructure only: ``make_golden.py`` installs this module as ``warp`` so
that the reference's own ``@wp.kernel`` / ``@wp.func`` source (``solver/core/*.py``,
``solver/processes/*.py``) can be executed on the CPU in this container, where the
real Warp (``warp-lang 1.14.0``, pinned at ``uv.lock:1002-1003``) is not installed.
The fixtures it produces are "the reference run here": the reference's kernel code,
unmodified, interpreted one thread index at a time.

Arithmetic model (what a fixture made through this module means):

* every kernel scalar is a numpy ``float32`` / ``float64`` scalar and every
  operation rounds once, IEEE round-to-nearest -- numpy 2's weak-scalar rule
  (NEP 50) keeps ``0.5 * x`` in float32 exactly as Warp types a Python literal
  next to a float32 operand;
* module-level float constants a kernel reads (``GRAVITY``, ``H_DRY``,
  ``SUBMERGED_SG`` ...) are float32 inside kernels, as Warp compiles them, while
  the host-side Python that shares the module still sees the float64 value;
* ``wp.pow`` is the C runtime's ``powf`` / ``pow`` (called through ctypes, as
  Warp's CPU build links it; numpy's own float32 power loop differs from it in
  about one input in five), ``wp.sqrt`` is the correctly rounded square root;
* ``wp.max(a, b)`` is ``a > b ? a : b``, ``wp.min`` is ``a < b ? a : b`` and
  ``wp.clamp(x, lo, hi)`` is ``min(max(lo, x), hi)`` -- the scalar builtins of
  Warp's native headers;
* there is no fused multiply-add and no fast-math reassociation. Warp's JIT may
  contract ``a*b+c`` on a real device; that is not reproduced here.

Launches loop over the launch dimension in row-major order. Every reference kernel
writes each output from one thread and reads only inputs (its determinism
invariant), so the loop order cannot change a result -- except for
``atomic_max``, which is order-independent.
"""

from __future__ import annotations

import builtins
import ctypes
import ctypes.util
import sys
import types

import numpy as np

float32 = np.float32
float64 = np.float64


def int32(x=0):
    return int(x)


uint32 = int32
int64 = int32

_DTYPES = {float32: np.float32, float64: np.float64, int32: np.int32}


class _Annotation:
    """What ``wp.array2d(dtype=...)`` evaluates to inside an annotation."""

    def __init__(self, dtype=None, ndim=1):
        self.dtype = dtype
        self.ndim = ndim


def array2d(dtype=None):
    return _Annotation(dtype, 2)


class FakeArray(np.ndarray):
    """A numpy array with the few Warp array methods the reference calls."""

    def numpy(self):
        # Warp's CPU device hands back a view of the array's own storage.
        return self.view(np.ndarray)

    def zero_(self):
        self[...] = 0

    def fill_(self, v):
        self[...] = v

    def assign(self, src):
        self[...] = np.asarray(src)

    @property
    def device(self):
        return "cpu"


def array(data=None, dtype=None, device=None, shape=None, copy=True, **_kw):
    if data is None and shape is None:
        return _Annotation(dtype, 1)  # used as ``wp.array(dtype=...)`` annotation
    npdt = _DTYPES.get(dtype, None)
    if data is None:
        return np.zeros(shape, dtype=npdt or np.float32).view(FakeArray)
    arr = np.array(data, dtype=npdt, copy=True)
    return arr.view(FakeArray)


def zeros(shape, dtype=float32, device=None, **_kw):
    return np.zeros(shape, dtype=_DTYPES.get(dtype, np.float32)).view(FakeArray)


def empty(shape, dtype=float32, device=None, **_kw):
    return zeros(shape, dtype, device)


def clone(a, device=None):
    return np.array(a, copy=True).view(FakeArray)


def init():
    return None


# --------------------------------------------------------------------------- #
# Kernel-side builtins.                                                        #
# --------------------------------------------------------------------------- #
def _kind(*vals):
    """The Warp scalar type an expression of these operands has."""
    if any(isinstance(v, np.float64) for v in vals):
        return np.float64
    if any(isinstance(v, (np.float32, float)) for v in vals):
        return np.float32
    return None


def _cast(kind, v):
    return kind(v) if kind is not None else v


def max(a, b):  # noqa: A001 -- Warp's name
    k = _kind(a, b)
    a, b = _cast(k, a), _cast(k, b)
    return a if a > b else b


def min(a, b):  # noqa: A001
    k = _kind(a, b)
    a, b = _cast(k, a), _cast(k, b)
    return a if a < b else b


def clamp(x, lo, hi):
    return min(max(lo, x), hi)


def abs(x):  # noqa: A001
    return builtins.abs(x)


def sqrt(x):
    k = _kind(x) or np.float32
    return k(np.sqrt(k(x)))


_LIBM = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_LIBM.powf.restype = ctypes.c_float
_LIBM.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_LIBM.pow.restype = ctypes.c_double
_LIBM.pow.argtypes = [ctypes.c_double, ctypes.c_double]


def pow(x, y):  # noqa: A001
    k = _kind(x, y) or np.float32
    if k is np.float64:
        return np.float64(_LIBM.pow(float(x), float(y)))
    return np.float32(_LIBM.powf(float(np.float32(x)), float(np.float32(y))))


def vec2f(a, b):
    return (np.float32(a), np.float32(b))


def vec3(a, b, c):
    return (np.float32(a), np.float32(b), np.float32(c))


vec2 = vec2f

_TID = [None]


def tid():
    return _TID[0]


def atomic_max(arr, idx, val):
    cur = arr[idx]
    if val > cur:
        arr[idx] = val
    return cur


def atomic_add(arr, idx, val):
    cur = arr[idx]
    arr[idx] = cur + val
    return cur


# --------------------------------------------------------------------------- #
# Decorators and launch.                                                       #
# --------------------------------------------------------------------------- #
_REGISTRY: dict[int, "_KernelFn"] = {}


class _KernelFn:
    """A ``@wp.func`` / ``@wp.kernel`` function, rebound to float32 globals."""

    def __init__(self, fn):
        self.fn = fn
        self.__name__ = fn.__name__
        self.__doc__ = fn.__doc__
        self._bound = None
        self._params = None

    def _bind(self):
        if self._bound is None:
            g = dict(self.fn.__globals__)
            for name, val in list(g.items()):
                if isinstance(val, float):
                    g[name] = np.float32(val)  # Warp compiles a float global as float32
                elif isinstance(val, _KernelFn):
                    g[name] = _DeviceCall(val)
            self._bound = types.FunctionType(
                self.fn.__code__, g, self.fn.__name__, self.fn.__defaults__, self.fn.__closure__
            )
        return self._bound

    def params(self):
        if self._params is None:
            import inspect

            sig = inspect.signature(self.fn)
            out = []
            for p in sig.parameters.values():
                ann = p.annotation
                if isinstance(ann, str):
                    ann = eval(ann, self.fn.__globals__)  # noqa: S307 -- reference source
                out.append(ann)
            self._params = out
        return self._params

    def __call__(self, *args):
        # Called from host Python (not from another kernel): run as a device call.
        return self._bind()(*args)


class _DeviceCall:
    def __init__(self, k):
        self.k = k

    def __call__(self, *args):
        return self.k._bind()(*args)


def func(fn):
    return _KernelFn(fn)


def kernel(fn=None, **_kw):
    if fn is None:
        return lambda f: _KernelFn(f)
    return _KernelFn(fn)


def _convert(ann, v):
    if ann is float32:
        return np.float32(v)
    if ann is float64:
        return np.float64(v)
    if ann is int32:
        return int(v)
    return v


def launch(kernel, dim, inputs=(), outputs=(), device=None, **_kw):
    body = kernel._bind()
    anns = kernel.params()
    args = [_convert(a, v) for a, v in zip(anns, list(inputs) + list(outputs), strict=True)]
    if isinstance(dim, int):
        for t in range(dim):
            _TID[0] = t
            body(*args)
    else:
        for t in np.ndindex(*dim):
            _TID[0] = t
            body(*args)
    _TID[0] = None


def synchronize():
    return None


def install() -> types.ModuleType:
    """Register this module as ``warp`` in ``sys.modules`` and return it."""
    mod = sys.modules[__name__]
    sys.modules["warp"] = mod
    return mod
