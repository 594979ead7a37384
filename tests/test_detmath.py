"""The deterministic powers of include/rb_detmath.h against a long-double reference.

The CUDA kernels and the oracle evaluate the reference's four fractional powers
(x^float32(7/3), x^float32(1/3), x^1.5, x^float32(4/3)) with these functions, so
they agree bit for bit; this pins how close they are to the exact powers: the
float rounding of x**p computed in x87 long double (64-bit mantissa).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

import oracle

P = {0: np.float32(7.0 / 3.0), 1: np.float32(1.0 / 3.0), 2: np.float32(1.5), 3: np.float32(4.0 / 3.0)}


@pytest.fixture(scope="module")
def detpow():
    f = oracle.lib(np.float32).rbo_pow_f32
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float, ctypes.c_int]
    oracle.set_pow_mode(1)
    yield f
    oracle.set_pow_mode(0)


@pytest.mark.parametrize("which", [0, 1, 2, 3])
def test_powers_are_correctly_rounded_on_a_wide_sample(detpow, which):
    rng = np.random.default_rng(100 + which)
    hi = 1e15 if which != 1 else 1e37
    xs = np.exp(rng.uniform(math.log(1e-30), math.log(hi), 120_000)).astype(np.float32)
    xs = np.concatenate([xs, np.float32([1e-3, 1.0, 2.0, 8.0, 10.0, 0.5, 1.17549435e-38])])
    got = np.array([detpow(float(x), which) for x in xs], np.float32)
    ref = np.power(xs.astype(np.longdouble), np.longdouble(P[which])).astype(np.float32)
    ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert (ulp > 0).sum() <= len(xs) // 10_000


@pytest.mark.parametrize("which", [0, 1, 3])
def test_special_values(detpow, which):
    assert detpow(0.0, which) == 0.0
    assert math.isinf(detpow(float("inf"), which))
    assert math.isnan(detpow(-1.0, which)) and math.isnan(detpow(float("nan"), which))
    assert math.isnan(detpow(-1.0, 2)) and detpow(0.0, 2) == 0.0
