"""Accuracy of the oracle's portable math (the EXACT-mode functions, restated
from the reference's pmath.hpp) against the platform library in double
precision: the cases of the reference's tests/test_pmath.cpp:25-80 (CPU)."""
import ctypes
import math

import numpy as np


def _ulp_error(value, reference):
    ref_f = np.float32(reference)
    ulp = float(np.nextafter(np.abs(ref_f), np.float32(np.inf)) - np.abs(ref_f))
    return abs(value - reference) / ulp


def test_portable_log(oracle):
    f = oracle.lib().oracle_portable_log
    worst = 0.0
    for k in range(1, (1 << 24) + 1, 97):  # every generator deviate has the form k * 2^-24
        u = float(np.float32(k * (1.0 / 16777216.0)))
        if u > 0.999:
            continue
        worst = max(worst, _ulp_error(f(u), math.log(u)))
    assert worst < 4.0, worst
    assert f(1.0) == 0.0
    for x in (0.9999999, 0.99999, 1.5, 1000.0, 1e-30):
        x = float(np.float32(x))
        assert abs(f(x) - math.log(x)) < 4e-7 * max(1.0, abs(math.log(x)))


def test_portable_sincos_turns(oracle):
    f = oracle.lib().oracle_portable_sincos_turns
    s, c = ctypes.c_float(), ctypes.c_float()
    worst = 0.0
    for k in range(1, (1 << 24) + 1, 101):
        u = float(np.float32(k * (1.0 / 16777216.0)))
        f(u, ctypes.byref(s), ctypes.byref(c))
        worst = max(worst, abs(s.value - math.sin(2 * math.pi * u)), abs(c.value - math.cos(2 * math.pi * u)))
    assert worst < 3e-7, worst
    f(0.25, ctypes.byref(s), ctypes.byref(c))
    assert (s.value, c.value) == (1.0, 0.0)
    f(1.0, ctypes.byref(s), ctypes.byref(c))
    assert (s.value, c.value) == (0.0, 1.0)


def test_portable_cbrt(oracle):
    f = oracle.lib().oracle_portable_cbrt
    worst = 0.0
    x = np.float32(0.01)
    while x < 10.0:
        worst = max(worst, _ulp_error(f(float(x)), float(x) ** (1.0 / 3.0)))
        x = np.float32(x * np.float32(1.0001))
    assert worst < 2.0, worst
    assert f(8.0) == 2.0 and f(1.0) == 1.0
