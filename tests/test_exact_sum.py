"""The deterministic mode's exact accumulator (tortoise_b200/csrc/tb_exact.cuh)
built for the host: each value is rounded once to the 2^-112 grid, sums of
those words do not depend on the order of the adds, and the single rounding
back to FP64 is round-to-nearest-even of the exact sum."""
import ctypes as C
import os
import random
import subprocess
from fractions import Fraction

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GRID = Fraction(1, 2 ** 112)


@pytest.fixture(scope="module")
def fx(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fx") / "libfx_host.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out,
                           os.path.join(HERE, "fx_host.cpp")])
    L = C.CDLL(out)
    u64p = C.POINTER(C.c_ulonglong)
    L.fx_host_of.argtypes = [C.c_double, u64p]
    L.fx_host_value.restype = C.c_double
    L.fx_host_value.argtypes = [u64p]
    L.fx_host_sum.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_longlong, u64p]
    L.fx_host_clamp.restype = C.c_double
    return L


def words_of(fx, v):
    w = (C.c_ulonglong * 3)()
    ok = fx.fx_host_of(v, w)
    return ok, list(w)


def signed(words):
    x = words[0] | (words[1] << 64) | (words[2] << 128)
    return x - (1 << 192) if words[2] >> 63 else x


def grid_round(v):
    """v rounded to the nearest multiple of 2^-112, halves away from zero."""
    q = Fraction(v) / GRID
    n = int(abs(q) + Fraction(1, 2))
    return n if v >= 0 else -n


def test_conversion_matches_the_grid(fx):
    rng = random.Random(1)
    vals = [0.0, -0.0, 1.0, -1.0, 2.0 ** -112, 2.0 ** -113, 3 * 2.0 ** -114, -(2.0 ** -113), 1e-300, 5e-324,
            2.0 ** 63, -(2.0 ** 63), 2.0 ** 64 * (1 - 2.0 ** -53), 0.1, -0.3]
    vals += [rng.uniform(-1, 1) * 10.0 ** rng.randint(-40, 18) for _ in range(2000)]
    for v in vals:
        ok, w = words_of(fx, v)
        assert ok, v
        assert signed(w) == grid_round(v), v


def test_values_beyond_the_range_are_refused(fx):
    for v in (2.0 ** 64, -(2.0 ** 64), 1e300, float("inf"), float("-inf"), float("nan")):
        ok, w = words_of(fx, v)
        assert not ok and w == [0, 0, 0], v


def test_clamp_is_the_largest_value_on_the_grid(fx):
    """Finite contributions of 2^64 or more are clamped to the largest double
    below 2^64: held exactly, and many of them still sum exactly (the words
    reach 2^79)."""
    c = fx.fx_host_clamp()
    assert c == 2.0 ** 64 * (1 - 2.0 ** -53) and np.nextafter(c, np.inf) == 2.0 ** 64
    ok, w = words_of(fx, c)
    assert ok and signed(w) == int(c) * 2 ** 112
    ok, w = words_of(fx, -c)
    assert ok and signed(w) == -int(c) * 2 ** 112
    n = 1000
    v = (C.c_double * n)(*([c] * (n - 1) + [-c]))
    order = (C.c_longlong * n)(*range(n))
    acc = (C.c_ulonglong * 3)()
    assert fx.fx_host_sum(v, order, n, acc) == 0
    assert signed(list(acc)) == (n - 2) * int(c) * 2 ** 112
    assert fx.fx_host_value(acc) == (n - 2) * c


def test_round_trip_is_exact_on_the_grid(fx):
    rng = random.Random(2)
    for _ in range(2000):
        v = rng.choice((-1, 1)) * rng.uniform(1, 10) * 10.0 ** rng.randint(-18, 18)   # |v| >= 2^-60: on the grid
        ok, w = words_of(fx, v)
        assert ok and fx.fx_host_value((C.c_ulonglong * 3)(*w)) == v, v


def test_sum_is_order_independent_and_correctly_rounded(fx):
    rng = np.random.default_rng(3)
    n = 4000
    # gain and loss terms of very different sizes that nearly cancel
    mags = 10.0 ** rng.integers(-30, 6, n)
    v = rng.standard_normal(n) * mags
    v = np.concatenate([v, -v[: n // 2] * (1 + 1e-9)])
    exact = sum(Fraction(grid_round(float(x))) for x in v) * GRID
    results = set()
    for seed in range(6):
        order = np.random.default_rng(seed).permutation(v.size).astype(np.int64)
        acc = (C.c_ulonglong * 3)()
        bad = fx.fx_host_sum(v.ctypes.data_as(C.POINTER(C.c_double)), order.ctypes.data_as(C.POINTER(C.c_longlong)),
                             v.size, acc)
        assert bad == 0
        assert Fraction(signed(list(acc))) * GRID == exact
        results.add((tuple(acc), fx.fx_host_value(acc)))
    assert len(results) == 1
    (_, value), = results
    assert value == float(exact)          # Python rounds a Fraction to nearest even
    # an FP64 sum in two orders for comparison: it does depend on the order
    s1 = float(np.sum(v))
    s2 = float(np.sum(v[::-1]))
    assert abs(value - float(exact)) <= abs(s1 - float(exact)) + abs(s2 - float(exact))


def test_negative_totals_and_carries(fx):
    # carries through every word in both directions
    v = np.array([2.0 ** 60, 2.0 ** -100, -(2.0 ** 60), -(2.0 ** -100), -(2.0 ** -112), 2.0 ** 10, -(2.0 ** 11)])
    order = np.arange(v.size, dtype=np.int64)
    acc = (C.c_ulonglong * 3)()
    fx.fx_host_sum(v.ctypes.data_as(C.POINTER(C.c_double)), order.ctypes.data_as(C.POINTER(C.c_longlong)), v.size, acc)
    assert fx.fx_host_value(acc) == float(Fraction(2 ** 10 - 2 ** 11) - GRID)
