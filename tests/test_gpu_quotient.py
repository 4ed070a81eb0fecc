"""GPU: the correctly rounded FP64 quotient the step kernels form from one
approximate reciprocal per divisor (clover_div.cuh, through
clover_gpu_quotient_selftest) equals IEEE division bit for bit: on random
operands, on quotients within a few 2^-53 ulp of a midpoint
(tests/quotient_cases.py), on divisors around the largest significand it
accepts, and on zeros, infinities, NaN and out-of-range values (which take the
IEEE division inside the self-test, as they do in the kernels)."""
import ctypes

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import quotient_cases as Q

pytestmark = pytest.mark.gpu


def _run(x, b):
    L = C.lib()
    f = L.clover_gpu_quotient_selftest
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_longlong]
    f.restype = ctypes.c_int
    x = np.ascontiguousarray(x, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    q = np.empty_like(x)
    fast = np.empty(len(x), dtype=np.int32)
    assert f(x.ctypes.data, b.ctypes.data, q.ctypes.data, fast.ctypes.data, len(x)) == 0
    with np.errstate(all="ignore"):
        ref = x / b
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(q), nan)
    same = q.view(np.uint64) == ref.view(np.uint64)
    bad = np.flatnonzero(~same & ~nan)
    assert len(bad) == 0, [(x[i], b[i], q[i], ref[i], fast[i]) for i in bad[:5]]
    return fast


def test_random_operands():
    x, b = Q.random_cases(8_000_000, 21)
    fast = _run(x, b)
    assert fast.mean() > 0.999
    x, b = Q.random_cases(2_000_000, 22, span=1000)
    _run(x, b)


def test_divisors_around_the_largest_accepted_significand():
    rng = np.random.default_rng(23)
    n = 2_000_000
    m = 2.0 - np.ldexp(rng.uniform(0.0, 1.0, n), -19)  # in (2 - 2^-19, 2]
    b = np.ldexp(m, rng.integers(-30, 30, n)) * rng.choice([-1.0, 1.0], n)
    x = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-30, 30, n)) * rng.choice([-1.0, 1.0], n)
    fast = _run(x, b)
    assert 0.2 < fast.mean() < 1.0  # the top of the range takes the IEEE division


def test_quotients_next_to_midpoints():
    x, b = Q.hard_cases(60_000, 24)
    assert _run(x, b).all()
    x, b = Q.hard_cases(20_000, 25, top_divisors=True)
    assert _run(x, b).all()


def test_special_values():
    x, b = Q.special_cases()
    fast = _run(x, b)
    assert 0 < fast.sum() < len(fast)
