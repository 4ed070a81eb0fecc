"""CPU: the shared-reciprocal FP64 quotient (clover_div.cuh) gives the IEEE
quotient bit for bit. Restated in exact arithmetic (tests/quotient_cases.py) on
random inputs and on quotients within a few 2^-53 ulp of a midpoint, where the
product with the reciprocal alone often rounds the wrong way; and the header
itself, compiled for the host (tests/quotient_host.cpp), on millions of them."""
import ctypes
import math
import os
import shutil
import subprocess
from fractions import Fraction

import pytest

import numpy as np

import quotient_cases as Q


def _bits(v):
    return np.array([v], dtype=np.float64).view(np.uint64)[0]


def _check(xs, bs):
    fast = 0
    for x, b in zip(xs.tolist(), bs.tolist()):
        y, ok = Q.recip_for(b)
        if not (ok and Q.quot_in_range(x)):
            continue
        fast += 1
        q = Q.quot_rn(x, b, y)
        assert _bits(q) == _bits(x / b), (x, b, q, x / b)
    return fast


def test_hard_cases_sit_next_to_midpoints():
    xs, bs = Q.hard_cases(200, 1)
    for x, b in zip(xs.tolist(), bs.tolist()):
        q = x / b
        exact = Fraction(x) / Fraction(b)
        # distance from the nearest midpoint, in ulps: at most 8 * 2^-53
        frac = abs(exact - Fraction(q)) / Fraction(math.ulp(q))
        assert abs(frac - Fraction(1, 2)) < Fraction(8, 2 ** 53), (x, b)


def test_exact_restatement_equals_ieee_division():
    assert _check(*Q.random_cases(1500, 2)) == 1500
    assert _check(*Q.hard_cases(1500, 3)) == 1500
    assert _check(*Q.hard_cases(300, 4, top_divisors=True)) == 300
    xs, bs = Q.special_cases()
    assert _check(xs, bs) > 200


def test_corrections_decide_the_hard_cases():
    """The product x * y with the reciprocal alone rounds the wrong way on
    about half of the quotients next to a midpoint."""
    xs, bs = Q.hard_cases(400, 5)
    wrong = 0
    for x, b in zip(xs.tolist(), bs.tolist()):
        y, _ = Q.recip_for(b)
        wrong += x * y != x / b
    assert wrong > 100


def test_range_flags():
    assert not Q.recip_for(2.0 - 2.0 ** -52)[1]  # 20 leading fraction bits all ones
    assert not Q.recip_for(2.0 - 2.0 ** -20)[1]
    assert Q.recip_for(2.0 - 2.0 ** -19)[1]
    assert not Q.recip_for(2.0 ** 101)[1] and Q.recip_for(-(2.0 ** 100))[1]
    assert Q.quot_in_range(-0.0) and not Q.quot_in_range(math.inf)
    assert not Q.quot_in_range(math.nan) and not Q.quot_in_range(2.0 ** -801)


HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def host_quotient(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    so = str(tmp_path_factory.mktemp("quot") / "libquot.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o", so,
                    os.path.join(HERE, "quotient_host.cpp")], check=True)
    f = ctypes.CDLL(so).quotient_batch
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_longlong]
    f.restype = None

    def run(x, b):
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        q = np.empty_like(x)
        fast = np.empty(len(x), dtype=np.int32)
        f(x.ctypes.data, b.ctypes.data, q.ctypes.data, fast.ctypes.data, len(x))
        with np.errstate(all="ignore"):
            ref = x / b
        nan = np.isnan(ref)
        assert np.array_equal(np.isnan(q), nan)
        bad = np.flatnonzero((q.view(np.uint64) != ref.view(np.uint64)) & ~nan)
        assert len(bad) == 0, [(x[i], b[i], q[i], ref[i]) for i in bad[:5]]
        return fast
    return run


def test_header_on_the_host_equals_ieee_division(host_quotient):
    assert host_quotient(*Q.random_cases(4_000_000, 31)).mean() > 0.999
    host_quotient(*Q.random_cases(1_000_000, 32, span=1000))
    assert host_quotient(*Q.hard_cases(20_000, 33)).all()
    assert host_quotient(*Q.hard_cases(5_000, 34, top_divisors=True)).all()
    xs, bs = Q.special_cases()
    fast = host_quotient(xs, bs)
    assert 0 < fast.sum() < len(fast)
