"""Test inputs for the correctly rounded FP64 quotient of the step kernels
(clover_div.cuh: recip_for + quot_rn), and an exact CPU restatement of it.

hard_cases() builds numerators x and divisors b whose quotient x/b lies as
close to a midpoint between two doubles as doubles allow: with b = B 2^(eb-52)
(B odd) and the midpoint m = M 2^(eQ-53) (M odd), x = (B M + d) 2^(eb+eQ-105)
is a double when B M + d is a multiple of 2^53 (or 2^54) with a 53-bit
quotient, and then x/b - m = d 2^(eb+eQ-105) / b: a few units of 2^-53 ulp.
These are the quotients whose rounding the correction steps decide.
"""
import math
from fractions import Fraction

import numpy as np


def _hard_one(B, d, eb, eq):
    inv = pow(B, -1, 1 << 53)
    m0 = (-d * inv) % (1 << 53)
    M = m0 + (1 << 53)  # odd when d is odd, in [2^53, 2^54)
    n = B * M + d
    for s in (53, 54):
        if n % (1 << s) == 0 and (1 << 52) <= n >> s < (1 << 53):
            x = math.ldexp(n >> s, eb + eq - 105 + s)
            b = math.ldexp(B, eb - 52)
            return x, b
    return None


def hard_cases(count, seed, top_divisors=False):
    """count (x, b) pairs with x/b within a few 2^-53 ulp of a midpoint.
    top_divisors: divisors whose significand is just below 2 - 2^-20 (the
    largest the fast quotient accepts)."""
    rng = np.random.default_rng(seed)
    xs, bs = [], []
    while len(xs) < count:
        if top_divisors:
            B = (1 << 53) - (1 << 32) - 1 - 2 * int(rng.integers(0, 1 << 20))
        else:
            B = (1 << 52) | int(rng.integers(0, 1 << 52)) | 1
        d = int(rng.choice([-7, -5, -3, -1, 1, 3, 5, 7]))
        eb = int(rng.integers(-60, 60))
        eq = int(rng.integers(-60, 60))
        r = _hard_one(B, d, eb, eq)
        if r is None:
            continue
        x, b = r
        if rng.integers(0, 2):
            x = -x
        if rng.integers(0, 2):
            b = -b
        xs.append(x)
        bs.append(b)
    return np.array(xs), np.array(bs)


def random_cases(count, seed, span=40):
    """Random significands with exponents within +-span, both signs."""
    rng = np.random.default_rng(seed)
    sig = lambda: rng.uniform(1.0, 2.0, count)
    x = np.ldexp(sig(), rng.integers(-span, span, count)) * rng.choice([-1.0, 1.0], count)
    b = np.ldexp(sig(), rng.integers(-span, span, count)) * rng.choice([-1.0, 1.0], count)
    return x, b


def special_cases():
    """Zeros, exact quotients, powers of two, and values outside the fast
    quotient's range (which take the IEEE division)."""
    xs, bs = [], []
    for x in (0.0, -0.0, 1.0, -3.0, 0.1, 1e-300, -1e-300, 1e300, 2.0 ** -801, 2.0 ** 801,
              math.inf, -math.inf, math.nan, 5e-324):
        for b in (1.0, 3.0, 0.1, -7.5, 2.0 ** -100, 2.0 ** 100, 2.0 ** -101, 2.0 ** 101,
                  2.0 - 2.0 ** -52, 2.0 - 2.0 ** -20, 2.0 - 2.0 ** -21, 1e-320, math.inf):
            xs.append(x)
            bs.append(b)
    for k in range(1, 200):
        b = 1.0 + k / 256.0
        xs.append(b * k)
        bs.append(b)
    return np.array(xs), np.array(bs)


# ---------------------------------------------------------------------------
# The algorithm in exact arithmetic: every operation rounded once to the
# nearest double (Python's int / int is correctly rounded), fma(a, b, c) as
# RN(a*b + c) of the exact product and sum. The FP32 seed is numpy's correctly
# rounded FP32 reciprocal, inside the 1 ulp the GPU's approximate reciprocal
# is allowed.

def _rn(v):
    return float(v)


def _fma(a, b, c):
    return _rn(Fraction(a) * Fraction(b) + Fraction(c))


def recip_for(b):
    if not (2.0 ** -100 <= abs(b) <= 2.0 ** 100):
        return math.nan, False  # the quotient is not used: IEEE division
    with np.errstate(all="ignore"):
        yf = np.float32(1.0) / np.float32(b)
    y = float(yf)
    e = _fma(-b, y, 1.0)
    y = _fma(y, e, y)
    e = _fma(-b, y, 1.0)
    y = _fma(y, e, y)
    hi = int(np.array([b]).view(np.uint64)[0] >> np.uint64(32))
    ok = (hi & 0xFFFFF) != 0xFFFFF
    return y, ok


def quot_in_range(x):
    return x == 0.0 or 2.0 ** -800 <= abs(x) <= 2.0 ** 800


def quot_rn(x, b, y):
    """The quotient's steps."""
    q0 = x * y  # one IEEE rounding (keeps the sign of a zero)
    r0 = _fma(-b, q0, x)
    q1 = _fma(r0, y, q0)
    r1 = _fma(-b, q1, x)
    q = _fma(r1, y, q1)
    return q0 if x == 0.0 else q
