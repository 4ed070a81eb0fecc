"""The GPU kernels' correctly rounded FP64 quotients without the IEEE division
sequence (cloverleaf3d_ref_b200/csrc/clover_div.cuh) give the IEEE quotient
bit for bit. Both are built for the host from the same header with glibc's
correctly rounded fma and checked against plain division:
- div6(x) = x / 6 (the momentum limiter's literal) on random, near-midpoint,
  exact-quotient, consecutive-mantissa and edge inputs;
- div_rn(a, b, RN(1/b)) = a / b on random operands, quotients built exactly
  next to midpoints (the 107-bit product of b and a midpoint, rounded to its
  neighbouring doubles), exact quotients, the hydro cycle's value ranges and
  edge inputs (zeros, subnormals, the fast path's limits, infinities, NaN)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name,count", [("div6_check", "8000000"), ("div_rn_check", "4000000")])
def test_quotients_match_ieee_division(tmp_path, name, count):
    exe = str(tmp_path / name)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math",
                           "-o", exe, os.path.join(HERE, "native", name + ".cc"), "-lm"])
    r = subprocess.run([exe, count], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    assert " bad 0" in r.stdout
