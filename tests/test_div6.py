"""The momentum limiter's division by 6 (clover_div.cuh, used by the GPU
kernels in place of the IEEE division sequence) gives the IEEE quotient bit
for bit: built for the host from the same header with glibc's correctly
rounded fma and checked against x / 6.0 on random, near-midpoint,
exact-quotient, consecutive-mantissa and edge inputs (zeros, subnormals,
the correction's range limits, infinities, NaN)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_div6_matches_ieee_division(tmp_path):
    exe = str(tmp_path / "div6_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math",
                           "-o", exe, os.path.join(HERE, "native", "div6_check.cc"), "-lm"])
    r = subprocess.run([exe, "8000000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    assert " bad 0" in r.stdout
