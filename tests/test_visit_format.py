"""The E12.4 formatting of the VTK writer (visit.f90 writes every value with
WRITE(u,'(e12.4)')): a 0.dddd mantissa, a two-digit exponent after E (three
digits without the E), right-aligned in 12 characters. Host code only."""
import pytest

import cloverleaf3d_ref_b200 as C

CASES = [
    (1.0, "  0.1000E+01"),
    (0.0, "  0.0000E+00"),
    (-0.5, " -0.5000E+00"),
    (0.2, "  0.2000E+00"),
    (123.456, "  0.1235E+03"),
    (9.99996, "  0.1000E+02"),
    (1.0e-8, "  0.1000E-07"),
    (-2.5e-3, " -0.2500E-02"),
    (12345678.9, "  0.1235E+08"),
    (1.5e100, "  0.1500+101"),
    (3.0e-120, "  0.3000-119"),
]


@pytest.mark.parametrize("value,text", CASES)
def test_e12_4(value, text):
    assert C.format_e12_4(value) == text
