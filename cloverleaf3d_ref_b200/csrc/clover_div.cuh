// Correctly rounded FP64 quotients without an IEEE division sequence: x / 6,
// and a / b given the correctly rounded reciprocal of b.
//
// The momentum limiter divides by the literal 6.0_8 (advec_mom_kernel.f90:320
// and its y/z forms). For a divisor known in advance, a multiplication by its
// correctly rounded reciprocal and one FMA correction give the correctly
// rounded quotient (P. Markstein, IBM J. Res. Dev. 34 (1990) 111-119; N.
// Brisebarre, J.-M. Muller, "Accelerating correctly rounded floating-point
// division when the divisor is known in advance", IEEE Trans. Computers 53
// (2004)). For b = 6, with z = RN(1/6) and binary64 (p = 53):
//   q  = RN(x z)            faithful: 1/6 = 1.0101..b * 2^-3 rounds down by a
//                           third of an ulp, so z = (1/6)(1 - 2^-54) and
//                           |q - x/6| < ulp/2 + |x/6| 2^-54 < 1 ulp(x/6);
//   r  = RN(x - 6q) = x - 6q exactly: q and x/6 share an exponent e (or q sits
//                           on the power of two above), x is a multiple of
//                           2^(e-50) and 6q of 2^(e-51), and |x - 6q| < 3 *
//                           2^(e-51);
//   q1 = RN(q + r z)        q + r z = x/6 - (x/6 - q) 2^-54 lies within
//                           2^-54 ulp of x/6, while x/6 is never a midpoint
//                           and lies at least ulp/6 from one (x - 6 mid is a
//                           nonzero multiple of 2^(e-52)), so q1 = RN(x/6).
// The argument needs q normal and x finite: |x| in [2^-1019, DBL_MAX]. Other
// inputs (zeros, whose sign the correction would lose, subnormal quotients,
// infinities, NaN) take the IEEE division. The FMAs are explicit calls, which
// -fmad=false (no contraction of separate operations) leaves fused.
#pragma once

#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define CLOVER_HD __host__ __device__ __forceinline__
#else
#define CLOVER_HD inline
#endif

namespace clover {

CLOVER_HD double div6(double x) {
  const double z = 0x1.5555555555555p-3;  // RN(1/6)
  const double ax = fabs(x);
  if (ax >= 0x1p-1019 && ax <= DBL_MAX) {
    const double q = x * z;
    const double r = fma(-q, 6.0, x);
    return fma(r, z, q);
  }
  return x / 6.0;
}

// single precision: the mixed path's limiter divides as its build divides
CLOVER_HD float div6(float x) { return x / 6.0f; }

// a / b correctly rounded, given y = RN(1/b) (an IEEE division formed once
// for several quotients by the same b, or a reciprocal table entry):
//   q0 = RN(a y)              |q0 - a/b| < 1.5 ulp (y within half an ulp)
//   q1 = RN(q0 + RN(a - b q0) y)   within half an ulp plus 2^-51 ulp of a/b:
//                             faithful
//   q2 = RN(q1 + (a - b q1) y) = RN(a/b)   a - b q1 is exact for a faithful
//                             q1, and by Markstein's theorem (IBM J. Res.
//                             Dev. 34 (1990); see also Cornea, Golliver,
//                             Markstein, ARITH 14 (1999)) the last step
//                             rounds correctly when y is within half an ulp
//                             of 1/b: near a midpoint m, |a/b - q1| is about
//                             ulp/2 and the step moves a/b by at most that
//                             times 2^-53, less than |a/b - m| >= 2^-54 ulp /
//                             (1 - 2^-53) (a - b m is a nonzero multiple of
//                             2^(eb+em)).
// The argument needs normal quotients and exact remainders: a and b with
// binary exponents in [-500, 500] (every value the hydro cycle divides by
// and into, by far); zeros (whose sign the FMAs would not keep), other
// magnitudes, infinities and NaN take the IEEE division.
CLOVER_HD bool div_rn_fast(double a, double b) {
  const double aa = fabs(a), ab = fabs(b);
  return aa >= 0x1p-500 && aa <= 0x1p+500 && ab >= 0x1p-500 && ab <= 0x1p+500;
}

CLOVER_HD double div_rn(double a, double b, double y) {
  if (!div_rn_fast(a, b)) return a / b;
  const double q0 = a * y;
  const double r0 = fma(-q0, b, a);
  const double q1 = fma(r0, y, q0);
  const double r1 = fma(-q1, b, a);
  return fma(r1, y, q1);
}

// single precision: as the build divides
CLOVER_HD float div_rn(float a, float b, float) { return a / b; }

}  // namespace clover
