// x / 6 correctly rounded without an IEEE division sequence.
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

}  // namespace clover
