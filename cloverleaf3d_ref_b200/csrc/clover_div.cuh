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
#include <cstdint>
#include <cstring>

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

// ---------------------------------------------------------------------------
// x / b correctly rounded for a divisor known only at run time, from one
// approximate reciprocal of b shared by every quotient with that divisor.
//
// The reciprocal: an FP32 seed (rcp.approx.ftz.f32 of RN32(b), relative error
// below 2^-22: the instruction's 1 ulp plus the rounding of b) and two Newton
// steps e = 1 - b y, y' = y + y e with FMAs. The first leaves a relative error
// |b y - 1| below 2^-44.7; the second forms y + y e = (1/b)(1 - d^2 - d rho)
// (d the error before the step, rho the rounding of e) within 2^-36 ulp of
// 1/b, so after its rounding |y - 1/b| <= (1/2 + 2^-36) ulp(1/b), that is
// |b y - 1| <= m 2^-54 (1 + 2^-35) with m in [1, 2) the significand of |b|.
//
// A quotient Q = x/b (u = ulp(Q), delta = b y - 1): q0 = RN(x y) is within 2u
// of Q. The residual r0 = RN(x - b q0) = b (Q - q0)(1 + rho) (rho its
// rounding, |rho| <= 2^-53) and q1 = RN(q0 + r0 y) =
// RN(Q + (Q - q0)(rho + delta + rho delta)), so |q1 - Q| <= (1/2 + 2^-50) u:
// q1 is a faithful rounding of Q. Then x - b q1 is representable (a multiple
// of 2^(e_b + e_Q - 104) below |b| u in magnitude, and no underflow in the
// ranges below), r1 = fma(-b, q1, x) is exact, and q1 + r1 y = Q + (Q - q1)
// delta lies within (1/2 + 2^-50) m 2^-54 (1 + 2^-35) u of Q (the correction
// step of P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34 (1990) 111-119). A midpoint
// between doubles is never Q, and lies at least u 2^-53 / m from it: x - b mid
// is a nonzero multiple of 2^(e_b + e_Q - 105). The bound is the smaller of
// the two while m < 2 - 2^-34, so q = RN(q1 + r1 y) = RN(Q).
//
// Ranges (else the caller takes the IEEE division): |b| in [2^-100, 2^100]
// with the 20 leading fraction bits of b not all ones (m < 2 - 2^-20), and x
// zero or |x| in [2^-800, 2^800]. A zero x returns x * y, the zero IEEE
// division gives. The FMAs are explicit calls, which -fmad=false leaves
// fused; the library's other operations stay uncontracted. The kernels use it
// where it measured faster than the IEEE division sequence (the momentum
// updates and Courant numbers, the cell Courant numbers, the PdV predictor and
// the equation of state); elsewhere they divide. The host form (for tests on
// the CPU) takes its seed from the correctly rounded FP32 reciprocal, which
// lies within the same 1 ulp.
struct Recip {
  double b, y;
  bool ok;  // b lies in the range above
};

CLOVER_HD Recip recip_for(double b) {
  Recip r;
  r.b = b;
#ifdef __CUDA_ARCH__
  const float bf = __double2float_rn(b);
  float yf;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(bf));
  const unsigned hi = (unsigned)__double2hiint(b);
#else
  const float yf = 1.0f / (float)b;
  std::uint64_t bits;
  std::memcpy(&bits, &b, sizeof bits);
  const unsigned hi = (unsigned)(bits >> 32);
#endif
  double y = (double)yf;
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  r.y = fma(y, e, y);
  const double ab = fabs(b);
  r.ok = ab >= 0x1p-100 && ab <= 0x1p100 && (hi & 0xFFFFFu) != 0xFFFFFu;
  return r;
}

// x lies in the range above
CLOVER_HD bool quot_in_range(double x) {
  const double ax = fabs(x);
  return (ax >= 0x1p-800 && ax <= 0x1p800) || x == 0.0;
}

// RN(x / r.b) when r.ok and quot_in_range(x)
CLOVER_HD double quot_rn(double x, const Recip& r) {
  const double q0 = x * r.y;
  const double r0 = fma(-r.b, q0, x);
  const double q1 = fma(r0, r.y, q0);
  const double r1 = fma(-r.b, q1, x);
  const double q = fma(r1, r.y, q1);
  return x == 0.0 ? q0 : q;  // q0 = x * y: a zero with the IEEE quotient's sign
}

#ifdef __CUDACC__

// x / b correctly rounded: in FP64 through quot_rn where x and b lie in its
// range, else by IEEE division; in FP32 by division.
__device__ __forceinline__ double div_rn(double x, double b) {
  const Recip r = recip_for(b);
  if (r.ok && quot_in_range(x)) return quot_rn(x, r);
  return x / b;
}
__device__ __forceinline__ float div_rn(float x, float b) { return x / b; }

// x / b + y / b with each quotient correctly rounded (PdV_kernel.f90:105-107:
// pressure and viscosity over density0), from one reciprocal in FP64.
__device__ __forceinline__ double quot_pair_sum(double x, double y, double b) {
  const Recip r = recip_for(b);
  if (r.ok && quot_in_range(x) && quot_in_range(y)) return quot_rn(x, r) + quot_rn(y, r);
  return x / b + y / b;
}
__device__ __forceinline__ float quot_pair_sum(float x, float y, float b) { return x / b + y / b; }

// v[q] / b for q = 0, 1, 2, each correctly rounded: in FP64 from one shared
// reciprocal of b (quot_rn above) where b and all three numerators lie in its
// range, else by IEEE division; in FP32 by division.
__device__ __forceinline__ void div3_rn(double (&v)[3], double b) {
  const Recip r = recip_for(b);
  if (r.ok && quot_in_range(v[0]) && quot_in_range(v[1]) && quot_in_range(v[2])) {
#pragma unroll
    for (int q = 0; q < 3; q++) v[q] = quot_rn(v[q], r);
  } else {
#pragma unroll
    for (int q = 0; q < 3; q++) v[q] = v[q] / b;
  }
}
__device__ __forceinline__ void div3_rn(float (&v)[3], float b) {
#pragma unroll
  for (int q = 0; q < 3; q++) v[q] = v[q] / b;
}
#endif

}  // namespace clover
