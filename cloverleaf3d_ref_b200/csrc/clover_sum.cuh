// Compensated FP64 sums of the field summary (field_summary_kernel.f90:57-77).
//
// The reference adds its five quantities with an OpenMP REDUCTION(+), whose
// order is unspecified. Here every partial sum carries Neumaier's compensation
// (A. Neumaier, ZAMM 54 (1974) 39-51): a running sum s and the running sum c
// of the rounding errors of the additions into s. The error of each addition
// is formed exactly by Knuth's TwoSum (TAOCP vol. 2, 4.2.2, Theorem B), which
// needs no comparison of magnitudes; the result is s + c, within about one
// rounding of the exact sum of the terms (plus n eps^2 times their absolute
// sum). Partial sums are merged pairwise (s of both with TwoSum, c added), so
// a fixed tree and a fixed second stage keep the result the same on every run.
// The error terms are exact only if a + b is neither contracted nor
// reassociated: the library is compiled with -fmad=false.
#pragma once

#include <cuda_runtime.h>

namespace clover {

constexpr int kSumQ = 5;  // vol, mass, ie, ke, press

// s + x into s, its rounding error into c
__device__ __forceinline__ void csum_add(double& s, double& c, double x) {
  const double t = s + x;
  const double xp = t - s;
  const double sp = t - xp;
  const double e = (s - sp) + (x - xp);
  s = t;
  c = c + e;
}

// the partial sum (s2, c2) into (s, c)
__device__ __forceinline__ void csum_merge(double& s, double& c, double s2, double c2) {
  csum_add(s, c, s2);
  c = c + c2;
}

// A block's kSumQ compensated partials reduced over its T threads in a fixed
// tree (sh: 2 * kSumQ * T doubles); thread 0 ends with the block's (s, c).
template <int T>
__device__ __forceinline__ void block_csum(double s[kSumQ], double c[kSumQ], double* sh) {
  const int t = threadIdx.x;
  double* ss = sh;
  double* cc = sh + kSumQ * T;
#pragma unroll
  for (int q = 0; q < kSumQ; q++) {
    ss[q * T + t] = s[q];
    cc[q * T + t] = c[q];
  }
  __syncthreads();
  for (int h = T / 2; h > 0; h >>= 1) {
    if (t < h)
#pragma unroll
      for (int q = 0; q < kSumQ; q++) {
        double a = ss[q * T + t], b = cc[q * T + t];
        csum_merge(a, b, ss[q * T + t + h], cc[q * T + t + h]);
        ss[q * T + t] = a;
        cc[q * T + t] = b;
      }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < kSumQ; q++) {
    s[q] = ss[q * T];
    c[q] = cc[q * T];
  }
}

}  // namespace clover
