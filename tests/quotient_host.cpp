// Host build of the step kernels' shared-reciprocal quotient: the functions of
// cloverleaf3d_ref_b200/csrc/clover_div.cuh compiled for the CPU (its host form
// seeds the reciprocal with the correctly rounded FP32 reciprocal). Built and
// loaded by tests/test_quotient.py.
#include "../cloverleaf3d_ref_b200/csrc/clover_div.cuh"

extern "C" void quotient_batch(const double* x, const double* b, double* q, int* fast, long long n) {
  for (long long i = 0; i < n; i++) {
    const clover::Recip r = clover::recip_for(b[i]);
    const bool ok = r.ok && clover::quot_in_range(x[i]);
    q[i] = ok ? clover::quot_rn(x[i], r) : x[i] / b[i];
    fast[i] = ok ? 1 : 0;
  }
}
