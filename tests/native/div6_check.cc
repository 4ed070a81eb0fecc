// CPU check of clover::div6 (cloverleaf3d_ref_b200/csrc/clover_div.cuh)
// against IEEE x / 6.0: every case must give the same bits. Test
// infrastructure, built and run by tests/test_div6.py.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

#include "../../cloverleaf3d_ref_b200/csrc/clover_div.cuh"

static uint64_t bits(double v) {
  uint64_t b;
  memcpy(&b, &v, 8);
  return b;
}
static double from_bits(uint64_t b) {
  double v;
  memcpy(&v, &b, 8);
  return v;
}

static long long checked = 0, bad = 0;

static void check(double x) {
  checked++;
  const double want = x / 6.0, got = clover::div6(x);
  if (bits(want) != bits(got) && !(want != want && got != got)) {
    if (bad < 10) printf("MISMATCH x=%a want=%a got=%a\n", x, want, got);
    bad++;
  }
}

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : 20000000;
  std::mt19937_64 rng(12345);
  // 1. random mantissas and exponents over the whole finite range, both signs
  for (long long i = 0; i < n; i++) {
    const uint64_t m = rng() & 0x000FFFFFFFFFFFFFull;
    const uint64_t e = rng() % 2047;  // includes subnormals (e == 0)
    const uint64_t s = (rng() & 1) << 63;
    check(from_bits(s | (e << 52) | m));
  }
  // 2. quotients near midpoints: the doubles around 6 * mid
  for (long long i = 0; i < n / 4; i++) {
    const uint64_t M = (1ull << 52) | (rng() & 0x000FFFFFFFFFFFFFull);
    const int e = (int)(rng() % 1800) - 900;
    const long double mid = ldexpl((long double)(2 * M + 1), e - 53);
    const double x = (double)(6.0L * mid);
    check(x);
    check(nextafter(x, 0.0));
    check(nextafter(x, 1e308));
  }
  // 3. exact quotients (x = 6 y with y of at most 50 significant bits)
  for (long long i = 0; i < n / 4; i++) {
    const uint64_t m = rng() & 0x000FFFFFFFFFFFF8ull;
    const uint64_t e = 1 + rng() % 2000;
    check(6.0 * from_bits((e << 52) | m));
  }
  // 4. consecutive mantissas at both ends of a binade and in its middle
  for (int k : {-1000, -3, 0, 1, 7, 500, 1000})
    for (uint64_t base : {0ull, 0x8000000000000ull, 0xFFFFFFFF00000ull})
      for (uint64_t i = 0; i < 1000000; i++) {
        const uint64_t m = (base + i) & 0x000FFFFFFFFFFFFFull;
        check(ldexp(from_bits((1023ull << 52) | m), k));
      }
  // 5. the edges: the range limits of the correction, subnormals, zeros,
  //    infinities, NaN, the largest finite values, 3 * 2^k
  const double edge[] = {0x1p-1019, 0x1.fffffffffffffp-1020, 0x1.0000000000001p-1019, 0x1p-1022,
                         0x1p-1074, 0x1.8p-1070, 4.9e-324, 2.2250738585072014e-308, 0.0, -0.0,
                         DBL_MAX, -DBL_MAX, 0x1.ffffffffffffep+1023, 1.0 / 0.0, -1.0 / 0.0,
                         0.0 / 0.0, 6.0, 3.0, 1.0, 0.1, 1e-300, 1e300};
  for (double x : edge) {
    check(x);
    check(-x);
  }
  for (int k = -1074; k <= 1022; k++) {
    check(ldexp(3.0, k));
    check(ldexp(1.0, k));
    check(ldexp(5.0, k));
  }
  printf("checked %lld bad %lld\n", checked, bad);
  return bad != 0;
}
