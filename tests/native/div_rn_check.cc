// CPU check of clover::div_rn (cloverleaf3d_ref_b200/csrc/clover_div.cuh):
// a / b from y = RN(1/b) against IEEE a / b, same bits required. Test
// infrastructure, built and run by tests/test_div6.py.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
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

static void check(double a, double b) {
  checked++;
  const double want = a / b, got = clover::div_rn(a, b, 1.0 / b);
  if (bits(want) != bits(got) && !(want != want && got != got)) {
    if (bad < 10) printf("MISMATCH a=%a b=%a want=%a got=%a\n", a, b, want, got);
    bad++;
  }
}

static double rnd(std::mt19937_64& rng, int emin, int emax) {
  const uint64_t m = rng() & 0x000FFFFFFFFFFFFFull;
  const uint64_t e = (uint64_t)(1023 + emin + (int)(rng() % (uint64_t)(emax - emin + 1)));
  return from_bits(((rng() & 1) << 63) | (e << 52) | m);
}

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : 10000000;
  std::mt19937_64 rng(2024);
  // 1. random operands over the fast path's range and beyond it
  for (long long i = 0; i < n; i++) check(rnd(rng, -520, 520), rnd(rng, -520, 520));
  // 2. quotients at and near midpoints: a = RN(b * m) and its neighbours for
  //    a midpoint m between two doubles (the cases where a wrong last step
  //    would show), b with random and with all-ones / all-zeros significands
  for (long long i = 0; i < n; i++) {
    double b = rnd(rng, -60, 60);
    if (i % 7 == 1) b = from_bits((bits(b) & 0xFFF0000000000000ull) | 0x000FFFFFFFFFFFFFull);
    if (i % 7 == 2) b = from_bits((bits(b) & 0xFFF0000000000000ull) | (rng() & 0xFull));
    const double q = rnd(rng, -60, 60);
    const long double m = (long double)q + (long double)(nextafter(q, 2 * q) - q) / 2.0L;
    const double a = (double)((long double)b * m);
    check(a, b);
    check(nextafter(a, 0.0), b);
    check(nextafter(a, 1e300), b);
    check(nextafter(nextafter(a, 1e300), 1e300), b);
  }
  // 2b. the hardest ones, built exactly: significands B (b = B 2^-52) and Q,
  //     the midpoint m = (2Q + 1) 2^-53 between Q 2^-52 and (Q + 1) 2^-52,
  //     the 107-bit product P = B (2Q + 1) = b m 2^105, and a = the doubles
  //     nearest P 2^-105 (a - b m is then as small as it can get)
  for (long long i = 0; i < n; i++) {
    const unsigned long long B = (1ull << 52) | (rng() & 0x000FFFFFFFFFFFFFull);
    const unsigned long long Q = (1ull << 52) | (rng() & 0x000FFFFFFFFFFFFFull);
    const unsigned __int128 P = (unsigned __int128)B * (2 * Q + 1);
    const int bitsP = 128 - (int)(P >> 64 ? __builtin_clzll((unsigned long long)(P >> 64))
                                           : 64 + __builtin_clzll((unsigned long long)P));
    const int sh = bitsP - 53;
    const unsigned long long A = (unsigned long long)((P + ((unsigned __int128)1 << (sh - 1))) >> sh);
    const int e = (int)(rng() % 80) - 40;
    const double b = ldexp((double)B, -52 + e);
    for (long long d = -2; d <= 2; d++) check(ldexp((double)(A + d), sh - 105 + e), b);
  }
  // 3. exact quotients (a = b * q with short significands) and small integers
  for (long long i = 0; i < n / 4; i++) {
    const double b = from_bits((bits(rnd(rng, -40, 40)) & 0xFFFFFFF000000000ull));
    const double q = from_bits((bits(rnd(rng, -40, 40)) & 0xFFFFFFF000000000ull));
    check(b * q, b);
    check((double)(rng() % 100000), (double)(1 + rng() % 1000));
  }
  // 4. the values the hydro cycle divides: node masses, cell widths, volumes
  for (long long i = 0; i < n / 4; i++) {
    std::uniform_real_distribution<double> u(-3.0, 3.0), w(1e-4, 10.0);
    check(u(rng), w(rng));
    check(u(rng) * w(rng), w(rng) * w(rng) * w(rng));
  }
  // 5. edges: zeros of both signs, the fast path's limits, subnormals,
  //    infinities, NaN, huge and tiny magnitudes
  const double edge[] = {0.0, -0.0, 0x1p-500, 0x1.fffffffffffffp-501, 0x1p+500,
                         0x1.0000000000001p+500, 4.9e-324, 2.2250738585072014e-308, 1e308,
                         1.0 / 0.0, -1.0 / 0.0, 0.0 / 0.0, 1.0, 3.0, 0.1, 6.0, 1e-300, 1e300};
  for (double a : edge)
    for (double b : edge) {
      check(a, b);
      check(-a, b);
      check(a, -b);
    }
  printf("checked %lld bad %lld\n", checked, bad);
  return bad != 0;
}
