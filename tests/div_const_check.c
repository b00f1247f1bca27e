/* SPDX-License-Identifier: GPL-3.0-or-later
 * TEST INFRASTRUCTURE: compares cw_div_const(x, c, RN(1/c)) (cppwrf_b200/csrc/cw_pow.h) with the IEEE division x / c
 * bit for bit, for c = 60 and 12, on n operands of each of three kinds drawn from a seed:
 *   0: random bit patterns over every exponent (subnormals, both guard limits, infinities and NaN included);
 *   1: operands whose quotient lies next to a midpoint between two doubles (x = RN(c (q + ulp(q) / 2)), the cases
 *      where a correction that is not exact would round the wrong way);
 *   2: small integers and multiples of c, +-1 and +-2 ulp (exact quotients, sign of zero).
 * Prints "mismatches <count> checked <count>" and the first mismatch, if any.
 *   div_const_check <n> <seed> */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../cppwrf_b200/csrc/cw_pow.h"

static uint64_t sm(uint64_t* s) { /* splitmix64 */
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double from_bits(uint64_t u) {
  double d;
  memcpy(&d, &u, 8);
  return d;
}
static uint64_t to_bits(double d) {
  uint64_t u;
  memcpy(&u, &d, 8);
  return u;
}

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  const long long n = atoll(argv[1]);
  uint64_t s = strtoull(argv[2], NULL, 10);
  const double cs[2] = {60.0, 12.0};
  long long bad = 0, checked = 0;
  for (int ci = 0; ci < 2; ++ci) {
    const double c = cs[ci], r = 1.0 / c;
    for (long long t = 0; t < n; ++t) {
      const int kind = (int)(t % 3);
      double x;
      const uint64_t u = sm(&s);
      if (kind == 0) {
        x = from_bits(u);
      } else if (kind == 1) {
        /* q with an exponent in [-900, 900] */
        const uint64_t e = (uint64_t)(1023 - 900 + (int)(sm(&s) % 1801));
        const double q = from_bits((u & 0x800FFFFFFFFFFFFFull) | (e << 52));
        const double ulp = nextafter(fabs(q), INFINITY) - fabs(q);
        x = fma(c, q, copysign(c * ulp * 0.5, q));
      } else {
        const long long m = (long long)(sm(&s) % 2000001) - 1000000;
        const double base = (u & 1) ? (double)m : c * (double)m;
        const int steps = (int)((u >> 1) % 5) - 2;
        x = base;
        for (int k = 0; k < (steps < 0 ? -steps : steps); ++k) x = nextafter(x, steps < 0 ? -INFINITY : INFINITY);
      }
      const double a = cw_div_const(x, c, r), b = x / c;
      ++checked;
      if (to_bits(a) != to_bits(b) && !(isnan(a) && isnan(b))) {
        if (!bad) printf("first mismatch: c %g x %a got %a want %a\n", c, x, a, b);
        ++bad;
      }
    }
  }
  printf("mismatches %lld checked %lld\n", bad, checked);
  return 0;
}
