/* Host restatement of div_fixed (mit_jax_b200/csrc/cg2d_pressure.cu): a / b for a divisor b fixed over a launch,
 * from y = RN(1/b) by Markstein's correction, q = RN(a y), RN(q + (a - q b) y) with the remainder exact by FMA.
 * Compared bit for bit with the IEEE quotient a / b on pseudo-random dividends over magnitudes 2^-800..2^800 (both
 * signs, zeros) and on divisors that are time steps (60 s .. 1 day), mantissas of all ones, all but one zero, and
 * random. Usage: div_fixed_check SAMPLES_PER_DIVISOR; exit status 1 and the first mismatches when any differ. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t st = 88172645463325252ull;
static uint64_t next(void) {
  st ^= st << 13;
  st ^= st >> 7;
  st ^= st << 17;
  return st;
}
static double unit(void) { return (double)(next() >> 11) * 0x1p-53; }

static double div_fixed(double a, double b, double y) {
  if (a == 0.0) return a * y;
  const double m = fabs(a);
  if (!(m >= 0x1p-900 && m <= 0x1p900) || y == 0.0) return a / b;
  const double q = a * y;
  return fma(fma(-q, b, a), y, q);
}

int main(int argc, char** argv) {
  const long n = argc > 1 ? atol(argv[1]) : 100000;
  const double fixed[] = {60.0, 100.0, 300.0, 450.0, 900.0, 1200.0, 1800.0, 3600.0, 10800.0, 43200.0, 86400.0,
                          0.1, 3.0, 7.0, 1e-3, 0x1.fffffffffffffp0, 0x1.0000000000001p0, 0x1.fffffffffffffp10,
                          0x1.5555555555555p0, 0x1.aaaaaaaaaaaabp3};
  const int nfixed = (int)(sizeof fixed / sizeof fixed[0]);
  long bad = 0, total = 0;
  for (int d = 0; d < nfixed + 40; ++d) {
    const double b = d < nfixed ? fixed[d] : ldexp(1.0 + unit(), (int)(next() % 80) - 40);
    const double y = 1.0 / b;
    for (long k = 0; k < n; ++k) {
      double a = k % 97 == 0 ? 0.0 : ldexp(1.0 + unit(), (int)(next() % 1601) - 800);
      if (next() & 1) a = -a;
      const double r0 = a / b, r1 = div_fixed(a, b, y);
      ++total;
      if (memcmp(&r0, &r1, sizeof r0) != 0) {
        if (bad < 5) printf("a=%a b=%a: %a != %a\n", a, b, r1, r0);
        ++bad;
      }
    }
  }
  printf("%ld of %ld quotients differ\n", bad, total);
  return bad != 0;
}
