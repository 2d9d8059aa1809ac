// Host check of csrc/fastdiv.h: fdiv(n, make_fastdiv(d)) == n / d over edge
// cases and random numerators below 2^63.  Prints the number of mismatches.
#include <stdint.h>
#include <stdio.h>

#include "fastdiv.h"

static unsigned long long rng = 0x9E3779B97F4A7C15ull;
static unsigned long long next() {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return rng;
}

int main() {
  long long bad = 0, checked = 0;
  int divisors[400];
  int nd = 0;
  for (int d = 1; d <= 300; d++) divisors[nd++] = d;
  for (int s = 9; s <= 30; s++) {
    divisors[nd++] = 1 << s;
    divisors[nd++] = (1 << s) + 1;
    divisors[nd++] = (1 << s) - 1;
  }
  divisors[nd++] = 1920;
  divisors[nd++] = 2147483647;
  const unsigned long long top = (1ull << 63) - 1;
  for (int i = 0; i < nd; i++) {
    const unsigned long long d = (unsigned long long)divisors[i];
    const mbr::FastDiv f = mbr::make_fastdiv(divisors[i]);
    unsigned long long cases[12] = {0, 1, d - 1, d, d + 1, 2 * d - 1, 2 * d, top, top - 1, top / d * d, top / d * d - 1,
                                    (1ull << 31) * d - 1};
    for (int c = 0; c < 12; c++) {
      const unsigned long long n = cases[c] & top;
      checked++;
      if (mbr::fdiv(n, f) != n / d) bad++;
    }
    for (int r = 0; r < 20000; r++) {
      unsigned long long n = next() & top;
      if (r & 1) n >>= (r % 62);          // small numerators too
      if (r % 3 == 0) n = n / d * d;      // exact multiples
      if (r % 5 == 0 && n) n -= 1;        // one below a multiple
      checked++;
      if (mbr::fdiv(n, f) != n / d) bad++;
    }
  }
  printf("%lld %lld\n", bad, checked);
  return bad != 0;
}
