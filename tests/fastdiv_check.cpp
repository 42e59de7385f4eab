// Host check of pfdd::FastDiv (csrc/pfdd_fastdiv.h) against / and % for every
// divisor 1..70000: seeded pseudo-random dividends below 2^31, the dividends
// k d - 1, k d, k d + 1 around each quotient, and the top of the range.
// Exit status 0 when every quotient and remainder agrees.
#include <cstdio>

#include "pfdd_fastdiv.h"

int main() {
  long bad = 0;
  for (int d = 1; d <= 70000; ++d) {
    const pfdd::FastDiv f(d);
    unsigned s = 12345u * (unsigned)d;
    for (int t = 0; t < 2000; ++t) {
      s = s * 1664525u + 1013904223u;
      const int n = (int)(s >> 1);
      if (f.div(n) != n / d || f.mod(n) != n % d) ++bad;
      const long k = n / d;
      for (int e = -1; e <= 1; ++e) {
        const long m = k * d + e;
        if (m >= 0 && m < (1L << 31) && f.div((int)m) != (int)(m / d)) ++bad;
      }
    }
    for (long n = (1L << 31) - 3L * d; n < (1L << 31); n += (d > 3 ? d / 3 : 1))
      if (n >= 0 && f.div((int)n) != (int)(n / d)) ++bad;
  }
  std::printf("mismatches %ld\n", bad);
  return bad != 0;
}
