// Division of non-negative ints below 2^31 by a divisor fixed at set-up,
// as one high multiply, an add and a shift: the round-up method of
// Granlund and Montgomery ("Division by invariant integers using
// multiplication", PLDI 1994, section 4) with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(m, n) + n) >> l.  For
// n < 2^31 the sum cannot overflow 32 bits.  Powers of two get m = 1, which
// makes umulhi vanish, so q = n >> l.  The constructor does a 64-bit
// division: build divisors on the host (or once per kernel), not per item.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define PFDD_HD __host__ __device__ __forceinline__
#else
#define PFDD_HD inline
#endif

namespace pfdd {

struct FastDiv {
  uint32_t d, m;
  int l;
  PFDD_HD FastDiv() : d(1), m(1), l(0) {}
  PFDD_HD explicit FastDiv(int v) : d((uint32_t)(v > 0 ? v : 1)), m(1), l(0) {
    while ((1u << l) < d) ++l;
    m = (uint32_t)(((uint64_t)1 << 32) * (((uint64_t)1 << l) - d) / d + 1);
  }
  PFDD_HD int div(int x) const {
#ifdef __CUDA_ARCH__
    const uint32_t hi = __umulhi(m, (uint32_t)x);
#else
    const uint32_t hi = (uint32_t)(((uint64_t)m * (uint32_t)x) >> 32);
#endif
    return (int)((hi + (uint32_t)x) >> l);
  }
  PFDD_HD int mod(int x) const { return x - div(x) * (int)d; }
};

}  // namespace pfdd
