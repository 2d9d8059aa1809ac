// fastdiv.h - exact unsigned division by a divisor fixed at launch time.
//
// The work queues hand out flat indices that the kernels split into (hit,
// task) or (row, column) pairs.  A 64-bit integer division on the GPU is a
// called software routine of about a hundred instructions; here it is one
// 64-bit multiply-high and a shift, with the multiplier computed on the host
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, the round-up method with N = 63):
//
//   for 0 <= n < 2^63 and d >= 1, with l = ceil(log2 d) and
//   m = ceil(2^(63+l) / d)  (m < 2^64 because d > 2^(l-1)),
//   floor(n / d) = floor(m * n / 2^(63+l)) = mulhi64(n, m) >> (l - 1).
//
// The error term of m*n/2^(63+l) over n/d is below n*d/(d*2^63) * 2^l/2^l < 1/d,
// so the floor cannot cross the next integer.  d = 1 (l = 0) is the identity.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define MBR_HD __host__ __device__
#else
#define MBR_HD
#endif

namespace mbr {

struct FastDiv {
  unsigned long long m;  // multiplier
  int32_t sh;            // right shift after the multiply-high; -1 for d == 1
  int32_t d;             // the divisor (1 .. 2^31 - 1)
};

// Host: the multiplier of divisor d (1 <= d < 2^31).
inline FastDiv make_fastdiv(int32_t d) {
  FastDiv f;
  f.d = d < 1 ? 1 : d;
  int l = 0;
  while ((1ull << l) < (unsigned long long)f.d) l++;
  if (l == 0) {
    f.m = 0;
    f.sh = -1;
    return f;
  }
  const unsigned __int128 num = (unsigned __int128)1 << (63 + l);
  f.m = (unsigned long long)((num + (unsigned __int128)(f.d - 1)) / (unsigned __int128)f.d);
  f.sh = l - 1;
  return f;
}

MBR_HD inline unsigned long long mulhi64(unsigned long long a, unsigned long long b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (unsigned long long)(((unsigned __int128)a * b) >> 64);
#endif
}

// floor(n / d) for 0 <= n < 2^63.
MBR_HD inline unsigned long long fdiv(unsigned long long n, const FastDiv &f) {
  return f.sh < 0 ? n : (mulhi64(n, f.m) >> f.sh);
}

}  // namespace mbr
