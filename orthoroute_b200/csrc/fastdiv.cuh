// Division of 32-bit unsigned integers by a run-time invariant divisor with a
// multiply-high and shifts, after T. Granlund and P. L. Montgomery, "Division
// by invariant integers using multiplication" (PLDI 1994), Figure 4.1:
//   m = floor(2^32 * (2^l - d) / d) + 1,  l = ceil(log2 d)
//   q = (t + ((n - t) >> 1)) >> (l - 1),  t = mulhi(m, n)      (d >= 2)
// Valid for every n < 2^32 and 1 <= d <= 2^31.
#pragma once
#include <stdint.h>

struct FastDiv {
  uint32_t d;
  uint32_t m;
  uint32_t l;

  __host__ __device__ __forceinline__ static uint32_t ceil_log2(uint32_t x) {
    // x >= 2
#ifdef __CUDA_ARCH__
    return 32u - (uint32_t)__clz((int)(x - 1u));
#else
    return 32u - (uint32_t)__builtin_clz(x - 1u);
#endif
  }

  __host__ __device__ __forceinline__ void init(uint32_t dd) {
    d = dd;
    if (dd <= 1u) {
      m = 0u;
      l = 0u;
      return;
    }
    l = ceil_log2(dd);
    m = (uint32_t)(((uint64_t)1 << 32) * (((uint64_t)1 << l) - dd) / dd) + 1u;
  }

  __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
    if (d <= 1u) return n;
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(n, m);
#else
    const uint32_t t = (uint32_t)(((uint64_t)n * m) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> (l - 1u);
  }
};
