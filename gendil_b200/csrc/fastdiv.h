// Division of 32-bit unsigned integers by a run-time-invariant divisor with one multiply-high,
// after Granlund & Montgomery, "Division by invariant integers using multiplication" (PLDI 1994,
// Fig. 4.1): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
//   q = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0),   t = mulhi(m, n),  for every n < 2^32.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define DGOP_HD __host__ __device__
#else
#define DGOP_HD
#endif

namespace dgop {

struct FastDiv {
  uint32_t d = 1, m = 0;
  int sh1 = 0, sh2 = 0;

  FastDiv() = default;
  explicit FastDiv(uint32_t divisor) : d(divisor) {
    int l = 0;
    while ((uint64_t(1) << l) < divisor) ++l;
    m = (uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << l) - divisor)) / divisor + 1);
    sh1 = l < 1 ? l : 1;
    sh2 = l - 1 > 0 ? l - 1 : 0;
  }

  DGOP_HD uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(m, n);
#else
    const uint32_t t = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
    return (t + ((n - t) >> sh1)) >> sh2;
  }
  DGOP_HD void divmod(uint32_t n, uint32_t& q, uint32_t& r) const {
    q = div(n);
    r = n - q * d;
  }
};

}  // namespace dgop
