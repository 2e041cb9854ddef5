// libm_dev.cuh -- device functions returning the host C library's log2f and
// exp2f results bit for bit (the table scheme is described in libm.h).
#pragma once

#include <cstdint>

#include "libm.h"

namespace cpsz {
namespace dev {

// Hard-case search radius on the GPU: the scan's 2^-18 ulp plus margin for the
// double-precision result's own error.
constexpr double kLibmHard = 1.0 / 262144.0 + 1.0 / 67108864.0;

// Binary search of x in the sorted a[lo, hi); returns its index or -1.
__device__ __forceinline__ int sorted_find(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi, uint32_t x) {
  const uint32_t end = hi;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < x) lo = mid + 1;
    else hi = mid;
  }
  return (lo < end && __ldg(a + lo) == x) ? (int)lo : -1;
}

// Adjacent float of a finite f towards +inf (up) or -inf.
__device__ __forceinline__ float adjacent_float(float f, bool up) {
  const uint32_t b = __float_as_uint(f);
  if ((b & 0x7fffffffu) == 0) return __uint_as_float(up ? 1u : 0x80000001u);
  const bool pos = (b >> 31) == 0;
  return __uint_as_float(pos == up ? b + 1 : b - 1);
}

// Host library's float result for input bits xb, given r = the function's
// value in double precision.
static __device__ __noinline__ float libm_round(double r, uint32_t xb, const LibmFn T) {
  const float f = __double2float_rn(r);
  const uint32_t key = xb >> 23;
  const double fd = (double)f;
  float g = f;
  double d = 0.5;
  bool hard = true;
  if (isfinite(f) && r != fd) {
    g = adjacent_float(f, r > fd);
    if (isfinite(g)) {
      const double gd = (double)g;
      d = fabs(r - 0.5 * (fd + gd)) / fabs(gd - fd);
      hard = d < kLibmHard;
    }
  }
  if (hard) {
    const uint32_t lo = __ldg(T.hard_off + key), hi = __ldg(T.hard_off + key + 1);
    const int at = sorted_find(T.hard_in, lo, hi, xb);
    if (at >= 0) return __uint_as_float(__ldg(T.hard_out + at));
    if (!isfinite(f) || !isfinite(g) || r == fd) return f;
  }
  if (d <= __ldg(T.band + key)) {
    const int s = __ldg(T.bmp_slot + key);
    bool m;
    if (s >= 0) {
      const uint32_t mant = xb & 0x7fffffu;
      m = (__ldg(T.bmp + ((size_t)s << 18) + (mant >> 5)) >> (mant & 31)) & 1u;
    } else {
      const uint32_t lo = __ldg(T.mis_off + key), hi = __ldg(T.mis_off + key + 1);
      m = sorted_find(T.mis, lo, hi, xb) >= 0;
    }
    if (m) return g;
  }
  return f;
}

// log2f(x) of the host library for x > 0 (NaN and +inf pass through).
__device__ __forceinline__ float host_log2f(float x, const LibmFn T) {
  return libm_round(log2((double)x), __float_as_uint(x), T);
}

// exp2f(x) of the host library for x >= -99 (the 3D decoder's domain).
__device__ __forceinline__ float host_exp2f(float x, const LibmFn T) {
  return libm_round(exp2((double)x), __float_as_uint(x), T);
}

}  // namespace dev
}  // namespace cpsz
