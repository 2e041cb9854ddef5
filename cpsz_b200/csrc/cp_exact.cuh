// cp_exact.cuh -- exact sign predicates for the critical-point checker.
//
// Two tools, both usable on host and device:
//   * Ival: interval arithmetic with directed rounding.  A polynomial in
//     float inputs evaluated on intervals encloses the exact value; when the
//     enclosure excludes zero its sign is certain (the fast path).
//   * Exp: Shewchuk expansions (a sum of doubles, nonoverlapping, increasing
//     magnitude) built with error-free two-sum / two-product; the sign of the
//     exact value is the sign of the largest component (the slow path, taken
//     only when the interval straddles zero).
// Products of two floats are exact in double (24 + 24 <= 53 bits), and a
// difference of two floats is exact as a two-sum pair, so every predicate
// below is decided exactly.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace cpsz {
namespace exact {

#define CPX_HD __host__ __device__

// ---- directed rounding ----------------------------------------------------------
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ double add_dn(double a, double b) { return __dadd_rd(a, b); }
__device__ __forceinline__ double add_up(double a, double b) { return __dadd_ru(a, b); }
__device__ __forceinline__ double mul_dn(double a, double b) { return __dmul_rd(a, b); }
__device__ __forceinline__ double mul_up(double a, double b) { return __dmul_ru(a, b); }
#else
// Host: the round-to-nearest result widened by one ulp is a valid enclosure.
inline double add_dn(double a, double b) { return std::nextafter(a + b, -INFINITY); }
inline double add_up(double a, double b) { return std::nextafter(a + b, INFINITY); }
inline double mul_dn(double a, double b) { return std::nextafter(a * b, -INFINITY); }
inline double mul_up(double a, double b) { return std::nextafter(a * b, INFINITY); }
#endif

struct Ival {
  double lo, hi;
};
CPX_HD inline Ival iv(double x) { return Ival{x, x}; }
CPX_HD inline Ival iv_diff(float a, float b) { return Ival{add_dn(a, -(double)b), add_up(a, -(double)b)}; }
CPX_HD inline Ival operator+(Ival a, Ival b) { return Ival{add_dn(a.lo, b.lo), add_up(a.hi, b.hi)}; }
CPX_HD inline Ival operator-(Ival a, Ival b) { return Ival{add_dn(a.lo, -b.hi), add_up(a.hi, -b.lo)}; }
CPX_HD inline Ival operator*(Ival a, Ival b) {
  const double p0 = mul_dn(a.lo, b.lo), p1 = mul_dn(a.lo, b.hi), p2 = mul_dn(a.hi, b.lo), p3 = mul_dn(a.hi, b.hi);
  const double q0 = mul_up(a.lo, b.lo), q1 = mul_up(a.lo, b.hi), q2 = mul_up(a.hi, b.lo), q3 = mul_up(a.hi, b.hi);
  return Ival{fmin(fmin(p0, p1), fmin(p2, p3)), fmax(fmax(q0, q1), fmax(q2, q3))};
}
CPX_HD inline Ival scale(Ival a, double k) {  // k > 0, a power of two (exact)
  return Ival{a.lo * k, a.hi * k};
}
// +1 / -1 when the enclosure excludes zero, 0 when undecided (or not finite)
CPX_HD inline int iv_sign(Ival a) {
  if (!(a.lo == a.lo) || !(a.hi == a.hi)) return 0;
  if (a.lo > 0) return 1;
  if (a.hi < 0) return -1;
  return 0;
}

// ---- expansions -------------------------------------------------------------------
CPX_HD inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
CPX_HD inline void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

// A nonoverlapping expansion with zero elimination, capacity CAP; `overflow`
// records a component that did not fit (the sign is then not trusted).
template <int CAP>
struct Exp {
  double c[CAP];
  int n = 0;
  bool overflow = false;
  // adds one double exactly (grow_expansion with zero elimination)
  CPX_HD void add(double b) {
    if (b == 0) return;
    double q = b;
    int m = 0;
    for (int i = 0; i < n; i++) {
      double s, e;
      two_sum(q, c[i], s, e);
      if (e != 0) c[m++] = e;
      q = s;
    }
    if (q != 0) {
      if (m < CAP) c[m++] = q;
      else overflow = true;
    }
    n = m;
  }
  template <int C2>
  CPX_HD void add(const Exp<C2>& b, double k = 1.0) {  // k: +-1 or a power of two
    for (int i = 0; i < b.n; i++) add(b.c[i] * k);
    overflow |= b.overflow;
  }
  // adds the exact product a * b
  template <int C1, int C2>
  CPX_HD void add_product(const Exp<C1>& a, const Exp<C2>& b, double k = 1.0) {
    for (int i = 0; i < a.n; i++)
      for (int j = 0; j < b.n; j++) {
        double p, e;
        two_prod(a.c[i], b.c[j], p, e);
        add(p * k);
        add(e * k);
      }
    overflow |= a.overflow | b.overflow;
  }
  // adds b * k for a small non-negative integer k, one exact power-of-two
  // scaling per set bit
  template <int C2>
  CPX_HD void add_times(const Exp<C2>& b, int k, double sgn = 1.0) {
    for (int bit = 0; k >> bit; bit++)
      if ((k >> bit) & 1) add(b, sgn * (double)(1 << bit));
  }
  CPX_HD int sign() const {
    for (int i = n - 1; i >= 0; i--)
      if (c[i] != 0) return c[i] > 0 ? 1 : -1;
    return 0;
  }
};

}  // namespace exact
}  // namespace cpsz
