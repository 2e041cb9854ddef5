// eb_math.cuh -- per-simplex critical-point-preserving error bounds, device side.
//
// These functions reproduce the reference's CPU arithmetic bit for bit; the
// translation unit that includes them is compiled with -fmad=false so that no
// product is fused into a following sum.  Operand types follow the reference
// exactly: float*float products stay float and are widened to double, sums
// run left to right in the declared type, sqrt and division are IEEE
// round-to-nearest (CUDA's default for double, and for float without
// -use_fast_math).  MINF(a,b) = (a<b)?a:b and MAX(a,b) = (a>b)?a:b keep their
// NaN behaviour.
#pragma once

#include <cuda_runtime.h>

namespace cpsz {
namespace dev {

__device__ __forceinline__ double minf_d(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double max_d(double a, double b) { return (a > b) ? a : b; }

// accumulate(): include/sz_cp_preserve_utils.hpp:194-198
__device__ __forceinline__ void acc(double v, double& p, double& n) {
  if (v >= 0) p += v;
  else n += -v;
}

// max_eb_to_keep_sign, degree 1 / 2: include/sz_cp_preserve_utils.hpp:61-92
__device__ __forceinline__ double keep_sign1(double P, double N) {
  if ((N == 0) || (P == 0)) return 1;
  return fabs(P - N) / (P + N);
}
__device__ __forceinline__ double keep_sign2(double positive, double negative) {
  if ((negative == 0) || (positive == 0)) return 1;
  double P = sqrt(positive), N = sqrt(negative);
  return fabs(P - N) / (P + N);
}

// max_eb_to_keep_sign_2d_offline_2 / _4 (T = double):
// src/sz_compress_cp_preserve_2d.cpp:31-49
__device__ __forceinline__ double off2(double a, double b) {
  double p = 0, n = 0;
  acc(a, p, n);
  acc(b, p, n);
  return keep_sign2(p, n);
}
__device__ __forceinline__ double off4(double a, double b, double c, double d) {
  double p = 0, n = 0;
  acc(a, p, n);
  acc(b, p, n);
  acc(c, p, n);
  acc(d, p, n);
  return keep_sign2(p, n);
}

// max_eb_to_keep_sign_det2x2<float>: src/sz_compress_cp_preserve_2d.cpp:18-29
__device__ __forceinline__ double keep_sign_det2x2(float u0, float u1, float u2, float v0, float v1, float v2) {
  double p = 0, n = 0;
  acc((double)(u0 * v1), p, n);
  acc((double)(-u0 * v2), p, n);
  acc((double)(u1 * v2), p, n);
  acc((double)(-u1 * v0), p, n);
  acc((double)(u2 * v0), p, n);
  acc((double)(-u2 * v1), p, n);
  return keep_sign2(p, n);
}

// max_eb_to_keep_sign_eigen_delta_2<float>: src/sz_compress_cp_preserve_2d.cpp:79-123.
// The triangle coordinates are compile-time constants of the two triangle
// kinds; the adjugate entries c[] are passed precomputed (float, exactly as
// get_adjugate_matrix_for_position produces them, including signed zeros).
static __device__ __noinline__ double keep_sign_eigen(float u0, float u1, float u2, float v0, float v1, float v2, float c0,
                                               float c1, float c2, float c3) {
  double eb;
  {
    double p = 0, n = 0;
    acc((double)(c0 * u0), p, n);
    acc((double)(c1 * u1), p, n);
    acc((double)(-(c0 + c1) * u2), p, n);
    acc((double)(c2 * v0), p, n);
    acc((double)(c3 * v1), p, n);
    acc((double)(-(c2 + c3) * v2), p, n);
    eb = keep_sign1(p, n);
    eb = minf_d(eb, keep_sign_det2x2(u0, u1, u2, v0, v1, v2));
  }
  float m = c1 * c2 - c0 * c3;
  float C = (-m) * (u0 * v1 - u0 * v2 + u1 * v2 - u1 * v0 + u2 * v0 - u2 * v1);
  if (C == 0) return 0;
  if (C < 0) return eb;
  float co[6];
  co[0] = c0 * u0;
  co[1] = c1 * u1;
  co[2] = -(c1 + c0) * u2;
  co[3] = c2 * v0;
  co[4] = c3 * v1;
  co[5] = -(c3 + c2) * v2;
  double p = 0, n = 0;
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) acc((double)(co[i] * co[j]), p, n);
  acc((double)(-4 * m * u1 * v0), p, n);
  acc((double)(4 * m * u2 * v0), p, n);
  acc((double)(4 * m * u0 * v1), p, n);
  acc((double)(-4 * m * u2 * v1), p, n);
  acc((double)(-4 * m * u0 * v2), p, n);
  acc((double)(4 * m * u1 * v2), p, n);
  return minf_d(eb, keep_sign2(p, n));
}

// Adjugate of the triangle coordinate matrix (get_adjugate_matrix_for_position,
// src/sz_compress_cp_preserve_2d.cpp:55-63) for the reversed coordinates the
// offline loop passes (:204-206), evaluated in float.
__device__ __forceinline__ void adjugate(float x0, float x1, float x2, float y0, float y1, float y2, float c[4]) {
  float det = (x0 - x2) * (y1 - y2) - (x1 - x2) * (y0 - y2);
  c[0] = (y1 - y2) / det;
  c[1] = -(y0 - y2) / det;
  c[2] = -(x1 - x2) / det;
  c[3] = (x0 - x2) / det;
}

// (det / x >= 1) of the reference for det != 0, decided exactly without a
// division: the rounded quotient is >= 1 iff the exact one is >= 1 - 2^-54
// (the midpoint below 1, which rounds to the even neighbour 1).
__device__ __forceinline__ bool quotient_at_least_one(double det, double x) {
  if (!isfinite(det) || !isfinite(x)) return det / x >= 1;
  if (x == 0) return signbit(x) ? det < 0 : det > 0;  // det / (+-0) = +-inf
  if ((det < 0) != (x < 0)) return false;
  const double a = fabs(det), b = fabs(x);
  if (a >= b) return true;
  if (a < 0.5 * b) return false;
  // b/2 <= a < b: b - a is exact (Sterbenz), and so is the scaling by 2^54
  return (b - a) * 18014398509481984.0 <= b;
}

// max_eb_to_keep_position_and_type<float>: src/sz_compress_cp_preserve_2d.cpp:125-172.
// kind 0 = "upper" triangle X = {{0,0},{1,0},{1,1}}, kind 1 = "lower"
// X = {{0,0},{0,1},{1,1}}, passed as x = X[.][1], y = X[.][0].
__device__ __forceinline__ double tri_eb(float u0, float u1, float u2, float v0, float v1, float v2, int kind) {
  double u0v1 = (double)(u0 * v1);
  double u1v0 = (double)(u1 * v0);
  double u0v2 = (double)(u0 * v2);
  double u2v0 = (double)(u2 * v0);
  double u1v2 = (double)(u1 * v2);
  double u2v1 = (double)(u2 * v1);
  double det = u0v1 - u1v0 + u1v2 - u2v1 + u2v0 - u0v2;
  double eb = 0;
  if (det != 0) {
    bool f1 = quotient_at_least_one(det, u2v0 - u0v2);
    bool f2 = quotient_at_least_one(det, u1v2 - u2v1);
    bool f3 = quotient_at_least_one(det, u0v1 - u1v0);
    if (f1 && f2 && f3) {
      double eb1 = minf_d(off2(u2v0, -u0v2), off4(u0v1, -u1v0, u1v2, -u2v1));
      double eb2 = minf_d(off2(u1v2, -u2v1), off4(u0v1, -u1v0, u2v0, -u0v2));
      double eb3 = minf_d(off2(u0v1, -u1v0), off4(u1v2, -u2v1, u2v0, -u0v2));
      float c[4];
      if (kind == 0) adjugate(0.f, 0.f, 1.f, 0.f, 1.f, 1.f, c);
      else adjugate(0.f, 1.f, 1.f, 0.f, 0.f, 1.f, c);
      double eb4 = minf_d(eb3, keep_sign_eigen(u0, u1, u2, v0, v1, v2, c[0], c[1], c[2], c[3]));
      eb = minf_d(eb1, eb2);
      eb = minf_d(eb, eb4);
    } else if (isfinite(u0v1) && isfinite(u1v0) && isfinite(u0v2) && isfinite(u2v0) && isfinite(u1v2) &&
               isfinite(u2v1)) {
      // All products finite: every keep-sign bound is a finite non-negative
      // double, MAX / MINF are plain max / min, and a flag whose first bound
      // cannot raise eb leaves it unchanged without its second bound.
      eb = 0;
      if (!f1) {
        const double e1 = off2(u2v0, -u0v2);
        if (e1 > eb) eb = max_d(eb, minf_d(e1, off4(u0v1, -u1v0, u1v2, -u2v1)));
      }
      if (!f2) {
        const double e1 = off2(u1v2, -u2v1);
        if (e1 > eb) eb = max_d(eb, minf_d(e1, off4(u0v1, -u1v0, u2v0, -u0v2)));
      }
      if (!f3) {
        const double e1 = off2(u0v1, -u1v0);
        if (e1 > eb) eb = max_d(eb, minf_d(e1, off4(u1v2, -u2v1, u2v0, -u0v2)));
      }
    } else {
      eb = 0;
      if (!f1) eb = max_d(eb, minf_d(off2(u2v0, -u0v2), off4(u0v1, -u1v0, u1v2, -u2v1)));
      if (!f2) eb = max_d(eb, minf_d(off2(u1v2, -u2v1), off4(u0v1, -u1v0, u2v0, -u0v2)));
      if (!f3) eb = max_d(eb, minf_d(off2(u0v1, -u1v0), off4(u1v2, -u2v1, u2v0, -u0v2)));
    }
  }
  return eb;
}

static __device__ __noinline__ double tri_eb_exact(float u0, float u1, float u2, float v0, float v1, float v2,
                                                   int kind) {
  return tri_eb(u0, u1, u2, v0, v1, v2, kind);
}

// ---- approximate float operations of the filtered bounds -----------------------
// (error maxima measured exhaustively on the device by selfcheck.cu)
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// ---- float-filtered 2D bound ------------------------------------------------------
// The compression path's triangle bound in single precision, for the
// ordinary triangles: no critical point, every quantity finite and away from
// the degenerate cases.  It returns false for the others, which take the
// exact double path.  Every quantity below is a function of the six float
// products p_ij = u_i * v_j, which the reference itself forms in float (its
// products are float*float; src/sz_compress_cp_preserve_2d.cpp:128-133), so
// they are the reference's values exactly.  Write S = sum |p|, u = 2^-24.
//
//  * exact differences.  x1 = p20 - p02, x2 = p12 - p21, x3 = p01 - p10 (the
//    reference's denominators) are formed with their rounding errors
//    (Knuth's two-sum: x_k + e_k is the difference exactly), and so are
//    s1 = x2 + x3, s2 = x1 + x3, s3 = x1 + x2 and det = x1 + x2 + x3: each is a
//    float within 2u of its exact value, relative (the error terms are
//    summed in float, at most u^2 S off).
//  * flags.  In real arithmetic det / x_k >= 1 iff s_k = det - x_k and x_k
//    have the same sign (or s_k = 0).  The reference evaluates det and x_k in
//    double (errors below 5 * 2^-53 S) and the quotient rounded; with the
//    margin T = 2^-44 S, when |s_k| > T, x_k != 0 and |det| > T the
//    reference's flag equals (sign s_k == sign x_k) and its det is not zero.
//    Otherwise, and when all three flags hold (a critical point), the
//    triangle is exact.
//  * bounds.  keep_sign2(P, N) = |sqrt P - sqrt N| / (sqrt P + sqrt N) =
//    |P - N| / (sqrt P + sqrt N)^2 (1 when P or N is 0), P and N the sums of
//    the positive / negated negative terms.  Its numerator P - N is one of the
//    accurate values above: x_k for the two-term bounds, s_k for the
//    four-term ones (p01 - p10 + p12 - p21 = x3 + x2, and so on).  The
//    denominator d = P + N + 2 sqrt(P N) comes from float sums of the terms
//    (3u relative each) and sqrt.approx: within 2^-20 relative.  Each value
//    is |D| times rcp.approx(d) (at most 9.9e-8 relative on these operands,
//    measured with the other premises) rounded once: within 2^-19.6 of the
//    real one.  The triangle's bound is the max over failing flags of the
//    min of two such values, both exact, so it too is within 2^-19.6 of the
//    real value's; the result t is within 2^-18 t of the real value, and the
//    reference's double value within 2^-50 r + 2^-52 of it; the enclosure
//    uses 2^-16 relative and 2^-40 absolute.
//  * range.  Exact path when S is not finite, S > 2^40 or S < 2^-60, or a
//    product P N is below 2^-110 and not 0 (sqrt of a subnormal product).
constexpr float FFILT_REL = 1.0f / 65536.0f;           // 2^-16
constexpr float FFILT_ABS = 9.09494702e-13f;           // 2^-40

__device__ __forceinline__ float pos_part(float t) { return t > 0.f ? t : 0.f; }
__device__ __forceinline__ float neg_part(float t) { return t < 0.f ? -t : 0.f; }

// ---- both triangles of a cell at once --------------------------------------------
// Cell (a, b) of the grid holds the "upper" triangle {(a,b), (a+1,b), (a+1,b+1)}
// and the "lower" one {(a,b), (a,b+1), (a+1,b+1)}: vertices 0 and 2 are
// shared, so p02, p20, x1 and the two-term bound of x1 are the same for both.
// cell_eb_float runs the filter above for the two triangles together, the
// upper one in the low word and the lower one in the high word of packed
// f32x2 operands: add / sub / mul.rn.f32x2 round each word exactly as the
// scalar instruction does, so every quantity is the one-triangle filter's
// (the two-sum error of a difference a - c is formed as (a - (s - bb)) -
// (c + bb), the scalar two_sum(a, -c)'s value up to the sign of a zero, which
// no later decision sees: a sum that is exactly zero fails its |.| > T test
// either way).  One instruction issue covers both words; comparisons and
// selects act on each word.
typedef unsigned long long f32x2;  // low word .x (upper triangle), high word .y (lower)
__device__ __forceinline__ f32x2 pk2(float x, float y) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void unpk2(f32x2 r, float& x, float& y) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(r));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 c;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(c) : "l"(a), "l"(b));
  return c;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 c;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(c) : "l"(a), "l"(b));
  return c;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 c;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(c) : "l"(a), "l"(b));
  return c;
}
// a + b = s + e exactly, word by word
__device__ __forceinline__ void two_sum2(f32x2 a, f32x2 b, f32x2& s, f32x2& e) {
  s = add2(a, b);
  const f32x2 bb = sub2(s, a);
  e = add2(sub2(a, sub2(s, bb)), sub2(b, bb));
}
// a - c = s + e exactly, word by word
__device__ __forceinline__ void two_diff2(f32x2 a, f32x2 c, f32x2& s, f32x2& e) {
  s = sub2(a, c);
  const f32x2 bb = sub2(s, a);
  e = sub2(sub2(a, sub2(s, bb)), add2(c, bb));
}
// keep_sign2 of both words: 1 where P or N is 0, else +-|D| / d with
// d = (P + N) + 2 sqrt(P N) (PpN = P + N) as D * rcp.approx(d); the sign is
// D's (callers take |.|)
__device__ __forceinline__ f32x2 ks2_val2(f32x2 D, f32x2 P, f32x2 N, f32x2 PpN, bool& bad_x, bool& bad_y) {
  const f32x2 pn = mul2(P, N);
  float P0, P1, N0, N1, q0, q1;
  unpk2(P, P0, P1);
  unpk2(N, N0, N1);
  unpk2(pn, q0, q1);
  const bool one0 = P0 == 0.f || N0 == 0.f, one1 = P1 == 0.f || N1 == 0.f;
  bad_x |= !one0 && !(q0 >= 1.2924697e-33f);  // 2^-110
  bad_y |= !one1 && !(q1 >= 1.2924697e-33f);
  const f32x2 sq = pk2(sqrt_approx(q0), sqrt_approx(q1));
  float d0, d1, v0, v1;
  unpk2(add2(PpN, add2(sq, sq)), d0, d1);
  unpk2(mul2(D, pk2(rcp_approx(d0), rcp_approx(d1))), v0, v1);
  return pk2(one0 ? 1.f : v0, one1 ? 1.f : v1);
}
__device__ __forceinline__ f32x2 pos2(f32x2 t) {
  float a, b;
  unpk2(t, a, b);
  return pk2(pos_part(a), pos_part(b));
}
__device__ __forceinline__ f32x2 neg2(f32x2 t) {
  float a, b;
  unpk2(t, a, b);
  return pk2(neg_part(a), neg_part(b));
}
// The float bounds of the cell's upper (t_up) and lower (t_lo) triangles, with
// ok_* false for a triangle that takes the exact path.  Vertices: U00 = (a,b),
// U10 = (a+1,b), U01 = (a,b+1), U11 = (a+1,b+1); the upper triangle is
// (U00, U10, U11), the lower (U00, U01, U11) -- tri_eb's (u0, u1, u2).
//
// Sums of parts.  Every bound's P and N are sums of the positive / negated
// negative parts of two or four of the terms (p20, -p02), (p12, -p21),
// (p01, -p10), whose pairs give P_k = pos(a) + neg(c), N_k = neg(a) + pos(c)
// for edge k = (a, -c): the two-term bound of x_k uses P_k, N_k, the
// four-term bound of s_k = x_i + x_j uses P_i + P_j, N_i + N_j, and
// S = (PN_1 + PN_2) + PN_3 with PN_k = P_k + N_k = |a| + |c|.  Summed in
// pairs, each is within 2u of its exact value (the filter allows 3u).
__device__ __forceinline__ void cell_eb_float(float U00, float U10, float U01, float U11, float V00, float V10,
                                              float V01, float V11, float& t_up, float& t_lo, bool& ok_up,
                                              bool& ok_lo) {
  const f32x2 u0 = pk2(U00, U00), u1 = pk2(U10, U01), u2 = pk2(U11, U11);
  const f32x2 v0 = pk2(V00, V00), v1 = pk2(V10, V01), v2 = pk2(V11, V11);
  const f32x2 p01 = mul2(u0, v1), p10 = mul2(u1, v0), p02 = mul2(u0, v2), p20 = mul2(u2, v0), p12 = mul2(u1, v2),
              p21 = mul2(u2, v1);
  f32x2 x1, e1, x2, e2, x3, e3;
  two_diff2(p20, p02, x1, e1);
  two_diff2(p12, p21, x2, e2);
  two_diff2(p01, p10, x3, e3);
  f32x2 h1, g1, h2, g2, h3, g3, hd, gd;
  two_sum2(x2, x3, h1, g1);
  two_sum2(x1, x3, h2, g2);
  two_sum2(x1, x2, h3, g3);
  two_sum2(h1, x1, hd, gd);
  const f32x2 e12 = add2(e1, e2);
  const f32x2 s1 = add2(h1, add2(g1, add2(e2, e3)));
  const f32x2 s2 = add2(h2, add2(g2, add2(e1, e3)));
  const f32x2 s3 = add2(h3, add2(g3, e12));
  const f32x2 det = add2(hd, add2(gd, add2(g1, add2(e12, e3))));
  const f32x2 P1 = add2(pos2(p20), neg2(p02)), N1 = add2(neg2(p20), pos2(p02));
  const f32x2 P2 = add2(pos2(p12), neg2(p21)), N2 = add2(neg2(p12), pos2(p21));
  const f32x2 P3 = add2(pos2(p01), neg2(p10)), N3 = add2(neg2(p01), pos2(p10));
  const f32x2 PN1 = add2(P1, N1), PN2 = add2(P2, N2), PN3 = add2(P3, N3);
  float S[2], X1[2], X2[2], X3[2], S1[2], S2[2], S3[2], DT[2];
  unpk2(add2(add2(PN1, PN2), PN3), S[0], S[1]);
  unpk2(x1, X1[0], X1[1]);
  unpk2(x2, X2[0], X2[1]);
  unpk2(x3, X3[0], X3[1]);
  unpk2(s1, S1[0], S1[1]);
  unpk2(s2, S2[0], S2[1]);
  unpk2(s3, S3[0], S3[1]);
  unpk2(det, DT[0], DT[1]);
  bool bad[2], f1[2], f2[2], f3[2];
#pragma unroll
  for (int w = 0; w < 2; w++) {
    // x1 is bitwise the same in both words: word 0's serves both
    const float T = S[w] * 5.68434189e-14f;  // 2^-44
    bool b = !(S[w] >= 8.67361738e-19f && S[w] <= 1.09951163e12f);  // [2^-60, 2^40], false for NaN
    b |= !(fabsf(S1[w]) > T && fabsf(S2[w]) > T && fabsf(S3[w]) > T && fabsf(DT[w]) > T);
    b |= X1[0] == 0.f || X2[w] == 0.f || X3[w] == 0.f;
    f1[w] = (S1[w] > 0.f) == (X1[0] > 0.f);
    f2[w] = (S2[w] > 0.f) == (X2[w] > 0.f);
    f3[w] = (S3[w] > 0.f) == (X3[w] > 0.f);
    bad[w] = b || (f1[w] && f2[w] && f3[w]);  // a critical point: exact path
  }
  // max over failing flags of min(two-term, four-term bound), all three
  // evaluated (no divergence); the two-term bound of x1 is the same for both
  // triangles and is evaluated once
  float k1;
  {
    float P1w, N1w, PN1w, unused;
    unpk2(P1, P1w, unused);
    unpk2(N1, N1w, unused);
    unpk2(PN1, PN1w, unused);
    const bool one = P1w == 0.f || N1w == 0.f;
    const float q = P1w * N1w;
    const bool b1 = !one && !(q >= 1.2924697e-33f);  // 2^-110
    bad[0] |= b1;
    bad[1] |= b1;
    k1 = one ? 1.f : X1[0] * rcp_approx(PN1w + 2.f * sqrt_approx(q));
  }
  float a1[2], a2[2], a3[2], b2[2], b3[2];
  unpk2(ks2_val2(s1, add2(P2, P3), add2(N2, N3), add2(PN2, PN3), bad[0], bad[1]), a1[0], a1[1]);
  unpk2(ks2_val2(x2, P2, N2, PN2, bad[0], bad[1]), a2[0], a2[1]);
  unpk2(ks2_val2(s2, add2(P1, P3), add2(N1, N3), add2(PN1, PN3), bad[0], bad[1]), b2[0], b2[1]);
  unpk2(ks2_val2(x3, P3, N3, PN3, bad[0], bad[1]), a3[0], a3[1]);
  unpk2(ks2_val2(s3, add2(P1, P2), add2(N1, N2), add2(PN1, PN2), bad[0], bad[1]), b3[0], b3[1]);
  float t[2];
#pragma unroll
  for (int w = 0; w < 2; w++) {
    float e = 0.f;
    if (!f1[w]) e = fmaxf(e, fminf(fabsf(k1), fabsf(a1[w])));
    if (!f2[w]) e = fmaxf(e, fminf(fabsf(a2[w]), fabsf(b2[w])));
    if (!f3[w]) e = fmaxf(e, fminf(fabsf(a3[w]), fabsf(b3[w])));
    t[w] = e;
  }
  t_up = t[0];
  t_lo = t[1];
  ok_up = !bad[0];
  ok_lo = !bad[1];
}

// ---- 3D (src/sz_compress_cp_preserve_3d.cpp:266-358) --------------------------

// acbrt1: include/sz_cp_preserve_utils.hpp:173-184 (the reference's own
// bit-level initial guess and two float Newton steps).
__device__ __forceinline__ float acbrt1(float x0) {
  int ix = __float_as_int(x0);
  ix = ix / 4 + ix / 16;
  ix = ix + ix / 16;
  ix = ix + ix / 256;
  ix = 0x2a5137a0 + ix;
  float x = __int_as_float(ix);
  x = 0.33333333f * (2.0f * x + x0 / (x * x));
  x = 0.33333333f * (2.0f * x + x0 / (x * x));
  return x;
}

__device__ __forceinline__ float keep_sign_3d(float positive, float negative) {
  if (positive == 0 && negative == 0) return 0;
  float P = acbrt1(positive), N = acbrt1(negative);
  return fabsf(P - N) / (P + N);
}

// acbrt1 for x0 >= +0 (finite or not): the bit pattern is a non-negative int,
// for which the divisions by 4, 16 and 256 are exact right shifts.
__device__ __forceinline__ float acbrt1_nonneg(float x0) {
  int ix = __float_as_int(x0);
  ix = (ix >> 2) + (ix >> 4);
  ix = ix + (ix >> 4);
  ix = ix + (ix >> 8);
  ix = 0x2a5137a0 + ix;
  float x = __int_as_float(ix);
  x = 0.33333333f * (2.0f * x + x0 / (x * x));
  x = 0.33333333f * (2.0f * x + x0 / (x * x));
  return x;
}
// keep_sign_3d for non-negative arguments (every sum of magnitudes)
__device__ __forceinline__ float keep_sign_3d_nonneg(float positive, float negative) {
  if (positive == 0 && negative == 0) return 0;
  float P = acbrt1_nonneg(positive), N = acbrt1_nonneg(negative);
  return fabsf(P - N) / (P + N);
}

// ---- filtered 3D sign-keeping bounds -----------------------------------------
// A tet's bound with finite magnitudes is max over the unflagged minors i of
// min(K(p_i, n_i), K(sp_i, sn_i)), K = keep_sign_3d: one of its (up to) 8
// values.  Each K gets a cheap enclosure [k~ - DELTA, k~ + DELTA]; only the
// values the enclosures cannot rule out are computed exactly (one per tet
// in 97 % of the tets of a smooth field, against seven), and the result is
// the reference's float.
//
// Enclosure.  For normal P, N > 0 write c = acbrt1 = cbrt (1 + e); over every
// normal float e lies in [-7.14e-8, 1.21e-6] (checked exhaustively against a
// double cube root), so l = ln(c(P) / c(N)) = ln(P / N) / 3 + ln(1 + e_P) -
// ln(1 + e_N) is within 1.28e-6 of ln(P / N) / 3.  The exact-arithmetic
// value |c(P) - c(N)| / (c(P) + c(N)) is tanh(|l| / 2), whose slope in l is
// (1 - K^2) / 2 <= 1/2; the reference's float evaluation (difference, sum,
// quotient) adds at most 3u (u = 2^-24).  The approximation: r = min / max
// (rcp.approx and a product), d = |lg2(r)| (lg2.approx), s = 2^(-d / 3)
// (a product by -1/3 and ex2.approx), k~ = (1 - s) / (1 + s) (rcp.approx).
// Exhaustive maxima of the .ftz.f32 approximations over the inputs they get
// here: rcp relative 9.9e-8 on all normal floats below 2^126; ex2 relative
// 1.44e-7 on [-87, 0]; lg2 absolute, per binade of r, 1.6e-7 on [1, 2),
// 2.2e-7 on [1/2, 1), 2.7e-7 on [1/4, 1/2), then about one ulp of the result
// (3.9e-7 on [2^-4, 2^-2), 6.3e-7 down to 2^-8, ..., 7.8e-6 below 2^-64).
// Distance of k~ to the exact-arithmetic value, term by term: 6.4e-7 (the
// cube roots, above); (ln 2 / 6) (1 - K^2) (2.3e-7 + lg2 error) for r and
// d, at most 8.1e-8 (on [2^-5, 2^-4)) since 1 - K^2 <= 4 s / (1 + s)^2
// falls faster than the lg2 error grows; 4.0e-8 (the product by -1/3, also
// damped); 7.2e-8 (ex2, through the slope 2 s / (1 + s)^2 <= 1/2); 3u +
// 9.9e-8 (the last three operations).  With the reference's 3u: 1.29e-6 in
// all, below DELTA less the rounding of k~ +- DELTA (6e-8).
//
// Other operands.  A ratio below 2^-126 flushes to 0 and gives k~ = 1; the
// cube roots then differ by a factor above 2^41, and K is 1 exactly.  Both
// zero: k~ = 0 = K.  One zero and the other >= 2^-60: k~ = 1 (r = 0) and K
// >= 1 - 2 acbrt1(0) / acbrt1(2^-60) - 3u > 1 - 4e-7.  No enclosure (the
// value is always computed exactly): a subnormal operand, a zero beside a
// value below 2^-60, and a larger operand >= 2^126 (its rcp.approx flushes).
constexpr float KS3_DELTA = 1.5e-6f;

__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// Enclosure [lo, hi] of keep_sign_3d(P, N) for finite P, N >= 0 ([-1, 2]
// where there is none: every K lies in [0, 1]).  On non-negative floats the
// order of the bit patterns is the order of the values.
__device__ __forceinline__ void ks3_enclose(float P, float N, float& lo, float& hi) {
  const unsigned bp = __float_as_uint(P), bn = __float_as_uint(N);
  const unsigned mn = umin(bp, bn), mx = umax(bp, bn);
  const float r = __uint_as_float(mn) * rcp_approx(__uint_as_float(mx));
  const float d = fabsf(lg2_approx(r));
  const float s = ex2_approx(d * -0.333333343f);
  const float k = mx == 0u ? 0.f : (1.f - s) * rcp_approx(1.f + s);
  const bool known = (mn >= 0x00800000u && mx < 0x7e800000u) || (mn == 0u && (mx == 0u || mx >= (67u << 23)));
  lo = known ? k - KS3_DELTA : -1.f;
  hi = known ? k + KS3_DELTA : 2.f;
}

__device__ __forceinline__ int sgnf(float v) { return (0.0f < v) - (v < 0.0f); }
__device__ __forceinline__ bool same_direction(float a, float b, float c, float d) {
  int s = sgnf(a);
  if (s == 0) return false;
  return (s == sgnf(b)) && (s == sgnf(c)) && (s == sgnf(d));
}

__device__ __forceinline__ float maxf_(float a, float b) { return (a > b) ? a : b; }
__device__ __forceinline__ float minf_(float a, float b) { return (a < b) ? a : b; }

// (M / Mi > 1) of the reference for nonzero doubles M, Mi, decided exactly
// without a division: the rounded quotient exceeds 1 iff the exact one
// exceeds 1 + 2^-53 (1 + 2^-53 itself rounds to the even neighbour 1).
__device__ __forceinline__ bool quotient_above_one(double M, double Mi) {
  if (!isfinite(M) || !isfinite(Mi)) return M / Mi > 1;
  if ((M < 0) != (Mi < 0)) return false;
  const double a = fabs(M), b = fabs(Mi);
  if (a > 2.0 * b) return true;
  if (a < b) return false;
  // b <= a <= 2b: a - b is exact (Sterbenz), and so is the scaling by 2^53
  return (a - b) * 9007199254740992.0 > b;
}

static __device__ __forceinline__ double tet_eb(float u0, float u1, float u2, float u3, float v0, float v1, float v2, float v3,
                                      float w0, float w1, float w2, float w3) {
  double u3v1w2 = u3 * v1 * w2, u3v2w1 = u3 * v2 * w1, u3v2w0 = u3 * v2 * w0, u3v0w2 = u3 * v0 * w2,
         u3v0w1 = u3 * v0 * w1, u3v1w0 = u3 * v1 * w0;
  double u1v3w2 = u1 * v3 * w2, u2v3w1 = u2 * v3 * w1, u2v3w0 = u2 * v3 * w0, u0v3w2 = u0 * v3 * w2,
         u0v3w1 = u0 * v3 * w1, u1v3w0 = u1 * v3 * w0;
  double u1v2w3 = u1 * v2 * w3, u2v1w3 = u2 * v1 * w3, u0v2w3 = u0 * v2 * w3, u2v0w3 = u2 * v0 * w3,
         u0v1w3 = u0 * v1 * w3, u1v0w3 = u1 * v0 * w3;
  double u0v1w2 = u0 * v1 * w2, u0v2w1 = u0 * v2 * w1, u1v2w0 = u1 * v2 * w0, u1v0w2 = u1 * v0 * w2,
         u2v0w1 = u2 * v0 * w1, u2v1w0 = u2 * v1 * w0;
  double u3_0 = -u3v1w2 + u3v2w1, u3_1 = -u3v2w0 + u3v0w2, u3_2 = -u3v0w1 + u3v1w0;
  double v3_0 = u1v3w2 - u2v3w1, v3_1 = u2v3w0 - u0v3w2, v3_2 = u0v3w1 - u1v3w0;
  double w3_0 = -u1v2w3 + u2v1w3, w3_1 = u0v2w3 - u2v0w3, w3_2 = -u0v1w3 + u1v0w3;
  double c_4 = u0v1w2 - u0v2w1 + u1v2w0 - u1v0w2 + u2v0w1 - u2v1w0;
  double M0 = u3_0 + v3_0 + w3_0;
  double M1 = u3_1 + v3_1 + w3_1;
  double M2 = u3_2 + v3_2 + w3_2;
  double M3 = c_4;
  double M = M0 + M1 + M2 + M3;
  if (M == 0) return 0;
  bool flag0 = (M0 == 0) || quotient_above_one(M, M0);
  bool flag1 = (M1 == 0) || quotient_above_one(M, M1);
  bool flag2 = (M2 == 0) || quotient_above_one(M, M2);
  bool flag3 = (M3 == 0) || quotient_above_one(M, M3);
  if (flag0 && flag1 && flag2 && flag3) {
    if (same_direction(u0, u1, u2, u3) || same_direction(v0, v1, v2, v3) || same_direction(w0, w1, w2, w3)) return 1;
    return 0;
  }
  float eb = 0;
  double pm0 = 0, nm0 = 0, pm1 = 0, nm1 = 0, pm2 = 0, nm2 = 0, pm3 = 0, nm3 = 0;
  acc(-u3v1w2, pm0, nm0); acc(u3v2w1, pm0, nm0); acc(u1v3w2, pm0, nm0);
  acc(-u2v3w1, pm0, nm0); acc(-u1v2w3, pm0, nm0); acc(u2v1w3, pm0, nm0);
  acc(-u3v2w0, pm1, nm1); acc(u3v0w2, pm1, nm1); acc(u2v3w0, pm1, nm1);
  acc(-u0v3w2, pm1, nm1); acc(u0v2w3, pm1, nm1); acc(-u2v0w3, pm1, nm1);
  acc(-u3v0w1, pm2, nm2); acc(u3v1w0, pm2, nm2); acc(u0v3w1, pm2, nm2);
  acc(-u1v3w0, pm2, nm2); acc(-u0v1w3, pm2, nm2); acc(u1v0w3, pm2, nm2);
  acc(u0v1w2, pm3, nm3); acc(-u0v2w1, pm3, nm3); acc(u1v2w0, pm3, nm3);
  acc(-u1v0w2, pm3, nm3); acc(u2v0w1, pm3, nm3); acc(-u2v1w0, pm3, nm3);
  float p_m0 = (float)pm0, p_m1 = (float)pm1, p_m2 = (float)pm2, p_m3 = (float)pm3;
  float n_m0 = (float)nm0, n_m1 = (float)nm1, n_m2 = (float)nm2, n_m3 = (float)nm3;
  // the "other three minors" sums, in the reference's left-to-right order
  const float sp0 = p_m1 + p_m2 + p_m3, sn0 = n_m1 + n_m2 + n_m3;
  const float sp1 = p_m0 + p_m2 + p_m3, sn1 = n_m0 + n_m2 + n_m3;
  const float sp2 = p_m0 + p_m1 + p_m3, sn2 = n_m0 + n_m1 + n_m3;
  const float sp3 = p_m0 + p_m1 + p_m2, sn3 = n_m0 + n_m1 + n_m2;
  if (isfinite(sp0) && isfinite(sp1) && isfinite(sp2) && isfinite(sp3) && isfinite(sn0) && isfinite(sn1) &&
      isfinite(sn2) && isfinite(sn3)) {
    // Every magnitude is finite (each appears in three of the sums), so every
    // keep_sign_3d value is a finite float in [0, 1] and MAX/MINF are plain
    // max/min: eb = max(0, max over unflagged i of min(A_i, B_i)), A_i =
    // K(p_i, n_i), B_i = K(sp_i, sn_i).  With enclosures of all eight
    // values, a minor whose min cannot reach the largest lower bound of a
    // min is dropped, and of a kept minor only a value that can be its min
    // is computed (value 2i + side is bit 2i + side of `need`).
    float lo[8], hi[8];
    ks3_enclose(p_m0, n_m0, lo[0], hi[0]);
    ks3_enclose(sp0, sn0, lo[1], hi[1]);
    ks3_enclose(p_m1, n_m1, lo[2], hi[2]);
    ks3_enclose(sp1, sn1, lo[3], hi[3]);
    ks3_enclose(p_m2, n_m2, lo[4], hi[4]);
    ks3_enclose(sp2, sn2, lo[5], hi[5]);
    ks3_enclose(p_m3, n_m3, lo[6], hi[6]);
    ks3_enclose(sp3, sn3, lo[7], hi[7]);
    const bool unf[4] = {!flag0, !flag1, !flag2, !flag3};
    float LO = -2.f;  // a lower bound of the result
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (unf[i]) LO = fmaxf(LO, fminf(lo[2 * i], lo[2 * i + 1]));
    unsigned need = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      if (!unf[i] || fminf(hi[2 * i], hi[2 * i + 1]) < LO) continue;
      if (lo[2 * i] <= hi[2 * i + 1]) need |= 1u << (2 * i);          // A_i can be the min
      if (lo[2 * i + 1] <= hi[2 * i]) need |= 1u << (2 * i + 1);      // B_i can be the min
    }
    // one exact evaluation per set bit, in ascending order (a minor's two
    // values are adjacent): the min within a minor, the max across minors
    float cur = 0.f;
    int cur_i = -1;
    while (need) {
      const int k = __ffs(need) - 1;
      need &= need - 1;
      const float P = (k & 4) ? ((k & 2) ? ((k & 1) ? sp3 : p_m3) : ((k & 1) ? sp2 : p_m2))
                              : ((k & 2) ? ((k & 1) ? sp1 : p_m1) : ((k & 1) ? sp0 : p_m0));
      const float N = (k & 4) ? ((k & 2) ? ((k & 1) ? sn3 : n_m3) : ((k & 1) ? sn2 : n_m2))
                              : ((k & 2) ? ((k & 1) ? sn1 : n_m1) : ((k & 1) ? sn0 : n_m0));
      const float v = keep_sign_3d_nonneg(P, N);
      if ((k >> 1) != cur_i) {
        eb = maxf_(eb, cur);
        cur = v;
        cur_i = k >> 1;
      } else {
        cur = minf_(cur, v);
      }
    }
    return maxf_(eb, cur);
  }
  if (!flag0) eb = maxf_(eb, minf_(keep_sign_3d(p_m0, n_m0), keep_sign_3d(sp0, sn0)));
  if (!flag1) eb = maxf_(eb, minf_(keep_sign_3d(p_m1, n_m1), keep_sign_3d(sp1, sn1)));
  if (!flag2) eb = maxf_(eb, minf_(keep_sign_3d(p_m2, n_m2), keep_sign_3d(sp2, sn2)));
  if (!flag3) eb = maxf_(eb, minf_(keep_sign_3d(p_m3, n_m3), keep_sign_3d(sp3, sn3)));
  return eb;
}

// Quantized-id lookup against host-computed thresholds t[1..n): the id is the
// number of thresholds <= e.  `guess` starts near the answer; the loops fix it.
// The 2D id of a float x under thresholds t[k] in (the float below 2^(2k-52),
// 2^(2k-52)]: -1 up to thr = 2^-52, else #{k >= 1 : x >= 2^(2k-52)} =
// (exponent(x) + 52) / 2 rounded down.  Floats from FLT_MAX's binade up (inf
// and nan: 90) give ids past the 2D range of 0..88.
__device__ __forceinline__ int pow4_id(float x) {
  if (x <= 2.220446049250313e-16f) return -1;
  const int e = (int)((__float_as_uint(x) >> 23) & 0xff) - 127;
  return (e + 52) >> 1;
}

__device__ __forceinline__ int count_thresholds(const double* t, int n, double e, int guess) {
  int g = guess < 0 ? 0 : (guess > n - 1 ? n - 1 : guess);
  while (g + 1 < n && e >= t[g + 1]) g++;
  while (g > 0 && e < t[g]) g--;
  return g;
}

}  // namespace dev
}  // namespace cpsz
