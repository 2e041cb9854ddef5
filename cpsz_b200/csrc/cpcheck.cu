// cpcheck.cu -- exact critical-point (CP) extraction and comparison.
//
// A cell holds a CP when the origin lies strictly inside the image of the
// cell's vertices in value space (the zero of the piecewise-linear field),
// decided with exact orientation signs.  Ties are broken by Simulation of
// Simplicity: the origin is moved to o = (e, e^2[, e^3]) for an infinitesimal
// e, so a zero on a shared edge or face belongs to exactly one cell.  A
// vertex whose value is exactly zero makes its cells CP-free, as in the
// reference's extraction tools (test/cp_extraction_2d.cpp:63-68,
// test/cp_extraction_3d.cpp:124-126).  Non-finite vertex values also make a
// cell CP-free.
//
// Cell numbering and simplices follow the reference's tools:
//   2D: cell 2*(i*(r2-1)+j)+k; k=0 {(i,j),(i+1,j),(i+1,j+1)} with unit
//       coordinates {(0,0),(0,1),(1,1)}, k=1 {(i,j),(i,j+1),(i+1,j+1)} with
//       {(0,0),(1,0),(1,1)} (test/cp_extraction_2d.cpp:117-147);
//   3D: cell 6*(cube index)+t, cube (i,j,k) of (r1-1)(r2-1)(r3-1), tet t with
//       the corners of test/cp_extraction_3d.cpp:39-77 (coordinates (dk,dj,di)).
// Types (output code = type + 1; 0 = no CP), from the Jacobian J of the
// linear interpolant:
//   2D (test/cp_extraction_2d.cpp:32-38): det J = 0 -> SINGULAR; real
//   eigenvalues (tr^2 - 4 det >= 0): det < 0 SADDLE, else tr < 0 ATTRACTING /
//   tr > 0 REPELLING; complex: tr < 0 ATTRACTING_FOCUS, tr > 0
//   REPELLING_FOCUS, tr = 0 CENTER.
//   3D (test/cp_extraction_3d.cpp:30-38): characteristic polynomial
//   l^3 + a2 l^2 + a1 l + a0 with discriminant d; SINGULAR if a0 = 0 or
//   d = 0; n = roots with negative real part, type = 1 + 2n + (d < 0).  For a
//   complex pair (d < 0) with real root r and real part al: r < 0 iff a0 > 0
//   and al < 0 iff h = a2 a1 - a0 > 0 (h = -2 al ((r + al)^2 + b^2); h = 0 is
//   SINGULAR); for three real roots Descartes' rule of signs counts them.
// Every sign is first taken from interval arithmetic and recomputed with
// exact expansions when the interval straddles zero.
#include "cp_exact.cuh"
#include "kernels.h"

namespace cpsz {

namespace {

using exact::Exp;
using exact::Ival;

// ---- 2D ---------------------------------------------------------------------------

// sign of det[Pa - o, Pb - o] = Dab + e (va - vb) + e^2 (ub - ua)
__device__ __forceinline__ int orient2(float ua, float va, float ub, float vb) {
  const double p = (double)ua * (double)vb, q = (double)ub * (double)va;  // exact
  if (p != q) return p > q ? 1 : -1;
  if (va != vb) return va > vb ? 1 : -1;
  if (ub != ua) return ub > ua ? 1 : -1;
  return 0;
}

__device__ __noinline__ void tri_signs_exact(const float* u, const float* v, int kind, int* s_tr, int* s_det,
                                             int* s_delta) {
  // a = du/dx, b = du/dy, c = dv/dx, d = dv/dy as exact float differences
  const int ax = kind ? 1 : 2, ax0 = kind ? 0 : 1, by = kind ? 2 : 1, by0 = kind ? 1 : 0;
  Exp<4> A, B, C, D;
  A.add(u[ax]);
  A.add(-(double)u[ax0]);
  B.add(u[by]);
  B.add(-(double)u[by0]);
  C.add(v[ax]);
  C.add(-(double)v[ax0]);
  D.add(v[by]);
  D.add(-(double)v[by0]);
  Exp<8> T;
  T.add(A);
  T.add(D);
  Exp<24> Dt;
  Dt.add_product(A, D);
  Dt.add_product(B, C, -1.0);
  Exp<8> E;
  E.add(A);
  E.add(D, -1.0);
  Exp<32> Dl;
  Dl.add_product(E, E);
  Dl.add_product(B, C, 4.0);
  *s_tr = T.sign();
  *s_det = Dt.sign();
  *s_delta = Dl.sign();
}

// Type code (1 + type) of a triangle known to hold a CP.
__device__ int tri_type(const float* u, const float* v, int kind) {
  const int ax = kind ? 1 : 2, ax0 = kind ? 0 : 1, by = kind ? 2 : 1, by0 = kind ? 1 : 0;
  const Ival a = exact::iv_diff(u[ax], u[ax0]), b = exact::iv_diff(u[by], u[by0]);
  const Ival c = exact::iv_diff(v[ax], v[ax0]), d = exact::iv_diff(v[by], v[by0]);
  int s_tr = exact::iv_sign(a + d);
  int s_det = exact::iv_sign(a * d - b * c);
  const Ival e = a - d;
  int s_delta = exact::iv_sign(e * e + exact::scale(b * c, 4.0));
  if (s_tr == 0 || s_det == 0 || s_delta == 0) tri_signs_exact(u, v, kind, &s_tr, &s_det, &s_delta);
  int type;
  if (s_det == 0) type = 0;  // SINGULAR
  else if (s_delta >= 0) type = (s_det < 0) ? 3 : (s_tr < 0 ? 1 : 2);
  else type = (s_tr < 0) ? 4 : (s_tr > 0 ? 5 : 6);
  return type + 1;
}

// 0 = no CP, else 1 + type.  Vertices in the reference's order.
__device__ int tri_cp(const float* u, const float* v, int kind) {
#pragma unroll
  for (int p = 0; p < 3; p++) {
    if (u[p] == 0.f && v[p] == 0.f) return 0;
    if (!isfinite(u[p]) || !isfinite(v[p])) return 0;
  }
  const int s0 = orient2(u[1], v[1], u[2], v[2]);
  const int s1 = orient2(u[2], v[2], u[0], v[0]);
  const int s2 = orient2(u[0], v[0], u[1], v[1]);
  if (s0 == 0 || s0 != s1 || s0 != s2) return 0;
  return tri_type(u, v, kind);
}

struct Tally {
  unsigned long long a = 0, b = 0, diff = 0, type = 0;
};

__device__ __forceinline__ void tally(Tally& t, int ca, int cb, bool with_b) {
  t.a += ca != 0;
  if (with_b) {
    t.b += cb != 0;
    t.diff += (ca != 0) != (cb != 0);
    t.type += (ca != 0) && (cb != 0) && (ca != cb);
  }
}

__device__ void flush(Tally t, unsigned long long* counts) {
  __shared__ unsigned long long red[4];
  if (threadIdx.x < 4) red[threadIdx.x] = 0;
  __syncthreads();
  unsigned long long v[4] = {t.a, t.b, t.diff, t.type};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    unsigned long long x = v[q];
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(&red[q], x);
  }
  __syncthreads();
  if (threadIdx.x < 4 && red[threadIdx.x]) atomicAdd(&counts[threadIdx.x], red[threadIdx.x]);
}

__global__ void __launch_bounds__(256) cp2d_kernel(const float* __restrict__ Ua, const float* __restrict__ Va,
                                                   const float* __restrict__ Ub, const float* __restrict__ Vb, int r1,
                                                   int r2, uint8_t* __restrict__ cells,
                                                   unsigned long long* __restrict__ counts, long long q0) {
  Tally t;
  const long long ncube = (long long)(r1 - 1) * (r2 - 1);
  const bool with_b = Ub != nullptr;
  for (long long q = q0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ncube;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / (r2 - 1)), j = (int)(q - (long long)i * (r2 - 1));
    const size_t p00 = (size_t)i * r2 + j, p10 = p00 + r2, p11 = p10 + 1, p01 = p00 + 1;
    int code[2][2];
    for (int f = 0; f < (with_b ? 2 : 1); f++) {
      const float* U = f ? Ub : Ua;
      const float* V = f ? Vb : Va;
      const float u00 = U[p00], u10 = U[p10], u11 = U[p11], u01 = U[p01];
      const float v00 = V[p00], v10 = V[p10], v11 = V[p11], v01 = V[p01];
      const float uk0[3] = {u00, u10, u11}, vk0[3] = {v00, v10, v11};
      const float uk1[3] = {u00, u01, u11}, vk1[3] = {v00, v01, v11};
      code[f][0] = tri_cp(uk0, vk0, 0);
      code[f][1] = tri_cp(uk1, vk1, 1);
    }
    if (cells) {
      cells[2 * q] = (uint8_t)code[0][0];
      cells[2 * q + 1] = (uint8_t)code[0][1];
    }
    for (int k = 0; k < 2; k++) tally(t, code[0][k], with_b ? code[1][k] : 0, with_b);
  }
  flush(t, counts);
}

// ---- 3D ---------------------------------------------------------------------------

// Corners of the 6 tets as (dk, dj, di); corner 0 is (0,0,0), corner 3 (1,1,1).
__constant__ int8_t c_cp_tet[6][4][3] = {
    {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {1, 1, 1}}, {{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
    {{0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}}, {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {1, 1, 1}},
    {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}}, {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}}};
// Inverses of the edge matrices X_[r][c] = X[c][r] - X[3][r] (integers).
__constant__ int8_t c_cp_xinv[6][3][3] = {
    {{0, 0, -1}, {0, -1, 1}, {-1, 1, 0}}, {{0, -1, 0}, {0, 1, -1}, {-1, 0, 1}},
    {{0, 0, -1}, {-1, 0, 1}, {1, -1, 0}}, {{-1, 0, 0}, {1, 0, -1}, {0, -1, 1}},
    {{0, -1, 0}, {-1, 1, 0}, {1, 0, -1}}, {{-1, 0, 0}, {1, -1, 0}, {0, 1, -1}}};

// exact sign of det[Pa, Pb, Pc] (columns are value triples)
__device__ __noinline__ int det3_exact(const float* a, const float* b, const float* c) {
  Exp<16> e;
  auto term = [&](float x, float y, float z, double s) {
    double p, err;
    exact::two_prod((double)x * (double)y, (double)z, p, err);
    e.add(s * p);
    e.add(s * err);
  };
  term(a[0], b[1], c[2], 1);
  term(a[0], b[2], c[1], -1);
  term(b[0], a[1], c[2], -1);
  term(b[0], a[2], c[1], 1);
  term(c[0], a[1], b[2], 1);
  term(c[0], a[2], b[1], -1);
  return e.sign();
}

// exact sign of a sum of six float*float products given as (x, y, sign) triples
__device__ __noinline__ int cross_sum_sign(const float* x, const float* y, const float* s) {
  Exp<8> e;
  for (int k = 0; k < 6; k++) e.add(s[k] * ((double)x[k] * (double)y[k]));
  return e.sign();
}

// sign of det[Pa - o, Pb - o, Pc - o] = D - e Nx - e^2 Ny - e^3 Nz,
// N = Pb x Pc + Pc x Pa + Pa x Pb
__device__ int orient3(const float* a, const float* b, const float* c) {
  // interval filter on D: each term (x*y exact) * z
  Ival d = exact::iv(0.0);
  auto term = [&](float x, float y, float z, bool neg) {
    const double p = (double)x * (double)y;
    Ival t{exact::mul_dn(p, z), exact::mul_up(p, z)};
    d = neg ? d - t : d + t;
  };
  term(a[0], b[1], c[2], false);
  term(a[0], b[2], c[1], true);
  term(b[0], a[1], c[2], true);
  term(b[0], a[2], c[1], false);
  term(c[0], a[1], b[2], false);
  term(c[0], a[2], b[1], true);
  int s = exact::iv_sign(d);
  if (s == 0) s = det3_exact(a, b, c);
  if (s != 0) return s;
  // N component k: sum over the cyclic pairs (P,Q) of (P x Q)_k
  const float* P[3] = {b, c, a};
  const float* Q[3] = {c, a, b};
  for (int comp = 0; comp < 3; comp++) {
    const int y = (comp + 1) % 3, z = (comp + 2) % 3;
    float xs[6], ys[6], ss[6];
    for (int r = 0; r < 3; r++) {
      xs[2 * r] = P[r][y];
      ys[2 * r] = Q[r][z];
      ss[2 * r] = 1.f;
      xs[2 * r + 1] = P[r][z];
      ys[2 * r + 1] = Q[r][y];
      ss[2 * r + 1] = -1.f;
    }
    const int n = cross_sum_sign(xs, ys, ss);
    if (n != 0) return -n;
  }
  return 0;
}

struct J3 {
  // entry (r, c): sum of up to two float differences, as four floats and signs
  float x[3][3][4];
};

__device__ __noinline__ void tet_signs_exact(const J3& J, int* s_a2, int* s_a1, int* s_a0, int* s_h, int* s_disc) {
  Exp<4> e[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      for (int q = 0; q < 4; q++) e[r][c].add(J.x[r][c][q]);
  Exp<12> tr;  // a2 = -tr
  tr.add(e[0][0]);
  tr.add(e[1][1]);
  tr.add(e[2][2]);
  Exp<24> c2;  // a1: sum of principal 2x2 minors
  c2.add_product(e[0][0], e[1][1]);
  c2.add_product(e[0][1], e[1][0], -1.0);
  c2.add_product(e[0][0], e[2][2]);
  c2.add_product(e[0][2], e[2][0], -1.0);
  c2.add_product(e[1][1], e[2][2]);
  c2.add_product(e[1][2], e[2][1], -1.0);
  Exp<24> m0, m1, m2;  // cofactors of the first row
  m0.add_product(e[1][1], e[2][2]);
  m0.add_product(e[1][2], e[2][1], -1.0);
  m1.add_product(e[1][0], e[2][2]);
  m1.add_product(e[1][2], e[2][0], -1.0);
  m2.add_product(e[1][0], e[2][1]);
  m2.add_product(e[1][1], e[2][0], -1.0);
  Exp<32> det;  // a0 = -det
  det.add_product(e[0][0], m0);
  det.add_product(e[0][1], m1, -1.0);
  det.add_product(e[0][2], m2);
  Exp<12> a2;
  a2.add(tr, -1.0);
  Exp<32> a0;
  a0.add(det, -1.0);
  // h = a2 a1 - a0
  Exp<32> h;
  h.add_product(a2, c2);
  h.add(a0, -1.0);
  // discriminant 18 a2 a1 a0 - 4 a2^3 a0 + a2^2 a1^2 - 4 a1^3 - 27 a0^2
  Exp<32> a2a1;
  a2a1.add_product(a2, c2);
  Exp<24> a2sq;
  a2sq.add_product(a2, a2);
  Exp<32> a1sq;
  a1sq.add_product(c2, c2);
  Exp<40> t1, t2, t3, t4, t5;
  t1.add_product(a2a1, a0);  // x18
  Exp<32> a2cube;
  a2cube.add_product(a2sq, a2);
  t2.add_product(a2cube, a0);  // x(-4)
  t3.add_product(a2sq, a1sq);  // x1
  t4.add_product(a1sq, c2);    // x(-4)
  t5.add_product(a0, a0);      // x(-27)
  Exp<48> disc;
  disc.add_times(t1, 18);
  disc.add_times(t2, 4, -1.0);
  disc.add(t3);
  disc.add_times(t4, 4, -1.0);
  disc.add_times(t5, 27, -1.0);
  *s_a2 = a2.sign();
  *s_a1 = c2.overflow ? 0 : c2.sign();
  *s_a0 = a0.sign();
  *s_h = h.sign();
  // an expansion that outgrew its capacity leaves the sign undecided
  // (classified SINGULAR); none does for float inputs in practice
  *s_disc = (disc.overflow || t1.overflow || t2.overflow || t3.overflow || t4.overflow || t5.overflow) ? 0 : disc.sign();
  if (h.overflow) *s_h = 0;
  if (a0.overflow) *s_a0 = 0;
}

__device__ int tet_type(const float P[4][3], int t) {
  // J = X_^{-1} U_, U_[k][c] = P[c][k] - P[3][k] (test/cp_extraction_3d.cpp:80-95)
  J3 J;
  Ival iJ[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      Ival acc = exact::iv(0.0);
      int q = 0;
      for (int k = 0; k < 3; k++) {
        const int x = c_cp_xinv[t][r][k];
        if (!x) continue;
        const float hi = P[c][k], lo = P[3][k];
        J.x[r][c][q++] = x > 0 ? hi : -hi;
        J.x[r][c][q++] = x > 0 ? -lo : lo;
        const Ival dlt = exact::iv_diff(hi, lo);
        acc = x > 0 ? acc + dlt : acc - dlt;
      }
      for (; q < 4; q++) J.x[r][c][q] = 0.f;
      iJ[r][c] = acc;
    }
  const Ival tr = iJ[0][0] + iJ[1][1] + iJ[2][2];
  const Ival a2 = exact::iv(0.0) - tr;
  const Ival a1 = (iJ[0][0] * iJ[1][1] - iJ[0][1] * iJ[1][0]) + (iJ[0][0] * iJ[2][2] - iJ[0][2] * iJ[2][0]) +
                  (iJ[1][1] * iJ[2][2] - iJ[1][2] * iJ[2][1]);
  const Ival det = iJ[0][0] * (iJ[1][1] * iJ[2][2] - iJ[1][2] * iJ[2][1]) -
                   iJ[0][1] * (iJ[1][0] * iJ[2][2] - iJ[1][2] * iJ[2][0]) +
                   iJ[0][2] * (iJ[1][0] * iJ[2][1] - iJ[1][1] * iJ[2][0]);
  const Ival a0 = exact::iv(0.0) - det;
  const Ival h = a2 * a1 - a0;
  const Ival disc = exact::iv(18.0) * a2 * a1 * a0 - exact::iv(4.0) * a2 * a2 * a2 * a0 + a2 * a2 * a1 * a1 -
                    exact::iv(4.0) * a1 * a1 * a1 - exact::iv(27.0) * a0 * a0;
  int s_a2 = exact::iv_sign(a2), s_a1 = exact::iv_sign(a1), s_a0 = exact::iv_sign(a0), s_h = exact::iv_sign(h),
      s_disc = exact::iv_sign(disc);
  if (!s_a2 || !s_a1 || !s_a0 || !s_h || !s_disc) tet_signs_exact(J, &s_a2, &s_a1, &s_a0, &s_h, &s_disc);
  if (!s_a0 || !s_disc) return 0 + 1;  // SINGULAR
  if (s_disc < 0) {
    if (!s_h) return 0 + 1;
    const int neg = (s_a0 > 0) + 2 * (s_h > 0);
    return 1 + 2 * neg + 1 + 1;
  }
  // three distinct real roots: sign changes of (1, a2, a1, a0), zeros skipped
  int prev = 1, changes = 0;
  const int seq[3] = {s_a2, s_a1, s_a0};
  for (int q = 0; q < 3; q++)
    if (seq[q]) {
      changes += seq[q] != prev;
      prev = seq[q];
    }
  return 1 + 2 * (3 - changes) + 1;
}

// 0 = no CP, else 1 + type.  P: the tet's corners in the reference's order.
__device__ int tet_cp(const float P[4][3], int t) {
  for (int p = 0; p < 4; p++) {
    if (P[p][0] == 0.f && P[p][1] == 0.f && P[p][2] == 0.f) return 0;
    if (!isfinite(P[p][0]) || !isfinite(P[p][1]) || !isfinite(P[p][2])) return 0;
  }
  const int s0 = orient3(P[1], P[2], P[3]);
  if (s0 == 0) return 0;
  const int s1 = -orient3(P[0], P[2], P[3]);
  if (s1 != s0) return 0;
  const int s2 = orient3(P[0], P[1], P[3]);
  if (s2 != s0) return 0;
  const int s3 = -orient3(P[0], P[1], P[2]);
  if (s3 != s0) return 0;
  return tet_type(P, t);
}

__global__ void __launch_bounds__(128) cp3d_kernel(const float* __restrict__ Ua, const float* __restrict__ Va,
                                                   const float* __restrict__ Wa, const float* __restrict__ Ub,
                                                   const float* __restrict__ Vb, const float* __restrict__ Wb, int r1,
                                                   int r2, int r3, uint8_t* __restrict__ cells,
                                                   unsigned long long* __restrict__ counts) {
  Tally tl;
  const long long c1 = r3 - 1, c0 = (long long)(r2 - 1) * (r3 - 1);
  const long long ncube = (long long)(r1 - 1) * c0;
  const bool with_b = Ub != nullptr;
  const size_t d1 = (size_t)r3, d0 = (size_t)r2 * r3;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ncube;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / c0);
    const long long rem = q - i * c0;
    const int j = (int)(rem / c1), k = (int)(rem - j * c1);
    const size_t base = (size_t)i * d0 + (size_t)j * d1 + k;
    float cube[2][8][3];
    for (int f = 0; f < (with_b ? 2 : 1); f++) {
      const float* U = f ? Ub : Ua;
      const float* V = f ? Vb : Va;
      const float* W = f ? Wb : Wa;
      for (int c = 0; c < 8; c++) {
        const size_t at = base + (size_t)((c >> 2) & 1) * d0 + (size_t)((c >> 1) & 1) * d1 + (c & 1);
        cube[f][c][0] = U[at];
        cube[f][c][1] = V[at];
        cube[f][c][2] = W[at];
      }
    }
    for (int t = 0; t < 6; t++) {
      int code[2] = {0, 0};
      for (int f = 0; f < (with_b ? 2 : 1); f++) {
        float P[4][3];
        for (int p = 0; p < 4; p++) {
          // corner (dk, dj, di) -> cube slot di*4 + dj*2 + dk
          const int slot = c_cp_tet[t][p][2] * 4 + c_cp_tet[t][p][1] * 2 + c_cp_tet[t][p][0];
          P[p][0] = cube[f][slot][0];
          P[p][1] = cube[f][slot][1];
          P[p][2] = cube[f][slot][2];
        }
        code[f] = tet_cp(P, t);
      }
      if (cells) cells[6 * q + t] = (uint8_t)code[0];
      tally(tl, code[0], code[1], with_b);
    }
  }
  flush(tl, counts);
}

// ---- labels for the learned bound proposer ---------------------------------------
// For a vertex with analytic bound e_a: the largest t in [0, tmax] (bisection,
// `steps` halvings) such that moving the vertex alone to any corner of the box
// (u +- |u| e, v +- |v| e), e = e_a 2^t, leaves the CP codes of its six
// incident triangles unchanged.
__global__ void labels2d_kernel(const float* __restrict__ U, const float* __restrict__ V, int r1, int r2,
                                const double* __restrict__ eb_a, const int* __restrict__ idx, int n, int steps,
                                float tmax, float* __restrict__ out) {
  // incident triangles: cell offset (di, dj), kind, position of the vertex
  const int inc[6][4] = {{0, 0, 0, 0}, {0, 0, 1, 0}, {-1, 0, 0, 1}, {-1, -1, 0, 2}, {-1, -1, 1, 2}, {0, -1, 1, 1}};
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = idx[s];
    const int i = v / r2, j = v - (v / r2) * r2;
    float tu[6][3], tv[6][3];
    int kind[6], pos[6], orig[6], nt = 0;
    for (int q = 0; q < 6; q++) {
      const int ci = i + inc[q][0], cj = j + inc[q][1], k = inc[q][2];
      if (ci < 0 || cj < 0 || ci > r1 - 2 || cj > r2 - 2) continue;
      const int pi[3] = {ci, ci + (k == 0), ci + 1};
      const int pj[3] = {cj, cj + (k == 1), cj + 1};
      for (int p = 0; p < 3; p++) {
        tu[nt][p] = U[(size_t)pi[p] * r2 + pj[p]];
        tv[nt][p] = V[(size_t)pi[p] * r2 + pj[p]];
      }
      kind[nt] = k;
      pos[nt] = inc[q][3];
      orig[nt] = tri_cp(tu[nt], tv[nt], k);
      nt++;
    }
    const float u0 = U[v], v0 = V[v];
    const double e0 = eb_a[v];
    float lo = 0.f, hi = tmax;
    for (int it = 0; it < steps; it++) {
      const float mid = 0.5f * (lo + hi);
      const double e = e0 * exp2((double)mid);
      bool pass = e == e;
      for (int c = 0; c < 4 && pass; c++) {
        const float cu = (float)((double)u0 + ((c & 1) ? 1.0 : -1.0) * fabs((double)u0) * e);
        const float cv = (float)((double)v0 + ((c & 2) ? 1.0 : -1.0) * fabs((double)v0) * e);
        for (int q = 0; q < nt && pass; q++) {
          float a[3] = {tu[q][0], tu[q][1], tu[q][2]}, b[3] = {tv[q][0], tv[q][1], tv[q][2]};
          a[pos[q]] = cu;
          b[pos[q]] = cv;
          pass = tri_cp(a, b, kind[q]) == orig[q];
        }
      }
      if (pass) lo = mid;
      else hi = mid;
    }
    out[s] = lo;
  }
}

}  // namespace

int launch_cp_check_2d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Ub, const float* Vb, int r1,
                       int r2, uint8_t* cells, unsigned long long* counts, int row0) {
  if (r1 < 2 || r2 < 2) return CPSZ_OK;
  if (row0 < 0) row0 = 0;
  if (row0 >= r1 - 1) return CPSZ_OK;
  const long long q0 = (long long)row0 * (r2 - 1);
  const long long n = (long long)(r1 - 1) * (r2 - 1) - q0;
  long long g = (n + 255) / 256;
  if (g > (long long)ctx->num_sms * 16) g = (long long)ctx->num_sms * 16;
  cp2d_kernel<<<(int)g, 256, 0, ctx->stream>>>(Ua, Va, Ub, Vb, r1, r2, cells, counts, q0);
  count_launch(ctx);
  return check_launch("cp2d_kernel");
}

int launch_labels_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, const double* eb_a,
                     const int* idx, int n, int steps, float tmax, float* out) {
  if (n <= 0) return CPSZ_OK;
  int g = (n + 127) / 128;
  if (g > ctx->num_sms * 8) g = ctx->num_sms * 8;
  labels2d_kernel<<<g, 128, 0, ctx->stream>>>(U, V, r1, r2, eb_a, idx, n, steps, tmax, out);
  count_launch(ctx);
  return check_launch("labels2d_kernel");
}

int launch_cp_check_3d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Wa, const float* Ub,
                       const float* Vb, const float* Wb, int r1, int r2, int r3, uint8_t* cells,
                       unsigned long long* counts) {
  if (r1 < 2 || r2 < 2 || r3 < 2) return CPSZ_OK;
  const long long n = (long long)(r1 - 1) * (r2 - 1) * (r3 - 1);
  long long g = (n + 127) / 128;
  if (g > (long long)ctx->num_sms * 32) g = (long long)ctx->num_sms * 32;
  cp3d_kernel<<<(int)g, 128, 0, ctx->stream>>>(Ua, Va, Wa, Ub, Vb, Wb, r1, r2, r3, cells, counts);
  count_launch(ctx);
  return check_launch("cp3d_kernel");
}

}  // namespace cpsz
