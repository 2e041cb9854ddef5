// wave3d.cu -- the 3D Lorenzo recursion of the offline (log) path on
// reconstructed log values (src/sz_compress_cp_preserve_3d.cpp:441-520,
// src/sz_decompress_cp_preserve_3d.cpp:52-104).
//
// A point's predictor reads its seven lower neighbours (i-1 / j-1 / k-1
// combinations), so all points of an anti-diagonal plane i + j + k = s are
// independent.  One launch finishes one plane; the planes run in order on the
// stream, so every neighbour a launch reads was written by an earlier launch.
// A point is handled by one thread, which couples the three components the
// way the reference does: the point is predictable only if all three are.
//
// Step arithmetic (all float; equal to the reference's float/double mix, see
// the wavefront notes in wave2d.cu): with p = 2^(id-23) and y = |x - pred| / p
// exact, the reference's capacity test is y < 65535, the code is
// 32768 +- ((int)y + 1) >> 1, and (float)(pred + 2 q p) equals the float sum
// pred + (2q) p.  The decoder's (float)(pred + 2 (code - 32768) p) is likewise
// pred + addend with the addend precomputed exactly in float.
#include "kernels.h"
#include "libm_dev.cuh"

namespace cpsz {

namespace {

constexpr int PLANE_NT = 128;

__device__ __forceinline__ float small_int_to_float(int v) {
  return __int_as_float(0x4B400000 + v) - 12582912.0f;
}

struct Nb {
  float4 q[7];
};

// Neighbours q0..q6 of the reference's predictor
//   pred = q0 + q3 + q5 + q6 - q1 - q2 - q4
// (q0 = (i-1,j-1,k-1), q1 = (i-1,j-1,k), q2 = (i-1,j,k-1), q3 = (i-1,j,k),
//  q4 = (i,j-1,k-1), q5 = (i,j-1,k), q6 = (i,j,k-1)); zero outside the field.
__device__ __forceinline__ void load_nb(const float4* __restrict__ rec, size_t idx, int i, int j, int k, size_t d0,
                                        size_t d1, Nb& n) {
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  n.q[0] = (i && j && k) ? rec[idx - d0 - d1 - 1] : z;
  n.q[1] = (i && j) ? rec[idx - d0 - d1] : z;
  n.q[2] = (i && k) ? rec[idx - d0 - 1] : z;
  n.q[3] = i ? rec[idx - d0] : z;
  n.q[4] = (j && k) ? rec[idx - d1 - 1] : z;
  n.q[5] = j ? rec[idx - d1] : z;
  n.q[6] = k ? rec[idx - 1] : z;
}

__device__ __forceinline__ float comp(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

__device__ __forceinline__ float predict(const Nb& n, int c) {
  float p = comp(n.q[0], c) + comp(n.q[3], c);
  p = p + comp(n.q[5], c);
  p = p + comp(n.q[6], c);
  p = p - comp(n.q[1], c);
  p = p - comp(n.q[2], c);
  p = p - comp(n.q[4], c);
  return p;
}

// Maps thread t of a plane launch to its point; false if none.
__device__ __forceinline__ bool plane_point(int s, int i_lo, int r1, int r2, int r3, int& i, int& j, int& k) {
  const long long t = (long long)blockIdx.x * PLANE_NT + threadIdx.x;
  const long long row = t / r2;
  if (row > r1) return false;
  i = i_lo + (int)row;
  j = (int)(t - row * r2);
  k = s - i - j;
  return i < r1 && k >= 0 && k < r3;
}

__global__ void __launch_bounds__(PLANE_NT) wave3d_compress_plane(const float4* __restrict__ in,
                                                                  float4* __restrict__ rec,
                                                                  ushort4* __restrict__ codes, int r1, int r2,
                                                                  int r3, int s, int i_lo) {
  int i, j, k;
  if (!plane_point(s, i_lo, r1, r2, r3, i, j, k)) return;
  const size_t d1 = (size_t)r3, d0 = (size_t)r2 * r3;
  const size_t idx = (size_t)i * d0 + (size_t)j * d1 + k;
  const float4 x = in[idx];
  Nb nb;
  load_nb(rec, idx, i, j, k, d0, d1, nb);
  const float inv = x.w;  // NaN: precision 0 (unpredictable)
  const float p = __int_as_float(0x7F000000 - __float_as_int(inv));
  bool ok = true;
  float dec[3];
  int q[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float pred = predict(nb, c);
    const float xc = comp(x, c);
    const float diff = xc - pred;
    const float y = fabsf(diff) * inv;
    const int qa = ((int)fminf(y, 65536.0f) + 1) >> 1;
    q[c] = (diff > 0.f) ? qa : -qa;
    dec[c] = pred + small_int_to_float(2 * q[c]) * p;
    ok = ok & (y < 65535.0f) & (fabsf(dec[c] - xc) < p);
  }
  if (ok) {
    rec[idx] = make_float4(dec[0], dec[1], dec[2], 0.f);
    codes[idx] = make_ushort4((unsigned short)(q[0] + 32768), (unsigned short)(q[1] + 32768),
                              (unsigned short)(q[2] + 32768), 0);
  } else {
    rec[idx] = make_float4(x.x, x.y, x.z, 0.f);
    codes[idx] = make_ushort4(0, 0, 0, 0);
  }
}

__global__ void __launch_bounds__(PLANE_NT) wave3d_decompress_plane(const float4* __restrict__ in,
                                                                    float4* __restrict__ rec,
                                                                    const uint8_t* __restrict__ signs,
                                                                    size_t sign_bytes, LibmFn Lg, LibmFn Ex,
                                                                    float* __restrict__ U, float* __restrict__ V,
                                                                    float* __restrict__ W, int r1, int r2, int r3,
                                                                    int s, int i_lo) {
  int i, j, k;
  if (!plane_point(s, i_lo, r1, r2, r3, i, j, k)) return;
  const size_t d1 = (size_t)r3, d0 = (size_t)r2 * r3;
  const size_t idx = (size_t)i * d0 + (size_t)j * d1 + k;
  const float4 x = in[idx];
  float lg[3], out[3];
  if (__float_as_int(x.w) != 0) {
    // raw point: the stored float, and its log for the neighbours' predictors
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float r = comp(x, c);
      out[c] = r;
      lg[c] = (r == 0.f) ? -100.f : dev::host_log2f(fabsf(r), Lg);
    }
  } else {
    Nb nb;
    load_nb(rec, idx, i, j, k, d0, d1, nb);
    const unsigned byte = (unsigned)(idx >> 3), bit = 7u - (unsigned)(idx & 7);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      lg[c] = predict(nb, c) + comp(x, c);
      const bool pos = (signs[(size_t)c * sign_bytes + byte] >> bit) & 1u;
      if (lg[c] < -99.f) {
        out[c] = 0.f;
      } else {
        const float e = dev::host_exp2f(lg[c], Ex);
        out[c] = pos ? e : -e;
      }
    }
  }
  rec[idx] = make_float4(lg[0], lg[1], lg[2], 0.f);
  U[idx] = out[0];
  V[idx] = out[1];
  W[idx] = out[2];
}

}  // namespace

int launch_wave3d_planes(cpsz_b200_ctx* ctx, bool decompress, const float4* in, float4* rec, ushort4* codes,
                         const uint8_t* signs, size_t sign_bytes, const LibmTables* L, float* U, float* V, float* W,
                         int r1, int r2, int r3) {
  const int planes = r1 + r2 + r3 - 2;
  for (int s = 0; s < planes; s++) {
    // rows i of plane s: max(0, s - (r2-1) - (r3-1)) .. min(r1-1, s)
    const int i_lo = max(0, s - (r2 - 1) - (r3 - 1));
    const int i_hi = min(r1 - 1, s);
    const long long threads = (long long)(i_hi - i_lo + 1) * r2;
    const int grid = (int)((threads + PLANE_NT - 1) / PLANE_NT);
    if (decompress)
      wave3d_decompress_plane<<<grid, PLANE_NT, 0, ctx->stream>>>(in, rec, signs, sign_bytes, L->log2f, L->exp2f, U,
                                                                  V, W, r1, r2, r3, s, i_lo);
    else
      wave3d_compress_plane<<<grid, PLANE_NT, 0, ctx->stream>>>(in, rec, codes, r1, r2, r3, s, i_lo);
  }
  count_launch(ctx, planes);
  return check_launch(decompress ? "wave3d_decompress_plane" : "wave3d_compress_plane");
}

}  // namespace cpsz
