// kernels3d.cu -- element-parallel kernels of the 3D offline (log) path:
//   eb3d     per-vertex error bound over the 24 tetrahedra around it
//            (src/sz_compress_cp_preserve_3d.cpp:366-418) and its quantized id
//   log3d    log transform with the host library's log2f and sign bitmaps
//            (include/sz_cp_preserve_utils.hpp:201-216), plus the
//            wavefront's per-point input (log values, 1/precision)
//   compact3d / prep3d   raster-order compaction of codes and unpredictable
//            values (compress) and its inverse (decompress)
#include <cfloat>

#include "eb_math.cuh"
#include "kernels.h"
#include "tuning.h"
#include "libm_dev.cuh"

namespace cpsz {

namespace {

// ---- eb3d ------------------------------------------------------------------------
// A CTA owns a 32 (k) x 8 (j) column of vertices and marches over i.  Per step
// it stages vertex plane i+1 (with a one-vertex halo towards -j/-k), evaluates
// the 6 tets of every cube of cube-plane i that touches the column (cubes
// j0-1..j0+7, k0-1..k0+31) into shared memory, and then finishes vertex plane
// i from cube-planes i-1 and i, replaying the reference's update order.
constexpr int EB_TK = 32, EB_TJ = 8, EB_NT = EB_TK * EB_TJ;
constexpr int VK = EB_TK + 2, VJ = EB_TJ + 2;
constexpr int CK = EB_TK + 1, CJ = EB_TJ + 1, NCELL = CK * CJ;

// Tet vertex offsets (dk, dj, di) within a cube; the 4th vertex is the cube
// corner (src/sz_compress_cp_preserve_3d.cpp:9-46, first six entries).
__constant__ int8_t c_tet[6][3][3] = {{{0, 0, 1}, {0, 1, 1}, {1, 1, 1}}, {{0, 1, 0}, {0, 1, 1}, {1, 1, 1}},
                                      {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}}, {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}},
                                      {{0, 1, 0}, {1, 1, 0}, {1, 1, 1}}, {{1, 0, 0}, {1, 1, 0}, {1, 1, 1}}};

__device__ __forceinline__ double min_ref(double s, double cur) { return (s < cur) ? s : cur; }

__global__ void __launch_bounds__(EB_NT, 3) eb3d_kernel(const float* __restrict__ U, const float* __restrict__ V,
                                                     const float* __restrict__ W, int r1, int r2, int r3,
                                                     int i_chunk, double max_pwr_eb, const double* __restrict__ thr,
                                                     int thr_n, uint8_t* __restrict__ id_q,
                                                     double* __restrict__ eb_out, int* __restrict__ flag) {
  __shared__ float vtx[2][3][VJ][VK];
  __shared__ float tets[2][6][CJ][CK];
  const int k0 = blockIdx.x * EB_TK, j0 = blockIdx.y * EB_TJ;
  const int i_begin = blockIdx.z * i_chunk, i_end = min(r1, i_begin + i_chunk);
  const size_t d1 = (size_t)r3, d0 = (size_t)r2 * r3;
  const bool cells = r1 >= 2 && r2 >= 2 && r3 >= 2;
  const int kl = threadIdx.x & 31, jl = threadIdx.x >> 5;
  const int j = j0 + jl, k = k0 + kl;
  int my_flag = 0;

  auto load_plane = [&](int i, int buf) {
    for (int e = threadIdx.x; e < VJ * VK; e += EB_NT) {
      const int jj = e / VK, kk = e - jj * VK;
      const int gj = j0 - 1 + jj, gk = k0 - 1 + kk;
      float u = 0.f, v = 0.f, w = 0.f;
      if (gj >= 0 && gj < r2 && gk >= 0 && gk < r3) {
        const size_t at = (size_t)i * d0 + (size_t)gj * d1 + gk;
        u = __ldg(U + at);
        v = __ldg(V + at);
        w = __ldg(W + at);
      }
      vtx[buf][0][jj][kk] = u;
      vtx[buf][1][jj][kk] = v;
      vtx[buf][2][jj][kk] = w;
    }
  };

  const int i_start = max(0, i_begin - 1);
  if (cells) load_plane(i_start, i_start & 1);
  for (int i = i_start; i < i_end; i++) {
    if (cells) {
      if (i + 1 < r1) load_plane(i + 1, (i + 1) & 1);
      __syncthreads();
      if (i <= r1 - 2) {
        const int a = i & 1, b = a ^ 1;  // vertex planes i (di = 0) and i + 1 (di = 1)
        for (int e = threadIdx.x; e < 6 * NCELL; e += EB_NT) {
          const int t = e / NCELL, c = e - t * NCELL;
          const int cj = c / CK, ck = c - cj * CK;
          const int gj = j0 - 1 + cj, gk = k0 - 1 + ck;
          float val = 0.f;
          if (gj >= 0 && gj <= r2 - 2 && gk >= 0 && gk <= r3 - 2) {
            float u[3], v[3], w[3];
#pragma unroll
            for (int x = 0; x < 3; x++) {
              const int dk = c_tet[t][x][0], dj = c_tet[t][x][1], di = c_tet[t][x][2];
              const int pl = di ? b : a;
              u[x] = vtx[pl][0][cj + dj][ck + dk];
              v[x] = vtx[pl][1][cj + dj][ck + dk];
              w[x] = vtx[pl][2][cj + dj][ck + dk];
            }
            val = (float)dev::tet_eb(u[0], u[1], u[2], vtx[a][0][cj][ck], v[0], v[1], v[2], vtx[a][1][cj][ck], w[0],
                                     w[1], w[2], vtx[a][2][cj][ck]);
          }
          tets[i & 1][t][cj][ck] = val;
        }
      }
      __syncthreads();
    }
    if (i < i_begin || j >= r2 || k >= r3) continue;
    double s = max_pwr_eb;
    if (cells) {
      // Updates in the reference's order: cubes by ascending linear index
      // (corner offsets (di,dj,dk) = 111,110,101,100,011,010,001,000), tets
      // ascending within a cube, only tets containing this vertex.
      const bool jm = j >= 1 && j - 1 <= r2 - 2, j0ok = j <= r2 - 2;
      const bool km = k >= 1 && k - 1 <= r3 - 2, k0ok = k <= r3 - 2;
#pragma unroll
      for (int oi = 1; oi >= 0; oi--) {
        const int ci = i - oi;
        if (ci < 0 || ci > r1 - 2) continue;
        const float(*T)[CJ][CK] = tets[ci & 1];
        if (oi == 1) {
          if (jm && km)
            for (int t = 0; t < 6; t++) s = min_ref(s, T[t][jl][kl]);
          if (jm && k0ok) {
            s = min_ref(s, T[0][jl][kl + 1]);
            s = min_ref(s, T[1][jl][kl + 1]);
          }
          if (j0ok && km) {
            s = min_ref(s, T[2][jl + 1][kl]);
            s = min_ref(s, T[3][jl + 1][kl]);
          }
          if (j0ok && k0ok) {
            s = min_ref(s, T[0][jl + 1][kl + 1]);
            s = min_ref(s, T[2][jl + 1][kl + 1]);
          }
        } else {
          if (jm && km) {
            s = min_ref(s, T[4][jl][kl]);
            s = min_ref(s, T[5][jl][kl]);
          }
          if (jm && k0ok) {
            s = min_ref(s, T[1][jl][kl + 1]);
            s = min_ref(s, T[4][jl][kl + 1]);
          }
          if (j0ok && km) {
            s = min_ref(s, T[3][jl + 1][kl]);
            s = min_ref(s, T[5][jl + 1][kl]);
          }
          if (j0ok && k0ok)
            for (int t = 0; t < 6; t++) s = min_ref(s, T[t][jl + 1][kl + 1]);
        }
      }
    }
    const size_t idx = (size_t)i * d0 + (size_t)j * d1 + k;
    int id = ID_ZERO;
    if (s > 0) {
      // id = (int)log2(log2(1 + s) / 2^-23); the guess only seeds the count
      const float g = __log2f(__double2float_rn(fmin(s, 1e30)) * 1.4426950f) + 23.0f;
      id = dev::count_thresholds(thr, thr_n, s, (int)fmaxf(g, 0.f));
      if (id >= ID_RAW_3D) my_flag |= FLAG_ID_OVERFLOW;
    }
    id_q[idx] = (uint8_t)id;
    if (eb_out) eb_out[idx] = s;
  }
  if (my_flag) atomicOr(flag, my_flag);
}

// ---- log3d -----------------------------------------------------------------------
__global__ void __launch_bounds__(256) log3d_kernel(const float* __restrict__ U, const float* __restrict__ V,
                                                    const float* __restrict__ W, const uint8_t* __restrict__ id_q,
                                                    size_t n, LibmFn L, float4* __restrict__ pairs,
                                                    uint32_t* __restrict__ signs, size_t sign_words) {
  const int lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t base = (size_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
    const size_t idx = base + lane;
    float x[3] = {0.f, 0.f, 0.f};
    int id = ID_ZERO;
    if (idx < n) {
      x[0] = __ldg(U + idx);
      x[1] = __ldg(V + idx);
      x[2] = __ldg(W + idx);
      id = __ldg(id_q + idx);
    }
    float lg[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const unsigned bal = __ballot_sync(0xffffffffu, x[c] > 0.f);
      if (lane == 0) signs[(size_t)c * sign_words + (base >> 5)] = __byte_perm(__brev(bal), 0, 0x0123);
      lg[c] = (x[c] != 0.f) ? dev::host_log2f(fabsf(x[c]), L) : -100.f;
    }
    if (idx < n) {
      // 1/precision = 2^(23 - id) for ids 1..23; NaN marks precision 0
      const float inv = (id >= 1 && id < ID_RAW_3D) ? __uint_as_float((uint32_t)(150 - id) << 23) : __uint_as_float(0x7fc00000u);
      pairs[idx] = make_float4(lg[0], lg[1], lg[2], inv);
    }
  }
}

// ---- raster compaction -------------------------------------------------------------
// Chunks of CH points per CTA (8 per thread); the predicted points of a chunk
// are counted first, the chunk counts scanned, and the write pass re-derives
// each thread's offset with a block scan.
constexpr int CH_NT = 256, CH_PER_T = 8, CH = CH_NT * CH_PER_T;

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* total) {
  __shared__ unsigned warp_sum[CH_NT / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[wid] = x;
  __syncthreads();
  unsigned before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < CH_NT / 32; w++) {
    const unsigned s = warp_sum[w];
    if (w < wid) before += s;
    all += s;
  }
  __syncthreads();
  *total = all;
  return before + x - v;
}

template <bool kCompress>
__device__ __forceinline__ bool is_pred(const void* src, size_t idx) {
  if (kCompress) return ((const ushort4*)src)[idx].x != 0;
  const int id = ((const uint8_t*)src)[idx];
  return id != 0 && id != ID_RAW_3D;
}

template <bool kCompress>
__global__ void __launch_bounds__(CH_NT) chunk_count_kernel(const void* __restrict__ src, size_t n,
                                                            unsigned* __restrict__ cnt) {
  const size_t base = (size_t)blockIdx.x * CH + (size_t)threadIdx.x * CH_PER_T;
  unsigned c = 0;
#pragma unroll
  for (int e = 0; e < CH_PER_T; e++)
    if (base + e < n) c += is_pred<kCompress>(src, base + e);
  unsigned total;
  block_exclusive_scan(c, &total);
  if (threadIdx.x == 0) cnt[blockIdx.x] = total;
}

__global__ void __launch_bounds__(CH_NT) compact3d_kernel(const ushort4* __restrict__ codes, uint8_t* __restrict__ ids,
                                                          const float* __restrict__ U, const float* __restrict__ V,
                                                          const float* __restrict__ W, size_t n,
                                                          const unsigned* __restrict__ chunk_off,
                                                          uint16_t* __restrict__ codes_out, float* __restrict__ unpred,
                                                          unsigned long long* __restrict__ hist_ids) {
  __shared__ unsigned h[32];
  if (threadIdx.x < 32) h[threadIdx.x] = 0;
  const size_t base = (size_t)blockIdx.x * CH + (size_t)threadIdx.x * CH_PER_T;
  ushort4 cv[CH_PER_T];
  unsigned c = 0;
#pragma unroll
  for (int e = 0; e < CH_PER_T; e++) {
    cv[e] = (base + e < n) ? codes[base + e] : make_ushort4(0, 0, 0, 0);
    c += cv[e].x != 0;
  }
  unsigned total;
  const unsigned off = block_exclusive_scan(c, &total);
  size_t pp = (size_t)chunk_off[blockIdx.x] + off;
  size_t up = base - pp;
#pragma unroll
  for (int e = 0; e < CH_PER_T; e++) {
    const size_t idx = base + e;
    if (idx >= n) break;
    const int q = ids[idx];
    int fin;
    if (cv[e].x != 0) {
      codes_out[3 * pp] = cv[e].x;
      codes_out[3 * pp + 1] = cv[e].y;
      codes_out[3 * pp + 2] = cv[e].z;
      pp++;
      fin = q;
    } else {
      unpred[3 * up] = U[idx];
      unpred[3 * up + 1] = V[idx];
      unpred[3 * up + 2] = W[idx];
      up++;
      fin = (q == ID_ZERO) ? 0 : ID_RAW_3D;
    }
    ids[idx] = (uint8_t)fin;
    atomicAdd(&h[fin & 31], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32 && h[threadIdx.x]) atomicAdd(&hist_ids[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}

__device__ __forceinline__ float small_int_to_float(int v) {
  // exact for |v| < 2^22: 1.5 * 2^23 + v has the integer in its low mantissa bits
  return __int_as_float(0x4B400000 + v) - 12582912.0f;
}

__global__ void __launch_bounds__(CH_NT) prep3d_kernel(const uint8_t* __restrict__ ids, size_t n,
                                                       const unsigned* __restrict__ chunk_off,
                                                       const uint16_t* __restrict__ codes, size_t n_codes,
                                                       const float* __restrict__ unpred, size_t n_unpred,
                                                       float4* __restrict__ pairs, int* __restrict__ flag) {
  const size_t base = (size_t)blockIdx.x * CH + (size_t)threadIdx.x * CH_PER_T;
  uint8_t iv[CH_PER_T];
  unsigned c = 0;
#pragma unroll
  for (int e = 0; e < CH_PER_T; e++) {
    iv[e] = (base + e < n) ? ids[base + e] : 0;
    c += (base + e < n) && iv[e] != 0 && iv[e] != ID_RAW_3D;
  }
  unsigned total;
  const unsigned off = block_exclusive_scan(c, &total);
  size_t pp = (size_t)chunk_off[blockIdx.x] + off;
  size_t up = base - pp;
  int bad = 0;
#pragma unroll
  for (int e = 0; e < CH_PER_T; e++) {
    const size_t idx = base + e;
    if (idx >= n) break;
    const int id = iv[e];
    float4 o;
    if (id != 0 && id != ID_RAW_3D) {
      // addend 2 (code - 32768) * 2^(id - 23), exact in float
      const float p = __uint_as_float((uint32_t)(104 + id) << 23);
      float a[3] = {0.f, 0.f, 0.f};
      if (3 * pp + 3 <= n_codes) {
#pragma unroll
        for (int x = 0; x < 3; x++) a[x] = small_int_to_float(2 * ((int)codes[3 * pp + x] - 32768)) * p;
      } else {
        bad = 1;
      }
      o = make_float4(a[0], a[1], a[2], 0.f);
      pp++;
    } else {
      float r[3] = {0.f, 0.f, 0.f};
      if (3 * up + 3 <= n_unpred) {
        r[0] = unpred[3 * up];
        r[1] = unpred[3 * up + 1];
        r[2] = unpred[3 * up + 2];
      } else {
        bad = 1;
      }
      o = make_float4(r[0], r[1], r[2], __int_as_float(1));
      up++;
    }
    pairs[idx] = o;
  }
  if (bad) atomicOr(flag, FLAG_RAW_RANGE);
}

__global__ void libm_eval_kernel(const float* __restrict__ in, size_t n, int which, LibmFn T,
                                 float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = which == 0 ? dev::host_log2f(in[i], T) : dev::host_exp2f(in[i], T);
}

int grid_for(size_t n, int per_block, int cap) {
  size_t g = (n + per_block - 1) / per_block;
  if (g > (size_t)cap) g = cap;
  return (int)(g ? g : 1);
}

}  // namespace

int launch_eb3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, int r1, int r2, int r3,
                double max_pwr_eb, const double* d_thr, int thr_n, uint8_t* id_q, double* eb_out) {
  dim3 grid((r3 + EB_TK - 1) / EB_TK, (r2 + EB_TJ - 1) / EB_TJ, 1);
  if (grid.y > 65535)
    return set_error(CPSZ_ERR_UNSUPPORTED, "3D field with r2 = %d exceeds the bound kernel's grid", r2);
  // split i so that the grid covers the GPU `fill` times (two CTAs per SM each)
  const long long cols = (long long)grid.x * grid.y;
  const size_t points = (size_t)r1 * r2 * r3;
  const int fill = tune_get(TUNE_EB3D_FILL, points), min_chunk = tune_get(TUNE_EB3D_MIN_CHUNK, points);
  long long want = ((long long)fill * ctx->num_sms * 2 + cols - 1) / cols;
  if (want < 1) want = 1;
  if (want > r1) want = r1;
  int chunk = (int)((r1 + want - 1) / want);
  if (chunk < min_chunk) chunk = min_chunk < r1 ? min_chunk : r1;
  grid.z = (r1 + chunk - 1) / chunk;
  eb3d_kernel<<<grid, EB_NT, 0, ctx->stream>>>(U, V, W, r1, r2, r3, chunk, max_pwr_eb, d_thr, thr_n, id_q, eb_out,
                                                ctx->d_flag);
  count_launch(ctx);
  return check_launch("eb3d_kernel");
}

int launch_log3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, const uint8_t* id_q, size_t n,
                 const LibmFn& L, float4* pairs, uint32_t* signs, size_t sign_words) {
  log3d_kernel<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(U, V, W, id_q, n, L, pairs, signs,
                                                                               sign_words);
  count_launch(ctx);
  return check_launch("log3d_kernel");
}

int launch_libm_eval(cpsz_b200_ctx* ctx, int which, const float* in, size_t n, const LibmTables& L, float* out) {
  libm_eval_kernel<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(in, n, which,
                                                                                   which ? L.exp2f : L.log2f, out);
  count_launch(ctx);
  return check_launch("libm_eval_kernel");
}

size_t chunk_count(size_t n) { return (n + CH - 1) / CH; }

int launch_chunk_count_3d(cpsz_b200_ctx* ctx, bool compress, const void* src, size_t n, unsigned* cnt) {
  const int g = (int)chunk_count(n);
  if (compress) chunk_count_kernel<true><<<g, CH_NT, 0, ctx->stream>>>(src, n, cnt);
  else chunk_count_kernel<false><<<g, CH_NT, 0, ctx->stream>>>(src, n, cnt);
  count_launch(ctx);
  return check_launch("chunk_count_kernel");
}

int launch_compact3d(cpsz_b200_ctx* ctx, const ushort4* codes, uint8_t* ids, const float* U, const float* V,
                     const float* W, size_t n, const unsigned* chunk_off, uint16_t* codes_out, float* unpred,
                     unsigned long long* hist_ids) {
  compact3d_kernel<<<(int)chunk_count(n), CH_NT, 0, ctx->stream>>>(codes, ids, U, V, W, n, chunk_off, codes_out,
                                                                    unpred, hist_ids);
  count_launch(ctx);
  return check_launch("compact3d_kernel");
}

int launch_prep3d(cpsz_b200_ctx* ctx, const uint8_t* ids, size_t n, const unsigned* chunk_off, const uint16_t* codes,
                  size_t n_codes, const float* unpred, size_t n_unpred, float4* pairs) {
  prep3d_kernel<<<(int)chunk_count(n), CH_NT, 0, ctx->stream>>>(ids, n, chunk_off, codes, n_codes, unpred, n_unpred,
                                                                 pairs, ctx->d_flag);
  count_launch(ctx);
  return check_launch("prep3d_kernel");
}

}  // namespace cpsz
