// blocks.cu -- 12x12 block-order plumbing of the 2D field blobs, and a
// generic device-wide exclusive scan.
//
// The reference emits quantization codes and unpredictable values in 12x12
// block order (blocks row-major, rows inside a block, src/sz_compress_3d.cpp:
// 126-193).  A "segment" is one row of one block (up to 12 points, contiguous
// in block order); segments are numbered in block order:
//   ord = bi*12*nby + bj*h + li,   h = rows of block-row bi (12, or the remainder),
// and element (i, j) sits at block-order position
//   bi*12*r2 + bj*12*h + li*w + lj,   w = columns of block bj.
#include <algorithm>

#include "kernels.h"

namespace cpsz {

namespace {

constexpr int BS = 12;
constexpr int NT = 256;

struct Seg {
  int i, j0, w;
  long long pos;  // block-order position of the segment's first element
};

__device__ __forceinline__ Seg seg_of(long long ord, int r1, int r2, int nby) {
  long long per_brow = (long long)BS * nby;
  int bi = (int)(ord / per_brow);
  int rem = (int)(ord - (long long)bi * per_brow);
  int h = min(BS, r1 - bi * BS);
  int bj = rem / h, li = rem - bj * h;
  int w = min(BS, r2 - bj * BS);
  Seg s;
  s.i = bi * BS + li;
  s.j0 = bj * BS;
  s.w = w;
  s.pos = (long long)bi * BS * r2 + (long long)bj * BS * h + (long long)li * w;
  return s;
}

__global__ void __launch_bounds__(NT) r2b_kernel(const uint16_t* __restrict__ raster, long long pitch, int r1, int r2,
                                                 int nby, long long nseg, uint16_t* __restrict__ blocks) {
  long long ord = (long long)blockIdx.x * NT + threadIdx.x;
  if (ord >= nseg) return;
  Seg s = seg_of(ord, r1, r2, nby);
  const uint16_t* src = raster + (long long)s.i * pitch + s.j0;
  for (int k = 0; k < s.w; k++) blocks[s.pos + k] = src[k];
}

// Decompression side of a point: the addend 2(code - 32768) * p that the
// wavefront adds to its prediction (p = 4^id * 2^-52, 0 for id 0;
// src/sz_decompress_cp_preserve_2d.cpp:30-34, include/sz_decompression_utils.hpp:65-73),
// or a raw flag for code 0 (the raw value is scattered in afterwards).
__global__ void __launch_bounds__(NT) b2r_kernel(const uint16_t* __restrict__ blocks, int r1, int r2, int nby,
                                                 long long nseg, uint16_t* __restrict__ raster, long long pitch,
                                                 const uint8_t* __restrict__ ids, float2* __restrict__ pair) {
  long long ord = (long long)blockIdx.x * NT + threadIdx.x;
  if (ord >= nseg) return;
  Seg s = seg_of(ord, r1, r2, nby);
  uint16_t* dst = raster + (long long)s.i * pitch + s.j0;
  for (int k = 0; k < s.w; k++) dst[k] = blocks[s.pos + k];
  if (pair) {
    const long long base = (long long)s.i * r2 + s.j0;
    for (int k = 0; k < s.w; k++) {
      const int code = blocks[s.pos + k];
      const int id = ids[base + k];
      const float p = id ? __int_as_float((2 * id - 52 + 127) << 23) : 0.f;
      pair[base + k] = make_float2((float)(2 * (code - 32768)) * p, __int_as_float(code == 0 ? 1 : 0));
    }
  }
}

__global__ void __launch_bounds__(NT) seg_count_kernel(const uint16_t* __restrict__ raster, long long pitch, int r1,
                                                       int r2, int nby, long long nseg, unsigned int* __restrict__ cnt) {
  long long ord = (long long)blockIdx.x * NT + threadIdx.x;
  if (ord >= nseg) return;
  Seg s = seg_of(ord, r1, r2, nby);
  const uint16_t* src = raster + (long long)s.i * pitch + s.j0;
  unsigned int c = 0;
  for (int k = 0; k < s.w; k++) c += (src[k] == 0);
  cnt[ord] = c;
}

__global__ void __launch_bounds__(NT) gather_kernel(const uint16_t* __restrict__ raster, long long pitch,
                                                    const float* __restrict__ x, long long x_pitch, int r1, int r2,
                                                    int nby, long long nseg, const unsigned int* __restrict__ off,
                                                    float* __restrict__ unpred) {
  long long ord = (long long)blockIdx.x * NT + threadIdx.x;
  if (ord >= nseg) return;
  Seg s = seg_of(ord, r1, r2, nby);
  const uint16_t* src = raster + (long long)s.i * pitch + s.j0;
  const float* xs = x + (long long)s.i * x_pitch + s.j0;
  unsigned int o = off[ord];
  for (int k = 0; k < s.w; k++)
    if (src[k] == 0) unpred[o++] = xs[k];
}

__global__ void __launch_bounds__(NT) scatter_kernel(const uint16_t* __restrict__ raster, long long pitch,
                                                     const float* __restrict__ unpred, unsigned long long n_unpred,
                                                     int r1, int r2, int nby, long long nseg,
                                                     const unsigned int* __restrict__ off,
                                                     float2* __restrict__ pairs, int* flag) {
  long long ord = (long long)blockIdx.x * NT + threadIdx.x;
  if (ord >= nseg) return;
  Seg s = seg_of(ord, r1, r2, nby);
  const uint16_t* src = raster + (long long)s.i * pitch + s.j0;
  float2* xs = pairs + (long long)s.i * r2 + s.j0;
  unsigned long long o = off[ord];
  for (int k = 0; k < s.w; k++)
    if (src[k] == 0) {
      if (o < n_unpred) xs[k].x = unpred[o];
      else atomicOr(flag, FLAG_RAW_RANGE);
      o++;
    }
}

// ---- generic exclusive scan (u32) ---------------------------------------------------
constexpr int SCAN_NT = 1024;
constexpr int SCAN_PER = 8;
constexpr int SCAN_CHUNK = SCAN_NT * SCAN_PER;

__device__ __forceinline__ unsigned int block_exclusive_scan(unsigned int v, unsigned int* warp_tot,
                                                             unsigned int* total) {
  unsigned int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) >= o) x += y;
  }
  if ((threadIdx.x & 31) == 31) warp_tot[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned int w = (threadIdx.x < blockDim.x / 32) ? warp_tot[threadIdx.x] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned int y = __shfl_up_sync(0xffffffffu, w, o);
      if (threadIdx.x >= o) w += y;
    }
    warp_tot[threadIdx.x] = w;
  }
  __syncthreads();
  unsigned int pre = (threadIdx.x >= 32 ? warp_tot[(threadIdx.x >> 5) - 1] : 0u) + x - v;
  if (total) *total = warp_tot[blockDim.x / 32 - 1];
  __syncthreads();
  return pre;
}

__global__ void __launch_bounds__(SCAN_NT) scan_reduce_kernel(const unsigned int* __restrict__ in, size_t n,
                                                              unsigned int* __restrict__ part) {
  __shared__ unsigned int warp_tot[32];
  size_t base = (size_t)blockIdx.x * SCAN_CHUNK;
  unsigned int s = 0;
  for (int k = 0; k < SCAN_PER; k++) {
    size_t i = base + (size_t)k * SCAN_NT + threadIdx.x;
    if (i < n) s += in[i];
  }
  unsigned int total;
  block_exclusive_scan(s, warp_tot, &total);
  if (threadIdx.x == 0) part[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_NT) scan_partials_kernel(unsigned int* __restrict__ part, size_t np) {
  __shared__ unsigned int warp_tot[32];
  __shared__ unsigned int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (size_t base = 0; base < np; base += SCAN_NT) {
    size_t i = base + threadIdx.x;
    unsigned int v = i < np ? part[i] : 0u;
    unsigned int total;
    unsigned int pre = block_exclusive_scan(v, warp_tot, &total);
    if (i < np) part[i] = carry + pre;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) part[np] = carry;
}

__global__ void __launch_bounds__(SCAN_NT) scan_down_kernel(const unsigned int* __restrict__ in, size_t n,
                                                            const unsigned int* __restrict__ part,
                                                            unsigned int* __restrict__ out) {
  __shared__ unsigned int warp_tot[32];
  size_t base = (size_t)blockIdx.x * SCAN_CHUNK + (size_t)threadIdx.x * SCAN_PER;
  unsigned int v[SCAN_PER];
  unsigned int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER; k++) {
    size_t i = base + k;
    v[k] = i < n ? in[i] : 0u;
    s += v[k];
  }
  unsigned int pre = block_exclusive_scan(s, warp_tot, nullptr) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_PER; k++) {
    size_t i = base + k;
    if (i < n) out[i] = pre;
    pre += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = part[gridDim.x];
}

// ---- strips: a 12-row block row cut into runs of STRIP_BLOCKS blocks ----------------
// A strip's blocks are consecutive in block order, so its block-order image is
// one contiguous range: the strip is staged in shared memory with coalesced
// row reads and written out with coalesced block-order writes.
constexpr int STRIP_BLOCKS = 32;
constexpr int STRIP_W = STRIP_BLOCKS * BS;  // 384 columns
constexpr int STRIP_NT = 256;

struct StripGeom {
  int bi, h, c0, W, nb, wl;
  long long out0;  // block-order position of the strip's first element
};
__device__ __forceinline__ StripGeom strip_geom(long long s, int r1, int r2, int nsc) {
  StripGeom g;
  g.bi = (int)(s / nsc);
  const int sc = (int)(s - (long long)g.bi * nsc);
  g.h = min(BS, r1 - g.bi * BS);
  g.c0 = sc * STRIP_W;
  g.W = min(STRIP_W, r2 - g.c0);
  g.nb = (g.W + BS - 1) / BS;
  g.wl = g.W - (g.nb - 1) * BS;  // width of the strip's last block (12 unless it ends the row)
  g.out0 = (long long)g.bi * BS * r2 + (long long)sc * STRIP_BLOCKS * BS * g.h;
  return g;
}
// block-order offset o inside the strip -> (row, column) inside the strip
__device__ __forceinline__ void strip_rc(const StripGeom& g, int o, int& li, int& col) {
  const int b = o / (BS * g.h);
  const int rem = o - b * BS * g.h;
  const int w = (b == g.nb - 1) ? g.wl : BS;
  li = rem / w;
  col = b * BS + (rem - li * w);
}

__global__ void __launch_bounds__(STRIP_NT) r2b_strip_kernel(const uint16_t* __restrict__ raster, long long pitch,
                                                             int r1, int r2, int nsc, uint16_t* __restrict__ blocks,
                                                             unsigned int* __restrict__ strip_cnt) {
  __shared__ uint16_t t[BS][STRIP_W + 2];
  __shared__ unsigned int wsum[STRIP_NT / 32];
  const StripGeom g = strip_geom(blockIdx.x, r1, r2, nsc);
  const uint16_t* src = raster + (long long)g.bi * BS * pitch + g.c0;
  for (int li = 0; li < g.h; li++)
    for (int c = threadIdx.x; c < g.W; c += STRIP_NT) t[li][c] = src[(long long)li * pitch + c];
  __syncthreads();
  unsigned int z = 0;
  uint16_t* dst = blocks + g.out0;
  const int n = g.h * g.W;
  for (int o = threadIdx.x; o < n; o += STRIP_NT) {
    int li, col;
    strip_rc(g, o, li, col);
    const uint16_t v = t[li][col];
    dst[o] = v;
    z += v == 0;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) z += __shfl_down_sync(0xffffffffu, z, d);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = z;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int tot = 0;
    for (int w = 0; w < STRIP_NT / 32; w++) tot += wsum[w];
    strip_cnt[blockIdx.x] = tot;
  }
}

// Unpredictable values (code 0) of each strip in block order, at the strip's
// offset (exclusive scan of the counts).  Strips without any return at once.
__global__ void __launch_bounds__(STRIP_NT) gather_strip_kernel(const uint16_t* __restrict__ raster, long long pitch,
                                                                const float* __restrict__ x, long long x_pitch,
                                                                int r1, int r2, int nsc,
                                                                const unsigned int* __restrict__ strip_off,
                                                                float* __restrict__ unpred) {
  __shared__ unsigned int wsum[STRIP_NT / 32];
  const unsigned int base = strip_off[blockIdx.x];
  if (strip_off[blockIdx.x + 1] == base) return;
  const StripGeom g = strip_geom(blockIdx.x, r1, r2, nsc);
  const int n = g.h * g.W;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned int run = base;
  for (int o0 = 0; o0 < n; o0 += STRIP_NT) {
    const int o = o0 + threadIdx.x;
    int li = 0, col = 0;
    bool z = false;
    if (o < n) {
      strip_rc(g, o, li, col);
      z = raster[(long long)(g.bi * BS + li) * pitch + g.c0 + col] == 0;
    }
    const unsigned int m = __ballot_sync(0xffffffffu, z);
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    unsigned int before = 0, tot = 0;
    for (int w = 0; w < STRIP_NT / 32; w++) {
      const unsigned int c = wsum[w];
      before += (w < warp) ? c : 0u;
      tot += c;
    }
    if (z) unpred[run + before + __popc(m & ((1u << lane) - 1u))] = x[(long long)(g.bi * BS + li) * x_pitch + g.c0 + col];
    run += tot;
    __syncthreads();
  }
}

inline long long nseg_of(int r1, int r2) { return (long long)r1 * ((r2 - 1) / BS + 1); }
inline unsigned grid_of(long long n) { return (unsigned)((n + NT - 1) / NT); }

}  // namespace

size_t scan_u32_tmp_bytes(size_t n) { return ((n + SCAN_CHUNK - 1) / SCAN_CHUNK + 2) * sizeof(unsigned int) + 256; }

int launch_scan_u32(cpsz_b200_ctx* ctx, const unsigned int* in, unsigned int* out, size_t n, void* tmp) {
  size_t nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  if (nb == 0) {
    cudaMemsetAsync(out, 0, sizeof(unsigned int), ctx->stream);
    return CPSZ_OK;
  }
  unsigned int* part = (unsigned int*)tmp;
  scan_reduce_kernel<<<(unsigned)nb, SCAN_NT, 0, ctx->stream>>>(in, n, part);
  scan_partials_kernel<<<1, SCAN_NT, 0, ctx->stream>>>(part, nb);
  scan_down_kernel<<<(unsigned)nb, SCAN_NT, 0, ctx->stream>>>(in, n, part, out);
  count_launch(ctx, 3);
  return check_launch("scan_u32");
}

int launch_raster_to_blocks_u16(cpsz_b200_ctx* ctx, const uint16_t* raster, long long pitch, int r1, int r2,
                                uint16_t* blocks, unsigned long long* hist) {
  long long nseg = nseg_of(r1, r2);
  int nby = (r2 - 1) / BS + 1;
  r2b_kernel<<<grid_of(nseg), NT, 0, ctx->stream>>>(raster, pitch, r1, r2, nby, nseg, blocks);
  count_launch(ctx);
  CPSZ_TRY(check_launch("r2b_kernel"));
  if (hist) return launch_hist_u16(ctx, blocks, (size_t)r1 * r2, hist);
  return CPSZ_OK;
}

int launch_blocks_to_raster_u16(cpsz_b200_ctx* ctx, const uint16_t* blocks, int r1, int r2, uint16_t* raster,
                                long long pitch, const uint8_t* ids, float2* pair) {
  long long nseg = nseg_of(r1, r2);
  int nby = (r2 - 1) / BS + 1;
  b2r_kernel<<<grid_of(nseg), NT, 0, ctx->stream>>>(blocks, r1, r2, nby, nseg, raster, pitch, ids, pair);
  count_launch(ctx);
  return check_launch("b2r_kernel");
}

size_t segment_scan_tmp_bytes(int r1, int r2) { return scan_u32_tmp_bytes((size_t)nseg_of(r1, r2)); }

size_t strip_count(int r1, int r2) {
  const long long nbx = (r1 + BS - 1) / BS, nsc = (r2 + STRIP_W - 1) / STRIP_W;
  return (size_t)(nbx * nsc);
}

int launch_r2b_strips(cpsz_b200_ctx* ctx, const uint16_t* raster, long long pitch, int r1, int r2, uint16_t* blocks,
                      unsigned int* strip_cnt, unsigned int* strip_off, void* scan_tmp) {
  const size_t ns = strip_count(r1, r2);
  if (ns == 0) return CPSZ_OK;
  if (ns > 0x7fffffffu) return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu strips", ns);
  const int nsc = (r2 + STRIP_W - 1) / STRIP_W;
  r2b_strip_kernel<<<(unsigned)ns, STRIP_NT, 0, ctx->stream>>>(raster, pitch, r1, r2, nsc, blocks, strip_cnt);
  count_launch(ctx);
  CPSZ_TRY(check_launch("r2b_strip_kernel"));
  return launch_scan_u32(ctx, strip_cnt, strip_off, ns, scan_tmp);
}

int launch_gather_strips(cpsz_b200_ctx* ctx, const uint16_t* raster, long long pitch, const float* x,
                         long long x_pitch, int r1, int r2, const unsigned int* strip_off, float* unpred) {
  const size_t ns = strip_count(r1, r2);
  if (ns == 0) return CPSZ_OK;
  const int nsc = (r2 + STRIP_W - 1) / STRIP_W;
  gather_strip_kernel<<<(unsigned)ns, STRIP_NT, 0, ctx->stream>>>(raster, pitch, x, x_pitch, r1, r2, nsc, strip_off,
                                                                  unpred);
  count_launch(ctx);
  return check_launch("gather_strip_kernel");
}

int launch_segment_scan(cpsz_b200_ctx* ctx, const uint16_t* codes_raster, long long pitch, int r1, int r2,
                        unsigned int* seg_count, unsigned int* seg_off, void* scan_tmp) {
  long long nseg = nseg_of(r1, r2);
  int nby = (r2 - 1) / BS + 1;
  seg_count_kernel<<<grid_of(nseg), NT, 0, ctx->stream>>>(codes_raster, pitch, r1, r2, nby, nseg, seg_count);
  count_launch(ctx);
  CPSZ_TRY(check_launch("seg_count_kernel"));
  return launch_scan_u32(ctx, seg_count, seg_off, (size_t)nseg, scan_tmp);
}

int launch_gather_unpred(cpsz_b200_ctx* ctx, const uint16_t* codes_raster, long long pitch, const float* x,
                         long long x_pitch, int r1, int r2, const unsigned int* seg_off, float* unpred) {
  long long nseg = nseg_of(r1, r2);
  int nby = (r2 - 1) / BS + 1;
  gather_kernel<<<grid_of(nseg), NT, 0, ctx->stream>>>(codes_raster, pitch, x, x_pitch, r1, r2, nby, nseg, seg_off,
                                                       unpred);
  count_launch(ctx);
  return check_launch("gather_kernel");
}

int launch_scatter_unpred(cpsz_b200_ctx* ctx, const uint16_t* codes_raster, long long pitch, const float* unpred,
                          unsigned long long n_unpred, int r1, int r2, const unsigned int* seg_off, float2* pairs) {
  long long nseg = nseg_of(r1, r2);
  int nby = (r2 - 1) / BS + 1;
  scatter_kernel<<<grid_of(nseg), NT, 0, ctx->stream>>>(codes_raster, pitch, unpred, n_unpred, r1, r2, nby, nseg,
                                                        seg_off, pairs, ctx->d_flag);
  count_launch(ctx);
  return check_launch("scatter_kernel");
}

}  // namespace cpsz
