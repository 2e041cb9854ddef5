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
// One pass per component.  A CTA takes the next strip in ticket order (tickets
// go out in the order CTAs start, so every earlier strip belongs to a CTA that
// is running or done), stages it, writes its block-order image, publishes its
// unpredictable count, finds the count of all earlier strips by a decoupled
// look-back over their published words (Merrill & Garland, "Single-pass
// Parallel Prefix Scan with Decoupled Look-back", 2016) and writes its
// unpredictable values in block order.  Status words: 2-bit state (0 = not
// yet, AGG = the strip's own count, PRE = inclusive prefix) over a 62-bit count.
constexpr unsigned long long ST_AGG = 1ull << 62, ST_PRE = 2ull << 62, ST_VAL = (1ull << 62) - 1;
constexpr long long LOOKBACK_SPIN = 1ll << 24;
constexpr unsigned FULLM = 0xffffffffu;

struct StripPass {
  const uint16_t* raster;
  const float* x;
  uint16_t* blocks;
  float* unpred;
  unsigned long long* status;  // ns words, then the ticket and the field total (u32 each); zeroed
};

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void __launch_bounds__(STRIP_NT) strip_pass_kernel(StripPass P0, StripPass P1, long long pitch,
                                                              long long x_pitch, int r1, int r2, int nsc,
                                                              unsigned int ns, int* flag) {
  __shared__ uint16_t t[BS][STRIP_W + 2];
  __shared__ unsigned int bz[STRIP_BLOCKS], bpre[STRIP_BLOCKS];
  __shared__ unsigned int s_idx;
  __shared__ unsigned long long s_excl;
  const StripPass P = blockIdx.y ? P1 : P0;
  unsigned int* ticket = reinterpret_cast<unsigned int*>(P.status + ns);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_idx = atomicAdd(ticket, 1u);
  __syncthreads();
  const unsigned int s = s_idx;
  const StripGeom g = strip_geom(s, r1, r2, nsc);
  const uint16_t* src = P.raster + (long long)g.bi * BS * pitch + g.c0;
  for (int li = 0; li < g.h; li++)
    for (int c = threadIdx.x; c < g.W; c += STRIP_NT) t[li][c] = src[(long long)li * pitch + c];
  __syncthreads();
  // block-order image, one warp per block: element k of block b is row k / w,
  // column k % w (w = 12 except a row's last block); the float quotient is
  // exact here because (k + 0.5) / w stays >= 1/24 away from an integer
  for (int b = warp; b < g.nb; b += STRIP_NT / 32) {
    const int w = (b == g.nb - 1) ? g.wl : BS;
    const float inv_w = 1.0f / (float)w;
    const int nk = g.h * w;
    uint16_t* dst = P.blocks + g.out0 + (long long)b * BS * g.h;
    unsigned int z = 0;
    for (int k = lane; k < nk; k += 32) {
      const int li = (int)(((float)k + 0.5f) * inv_w);
      const uint16_t v = t[li][b * BS + (k - li * w)];
      dst[k] = v;
      z += v == 0;
    }
    z = __reduce_add_sync(FULLM, z);
    if (lane == 0) bz[b] = z;
  }
  __syncthreads();
  if (warp == 0) {
    const unsigned int v = lane < g.nb ? bz[lane] : 0u;
    unsigned int inc = v;  // inclusive scan of the block counts
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned int y = __shfl_up_sync(FULLM, inc, d);
      if (lane >= d) inc += y;
    }
    bpre[lane] = inc - v;
    const unsigned long long tot = __shfl_sync(FULLM, inc, 31);
    unsigned long long excl = 0;
    if (s == 0) {
      if (lane == 0) st_release64(&P.status[0], ST_PRE | tot);
    } else {
      if (lane == 0) st_release64(&P.status[s], ST_AGG | tot);
      long long p = (long long)s - 1;
      long long spins = 0;
      for (;;) {
        const long long q = p - lane;
        const unsigned long long w = q >= 0 ? ld_acquire64(&P.status[q]) : ST_PRE;  // before strip 0: prefix 0
        const unsigned int pre_m = __ballot_sync(FULLM, (w & ~ST_VAL) == ST_PRE);
        const unsigned int none_m = __ballot_sync(FULLM, (w & ~ST_VAL) == 0);
        const int last = pre_m ? __ffs(pre_m) - 1 : 31;  // the nearest prefix, or the whole window
        const unsigned int upto = last == 31 ? FULLM : ((1u << (last + 1)) - 1u);
        if (none_m & upto) {  // a nearer strip has not published yet
          if (++spins > LOOKBACK_SPIN) {
            if (lane == 0) atomicOr(flag, FLAG_TIMEOUT);
            break;
          }
          __nanosleep(64);
          continue;
        }
        unsigned long long add = lane <= last ? (w & ST_VAL) : 0ull;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) add += __shfl_xor_sync(FULLM, add, d);
        excl += add;
        if (pre_m) break;
        p -= 32;
      }
      if (lane == 0) st_release64(&P.status[s], ST_PRE | (excl + tot));
    }
    if (lane == 0) {
      s_excl = excl;
      if (s == ns - 1) ticket[1] = (unsigned int)(excl + tot);
    }
  }
  __syncthreads();
  // unpredictable values, in block order
  const unsigned long long excl = s_excl;
  for (int b = warp; b < g.nb; b += STRIP_NT / 32) {
    if (bz[b] == 0) continue;
    const int w = (b == g.nb - 1) ? g.wl : BS;
    const float inv_w = 1.0f / (float)w;
    const int nk = g.h * w;
    unsigned long long run = excl + bpre[b];
    for (int k0 = 0; k0 < nk; k0 += 32) {
      const int k = k0 + lane;
      int li = 0, col = 0;
      bool z = false;
      if (k < nk) {
        li = (int)(((float)k + 0.5f) * inv_w);
        col = b * BS + (k - li * w);
        z = t[li][col] == 0;
      }
      const unsigned int m = __ballot_sync(FULLM, z);
      if (z)
        P.unpred[run + __popc(m & ((1u << lane) - 1u))] =
            P.x[(long long)(g.bi * BS + li) * x_pitch + g.c0 + col];
      run += __popc(m);
    }
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

size_t strip_scratch_bytes(int r1, int r2) { return 8 * strip_count(r1, r2) + 8; }

int launch_strip_pass(cpsz_b200_ctx* ctx, const uint16_t* const raster[2], long long pitch, const float* const x[2],
                      long long x_pitch, int r1, int r2, uint16_t* const blocks[2], float* const unpred[2],
                      void* const scratch[2]) {
  const size_t ns = strip_count(r1, r2);
  if (ns == 0) return CPSZ_OK;
  if (ns > 0x7fffffffu) return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu strips", ns);
  const int nsc = (r2 + STRIP_W - 1) / STRIP_W;
  StripPass P[2];
  for (int f = 0; f < 2; f++) {
    CPSZ_CUDA_TRY(cudaMemsetAsync(scratch[f], 0, strip_scratch_bytes(r1, r2), ctx->stream));
    P[f] = StripPass{raster[f], x[f], blocks[f], unpred[f], (unsigned long long*)scratch[f]};
  }
  strip_pass_kernel<<<dim3((unsigned)ns, 2), STRIP_NT, 0, ctx->stream>>>(P[0], P[1], pitch, x_pitch, r1, r2, nsc,
                                                                         (unsigned)ns, ctx->d_flag);
  count_launch(ctx);
  return check_launch("strip_pass_kernel");
}

const unsigned int* strip_total(const void* scratch, int r1, int r2) {
  return (const unsigned int*)((const char*)scratch + 8 * strip_count(r1, r2) + 4);
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
