// blocks.cu -- 12x12 block-order plumbing of the 2D field blobs, and a
// generic device-wide exclusive scan.
//
// The reference emits quantization codes and unpredictable values in 12x12
// block order (blocks row-major, rows inside a block, src/sz_compress_3d.cpp:
// 126-193): element (i, j) sits at block-order position
//   bi*12*r2 + bj*12*h + li*w + lj,   h = rows of block-row bi (12, or the
//   remainder), w = columns of block bj (12, or the remainder).
#include <algorithm>

#include "kernels.h"
#include "lookback.cuh"

namespace cpsz {

namespace {

constexpr int BS = 12;
constexpr unsigned FULLM = 0xffffffffu;

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
// one contiguous range.  A CTA stages the strip in shared memory as rows and
// moves it between the two orders with 16-byte global loads and stores on both
// sides (a thread issues all of its loads before it stores any: the kernels
// are bound by memory latency, not by instructions).
constexpr int STRIP_BLOCKS = 32;
constexpr int STRIP_W = STRIP_BLOCKS * BS;  // 384 columns
constexpr int STRIP_NT = 256;
constexpr int STRIP_TP = STRIP_W + 8;  // shared row pitch in u16: 784 bytes, 16-byte rows
constexpr int STRIP_VEC = (BS * STRIP_W / 8 + STRIP_NT - 1) / STRIP_NT;  // 16-byte vectors per thread: 3

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

// Element e of a strip's block-order image: block b, row li and column lj
// inside it (w = the block's width).  Every block but the last is 12 wide, so
// b = e / (12 h) clamped to the last block.
struct StripPos {
  int b, li, lj, w;
};
__device__ __forceinline__ StripPos strip_pos(const StripGeom& g, int e) {
  StripPos p;
  p.b = min(e / (BS * g.h), g.nb - 1);
  const int k = e - p.b * BS * g.h;
  p.w = p.b == g.nb - 1 ? g.wl : BS;
  p.li = k / p.w;
  p.lj = k - p.li * p.w;
  return p;
}
__device__ __forceinline__ void strip_next(const StripGeom& g, StripPos& p) {
  if (++p.lj == p.w) {
    p.lj = 0;
    if (++p.li == g.h) {
      p.li = 0;
      ++p.b;
      p.w = p.b == g.nb - 1 ? g.wl : BS;
    }
  }
}

// The scalar head and tail that align a strip's block-order range to 16
// bytes: elements [0, head) and [head + 8 nvec, E) go one by one, the nvec
// vectors between them 8 at a time.  An unaligned base takes the scalar path.
struct StripSplit {
  int E, head, nvec;
};
__device__ __forceinline__ StripSplit strip_split(const StripGeom& g, const uint16_t* base) {
  StripSplit sp;
  sp.E = g.h * g.W;
  sp.head = sp.E;
  sp.nvec = 0;
  if ((reinterpret_cast<uintptr_t>(base) & 15) == 0) {
    sp.head = min(sp.E, (int)((8 - (g.out0 & 7)) & 7));
    sp.nvec = (sp.E - sp.head) >> 3;
  }
  return sp;
}

// The strips' unpredictable counts are summed by decoupled look-back
// (lookback.cuh): a CTA takes the next strip in ticket order, so every
// earlier strip belongs to a CTA that is running or done.  One load per lane
// could not keep pace with tens of thousands of strips (windows of in-flight
// strips that had not yet published their prefix grew to hundreds), hence
// the look-back's several windows per round trip.
constexpr long long LOOKBACK_SPIN = 1ll << 24;

// Warp 0 of a strip's CTA: the exclusive prefix of its blocks' zero counts
// (bpre), its own count published, and the count of all earlier strips
// (s_excl); the last strip also stores the component's total beside the
// ticket.  A look-back that waits past its bound sets FLAG_TIMEOUT.
__device__ __forceinline__ void strip_prefix(unsigned long long* status, unsigned int s, unsigned int ns,
                                             const StripGeom& g, const unsigned int* bz, unsigned int* bpre,
                                             unsigned long long* s_excl, int lane, int* flag) {
  const unsigned int v = lane < g.nb ? bz[lane] : 0u;
  unsigned int inc = v;  // inclusive scan of the block counts
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned int y = __shfl_up_sync(FULLM, inc, d);
    if (lane >= d) inc += y;
  }
  bpre[lane] = inc - v;
  const unsigned long long tot = __shfl_sync(FULLM, inc, 31);
  if (lane == 0) lookback_publish(status, s, tot);
  const unsigned long long excl = lookback_warp(status, s, tot, lane, LOOKBACK_SPIN, flag);
  if (lane == 0) {
    *s_excl = excl;
    if (s == ns - 1) reinterpret_cast<unsigned int*>(status + ns)[1] = (unsigned int)(excl + tot);
  }
}

__device__ __forceinline__ unsigned int lanemask_lt(int lane) { return (1u << lane) - 1u; }

struct StripPass {
  const uint16_t* raster;
  const float* x;
  uint16_t* blocks;
  float* unpred;
  unsigned long long* status;  // ns words, then the ticket and the component total (u32 each); zeroed
};

// Compression, one launch for both components: codes raster -> block order,
// and the unpredictable values (code 0) in block order.
__global__ void __launch_bounds__(STRIP_NT) strip_pass_kernel(StripPass P0, StripPass P1, long long pitch,
                                                              long long x_pitch, int r1, int r2, int nsc,
                                                              unsigned int ns, int* flag) {
  __shared__ __align__(16) uint16_t t[BS][STRIP_TP];
  __shared__ unsigned int bz[STRIP_BLOCKS], bpre[STRIP_BLOCKS];
  __shared__ unsigned int s_idx;
  __shared__ unsigned long long s_excl;
  const StripPass P = blockIdx.y ? P1 : P0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_idx = atomicAdd(reinterpret_cast<unsigned int*>(P.status + ns), 1u);
  if (threadIdx.x < STRIP_BLOCKS) bz[threadIdx.x] = 0;
  __syncthreads();
  const unsigned int s = s_idx;
  const StripGeom g = strip_geom(s, r1, r2, nsc);

  // rows into shared memory
  const uint16_t* src = P.raster + (long long)g.bi * BS * pitch + g.c0;
  if (((reinterpret_cast<uintptr_t>(P.raster) | (uintptr_t)(2 * pitch)) & 15) == 0) {
    const int nv = g.W >> 3, tot = g.h * nv;  // c0 is a multiple of 8, so every row's vectors are aligned
    uint4 v[STRIP_VEC];
#pragma unroll
    for (int it = 0; it < STRIP_VEC; it++) {
      const int q = threadIdx.x + it * STRIP_NT;
      if (q < tot) {
        const int li = q / nv;
        v[it] = __ldg(reinterpret_cast<const uint4*>(src + (long long)li * pitch) + (q - li * nv));
      }
    }
#pragma unroll
    for (int it = 0; it < STRIP_VEC; it++) {
      const int q = threadIdx.x + it * STRIP_NT;
      if (q < tot) {
        const int li = q / nv;
        reinterpret_cast<uint4*>(&t[li][0])[q - li * nv] = v[it];
      }
    }
    const int rem = g.W - 8 * nv;  // the field's last columns
    for (int q = threadIdx.x; q < g.h * rem; q += STRIP_NT) {
      const int li = q / rem, c = 8 * nv + (q - li * rem);
      t[li][c] = src[(long long)li * pitch + c];
    }
  } else {
#pragma unroll 6
    for (int q = threadIdx.x; q < g.h * g.W; q += STRIP_NT) {
      const int li = q / g.W, c = q - li * g.W;
      t[li][c] = src[(long long)li * pitch + c];
    }
  }
  __syncthreads();

  // block-order image, 8 elements per 16-byte store; zero codes counted per
  // block (shared atomics only where a thread met zeros)
  uint16_t* dst = P.blocks + g.out0;
  const StripSplit sp = strip_split(g, dst);
  for (int q = threadIdx.x; q < sp.nvec; q += STRIP_NT) {
    const int e0 = sp.head + 8 * q;
    StripPos p = strip_pos(g, e0);
    unsigned int w32[4];
    int zb = p.b;
    unsigned int z = 0;
#pragma unroll
    for (int m = 0; m < 8; m++) {
      if (p.b != zb) {
        if (z) atomicAdd(&bz[zb], z);
        zb = p.b;
        z = 0;
      }
      const unsigned int v = t[p.li][p.b * BS + p.lj];
      z += v == 0;
      w32[m >> 1] = (m & 1) ? (w32[m >> 1] | (v << 16)) : v;
      strip_next(g, p);
    }
    if (z) atomicAdd(&bz[zb], z);
    *reinterpret_cast<uint4*>(dst + e0) = make_uint4(w32[0], w32[1], w32[2], w32[3]);
  }
  const int tail0 = sp.head + 8 * sp.nvec;
  for (int q = threadIdx.x; q < sp.head + (sp.E - tail0); q += STRIP_NT) {
    const int e = q < sp.head ? q : tail0 + (q - sp.head);
    const StripPos p = strip_pos(g, e);
    const uint16_t v = t[p.li][p.b * BS + p.lj];
    dst[e] = v;
    if (v == 0) atomicAdd(&bz[p.b], 1u);
  }
  __syncthreads();
  if (warp == 0) strip_prefix(P.status, s, ns, g, bz, bpre, &s_excl, lane, flag);
  __syncthreads();

  // unpredictable values, in block order
  const unsigned long long excl = s_excl;
  for (int b = warp; b < g.nb; b += STRIP_NT / 32) {
    if (bz[b] == 0) continue;
    const int w = (b == g.nb - 1) ? g.wl : BS;
    const int nk = g.h * w;
    unsigned long long run = excl + bpre[b];
    for (int k0 = 0; k0 < nk; k0 += 32) {
      const int k = k0 + lane;
      int li = 0, col = 0;
      bool z = false;
      if (k < nk) {
        li = k / w;
        col = b * BS + (k - li * w);
        z = t[li][col] == 0;
      }
      const unsigned int m = __ballot_sync(FULLM, z);
      if (z) P.unpred[run + __popc(m & lanemask_lt(lane))] = P.x[(long long)(g.bi * BS + li) * x_pitch + g.c0 + col];
      run += __popc(m);
    }
  }
}

struct StripUnpass {
  const uint16_t* blocks;      // block-order codes
  const uint8_t* ids;          // the component's error-bound ids, raster order (pitch r2)
  const float* unpred;         // unpredictable values, block order
  unsigned long long n_unpred;
  float2* pair;                // raster (pitch r2)
  unsigned long long* status;  // as in StripPass
  int id_shift;                // p = 2^(id_shift * id) * 2^-52: 2 (offline), 1 (offline_log)
};

// Decompression side of a point: the addend 2(code - 32768) * p that the
// wavefront adds to its prediction (p = 4^id * 2^-52 for the offline blob,
// 2^id * 2^-52 for the offline_log one, 0 for id 0;
// src/sz_decompress_cp_preserve_2d.cpp:30-34 and :76-80,
// include/sz_decompression_utils.hpp:65-73), or for code 0 the raw flag with
// the raw value in .x.
__device__ __forceinline__ float2 dec_pair(unsigned int code, unsigned int id, int shift) {
  const float p = id ? __int_as_float((int)(shift * (int)id - 52 + 127) << 23) : 0.f;
  return make_float2((float)(2 * ((int)code - 32768)) * p, __int_as_float(code == 0 ? 1 : 0));
}

// Decompression, one launch for both components: block-order codes -> the
// raster pairs the wavefront reads, with the unpredictable values (block
// order) scattered into the pairs of the zero codes.  The last strip stores
// the number of zero codes, which the host checks against the stored list.
__global__ void __launch_bounds__(STRIP_NT) strip_unpass_kernel(StripUnpass P0, StripUnpass P1, int r1, int r2,
                                                                int nsc, unsigned int ns, int* flag) {
  __shared__ __align__(16) uint16_t t[BS][STRIP_TP];
  __shared__ unsigned int bz[STRIP_BLOCKS], bpre[STRIP_BLOCKS];
  __shared__ unsigned int s_idx;
  __shared__ unsigned long long s_excl;
  const StripUnpass P = blockIdx.y ? P1 : P0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_idx = atomicAdd(reinterpret_cast<unsigned int*>(P.status + ns), 1u);
  if (threadIdx.x < STRIP_BLOCKS) bz[threadIdx.x] = 0;
  __syncthreads();
  const unsigned int s = s_idx;
  const StripGeom g = strip_geom(s, r1, r2, nsc);

  // block-order codes into shared rows, zero codes counted per block
  const uint16_t* src = P.blocks + g.out0;
  const StripSplit sp = strip_split(g, src);
  {
    uint4 v[STRIP_VEC];
#pragma unroll
    for (int it = 0; it < STRIP_VEC; it++) {
      const int q = threadIdx.x + it * STRIP_NT;
      if (q < sp.nvec) v[it] = __ldg(reinterpret_cast<const uint4*>(src + sp.head + 8 * q));
    }
#pragma unroll
    for (int it = 0; it < STRIP_VEC; it++) {
      const int q = threadIdx.x + it * STRIP_NT;
      if (q < sp.nvec) {
        const unsigned int w32[4] = {v[it].x, v[it].y, v[it].z, v[it].w};
        StripPos p = strip_pos(g, sp.head + 8 * q);
        int zb = p.b;
        unsigned int z = 0;
#pragma unroll
        for (int m = 0; m < 8; m++) {
          if (p.b != zb) {
            if (z) atomicAdd(&bz[zb], z);
            zb = p.b;
            z = 0;
          }
          const uint16_t c = (uint16_t)(w32[m >> 1] >> ((m & 1) * 16));
          t[p.li][p.b * BS + p.lj] = c;
          z += c == 0;
          strip_next(g, p);
        }
        if (z) atomicAdd(&bz[zb], z);
      }
    }
  }
  const int tail0 = sp.head + 8 * sp.nvec;
  for (int q = threadIdx.x; q < sp.head + (sp.E - tail0); q += STRIP_NT) {
    const int e = q < sp.head ? q : tail0 + (q - sp.head);
    const StripPos p = strip_pos(g, e);
    const uint16_t c = src[e];
    t[p.li][p.b * BS + p.lj] = c;
    if (c == 0) atomicAdd(&bz[p.b], 1u);
  }
  __syncthreads();
  if (warp == 0) strip_prefix(P.status, s, ns, g, bz, bpre, &s_excl, lane, flag);

  // raster pairs (the other warps start while warp 0 looks back)
  const long long row0 = (long long)g.bi * BS;
  if ((r2 & 3) == 0 && ((reinterpret_cast<uintptr_t>(P.ids) & 3) | (reinterpret_cast<uintptr_t>(P.pair) & 15)) == 0) {
    // 4 columns per item (W is a multiple of 4 here): one u32 of ids in, two 16-byte pair stores out
    constexpr int ROW_VEC = (BS * STRIP_W / 4 + STRIP_NT - 1) / STRIP_NT;  // 5
    const int nq = g.W >> 2, tot = g.h * nq;
    unsigned int idv[ROW_VEC];
#pragma unroll
    for (int u = 0; u < ROW_VEC; u++) {
      const int q = threadIdx.x + u * STRIP_NT;
      if (q < tot) {
        const int li = q / nq;
        idv[u] = __ldg(reinterpret_cast<const unsigned int*>(P.ids + (row0 + li) * r2 + g.c0) + (q - li * nq));
      }
    }
#pragma unroll
    for (int u = 0; u < ROW_VEC; u++) {
      const int q = threadIdx.x + u * STRIP_NT;
      if (q < tot) {
        const int li = q / nq, c = 4 * (q - li * nq);
        const uint2 cw = *reinterpret_cast<const uint2*>(&t[li][c]);
        const float2 a = dec_pair(cw.x & 0xffffu, idv[u] & 0xffu, P.id_shift),
                     b = dec_pair(cw.x >> 16, (idv[u] >> 8) & 0xffu, P.id_shift);
        const float2 d = dec_pair(cw.y & 0xffffu, (idv[u] >> 16) & 0xffu, P.id_shift),
                     e = dec_pair(cw.y >> 16, idv[u] >> 24, P.id_shift);
        float4* out = reinterpret_cast<float4*>(P.pair + (row0 + li) * r2 + g.c0 + c);
        out[0] = make_float4(a.x, a.y, b.x, b.y);
        out[1] = make_float4(d.x, d.y, e.x, e.y);
      }
    }
  } else {
#pragma unroll 6
    for (int q = threadIdx.x; q < g.h * g.W; q += STRIP_NT) {
      const int li = q / g.W, c = q - li * g.W;
      const long long gi = (row0 + li) * r2 + g.c0 + c;
      P.pair[gi] = dec_pair(t[li][c], P.ids[gi], P.id_shift);
    }
  }
  __syncthreads();  // the raw values below overwrite .x of pairs stored above

  // unpredictable values, in block order
  const unsigned long long excl = s_excl;
  for (int b = warp; b < g.nb; b += STRIP_NT / 32) {
    if (bz[b] == 0) continue;
    const int w = (b == g.nb - 1) ? g.wl : BS;
    const int nk = g.h * w;
    unsigned long long run = excl + bpre[b];
    for (int k0 = 0; k0 < nk; k0 += 32) {
      const int k = k0 + lane;
      int li = 0, col = 0;
      bool z = false;
      if (k < nk) {
        li = k / w;
        col = b * BS + (k - li * w);
        z = t[li][col] == 0;
      }
      const unsigned int m = __ballot_sync(FULLM, z);
      if (z) {
        const unsigned long long o = run + __popc(m & lanemask_lt(lane));
        if (o < P.n_unpred) P.pair[(row0 + li) * r2 + g.c0 + col].x = P.unpred[o];
        else atomicOr(flag, FLAG_RAW_RANGE);
      }
      run += __popc(m);
    }
  }
}

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

size_t strip_count(int r1, int r2) {
  const long long nbx = (r1 + BS - 1) / BS, nsc = (r2 + STRIP_W - 1) / STRIP_W;
  return (size_t)(nbx * nsc);
}

size_t strip_scratch_bytes(int r1, int r2) { return 8 * strip_count(r1, r2) + 8; }

const unsigned int* strip_total(const void* scratch, int r1, int r2) {
  return (const unsigned int*)((const char*)scratch + 8 * strip_count(r1, r2) + 4);
}

int launch_strip_pass(cpsz_b200_ctx* ctx, const uint16_t* const raster[2], long long pitch, const float* const x[2],
                      long long x_pitch, int r1, int r2, uint16_t* const blocks[2], float* const unpred[2],
                      void* const scratch[2]) {
  const size_t ns = strip_count(r1, r2);
  if (ns > 0x7fffffffu) return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu strips", ns);
  for (int f = 0; f < 2; f++)  // the totals of an empty field read 0
    CPSZ_CUDA_TRY(cudaMemsetAsync(scratch[f], 0, strip_scratch_bytes(r1, r2), ctx->stream));
  if (ns == 0) return CPSZ_OK;
  const int nsc = (r2 + STRIP_W - 1) / STRIP_W;
  StripPass P[2];
  for (int f = 0; f < 2; f++) P[f] = StripPass{raster[f], x[f], blocks[f], unpred[f], (unsigned long long*)scratch[f]};
  strip_pass_kernel<<<dim3((unsigned)ns, 2), STRIP_NT, 0, ctx->stream>>>(P[0], P[1], pitch, x_pitch, r1, r2, nsc,
                                                                         (unsigned)ns, ctx->d_flag);
  count_launch(ctx);
  return check_launch("strip_pass_kernel");
}

int launch_strip_unpass(cpsz_b200_ctx* ctx, const uint16_t* const blocks[2], const uint8_t* const ids[2],
                        const float* const unpred[2], const unsigned long long n_unpred[2], int r1, int r2,
                        float2* const pair[2], void* const scratch[2], int id_shift) {
  const size_t ns = strip_count(r1, r2);
  if (ns > 0x7fffffffu) return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu strips", ns);
  for (int f = 0; f < 2; f++)  // the totals of an empty field read 0
    CPSZ_CUDA_TRY(cudaMemsetAsync(scratch[f], 0, strip_scratch_bytes(r1, r2), ctx->stream));
  if (ns == 0) return CPSZ_OK;
  const int nsc = (r2 + STRIP_W - 1) / STRIP_W;
  StripUnpass P[2];
  for (int f = 0; f < 2; f++)
    P[f] = StripUnpass{blocks[f], ids[f], unpred[f], n_unpred[f], pair[f], (unsigned long long*)scratch[f], id_shift};
  strip_unpass_kernel<<<dim3((unsigned)ns, 2), STRIP_NT, 0, ctx->stream>>>(P[0], P[1], r1, r2, nsc, (unsigned)ns,
                                                                           ctx->d_flag);
  count_launch(ctx);
  return check_launch("strip_unpass_kernel");
}

}  // namespace cpsz
