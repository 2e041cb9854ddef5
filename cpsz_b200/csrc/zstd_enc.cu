// zstd_enc.cu -- the GPU lossless stage: Zstandard frames of device data.
//
// The reference applies ZSTD_compress(level 3) to every blob on the host
// (src/sz_lossless.cpp:11-26); here the same kind of frame is written on the
// GPU (format: zstd_format.h), readable by any Zstandard decoder and so by the
// reference's sz_lossless_decompress.  The input is cut into 8 KB blocks that
// are encoded independently, one warp each (16 warps an SM):
//   0. the warp stages its block in shared memory with 16-byte loads, so the
//      match loop below (a dependent chain: one step per match on the
//      Huffman bit streams of a blob, a match every few bytes) waits on
//      shared memory, not on global loads (32 KB blocks read from global
//      memory: 9.6 ms for a 89 MB blob; staged, with four warps an SM for
//      lack of shared memory: 17.7 ms);
//   1. greedy matching: the warp looks at 32 consecutive positions at a time,
//      each lane hashing the 4 bytes at its position into the warp's table of
//      last positions (shared memory, 2048 16-bit entries) and checking the
//      candidate; the first matching lane starts a match, which the warp
//      extends 32 bytes per step; positions before it enter the table.  With
//      no match the window advances 32 positions;
//   2. the block body: raw literals (the bytes no match covers, copied by the
//      warp) and the sequences section, coded by one lane with the predefined
//      FSE tables (every offset a real offset, so blocks share no state);
//      an all-equal block becomes an RLE block, a block that does not shrink
//      a raw block.
// Block sizes are scanned and a gather kernel places the blocks after the
// frame header.  Matches stay inside their block.
#include <cstring>

#include "kernels.h"
#include "zstd_format.h"

namespace cpsz {

namespace {

constexpr int ZBLK = 8 * 1024;
constexpr int ZHT_BITS = 11;
constexpr int ZWARPS = 8;  // blocks per CTA
constexpr int ZMAXSEQ = ZBLK / zstd::kMinMatch + 1;
constexpr int ZOUT = ZBLK + 16;  // per-block output slot: a raw block and its header fit
constexpr unsigned FULLMASK = 0xffffffffu;

__constant__ zstd::Tables c_tables;

__device__ __forceinline__ uint32_t load4(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
__device__ __forceinline__ uint32_t zhash(uint32_t v) { return (v * 2654435761u) >> (32 - ZHT_BITS); }

// Shared memory of one warp: its block's bytes and its hash table of
// block-local positions + 1 (0 = empty).
struct ZWarpSmem {
  uint8_t data[ZBLK];
  uint16_t ht[1 << ZHT_BITS];
};
constexpr size_t ZSMEM = sizeof(ZWarpSmem) * ZWARPS;

// One warp per block: the block staged in shared memory (16-byte loads), so
// the match loop's byte reads are shared-memory reads; matches, then the
// encoded block (header included) into its slot of `slots`; sizes[b] = the
// encoded block's bytes.
__global__ void __launch_bounds__(32 * ZWARPS) zstd_block_kernel(const uint8_t* __restrict__ src, size_t n,
                                                                 long long nblocks, zstd::Seq* __restrict__ seq_all,
                                                                 uint8_t* __restrict__ slots,
                                                                 unsigned int* __restrict__ sizes) {
  extern __shared__ __align__(16) uint8_t zsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long b = (long long)blockIdx.x * ZWARPS + warp;
  if (b >= nblocks) return;  // warp-uniform; only __syncwarp below
  ZWarpSmem& W = reinterpret_cast<ZWarpSmem*>(zsm)[warp];
  const size_t s0 = (size_t)b * ZBLK;
  const int len = (int)((n - s0) < (size_t)ZBLK ? (n - s0) : (size_t)ZBLK);
  {
    const uint8_t* g = src + s0;
    int k0 = 0;
    if (((uintptr_t)g & 15) == 0) {
      const int nv = len >> 4;
      for (int q = lane; q < nv; q += 32)
        reinterpret_cast<uint4*>(W.data)[q] = __ldcs(reinterpret_cast<const uint4*>(g) + q);
      k0 = nv << 4;
    }
    for (int i = k0 + lane; i < len; i += 32) W.data[i] = g[i];
    __syncwarp();
  }
  const uint8_t* blk = W.data;
  uint8_t* out = slots + (size_t)b * ZOUT;
  const bool last = b == nblocks - 1;
  uint16_t* ht = W.ht;

  // ---- RLE block: every byte equal ----
  {
    const uint8_t first = len > 0 ? blk[0] : 0;
    bool same = true;
    for (int i = lane; i < len && same; i += 32) same = blk[i] == first;
    if (__all_sync(FULLMASK, same) && len > 1) {
      if (lane == 0) {
        zstd::write_block_header(out, last, 1, (uint32_t)len);
        out[3] = first;
        sizes[b] = 4;
      }
      return;
    }
  }

  // ---- greedy matching ----
  for (int i = lane; i < (1 << ZHT_BITS); i += 32) ht[i] = 0;
  __syncwarp();
  zstd::Seq* seqs = seq_all + (size_t)b * ZMAXSEQ;
  int nseq = 0, anchor = 0, p = 0, nlit = 0;
  while (p + zstd::kMinMatch <= len) {
    const int pos = p + lane;
    const bool ok = pos + zstd::kMinMatch <= len;
    const uint32_t v = ok ? load4(blk + pos) : 0u;
    const uint32_t h = zhash(v);
    const uint32_t cand = ok ? ht[h] : 0u;  // position + 1 in the block, 0 = none
    const bool m = cand != 0u && load4(blk + cand - 1) == v;
    const unsigned bal = __ballot_sync(FULLMASK, m);
    const int f = bal ? __ffs(bal) - 1 : 32;
    __syncwarp();
    if (ok && lane <= f) ht[h] = (uint16_t)(pos + 1);
    __syncwarp();
    if (!bal) {
      p += 32;
      continue;
    }
    const int mpos = p + f;
    const int mref = (int)__shfl_sync(FULLMASK, cand, f) - 1;
    int L = zstd::kMinMatch;
    for (;;) {
      const int i = mpos + L + lane;
      const bool eq = i < len && blk[mref + L + lane] == blk[i];
      const unsigned ne = __ballot_sync(FULLMASK, !eq);
      if (ne) {
        L += __ffs(ne) - 1;
        break;
      }
      L += 32;
    }
    if (lane == 0) seqs[nseq] = zstd::Seq{(uint32_t)(mpos - anchor), (uint32_t)L, (uint32_t)(mpos - mref)};
    nseq++;
    nlit += mpos - anchor;
    anchor = mpos + L;
    p = anchor;
  }
  nlit += len - anchor;
  __syncwarp();

  // ---- block body: raw literals, then the sequences ----
  uint8_t* body = out + 3;
  const int cap = len - 1;  // a compressed body must be smaller than the raw block
  int k = 0;
  bool comp = nseq > 0 && nlit + 3 < cap;
  if (comp) {
    uint8_t hdr[3];
    k = (int)zstd::write_raw_literals_header((uint32_t)nlit, hdr);
    if (lane < k) body[lane] = hdr[lane];
    int at = 0;
    for (int q = 0; q <= nseq; q++) {
      int lit;
      if (q < nseq) {
        const zstd::Seq s = seqs[q];
        lit = (int)s.lit;
        for (int i = lane; i < lit; i += 32) body[k + i] = blk[at + i];
        at += lit + (int)s.ml;
      } else {
        lit = len - at;
        for (int i = lane; i < lit; i += 32) body[k + i] = blk[at + i];
      }
      k += lit;
    }
    __syncwarp();
    int total = 0;
    if (lane == 0) {
      const size_t sq = zstd::write_sequences(c_tables, seqs, nseq, body + k, (size_t)(cap - k));
      total = sq ? k + (int)sq : 0;
    }
    total = __shfl_sync(FULLMASK, total, 0);
    comp = total > 0 && total < len;
    if (comp && lane == 0) {
      zstd::write_block_header(out, last, 2, (uint32_t)total);
      sizes[b] = 3 + total;
    }
  }
  if (!comp) {
    __syncwarp();
    for (int i = lane; i < len; i += 32) body[i] = blk[i];
    if (lane == 0) {
      zstd::write_block_header(out, last, 0, (uint32_t)len);
      sizes[b] = 3 + len;
    }
  }
}

// Block b's bytes to dst + off[b] (one CTA per block).
__global__ void __launch_bounds__(256) zstd_gather_kernel(const uint8_t* __restrict__ slots,
                                                          const unsigned int* __restrict__ sizes,
                                                          const unsigned int* __restrict__ off,
                                                          uint8_t* __restrict__ dst) {
  const long long b = blockIdx.x;
  const uint8_t* s = slots + (size_t)b * ZOUT;
  uint8_t* d = dst + off[b];
  const unsigned int sz = sizes[b];
  for (unsigned int i = threadIdx.x; i < sz; i += blockDim.x) d[i] = s[i];
}

bool g_tables_ready[64] = {};
bool g_smem_set[64] = {};

}  // namespace

size_t zstd_frame_bound(size_t n) {
  const size_t nb = n ? (n + ZBLK - 1) / ZBLK : 1;
  return zstd::kFrameHeader + n + 4 * nb;
}

size_t zstd_tmp_bytes(size_t n) {
  const size_t nb = n ? (n + ZBLK - 1) / ZBLK : 1;
  auto al = [](size_t x) { return (x + 255) / 256 * 256 + 256; };
  return al(nb * ZMAXSEQ * sizeof(zstd::Seq)) + al(nb * ZOUT) + 2 * al(4 * (nb + 1)) + al(scan_u32_tmp_bytes(nb));
}

int launch_zstd_frame(cpsz_b200_ctx* ctx, const uint8_t* d_in, size_t n, uint8_t* d_out, size_t out_cap,
                      size_t* out_size, void* tmp) {
  cudaStream_t st = ctx->stream;
  if (!g_tables_ready[ctx->device & 63]) {
    zstd::Tables T;
    zstd::build_tables(&T);
    CPSZ_CUDA_TRY(cudaMemcpyToSymbol(c_tables, &T, sizeof(T)));
    g_tables_ready[ctx->device & 63] = true;
  }
  const long long nb = n ? (long long)((n + ZBLK - 1) / ZBLK) : 0;
  auto al = [](size_t x) { return (x + 255) / 256 * 256 + 256; };
  uint8_t* t = (uint8_t*)tmp;
  zstd::Seq* seqs = (zstd::Seq*)t;
  t += al((size_t)(nb ? nb : 1) * ZMAXSEQ * sizeof(zstd::Seq));
  uint8_t* slots = t;
  t += al((size_t)(nb ? nb : 1) * ZOUT);
  unsigned int* sizes = (unsigned int*)t;
  t += al(4 * (size_t)(nb + 1));
  unsigned int* off = (unsigned int*)t;
  t += al(4 * (size_t)(nb + 1));
  void* scan_tmp = t;
  uint8_t hdr[zstd::kFrameHeader + 3];
  size_t h = zstd::write_frame_header(hdr, n);
  if (nb == 0) {
    // an empty frame: one empty raw block
    zstd::write_block_header(hdr + h, true, 0, 0);
    h += 3;
    if (out_cap < h) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < frame size %zu", out_cap, h);
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d_out, hdr, h, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaStreamSynchronize(st));
    *out_size = h;
    return CPSZ_OK;
  }
  if (n > ((size_t)1 << 32) - 4 * (size_t)nb - 64)
    return set_error(CPSZ_ERR_UNSUPPORTED, "lossless stage input of %zu bytes exceeds 4 GB", n);
  if (!g_smem_set[ctx->device & 63]) {
    CPSZ_CUDA_TRY(cudaFuncSetAttribute(zstd_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZSMEM));
    g_smem_set[ctx->device & 63] = true;
  }
  zstd_block_kernel<<<(unsigned)((nb + ZWARPS - 1) / ZWARPS), 32 * ZWARPS, ZSMEM, st>>>(d_in, n, nb, seqs, slots,
                                                                                         sizes);
  count_launch(ctx);
  CPSZ_TRY(check_launch("zstd_block_kernel"));
  CPSZ_TRY(launch_scan_u32(ctx, sizes, off, (size_t)nb, scan_tmp));
  unsigned int total = 0;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(&total, off + nb, 4, cudaMemcpyDeviceToHost, st));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(st));
  const size_t fsize = h + total;
  *out_size = fsize;
  if (fsize > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < frame size %zu", out_cap, fsize);
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d_out, hdr, h, cudaMemcpyHostToDevice, st));
  zstd_gather_kernel<<<(unsigned)nb, 256, 0, st>>>(slots, sizes, off, d_out + h);
  count_launch(ctx);
  return check_launch("zstd_gather_kernel");
}

}  // namespace cpsz
