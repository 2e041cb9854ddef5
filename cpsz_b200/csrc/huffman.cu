// huffman.cu -- GPU side of the SZ-1.x Huffman codec used by the reference
// (src/sz_huffman.cpp): symbol histograms, the MSB-first bit packer and a
// self-synchronising parallel decoder.
//
// Encoder.  The reference's packer (encode, src/sz_huffman.cpp:217-320) emits
// the MSB-first concatenation of the codes, zero padded to a byte.  Here one
// persistent kernel reads every symbol once: a tile of 8192 consecutive
// symbols sums and scans its code lengths, finds its starting bit by a
// decoupled look-back over the earlier tiles' published bit counts, packs its
// codes into a shared-memory word buffer aligned to the global 32-bit word
// grid and stores it with coalesced stores (atomicOr for the two edge words,
// shared with the neighbouring tiles).  Words are stored byte-swapped so
// memory holds the big-endian byte stream the reference writes.
//
// Decoder.  The reference stream has no chunk index, so decoding uses
// self-synchronisation (after Weissenberger & Schmidt, ICPP 2018): the stream
// is cut into S-bit subsequences, each thread first decodes its subsequence
// from its nominal start (finding the codeword boundary at which it leaves),
// then subsequences whose assumed start differs from their predecessor's exit
// are re-decoded from that exit until nothing changes (prefix codes
// resynchronise within a few codewords, so this settles in one or two
// rounds), then counts are scanned and every thread decodes again, writing its
// symbols.  Lookup is a 2^12-entry first-level table with a bit-serial tree
// walk for longer codes.
#include "kernels.h"
#include "lookback.cuh"

namespace cpsz {

namespace {

// ---- encoder: one pass with decoupled look-back --------------------------------------
constexpr int PK_NT = 256;                  // threads per CTA
constexpr int PK_SPT = 32;                  // symbols per thread (a contiguous run)
constexpr int PK_TILE = PK_NT * PK_SPT;     // symbols per tile
constexpr int PK_WORDS = PK_TILE;           // staged words of a tile whose codes are at most 32 bits
constexpr int PK_WIN = 1536;                // codebook entries cached in shared memory: u16 symbols
constexpr int PK_WIN_LO = 32768 - PK_WIN / 2;  // [PK_WIN_LO, PK_WIN_LO + PK_WIN) (all 256 for u8)
constexpr int PK_CTAS_PER_SM = 4;
constexpr long long PK_SPIN_LIMIT = 1ll << 22;  // look-back polls before giving up (FLAG_TIMEOUT)

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

template <class Sym>
struct PackWin {
  static constexpr int lo = sizeof(Sym) == 1 ? 0 : PK_WIN_LO;
  static constexpr int n = sizeof(Sym) == 1 ? 256 : PK_WIN;
  static constexpr int per_word = 4 / (int)sizeof(Sym);  // symbols per 32-bit register
};

struct PackShared {
  uint32_t words[PK_WORDS];     // the tile's packed bits from its first bit (tile-relative)
  uint32_t lcode[PK_WIN];       // codes of at most 32 bits, left-aligned (0 for longer codes)
  uint8_t len[PK_WIN];
  unsigned int warp_bits[PK_NT / 32];
  unsigned long long excl;
  unsigned int tile;
};

// Code length of symbol s (the cached window, else the global table).
template <class Sym>
__device__ __forceinline__ unsigned pk_len(const PackShared& sh, unsigned s, const uint8_t* __restrict__ len) {
  if (sizeof(Sym) == 1) return sh.len[s];
  const unsigned d = s - (unsigned)PackWin<Sym>::lo;
  return d < (unsigned)PackWin<Sym>::n ? sh.len[d] : __ldg(len + s);
}
// Left-aligned code of symbol s whose length l is at most 32.
template <class Sym>
__device__ __forceinline__ uint32_t pk_lcode(const PackShared& sh, unsigned s, unsigned l,
                                             const unsigned long long* __restrict__ code) {
  if (sizeof(Sym) == 1) return sh.lcode[s];
  const unsigned d = s - (unsigned)PackWin<Sym>::lo;
  if (d < (unsigned)PackWin<Sym>::n) return sh.lcode[d];
  return l ? (uint32_t)(__ldg(code + s) << (32 - l)) : 0u;
}

// Persistent packer.  Tiles of PK_TILE symbols are taken in order from a
// ticket; thread t of a tile owns its symbols t*32 .. t*32+31.  Per tile:
//   1. code lengths (kept in registers) summed and scanned in the CTA; the
//      tile's bit count is published for the look-back (lookback.cuh);
//   2. the codes are packed tile-relative into the shared word buffer: each
//      thread appends its codes to a 64-bit register and stores every word
//      it completes (a word is completed by exactly one thread, which also
//      zeroes the bits of earlier threads in it); after a barrier each
//      thread ORs in its last, partial word;
//   3. warp 0 finds the tile's starting bit (by now the predecessors have
//      mostly published); the buffer goes out shifted onto the global word
//      grid with coalesced stores, the two edge words (shared with the
//      neighbouring tiles) by atomicOr.
// A tile with a code longer than 32 bits (possible only for skewed
// histograms) finds its starting bit first and ORs its words straight into
// global memory.  The stream starts at bit `bit0` (0-31) of out[0].
template <class Sym, bool MAP0>
__global__ void __launch_bounds__(PK_NT, PK_CTAS_PER_SM)
    pack_kernel(const Sym* __restrict__ sym, size_t n, const unsigned long long* __restrict__ code,
                const uint8_t* __restrict__ len, int nsym, uint32_t* __restrict__ out, size_t cap_words, int bit0,
                unsigned long long* __restrict__ state, unsigned int* __restrict__ ticket, unsigned long long ntiles,
                unsigned long long* __restrict__ d_total, int* __restrict__ flag) {
  using W = PackWin<Sym>;
  constexpr int NW = PK_SPT / W::per_word;  // registers of packed symbols
  constexpr int SB = 8 * (int)sizeof(Sym);
  constexpr unsigned SMASK = sizeof(Sym) == 1 ? 0xffu : 0xffffu;
  __shared__ PackShared sh;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < W::n; i += PK_NT) {
    const int s = W::lo + i;
    const unsigned l = s < nsym ? len[s] : 0u;
    sh.len[i] = (uint8_t)l;
    sh.lcode[i] = (l >= 1 && l <= 32) ? (uint32_t)(code[s] << (32 - l)) : 0u;
  }
  const bool vec_ok = ((uintptr_t)sym & 15) == 0;
  for (;;) {
    if (tid == 0) sh.tile = atomicAdd(ticket, 1u);
    __syncthreads();  // also: the codebook window is in place
    const unsigned long long tile = sh.tile;
    if (tile >= ntiles) break;
    const size_t my = (size_t)tile * PK_TILE + (size_t)tid * PK_SPT;
    const int cnt = my >= n ? 0 : (int)((n - my) < (size_t)PK_SPT ? (n - my) : (size_t)PK_SPT);
    uint32_t w[NW];
    if (cnt == PK_SPT && vec_ok) {
      const uint4* src = reinterpret_cast<const uint4*>(sym + my);
#pragma unroll
      for (int q = 0; q < NW / 4; q++) {
        const uint4 v = __ldcs(src + q);
        w[4 * q] = v.x;
        w[4 * q + 1] = v.y;
        w[4 * q + 2] = v.z;
        w[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < NW; q++) w[q] = 0;
#pragma unroll
      for (int k = 0; k < PK_SPT; k++)
        if (k < cnt) w[k / W::per_word] |= (uint32_t)sym[my + k] << (SB * (k % W::per_word));
    }
    auto sym_k = [&](int k) -> unsigned {
      unsigned s = (w[k / W::per_word] >> (SB * (k % W::per_word))) & SMASK;
      if (MAP0 && s == ID_ZERO) s = 0;
      return s;
    };
    // 1. lengths, 4 to a register
    uint32_t lw[PK_SPT / 4];
    unsigned int bits = 0;
    bool lng = false;
#pragma unroll
    for (int k = 0; k < PK_SPT; k++) {
      const unsigned l = k < cnt ? pk_len<Sym>(sh, sym_k(k), len) : 0u;
      bits += l;
      lng |= l > 32;
      lw[k / 4] = (k % 4) ? (lw[k / 4] | (l << (8 * (k % 4)))) : l;
    }
    unsigned int x = bits;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sh.warp_bits[warp] = x;
    const bool any_long = __syncthreads_or(lng) != 0;
    unsigned int wpre = 0, agg = 0;
#pragma unroll
    for (int q = 0; q < PK_NT / 32; q++) {
      const unsigned int v = sh.warp_bits[q];
      wpre += q < warp ? v : 0u;
      agg += v;
    }
    const unsigned int tpre = wpre + x - bits;
    auto len_k = [&](int k) -> unsigned { return (lw[k / 4] >> (8 * (k % 4))) & 255u; };
    unsigned long long excl;

    if (!any_long) {
      // 2. tile-relative packing; nobody completes the last partial word
      if (tid == 0) {
        lookback_publish(state, tile, agg);
        if (agg & 31) sh.words[agg >> 5] = 0;
      }
      int wi = (int)(tpre >> 5);
      int nacc = (int)(tpre & 31);  // leading bits of word wi belong to earlier threads
      unsigned long long acc = 0;   // pending bits, most significant first
#pragma unroll
      for (int k = 0; k < PK_SPT; k++) {
        if (k < cnt) {
          const unsigned l = len_k(k);
          acc |= (unsigned long long)pk_lcode<Sym>(sh, sym_k(k), l, code) << (32 - nacc);
          nacc += (int)l;
          if (nacc >= 32) {
            sh.words[wi++] = (uint32_t)(acc >> 32);
            acc <<= 32;
            nacc -= 32;
          }
        }
      }
      __syncthreads();  // every completed word is in place
      if (bits > 0 && nacc > 0) atomicOr(&sh.words[wi], (uint32_t)(acc >> 32));
      __syncthreads();
      // 3. the starting bit, then the words onto the global grid
      if (warp == 0) {
        const unsigned long long e = lookback_warp(state, tile, agg, lane, PK_SPIN_LIMIT, flag);
        if (lane == 0) sh.excl = e;
      }
      __syncthreads();
      excl = sh.excl;
      const unsigned long long s0 = (unsigned long long)bit0 + excl;
      const unsigned int shift = (unsigned int)(s0 & 31);
      const unsigned long long w_lo = s0 >> 5;
      const int nrel = (int)((agg + 31) >> 5);
      const int nout = agg ? (int)((shift + agg - 1) >> 5) + 1 : 0;
      for (int k = tid; k < nout; k += PK_NT) {
        const unsigned long long g = w_lo + (unsigned long long)k;
        if (g >= cap_words) {
          atomicOr(flag, FLAG_OUT_CAPACITY);
          break;
        }
        const uint32_t lo = k < nrel ? sh.words[k] : 0u;
        const uint32_t hi = k > 0 ? sh.words[k - 1] : 0u;
        const uint32_t v = bswap32(shift ? __funnelshift_r(lo, hi, shift) : lo);
        if (k == 0 || k == nout - 1) atomicOr(&out[g], v);  // shared with the neighbouring tiles
        else out[g] = v;
      }
    } else {
      // a code longer than 32 bits: the starting bit first, every word ORed
      if (warp == 0) {
        if (lane == 0) lookback_publish(state, tile, agg);
        const unsigned long long e = lookback_warp(state, tile, agg, lane, PK_SPIN_LIMIT, flag);
        if (lane == 0) sh.excl = e;
      }
      __syncthreads();
      excl = sh.excl;
      const unsigned long long s0 = (unsigned long long)bit0 + excl;
      const unsigned long long w_lo = s0 >> 5;
      const unsigned int pos = (unsigned int)(s0 & 31) + tpre;
      int wi = (int)(pos >> 5);
      int nacc = (int)(pos & 31);
      unsigned long long acc = 0;
      auto emit = [&]() {
        const unsigned long long g = w_lo + (unsigned long long)wi;
        if (g < cap_words) atomicOr(&out[g], bswap32((uint32_t)(acc >> 32)));
        else atomicOr(flag, FLAG_OUT_CAPACITY);
        wi++;
      };
      auto put = [&](uint32_t v, int l) {  // 1 <= l <= 32, v < 2^l
        acc |= (unsigned long long)v << (64 - nacc - l);
        nacc += l;
        if (nacc >= 32) {
          emit();
          acc <<= 32;
          nacc -= 32;
        }
      };
      for (int k = 0; k < cnt; k++) {
        unsigned s = (unsigned)sym[my + k];
        if (MAP0 && s == ID_ZERO) s = 0;
        const int l = __ldg(len + s);
        const unsigned long long c = __ldg(code + s);
        if (l > 32) {
          put((uint32_t)(c >> 32) & (uint32_t)((1ull << (l - 32)) - 1), l - 32);
          put((uint32_t)c, 32);
        } else if (l > 0) {
          put((uint32_t)c & (uint32_t)((1ull << l) - 1), l);
        }
      }
      if (bits > 0 && nacc > 0) emit();
    }
    if (tile == ntiles - 1 && tid == 0 && d_total) *d_total = excl + agg;
    __syncthreads();  // the shared buffers are reused by the next tile
  }
}

__global__ void __launch_bounds__(256) codebook_scatter_kernel(const HuffEntry* __restrict__ e, size_t n,
                                                               unsigned long long* __restrict__ code,
                                                               uint8_t* __restrict__ len) {
  const size_t i = (size_t)blockIdx.x * 256 + threadIdx.x;
  if (i < n) {
    const HuffEntry v = e[i];
    code[v.sym] = v.code;
    len[v.sym] = (uint8_t)v.len;
  }
}

size_t pack_scratch_words(size_t n) { return (n + PK_TILE - 1) / PK_TILE + 1; }

// scratch: pack_scratch_words(n) words (ticket, then one state per tile), zeroed here.
template <class Sym>
int pack_launch(int num_sms, cudaStream_t st, const Sym* sym, size_t n, bool map_id_zero, HuffEncTable tab,
                uint32_t* out, size_t out_cap_bytes, int bit0, unsigned long long* scratch,
                unsigned long long* d_total_bits, int* flag) {
  if (n == 0) return CPSZ_OK;
  if (bit0 < 0 || bit0 > 31) return set_error(CPSZ_ERR_INVALID, "internal: stream start bit %d", bit0);
  const unsigned long long ntiles = (n + PK_TILE - 1) / PK_TILE;
  CPSZ_CUDA_TRY(cudaMemsetAsync(scratch, 0, (ntiles + 1) * 8, st));
  const unsigned long long cap = (unsigned long long)num_sms * PK_CTAS_PER_SM;
  const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
  auto k = pack_kernel<Sym, false>;
  if constexpr (sizeof(Sym) == 1) {
    if (map_id_zero) k = pack_kernel<Sym, true>;
  }
  k<<<grid, PK_NT, 0, st>>>(sym, n, tab.code, tab.len, tab.nsym, out, out_cap_bytes / 4, bit0, scratch + 1,
                            reinterpret_cast<unsigned int*>(scratch), ntiles, d_total_bits, flag);
  return check_launch("pack_kernel");
}

template <class Sym>
int encode_impl(cpsz_b200_ctx* ctx, const Sym* sym, size_t n, bool map_id_zero, HuffEncTable tab, uint32_t* out,
                size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp, int bit0) {
  if (n == 0) return CPSZ_OK;
  CPSZ_TRY(pack_launch<Sym>(ctx->num_sms, ctx->stream, sym, n, map_id_zero, tab, out, out_cap_bytes, bit0,
                            (unsigned long long*)tmp, d_total_bits, ctx->d_flag));
  count_launch(ctx);
  return CPSZ_OK;
}

// Exclusive scan of the per-CTA bit counts (single CTA, sequential over chunks).
__global__ void __launch_bounds__(1024) scan_u64_kernel(const unsigned long long* __restrict__ in,
                                                        unsigned long long* __restrict__ out, size_t n) {
  __shared__ unsigned long long warp_tot[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (size_t base = 0; base < n; base += 1024) {
    size_t i = base + threadIdx.x;
    unsigned long long v = i < n ? in[i] : 0ull;
    unsigned long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) >= o) x += y;
    }
    if ((threadIdx.x & 31) == 31) warp_tot[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      unsigned long long w = warp_tot[threadIdx.x];
      for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (threadIdx.x >= o) w += y;
      }
      warp_tot[threadIdx.x] = w;
    }
    __syncthreads();
    unsigned long long pre = carry + (threadIdx.x >= 32 ? warp_tot[(threadIdx.x >> 5) - 1] : 0ull) + x - v;
    if (i < n) out[i] = pre;
    __syncthreads();
    if (threadIdx.x == 1023) carry = pre + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// ---- histogram -------------------------------------------------------------------
constexpr int HIST_NT = 512;
constexpr int HIST_LO = 32768 - 4096;  // shared window of the code histogram
constexpr int HIST_W = 8192;

// Codes concentrate on 32768 and its neighbours (prediction errors of zero and
// one quantum): those three are counted in registers and reduced once per
// warp, so the shared-memory atomics see only the spread-out remainder (no
// 32-way same-address conflicts).  Reads are 16-byte vectors where aligned.
template <bool SKIP0 = false>
__device__ __forceinline__ void hist_add(unsigned int* sh, unsigned long long* hist, unsigned v, unsigned& c_lo,
                                         unsigned& c_mid, unsigned& c_hi) {
  const unsigned d = v - 32767u;
  if (d < 3u) {
    c_lo += d == 0u;
    c_mid += d == 1u;
    c_hi += d == 2u;
  } else if (v == 0u) {
    if (!SKIP0) atomicAdd(&sh[HIST_W], 1u);
  } else if (v - (unsigned)HIST_LO < (unsigned)HIST_W) {
    atomicAdd(&sh[v - HIST_LO], 1u);
  } else {
    atomicAdd(&hist[v], 1ull);
  }
}

// Symbols t0, t0 + stride, ... of s[0, n) into the shared window / registers:
// the elements before the first 16-byte boundary, the vector body, the tail.
template <bool SKIP0 = false>
__device__ __forceinline__ void hist_span(unsigned* sh, unsigned long long* hist, const uint16_t* s, size_t n,
                                          size_t t0, size_t stride, unsigned& c_lo, unsigned& c_mid, unsigned& c_hi) {
  const size_t head = ((16 - ((uintptr_t)s & 15)) & 15) / 2;
  const size_t h = head < n ? head : n;
  if (t0 < h) hist_add<SKIP0>(sh, hist, s[t0], c_lo, c_mid, c_hi);
  const size_t nv = (n - h) / 8;
  const uint4* sv = reinterpret_cast<const uint4*>(s + h);
  for (size_t i = t0; i < nv; i += stride) {
    const uint4 w = __ldcs(sv + i);
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      hist_add<SKIP0>(sh, hist, ws[q] & 0xffffu, c_lo, c_mid, c_hi);
      hist_add<SKIP0>(sh, hist, ws[q] >> 16, c_lo, c_mid, c_hi);
    }
  }
  for (size_t i = h + nv * 8 + t0; i < n; i += stride) hist_add<SKIP0>(sh, hist, s[i], c_lo, c_mid, c_hi);
}
// The register counts and the shared window into the global histogram.
__device__ __forceinline__ void hist_flush(unsigned* sh, unsigned long long* hist, unsigned c_lo, unsigned c_mid,
                                           unsigned c_hi) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    c_lo += __shfl_down_sync(0xffffffffu, c_lo, o);
    c_mid += __shfl_down_sync(0xffffffffu, c_mid, o);
    c_hi += __shfl_down_sync(0xffffffffu, c_hi, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (c_lo) atomicAdd(&sh[32767 - HIST_LO], c_lo);
    if (c_mid) atomicAdd(&sh[32768 - HIST_LO], c_mid);
    if (c_hi) atomicAdd(&sh[32769 - HIST_LO], c_hi);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < HIST_W; k += HIST_NT)
    if (sh[k]) atomicAdd(&hist[HIST_LO + k], (unsigned long long)sh[k]);
  if (threadIdx.x == 0 && sh[HIST_W]) atomicAdd(&hist[0], (unsigned long long)sh[HIST_W]);
}

// Stream blockIdx.y (s0 / s1, n symbols each) into its histogram (h0 / h1);
// SKIP0: symbol 0 is not counted.
template <bool SKIP0>
__global__ void __launch_bounds__(HIST_NT) hist_u16_kernel(const uint16_t* __restrict__ s0,
                                                           const uint16_t* __restrict__ s1, size_t n,
                                                           unsigned long long* __restrict__ h0,
                                                           unsigned long long* __restrict__ h1) {
  const uint16_t* __restrict__ s = blockIdx.y ? s1 : s0;
  unsigned long long* __restrict__ hist = blockIdx.y ? h1 : h0;
  __shared__ unsigned int sh[HIST_W + 1];  // window + symbol 0
  for (int k = threadIdx.x; k <= HIST_W; k += HIST_NT) sh[k] = 0;
  __syncthreads();
  unsigned c_lo = 0, c_mid = 0, c_hi = 0;
  hist_span<SKIP0>(sh, hist, s, n, (size_t)blockIdx.x * HIST_NT + threadIdx.x, (size_t)gridDim.x * HIST_NT, c_lo,
                   c_mid, c_hi);
  hist_flush(sh, hist, c_lo, c_mid, c_hi);
}

// ---- histogram follower ----------------------------------------------------------
// Counts a field's code histograms while its wavefront is still running:
// blockIdx.y is the component; the CTAs take slices of FOLLOW_ROWS rows in
// row order from the component's ticket, wait for the slice's row group to
// be flagged done by the wavefront (thread 0 polls with acquire loads, the
// CTA then acquires), and count the slice.  The wavefront finishes its
// groups in row order, so most of the field is counted during the
// wavefront's tail and only the last group's slices remain once it ends.
// A wait that outlasts FOLLOW_WAIT_NS (the wavefront is not running: a tool
// serialises kernels) sets *gave_up and every CTA stops; the host counts
// the histograms again.
constexpr int FOLLOW_ROWS = 8;
constexpr long long FOLLOW_WAIT_NS = 100000000ll;  // 100 ms

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ long long follow_clock_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void __launch_bounds__(HIST_NT) hist_follow_kernel(const uint16_t* __restrict__ c0,
                                                              const uint16_t* __restrict__ c1,
                                                              const unsigned* __restrict__ d0,
                                                              const unsigned* __restrict__ d1, int r1, int r2,
                                                              unsigned long long* __restrict__ h0,
                                                              unsigned long long* __restrict__ h1,
                                                              unsigned* __restrict__ tickets, int* gave_up) {
  const uint16_t* __restrict__ codes = blockIdx.y ? c1 : c0;
  const unsigned* __restrict__ done = blockIdx.y ? d1 : d0;
  unsigned long long* __restrict__ hist = blockIdx.y ? h1 : h0;
  __shared__ unsigned int sh[HIST_W + 1];
  __shared__ int s_slice;
  for (int k = threadIdx.x; k <= HIST_W; k += HIST_NT) sh[k] = 0;
  unsigned c_lo = 0, c_mid = 0, c_hi = 0;
  const int nslices = (r1 + FOLLOW_ROWS - 1) / FOLLOW_ROWS;
  for (;;) {
    if (threadIdx.x == 0) {
      int sl = (int)atomicAdd(tickets + blockIdx.y, 1u);
      if (sl < nslices) {
        const unsigned* flag = done + (sl * FOLLOW_ROWS) / WAVE_GROUP_ROWS;
        if (!ld_acquire_u32(flag)) {
          const long long t0 = follow_clock_ns();
          while (!ld_acquire_u32(flag)) {
            if (*(volatile int*)gave_up || follow_clock_ns() - t0 > FOLLOW_WAIT_NS) {
              atomicOr(gave_up, 1);
              sl = nslices;
              break;
            }
            __nanosleep(1000);
          }
        }
      }
      s_slice = sl;
    }
    __syncthreads();
    const int sl = s_slice;
    if (sl >= nslices) break;
    (void)ld_acquire_u32(done + (sl * FOLLOW_ROWS) / WAVE_GROUP_ROWS);
    const int row0 = sl * FOLLOW_ROWS, rows = min(FOLLOW_ROWS, r1 - row0);
    hist_span(sh, hist, codes + (size_t)row0 * r2, (size_t)rows * r2, threadIdx.x, HIST_NT, c_lo, c_mid, c_hi);
    __syncthreads();  // s_slice is rewritten only after every thread has read it
  }
  hist_flush(sh, hist, c_lo, c_mid, c_hi);
}

// ---- decoder ---------------------------------------------------------------------
constexpr int DEC_S = 1024;  // bits per subsequence
constexpr int DEC_NT = 256;

struct BitReader {
  const uint32_t* w;  // big-endian words
  __device__ __forceinline__ uint32_t peek32(unsigned long long pos) const {
    size_t wi = pos >> 5;
    uint32_t a = bswap32(__ldg(w + wi)), b = bswap32(__ldg(w + wi + 1));
    return __funnelshift_l(b, a, (unsigned)(pos & 31));
  }
};

// Decodes one symbol at `pos`; returns its length in bits (0 on a corrupt walk).
__device__ __forceinline__ int decode_one(const BitReader& br, const uint32_t* lut, const HuffDecTable& T,
                                          unsigned long long pos, uint32_t* sym) {
  uint32_t p = br.peek32(pos);
  uint32_t e = lut[p >> (32 - HUFF_LUT_BITS)];
  if (!(e & 0x80)) {
    *sym = e >> 8;
    return (int)(e & 0x7f);
  }
  uint32_t node = e >> 8;
  int l = HUFF_LUT_BITS;
  while (l < 64) {
    uint32_t bit = (br.peek32(pos + l) >> 31) & 1u;
    node = T.child[2 * node + bit];
    l++;
    if (node == 0 || node >= (uint32_t)T.node_count) return 0;
    if (T.leaf[node]) {
      *sym = T.sym[node];
      return l;
    }
  }
  return 0;
}

// A sequential reader: the next bits MSB-first in a 64-bit register, refilled
// a word at a time, so a symbol found by the table costs no memory access.
// Holds at least 32 valid bits between symbols.
struct BitCursor {
  const uint32_t* w;
  unsigned long long buf;
  unsigned long long wi;  // the next word to load
  int nb;                 // valid bits in buf
  __device__ __forceinline__ void seek(unsigned long long pos) {
    wi = pos >> 5;
    const unsigned long long a = bswap32(__ldg(w + wi)), b = bswap32(__ldg(w + wi + 1));
    buf = ((a << 32) | b) << (pos & 31);
    nb = 64 - (int)(pos & 31);
    wi += 2;
  }
  __device__ __forceinline__ void skip(int l) {  // 1 <= l <= 32
    buf <<= l;
    nb -= l;
    if (nb <= 32) {
      buf |= (unsigned long long)bswap32(__ldg(w + wi)) << (32 - nb);
      nb += 32;
      wi++;
    }
  }
};

// decode_one on the cursor, which sits at `pos`; advances it past the symbol.
__device__ __forceinline__ int decode_cur(BitCursor& c, const BitReader& br, const uint32_t* lut,
                                          const HuffDecTable& T, unsigned long long pos, uint32_t* sym) {
  const uint32_t e = lut[(uint32_t)(c.buf >> (64 - HUFF_LUT_BITS))];
  if (!(e & 0x80)) {
    *sym = e >> 8;
    const int l = (int)(e & 0x7f);
    c.skip(l);
    return l;
  }
  const int l = decode_one(br, lut, T, pos, sym);  // a code longer than the table: walk the tree
  if (l > 0) c.seek(pos + l);
  return l;
}

__device__ __forceinline__ void load_lut(uint32_t* slut, const uint32_t* lut) {
  for (int k = threadIdx.x; k < (1 << HUFF_LUT_BITS); k += blockDim.x) slut[k] = lut[k];
  __syncthreads();
}

// Count word bit: the subsequence's decode ran into an invalid code (possible
// from an unsynchronised start; on the true path only in a corrupt stream).
constexpr unsigned int DEC_INVALID = 0x80000000u;

// Phase 1: decode subsequence t from its nominal start to its limit.
// Phase 2 (resync): subsequence t restarts from its predecessor's exit when
// that differs from its start.  Huffman codes resynchronise within a few
// symbols, so the new path runs in lockstep with the previous one (always
// advancing the one behind): once both reach the same bit position the rest
// equals the previous decode, whose exit and count (less the symbols before
// that position) carry over.
__global__ void __launch_bounds__(DEC_NT) dec_scan_kernel(BitReader br, HuffDecTable T, unsigned long long nbits,
                                                          int nsub, unsigned long long* __restrict__ start,
                                                          unsigned long long* __restrict__ end,
                                                          unsigned int* __restrict__ cnt, int resync,
                                                          int* __restrict__ changed, int* flag) {
  __shared__ uint32_t slut[1 << HUFF_LUT_BITS];
  int t = blockIdx.x * DEC_NT + threadIdx.x;
  // a resynchronisation round leaves at once the blocks with no start to
  // move (most of them after the first round), without loading the table
  if (resync && !__syncthreads_or(t > 0 && t < nsub && end[t - 1] != start[t])) return;
  load_lut(slut, T.lut);
  if (t >= nsub) return;
  unsigned long long lim = (unsigned long long)(t + 1) * DEC_S;
  if (lim > nbits) lim = nbits;
  uint32_t sym;
  if (!resync) {
    unsigned long long pos = (unsigned long long)t * DEC_S;
    start[t] = pos;
    BitCursor cur{br.w};
    cur.seek(pos);
    unsigned int c = 0;
    while (pos < lim) {
      const int l = decode_cur(cur, br, slut, T, pos, &sym);
      if (l == 0) {
        if (t == 0) atomicOr(flag, FLAG_HUFF_CORRUPT);
        c |= DEC_INVALID;
        pos = lim;
        break;
      }
      pos += l;
      c++;
    }
    end[t] = pos;
    cnt[t] = c;
    return;
  }
  if (t == 0) return;
  const unsigned long long s = end[t - 1], s_old = start[t];
  if (s == s_old) return;
  const unsigned long long e_old = end[t];
  const unsigned int c_old = cnt[t];
  start[t] = s;
  *changed = 1;
  unsigned long long a = s, b = s_old;  // the new path, the previous one
  unsigned int ca = 0, cb = 0;
  bool old_ok = true;
  while (a < lim) {
    if (old_ok && b < a) {  // b < a < lim: still on the previous decode
      const int l = decode_one(br, slut, T, b, &sym);
      if (l == 0) old_ok = false;
      b += l;
      cb++;
      continue;
    }
    if (old_ok && a == b) {
      if (c_old & DEC_INVALID) atomicOr(flag, FLAG_HUFF_CORRUPT);
      end[t] = e_old;
      cnt[t] = ca + ((c_old & ~DEC_INVALID) - cb);
      return;
    }
    const int l = decode_one(br, slut, T, a, &sym);
    if (l == 0) {
      atomicOr(flag, FLAG_HUFF_CORRUPT);
      a = lim;
      break;
    }
    a += l;
    ca++;
  }
  end[t] = a;
  cnt[t] = ca;
}

// Phase 3: subsequence t writes its symbols from output index off[t].  A
// thread's symbols are packed into aligned 64-bit stores (single stores at the
// unaligned head and tail of its range): one store per symbol, each to its
// own line, made the write rate the limit.
template <class Out>
__global__ void __launch_bounds__(DEC_NT) dec_write_kernel(BitReader br, HuffDecTable T, unsigned long long nbits,
                                                           int nsub, const unsigned long long* __restrict__ start,
                                                           const unsigned long long* __restrict__ off,
                                                           size_t n, Out* __restrict__ out) {
  constexpr int PER = 8 / sizeof(Out);
  constexpr int SB = 8 * sizeof(Out);
  __shared__ uint32_t slut[1 << HUFF_LUT_BITS];
  load_lut(slut, T.lut);
  int t = blockIdx.x * DEC_NT + threadIdx.x;
  if (t >= nsub) return;
  unsigned long long lim = (unsigned long long)(t + 1) * DEC_S;
  if (lim > nbits) lim = nbits;
  unsigned long long pos = start[t];
  unsigned long long o = off[t];
  const bool packed = (reinterpret_cast<uintptr_t>(out) & 7) == 0;
  BitCursor cur{br.w};
  cur.seek(pos);
  unsigned long long acc = 0;
  int na = 0;  // symbols in acc, which starts at an aligned index
  while (pos < lim && o < n) {
    uint32_t sym;
    const int l = decode_cur(cur, br, slut, T, pos, &sym);
    if (l == 0) break;
    pos += l;
    if (na == 0 && (!packed || (o % PER) != 0)) {
      out[o++] = (Out)sym;
      continue;
    }
    acc |= (unsigned long long)(Out)sym << (SB * na);
    o++;
    if (++na == PER) {
      *reinterpret_cast<unsigned long long*>(out + (o - PER)) = acc;
      acc = 0;
      na = 0;
    }
  }
  for (int k = 0; k < na; k++) out[o - na + k] = (Out)(acc >> (SB * k));
}

__global__ void fill_kernel_u8(uint8_t* out, size_t n, uint8_t v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) out[i] = v;
}
__global__ void fill_kernel_u16(uint16_t* out, size_t n, uint16_t v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) out[i] = v;
}

__global__ void u32_to_u64_kernel(const unsigned int* in, unsigned long long* out, int n, unsigned int mask) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] & mask;
}

__global__ void clear_invalid_kernel(unsigned int* cnt, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cnt[i] &= ~DEC_INVALID;
}

__global__ void check_total_kernel(const unsigned long long* off, int nsub, size_t n, int* flag) {
  if (off[nsub] < n) atomicOr(flag, FLAG_HUFF_CORRUPT);
}

}  // namespace

int launch_codebook_scatter(cpsz_b200_ctx* ctx, const HuffEntry* d_entries, size_t n, unsigned long long* code,
                            uint8_t* len) {
  if (n == 0) return CPSZ_OK;
  codebook_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d_entries, n, code, len);
  count_launch(ctx);
  return check_launch("codebook_scatter_kernel");
}

size_t huff_encode_tmp_bytes(size_t n) { return align_up(pack_scratch_words(n), 32) * sizeof(unsigned long long); }

int launch_huff_encode_u8(cpsz_b200_ctx* ctx, const uint8_t* sym, size_t n, bool map_id_zero, HuffEncTable tab,
                          uint32_t* out_words, size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp,
                          int bit0) {
  return encode_impl<uint8_t>(ctx, sym, n, map_id_zero, tab, out_words, out_cap_bytes, d_total_bits, tmp, bit0);
}

int launch_huff_encode_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, HuffEncTable tab, uint32_t* out_words,
                           size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp, int bit0) {
  return encode_impl<uint16_t>(ctx, sym, n, false, tab, out_words, out_cap_bytes, d_total_bits, tmp, bit0);
}

int launch_hist_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, unsigned long long* hist) {
  return launch_hist_u16_pair(ctx, sym, nullptr, n, hist, nullptr);
}
int launch_hist_u16_pair(cpsz_b200_ctx* ctx, const uint16_t* a, const uint16_t* b, size_t n, unsigned long long* ha,
                         unsigned long long* hb) {
  if (n == 0) return CPSZ_OK;
  const int k = b ? 2 : 1;
  int grid = ctx->num_sms * 2 / k;
  size_t need = (n + HIST_NT - 1) / HIST_NT;
  if ((size_t)grid > need) grid = (int)need;
  hist_u16_kernel<false><<<dim3(grid, k), HIST_NT, 0, ctx->stream>>>(a, b, n, ha, hb);
  count_launch(ctx);
  return check_launch("hist_u16_kernel");
}
int launch_hist_u16_nonzero(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, unsigned long long* hist) {
  if (n == 0) return CPSZ_OK;
  int grid = ctx->num_sms * 2;
  size_t need = (n + HIST_NT - 1) / HIST_NT;
  if ((size_t)grid > need) grid = (int)need;
  hist_u16_kernel<true><<<dim3(grid, 1), HIST_NT, 0, ctx->stream>>>(sym, nullptr, n, hist, nullptr);
  count_launch(ctx);
  return check_launch("hist_u16_kernel");
}

int launch_hist_follow(cpsz_b200_ctx* ctx, const uint16_t* const codes[2], const unsigned* const group_done[2], int r1,
                       int r2, unsigned long long* const hist[2], unsigned* tickets, int* gave_up, cudaStream_t stream) {
  if (r1 <= 0 || r2 <= 0) return CPSZ_OK;
  const int nslices = (r1 + FOLLOW_ROWS - 1) / FOLLOW_ROWS;
  const int grid = std::min(nslices, ctx->num_sms);
  hist_follow_kernel<<<dim3(grid, 2), HIST_NT, 0, stream>>>(codes[0], codes[1], group_done[0], group_done[1], r1, r2,
                                                            hist[0], hist[1], tickets, gave_up);
  count_launch(ctx);
  return check_launch("hist_follow_kernel");
}

size_t huff_decode_tmp_bytes(size_t nbits) {
  size_t nsub = (nbits + DEC_S - 1) / DEC_S + 1;
  return align_up(nsub + 1, 32) * 8 * 3 + align_up(nsub + 1, 32) * 4 * 2 + 4096 + scan_u32_tmp_bytes(nsub + 1);
}

int launch_huff_decode(cpsz_b200_ctx* ctx, const uint8_t* bytes, size_t nbytes, size_t n, HuffDecTable tab, void* out,
                       int out_bytes_per_sym, void* tmp) {
  if (n == 0) return CPSZ_OK;
  if (tab.root_is_leaf) {
    unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8);
    if (out_bytes_per_sym == 1) fill_kernel_u8<<<grid, 256, 0, ctx->stream>>>((uint8_t*)out, n, (uint8_t)tab.root_sym);
    else fill_kernel_u16<<<grid, 256, 0, ctx->stream>>>((uint16_t*)out, n, (uint16_t)tab.root_sym);
    count_launch(ctx);
    return check_launch("huffman fill");
  }
  unsigned long long nbits = (unsigned long long)nbytes * 8;
  int nsub = (int)((nbits + DEC_S - 1) / DEC_S);
  if (nsub == 0) return set_error(CPSZ_ERR_FORMAT, "empty Huffman stream for %zu symbols", n);
  char* p = (char*)tmp;
  size_t a = align_up((size_t)nsub + 1, 32);
  unsigned long long* start = (unsigned long long*)p;
  p += a * 8;
  unsigned long long* end = (unsigned long long*)p;
  p += a * 8;
  unsigned long long* off = (unsigned long long*)p;
  p += a * 8;
  unsigned int* cnt = (unsigned int*)p;
  p += a * 4;
  int* changed = (int*)p;
  BitReader br{(const uint32_t*)bytes};
  unsigned grid = (unsigned)((nsub + DEC_NT - 1) / DEC_NT);
  dec_scan_kernel<<<grid, DEC_NT, 0, ctx->stream>>>(br, tab, nbits, nsub, start, end, cnt, 0, changed, ctx->d_flag);
  count_launch(ctx);
  // resynchronisation rounds; each round fixes at least one more subsequence,
  // in practice the first round already converges.
  int* h_changed = (int*)ctx->pinned;
  for (int round = 0; round < nsub; round++) {
    cudaMemsetAsync(changed, 0, sizeof(int), ctx->stream);
    dec_scan_kernel<<<grid, DEC_NT, 0, ctx->stream>>>(br, tab, nbits, nsub, start, end, cnt, 1, changed, ctx->d_flag);
    count_launch(ctx);
    cudaMemcpyAsync(h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (!*h_changed) break;
  }
  // output offsets: a device-wide u32 scan when every offset fits 32 bits (a
  // subsequence decodes at most one symbol per bit, plus the one crossing its
  // end), else one CTA over 64-bit counts; the exits are no longer needed
  // after the final round, so their array holds the counts' copy
  if (nbits + (unsigned long long)nsub < (1ull << 32)) {
    unsigned int* off32 = reinterpret_cast<unsigned int*>(end);
    clear_invalid_kernel<<<(nsub + 255) / 256, 256, 0, ctx->stream>>>(cnt, nsub);
    CPSZ_TRY(launch_scan_u32(ctx, cnt, off32, (size_t)nsub, p + 256));  // off32[nsub] = the total
    u32_to_u64_kernel<<<(nsub + 256) / 256, 256, 0, ctx->stream>>>(off32, off, nsub + 1, 0xffffffffu);
  } else {
    unsigned long long* cnt64 = end;
    u32_to_u64_kernel<<<(nsub + 255) / 256, 256, 0, ctx->stream>>>(cnt, cnt64, nsub, ~DEC_INVALID);
    scan_u64_kernel<<<1, 1024, 0, ctx->stream>>>(cnt64, off, (size_t)nsub);
  }
  check_total_kernel<<<1, 1, 0, ctx->stream>>>(off, nsub, n, ctx->d_flag);
  if (out_bytes_per_sym == 1)
    dec_write_kernel<uint8_t><<<grid, DEC_NT, 0, ctx->stream>>>(br, tab, nbits, nsub, start, off, n, (uint8_t*)out);
  else
    dec_write_kernel<uint16_t><<<grid, DEC_NT, 0, ctx->stream>>>(br, tab, nbits, nsub, start, off, n, (uint16_t*)out);
  count_launch(ctx, 4);
  return check_launch("huffman decode");
}

// ---- Huffman packing without any allocation ---------------------------------------------
//
// Some callers cannot allocate device memory at the point where they encode:
// an in-situ analysis hook running inside a simulation that reserved all GPU
// memory for its own pool at start-up, a plugin that is only handed
// preallocated buffers by its host framework, or a real-time loop where a
// cudaMalloc (which may synchronise the device) is not allowed.  For them
// this entry point packs a symbol stream with the same kernel as
// cpsz_b200_huffman_encode_u16 but takes its scratch -- the tile ticket and
// the per-tile look-back states -- from a fixed array in this file instead of
// a context workspace.  The array (about 64 KB) lives on every GPU that loads
// the library until the process exits, and it bounds the stream length.

constexpr size_t kNoAllocMaxSymbols = size_t(1) << 26;  // 67,108,864 symbols per call
constexpr size_t kNoAllocTiles = kNoAllocMaxSymbols / PK_TILE;
// layout: [ticket][tile states: kNoAllocTiles][flag word]
static __device__ __align__(256) unsigned long long g_noalloc_scratch[1 + kNoAllocTiles + 1];

namespace {

// The array's device address in the calling thread's current context.  It is
// looked up on every call (a lookup, no allocation): an address cached once
// per device would go stale after a device reset, or in a context the caller
// created and made current itself, and kernels given it would write to memory
// that is no longer the array.
int noalloc_scratch(unsigned long long** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess)
    return set_error(e == cudaErrorNoDevice ? CPSZ_ERR_NO_DEVICE : CPSZ_ERR_CUDA,
                     "cudaGetSymbolAddress of the no-alloc scratch: %s", cudaGetErrorString(e));
  *out = (unsigned long long*)p;
  return CPSZ_OK;
}

}  // namespace

}  // namespace cpsz

extern "C" int cpsz_b200_huffman_encode_u16_noalloc(const uint16_t* sym, size_t n, const uint64_t* code,
                                                    const uint8_t* len, unsigned char* out, size_t out_cap,
                                                    uint64_t* total_bits, void* stream) {
  using namespace cpsz;
  clear_error();
  if (!sym || !code || !len || !out || !total_bits) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  if (((uintptr_t)out & 3) != 0) return set_error(CPSZ_ERR_INVALID, "output must be 4-byte aligned");
  // the packer stores whole 32-bit words: a capacity that is not a multiple of
  // 4 would leave its last bytes unwritten without the overflow rule noticing
  if (out_cap % 4 != 0) return set_error(CPSZ_ERR_INVALID, "out_cap (%zu) must be a multiple of 4", out_cap);
  if (n > kNoAllocMaxSymbols)
    return set_error(CPSZ_ERR_INVALID, "%zu symbols exceed the no-alloc maximum of %zu symbols per call", n,
                     kNoAllocMaxSymbols);
  unsigned long long* scratch = nullptr;
  CPSZ_TRY(noalloc_scratch(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  int* flag = (int*)(scratch + 1 + kNoAllocTiles);
  // the packer ORs the edge words of every tile: the output starts at zero
  CPSZ_CUDA_TRY(cudaMemsetAsync(out, 0, out_cap, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned long long), st));
  if (n == 0) {
    CPSZ_CUDA_TRY(cudaMemsetAsync(total_bits, 0, sizeof(uint64_t), st));
    return CPSZ_OK;
  }
  int dev = 0, sms = 0;
  CPSZ_CUDA_TRY(cudaGetDevice(&dev));
  CPSZ_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CPSZ_TRY(pack_launch<uint16_t>(sms, st, sym, n, false, HuffEncTable{(const unsigned long long*)code, len, 65536},
                                 (uint32_t*)out, out_cap, 0, scratch, (unsigned long long*)total_bits, flag));
  return check_launch("huffman no-alloc encode");
}
