// huffman.cu -- GPU side of the SZ-1.x Huffman codec used by the reference
// (src/sz_huffman.cpp): symbol histograms, the MSB-first bit packer and a
// self-synchronising parallel decoder.
//
// Encoder.  The reference's packer (encode, src/sz_huffman.cpp:217-320) emits
// the MSB-first concatenation of the codes, zero padded to a byte.  Here a CTA
// owns 4096 consecutive symbols: pass 1 sums code lengths per CTA, a scan gives
// every CTA its starting bit, pass 2 re-reads the symbols, scans the lengths
// inside the CTA, ORs the codes into a shared-memory word buffer aligned to
// the global 32-bit word grid, and stores it with plain coalesced stores except
// for the two edge words, which are shared with the neighbouring CTAs and use
// atomicOr.  Words are stored byte-swapped so memory holds the big-endian byte
// stream the reference writes.
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

namespace cpsz {

namespace {

constexpr int ENC_NT = 256;
constexpr int ENC_PER_THREAD = 16;
constexpr int ENC_PER_CTA = ENC_NT * ENC_PER_THREAD;

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

template <class Sym>
__device__ __forceinline__ int sym_at(const Sym* s, size_t i, bool map_id_zero) {
  int v = (int)s[i];
  if (map_id_zero && v == ID_ZERO) v = 0;
  return v;
}

template <class Sym>
__global__ void __launch_bounds__(ENC_NT) enc_count_kernel(const Sym* __restrict__ sym, size_t n, bool map_id_zero,
                                                           const uint8_t* __restrict__ len,
                                                           unsigned long long* __restrict__ cta_bits) {
  __shared__ unsigned int red[ENC_NT / 32];
  size_t base = (size_t)blockIdx.x * ENC_PER_CTA;
  unsigned int bits = 0;
#pragma unroll 4
  for (int k = 0; k < ENC_PER_THREAD; k++) {
    size_t i = base + (size_t)k * ENC_NT + threadIdx.x;
    if (i < n) bits += len[sym_at(sym, i, map_id_zero)];
  }
  for (int o = 16; o; o >>= 1) bits += __shfl_xor_sync(0xffffffffu, bits, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bits;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < ENC_NT / 32; w++) t += red[w];
    cta_bits[blockIdx.x] = t;
  }
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

template <class Sym>
__global__ void __launch_bounds__(ENC_NT) enc_write_kernel(const Sym* __restrict__ sym, size_t n, bool map_id_zero,
                                                           const unsigned long long* __restrict__ code,
                                                           const uint8_t* __restrict__ len,
                                                           const unsigned long long* __restrict__ cta_off,
                                                           uint32_t* __restrict__ out, size_t cap_words,
                                                           int* __restrict__ flag) {
  extern __shared__ uint32_t sbuf[];
  __shared__ unsigned int warp_tot[ENC_NT / 32];
  const size_t base = (size_t)blockIdx.x * ENC_PER_CTA;
  const unsigned long long start = cta_off[blockIdx.x];
  const unsigned long long end = cta_off[blockIdx.x + 1];
  if (start == end) return;
  const int shift = (int)(start & 31);
  const int nwords = (int)(((end - 1) >> 5) - (start >> 5) + 1);
  for (int k = threadIdx.x; k < nwords; k += ENC_NT) sbuf[k] = 0;
  // thread t owns symbols base + t*16 .. +15 (contiguous run for in-order packing)
  const size_t my = base + (size_t)threadIdx.x * ENC_PER_THREAD;
  int s_loc[ENC_PER_THREAD];
  unsigned int bits = 0;
#pragma unroll
  for (int k = 0; k < ENC_PER_THREAD; k++) {
    size_t i = my + k;
    s_loc[k] = (i < n) ? sym_at(sym, i, map_id_zero) : -1;
    if (s_loc[k] >= 0) bits += len[s_loc[k]];
  }
  unsigned int x = bits;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) >= o) x += y;
  }
  if ((threadIdx.x & 31) == 31) warp_tot[threadIdx.x >> 5] = x;
  __syncthreads();
  unsigned int pre = x - bits;
  for (int w = 0; w < (int)(threadIdx.x >> 5); w++) pre += warp_tot[w];
  unsigned int pos = (unsigned int)shift + pre;  // bit position inside sbuf
#pragma unroll
  for (int k = 0; k < ENC_PER_THREAD; k++) {
    if (s_loc[k] < 0) break;
    int l = len[s_loc[k]];
    unsigned long long c = code[s_loc[k]];
    while (l > 0) {
      int wi = pos >> 5, off = pos & 31;
      int room = 32 - off;
      int take = l < room ? l : room;
      uint32_t part = (uint32_t)((c >> (l - take)) & ((take == 32) ? 0xffffffffull : ((1ull << take) - 1)));
      atomicOr(&sbuf[wi], part << (room - take));
      pos += take;
      l -= take;
    }
  }
  __syncthreads();
  const size_t w0 = start >> 5;
  for (int k = threadIdx.x; k < nwords; k += ENC_NT) {
    if (w0 + k >= cap_words) {
      atomicOr(flag, FLAG_OUT_CAPACITY);
      break;
    }
    uint32_t v = bswap32(sbuf[k]);
    if (k == 0 || k == nwords - 1) atomicOr(&out[w0 + k], v);
    else out[w0 + k] = v;
  }
}

template <class Sym>
int encode_impl(cpsz_b200_ctx* ctx, const Sym* sym, size_t n, bool map_id_zero, HuffEncTable tab, uint32_t* out,
                size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp) {
  if (n == 0) return CPSZ_OK;
  size_t nb = (n + ENC_PER_CTA - 1) / ENC_PER_CTA;
  unsigned long long* cta_bits = (unsigned long long*)tmp;
  unsigned long long* cta_off = cta_bits + align_up(nb, 32);
  enc_count_kernel<Sym><<<(unsigned)nb, ENC_NT, 0, ctx->stream>>>(sym, n, map_id_zero, tab.len, cta_bits);
  scan_u64_kernel<<<1, 1024, 0, ctx->stream>>>(cta_bits, cta_off, nb);
  // shared word buffer for the worst case of 64-bit codes (32 KB)
  size_t smem = ((size_t)ENC_PER_CTA * 64) / 32 * 4 + 16;
  enc_write_kernel<Sym><<<(unsigned)nb, ENC_NT, smem, ctx->stream>>>(sym, n, map_id_zero, tab.code, tab.len,
                                                                       cta_off, out, out_cap_bytes / 4, ctx->d_flag);
  if (d_total_bits)
    cudaMemcpyAsync(d_total_bits, cta_off + nb, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, ctx->stream);
  count_launch(ctx, 3);
  return check_launch("huffman encode");
}

// ---- histogram -------------------------------------------------------------------
constexpr int HIST_NT = 512;
constexpr int HIST_LO = 32768 - 4096;  // shared window of the code histogram
constexpr int HIST_W = 8192;

// Codes concentrate on 32768 and its neighbours (prediction errors of zero and
// one quantum): those three are counted in registers and reduced once per
// warp, so the shared-memory atomics see only the spread-out remainder (no
// 32-way same-address conflicts).  Reads are 16-byte vectors where aligned.
__device__ __forceinline__ void hist_add(unsigned int* sh, unsigned long long* hist, unsigned v, unsigned& c_lo,
                                         unsigned& c_mid, unsigned& c_hi) {
  const unsigned d = v - 32767u;
  if (d < 3u) {
    c_lo += d == 0u;
    c_mid += d == 1u;
    c_hi += d == 2u;
  } else if (v == 0u) {
    atomicAdd(&sh[HIST_W], 1u);
  } else if (v - (unsigned)HIST_LO < (unsigned)HIST_W) {
    atomicAdd(&sh[v - HIST_LO], 1u);
  } else {
    atomicAdd(&hist[v], 1ull);
  }
}

__global__ void __launch_bounds__(HIST_NT) hist_u16_kernel(const uint16_t* __restrict__ s, size_t n,
                                                           unsigned long long* __restrict__ hist) {
  __shared__ unsigned int sh[HIST_W + 1];  // window + symbol 0
  for (int k = threadIdx.x; k <= HIST_W; k += HIST_NT) sh[k] = 0;
  __syncthreads();
  unsigned c_lo = 0, c_mid = 0, c_hi = 0;
  const size_t stride = (size_t)gridDim.x * HIST_NT;
  const size_t t0 = (size_t)blockIdx.x * HIST_NT + threadIdx.x;
  // elements before the first 16-byte boundary, the vector body, the tail
  const size_t head = ((16 - ((uintptr_t)s & 15)) & 15) / 2;
  const size_t h = head < n ? head : n;
  if (t0 < h) hist_add(sh, hist, s[t0], c_lo, c_mid, c_hi);
  const size_t nv = (n - h) / 8;
  const uint4* sv = reinterpret_cast<const uint4*>(s + h);
  for (size_t i = t0; i < nv; i += stride) {
    const uint4 w = __ldcs(sv + i);
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      hist_add(sh, hist, ws[q] & 0xffffu, c_lo, c_mid, c_hi);
      hist_add(sh, hist, ws[q] >> 16, c_lo, c_mid, c_hi);
    }
  }
  for (size_t i = h + nv * 8 + t0; i < n; i += stride) hist_add(sh, hist, s[i], c_lo, c_mid, c_hi);
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

size_t huff_encode_tmp_bytes(size_t n) {
  size_t nb = (n + ENC_PER_CTA - 1) / ENC_PER_CTA;
  return (align_up(nb, 32) + nb + 1 + 32) * sizeof(unsigned long long);
}

int launch_huff_encode_u8(cpsz_b200_ctx* ctx, const uint8_t* sym, size_t n, bool map_id_zero, HuffEncTable tab,
                          uint32_t* out_words, size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp) {
  return encode_impl<uint8_t>(ctx, sym, n, map_id_zero, tab, out_words, out_cap_bytes, d_total_bits, tmp);
}

int launch_huff_encode_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, HuffEncTable tab, uint32_t* out_words,
                           size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp) {
  return encode_impl<uint16_t>(ctx, sym, n, false, tab, out_words, out_cap_bytes, d_total_bits, tmp);
}

int launch_hist_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, unsigned long long* hist) {
  if (n == 0) return CPSZ_OK;
  int grid = ctx->num_sms * 2;
  size_t need = (n + HIST_NT - 1) / HIST_NT;
  if ((size_t)grid > need) grid = (int)need;
  hist_u16_kernel<<<grid, HIST_NT, 0, ctx->stream>>>(sym, n, hist);
  count_launch(ctx);
  return check_launch("hist_u16_kernel");
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
// this entry point packs a symbol stream with the same kernels as
// cpsz_b200_huffman_encode_u16 but takes its scratch -- the per-CTA bit
// counts and their scan -- from a fixed array in this file instead of a
// context workspace.  The array (about 260 KB) lives on every GPU that loads
// the library until the process exits, and it bounds the stream length.

constexpr size_t kNoAllocMaxSymbols = size_t(1) << 26;  // 67,108,864 symbols per call
constexpr size_t kNoAllocMaxCtas = kNoAllocMaxSymbols / ENC_PER_CTA;
constexpr size_t kNoAllocCounts = kNoAllocMaxCtas + 32;  // per-CTA bit counts (+ padding)
// layout: [counts: kNoAllocCounts][offsets: kNoAllocMaxCtas + 1][flag word]
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocCounts + kNoAllocMaxCtas + 1 + 1];

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
  unsigned long long* cta_bits = scratch;
  unsigned long long* cta_off = scratch + kNoAllocCounts;
  int* flag = (int*)(cta_off + kNoAllocMaxCtas + 1);
  // the packer ORs the edge words of every CTA: the output starts at zero
  CPSZ_CUDA_TRY(cudaMemsetAsync(out, 0, out_cap, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned long long), st));
  if (n == 0) {
    CPSZ_CUDA_TRY(cudaMemsetAsync(total_bits, 0, sizeof(uint64_t), st));
    return CPSZ_OK;
  }
  const size_t nb = (n + ENC_PER_CTA - 1) / ENC_PER_CTA;
  enc_count_kernel<uint16_t><<<(unsigned)nb, ENC_NT, 0, st>>>(sym, n, false, len, cta_bits);
  scan_u64_kernel<<<1, 1024, 0, st>>>(cta_bits, cta_off, nb);
  const size_t smem = ((size_t)ENC_PER_CTA * 64) / 32 * 4 + 16;
  enc_write_kernel<uint16_t><<<(unsigned)nb, ENC_NT, smem, st>>>(sym, n, false,
                                                                 (const unsigned long long*)code, len, cta_off,
                                                                 (uint32_t*)out, out_cap / 4, flag);
  CPSZ_CUDA_TRY(cudaMemcpyAsync(total_bits, cta_off + nb, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  return check_launch("huffman no-alloc encode");
}
