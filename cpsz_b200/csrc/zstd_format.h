// zstd_format.h -- writing Zstandard frames (RFC 8878), host and device code.
//
// The reference finishes every compression with ZSTD_compress(level 3) on the
// host (src/sz_lossless.cpp:11-26) and reads it back with ZSTD_decompress.
// The GPU lossless stage writes standard frames with the same decoder in mind,
// so the reference's sz_lossless_decompress reads them unchanged:
//   * frame header: magic, a window descriptor (no single segment), the
//     content size in 8 bytes, no dictionary, no checksum;
//   * blocks of at most 128 KB, each encoded on its own: raw literals and
//     sequences coded with the predefined FSE distributions (RFC 8878
//     section 3.1.1.3.2.2), every offset written as a real offset (offset
//     value = offset + 3), never a repeat code, so no state crosses blocks;
//   * a block whose compressed form is not smaller is stored raw, a block of
//     one repeated byte as an RLE block.
// The FSE encoding follows the published tANS construction (the decoding
// table of RFC 8878 section 4.1.1, read backwards): states in
// [table_size, 2 table_size), a symbol's transition emits the state's low
// bits and moves to the next state through the per-symbol (delta_nb_bits,
// delta_find_state) pair.
#pragma once

#include <cstddef>
#include <cstdint>

#ifdef __CUDACC__
#define ZHD __host__ __device__ __forceinline__
#else
#define ZHD inline
#endif

namespace cpsz {
namespace zstd {

constexpr uint32_t kMagic = 0xFD2FB528u;
constexpr int kBlockMax = 128 * 1024;
constexpr int kMinMatch = 4;   // matches the encoder emits (the format allows 3)
constexpr int kWindowLog = 22; // 4 MB window (offsets never exceed it)

// ---- sequence codes (RFC 8878 3.1.1.3.2.1.1) --------------------------------
// Literals length code -> baseline, extra bits; match length code -> baseline
// (of the length itself), extra bits.  Accessors (not namespace-scope arrays)
// so host and device code share them.
ZHD uint32_t ll_base(int c) {
  constexpr uint32_t t[36] = {0,  1,  2,  3,  4,  5,  6,  7,  8,   9,   10,  11,   12,   13,   14,    15,    16,   18,
                              20, 22, 24, 28, 32, 40, 48, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536};
  return t[c];
}
ZHD int ll_bits(int c) {
  constexpr uint8_t t[36] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  1,  1,
                             1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
  return t[c];
}
ZHD uint32_t ml_base(int c) {
  constexpr uint32_t t[53] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  12,  13,  14,  15,   16,   17,   18,   19,    20,
                              21, 22, 23, 24, 25, 26, 27, 28, 29,  30,  31,  32,  33,   34,   35,   37,   39,    41,
                              43, 47, 51, 59, 67, 83, 99, 131, 259, 515, 1027, 2051, 4099, 8195, 16387, 32771, 65539};
  return t[c];
}
ZHD int ml_bits(int c) {
  constexpr uint8_t t[53] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                             0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
  return t[c];
}

// Predefined distributions (RFC 8878 3.1.1.3.2.2); -1 = "less than 1".
constexpr int kLLLog = 6, kMLLog = 6, kOFLog = 5;
constexpr int16_t kLLNorm[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                 2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
constexpr int16_t kMLNorm[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};
constexpr int16_t kOFNorm[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};

ZHD int highbit32(uint32_t v) {
#ifdef __CUDA_ARCH__
  return 31 - __clz(v);
#else
  return 31 - __builtin_clz(v);
#endif
}

ZHD int ll_code(uint32_t ll) {
  if (ll < 16) return (int)ll;
  if (ll >= 65536) return 35;
  // codes 16..35 by baseline (monotone, 20 entries)
  int c = 16;
  while (c < 35 && ll_base(c + 1) <= ll) c++;
  return c;
}
// code of a match length (>= 3)
ZHD int ml_code(uint32_t ml) {
  const uint32_t b = ml - 3;
  if (b < 32) return (int)b;
  int c = 32;
  while (c < 52 && ml_base(c + 1) <= ml) c++;
  return c;
}

// ---- FSE compression table -------------------------------------------------------
struct FseSym {
  int32_t delta_find_state;
  uint32_t delta_nb_bits;
};
struct FseCTable {
  int table_log;
  int max_sym;
  uint16_t state[64];  // next-state table (state values table_size .. 2 table_size - 1)
  FseSym sym[64];
};

// Builds the compression table of a normalized distribution (host; the tables
// are small and constant).  The cell spread is the decoder's (RFC 8878 4.1.1):
// "less than 1" symbols take the last cells, the others are spread with step
// (size >> 1) + (size >> 3) + 3, skipping the cells of the former.
inline void fse_build(const int16_t* norm, int max_sym, int table_log, FseCTable* t) {
  const int size = 1 << table_log;
  int high = size - 1;
  uint8_t cell_sym[64];
  for (int s = 0; s <= max_sym; s++)
    if (norm[s] == -1) cell_sym[high--] = (uint8_t)s;
  const int step = (size >> 1) + (size >> 3) + 3, mask = size - 1;
  int pos = 0;
  for (int s = 0; s <= max_sym; s++)
    for (int i = 0; i < norm[s]; i++) {
      cell_sym[pos] = (uint8_t)s;
      do pos = (pos + step) & mask;
      while (pos > high);
    }
  // cumulative counts; cells of each symbol in increasing order -> encoder states
  int cum[65];
  cum[0] = 0;
  for (int s = 0; s <= max_sym; s++) cum[s + 1] = cum[s] + (norm[s] == -1 ? 1 : norm[s]);
  int fill[64];
  for (int s = 0; s <= max_sym; s++) fill[s] = cum[s];
  for (int u = 0; u < size; u++) t->state[fill[cell_sym[u]]++] = (uint16_t)(size + u);
  for (int s = 0; s <= max_sym; s++) {
    const int c = norm[s] == -1 ? 1 : norm[s];
    if (c == 0) {
      t->sym[s].delta_find_state = 0;
      t->sym[s].delta_nb_bits = ((uint32_t)(table_log + 1) << 16) - (uint32_t)size;
    } else if (c == 1) {
      t->sym[s].delta_find_state = cum[s] - 1;
      t->sym[s].delta_nb_bits = ((uint32_t)table_log << 16) - (uint32_t)size;
    } else {
      const int max_bits_out = table_log - highbit32((uint32_t)(c - 1));
      const uint32_t min_state_plus = (uint32_t)c << max_bits_out;
      t->sym[s].delta_nb_bits = ((uint32_t)max_bits_out << 16) - min_state_plus;
      t->sym[s].delta_find_state = cum[s] - c;
    }
  }
  t->table_log = table_log;
  t->max_sym = max_sym;
}

// ---- bit stream (forward writer; the decoder reads it backwards) ---------------
struct BitWriter {
  uint8_t* out;
  size_t cap, pos;
  uint64_t acc;
  int n;
  bool overflow;
};
ZHD void bw_init(BitWriter& w, uint8_t* out, size_t cap) {
  w.out = out;
  w.cap = cap;
  w.pos = 0;
  w.acc = 0;
  w.n = 0;
  w.overflow = false;
}
// appends the low `nb` bits of v (nb <= 32)
ZHD void bw_add(BitWriter& w, uint32_t v, int nb) {
  if (nb == 0) return;
  w.acc |= (uint64_t)(v & (uint32_t)((1ull << nb) - 1)) << w.n;
  w.n += nb;
  while (w.n >= 8) {
    if (w.pos < w.cap) w.out[w.pos] = (uint8_t)w.acc;
    else w.overflow = true;
    w.pos++;
    w.acc >>= 8;
    w.n -= 8;
  }
}
// end mark (one 1 bit) and the last partial byte; returns the stream's bytes
ZHD size_t bw_close(BitWriter& w) {
  bw_add(w, 1, 1);
  if (w.n > 0) {
    if (w.pos < w.cap) w.out[w.pos] = (uint8_t)w.acc;
    else w.overflow = true;
    w.pos++;
    w.acc = 0;
    w.n = 0;
  }
  return w.pos;
}

struct FseState {
  uint32_t value;
  const FseCTable* t;
};
ZHD void fse_init(FseState& s, const FseCTable* t, int sym) {
  const FseSym& tt = t->sym[sym];
  const uint32_t nb = (tt.delta_nb_bits + (1u << 15)) >> 16;
  const uint32_t v = (nb << 16) - tt.delta_nb_bits;
  s.t = t;
  s.value = t->state[(v >> nb) + tt.delta_find_state];
}
ZHD void fse_encode(BitWriter& w, FseState& s, int sym) {
  const FseSym& tt = s.t->sym[sym];
  const uint32_t nb = (s.value + tt.delta_nb_bits) >> 16;
  bw_add(w, s.value, (int)nb);
  s.value = s.t->state[(s.value >> nb) + tt.delta_find_state];
}
ZHD void fse_flush(BitWriter& w, const FseState& s) { bw_add(w, s.value, s.t->table_log); }

// The encoder's constant tables: the three predefined FSE tables and the
// sequence codes as lookups (device code reads them from constant memory; a
// length beyond the lookup takes the format's highbit rule).
struct Tables {
  FseCTable ll, ml, of;
  uint8_t ll_code[64];   // literals length -> code (>= 64: highbit + 19)
  uint8_t ml_code[128];  // match length - 3 -> code (>= 128: highbit + 36)
  uint8_t ll_bits[36], ml_bits[53];
};
inline void build_tables(Tables* t) {
  fse_build(kLLNorm, 35, kLLLog, &t->ll);
  fse_build(kMLNorm, 52, kMLLog, &t->ml);
  fse_build(kOFNorm, 28, kOFLog, &t->of);
  for (uint32_t v = 0; v < 64; v++) t->ll_code[v] = (uint8_t)ll_code(v);
  for (uint32_t v = 0; v < 128; v++) t->ml_code[v] = (uint8_t)ml_code(v + 3);
  for (int c = 0; c < 36; c++) t->ll_bits[c] = (uint8_t)ll_bits(c);
  for (int c = 0; c < 53; c++) t->ml_bits[c] = (uint8_t)ml_bits(c);
}
ZHD int ll_code_t(const Tables& T, uint32_t ll) { return ll < 64 ? T.ll_code[ll] : highbit32(ll) + 19; }
ZHD int ml_code_t(const Tables& T, uint32_t ml) {
  const uint32_t b = ml - 3;
  return b < 128 ? T.ml_code[b] : highbit32(b) + 36;
}

// One sequence: `lit` literals, then a match of `ml` (>= 3) bytes at distance `off`.
struct Seq {
  uint32_t lit, ml, off;
};

// Sequences section (RFC 8878 3.1.1.3.2): count, modes (all predefined), and
// the FSE bit stream written from the last sequence to the first.
// Returns bytes written, or 0 if `cap` was too small.
ZHD size_t write_sequences(const Tables& T, const Seq* seq, int nseq, uint8_t* out, size_t cap) {
  size_t p = 0;
  if (cap < 4) return 0;
  if (nseq < 128) {
    out[p++] = (uint8_t)nseq;
  } else if (nseq < 0x7F00) {
    out[p++] = (uint8_t)((nseq >> 8) + 128);
    out[p++] = (uint8_t)nseq;
  } else {
    out[p++] = 255;
    out[p++] = (uint8_t)(nseq - 0x7F00);
    out[p++] = (uint8_t)((nseq - 0x7F00) >> 8);
  }
  if (nseq == 0) return p;
  out[p++] = 0;  // predefined modes for literal lengths, offsets, match lengths
  BitWriter w;
  bw_init(w, out + p, cap - p);
  auto codes = [&T](const Seq& q, int& llc, int& mlc, int& ofc, uint32_t& ofv) {
    llc = ll_code_t(T, q.lit);
    mlc = ml_code_t(T, q.ml);
    ofv = q.off + 3;  // a real offset, never a repeat code
    ofc = highbit32(ofv);
  };
  int llc, mlc, ofc;
  uint32_t ofv;
  codes(seq[nseq - 1], llc, mlc, ofc, ofv);
  FseState sml, sof, sll;
  fse_init(sml, &T.ml, mlc);
  fse_init(sof, &T.of, ofc);
  fse_init(sll, &T.ll, llc);
  bw_add(w, seq[nseq - 1].lit, T.ll_bits[llc]);
  bw_add(w, seq[nseq - 1].ml - 3, T.ml_bits[mlc]);
  bw_add(w, ofv, ofc);
  for (int n = nseq - 2; n >= 0; n--) {
    codes(seq[n], llc, mlc, ofc, ofv);
    fse_encode(w, sof, ofc);
    fse_encode(w, sml, mlc);
    fse_encode(w, sll, llc);
    bw_add(w, seq[n].lit, T.ll_bits[llc]);
    bw_add(w, seq[n].ml - 3, T.ml_bits[mlc]);
    bw_add(w, ofv, ofc);
  }
  fse_flush(w, sml);
  fse_flush(w, sof);
  fse_flush(w, sll);
  const size_t nb = bw_close(w);
  if (w.overflow) return 0;
  return p + nb;
}

// Raw literals section header (RFC 8878 3.1.1.3.1.1) for `n` literals.
ZHD size_t write_raw_literals_header(uint32_t n, uint8_t* out) {
  if (n < 32) {
    out[0] = (uint8_t)(n << 3);
    return 1;
  }
  if (n < 4096) {
    out[0] = (uint8_t)(0x4 | ((n & 0xF) << 4));
    out[1] = (uint8_t)(n >> 4);
    return 2;
  }
  out[0] = (uint8_t)(0xC | ((n & 0xF) << 4));
  out[1] = (uint8_t)(n >> 4);
  out[2] = (uint8_t)(n >> 12);
  return 3;
}

// Block header: last flag, type (0 raw, 1 RLE, 2 compressed), 21-bit size.
ZHD void write_block_header(uint8_t* out, bool last, int type, uint32_t size) {
  const uint32_t h = (last ? 1u : 0u) | ((uint32_t)type << 1) | (size << 3);
  out[0] = (uint8_t)h;
  out[1] = (uint8_t)(h >> 8);
  out[2] = (uint8_t)(h >> 16);
}

// Frame header: magic, descriptor (8-byte content size, no single segment,
// no checksum, no dictionary), window descriptor.  Returns its size (14).
constexpr size_t kFrameHeader = 4 + 1 + 1 + 8;
inline size_t write_frame_header(uint8_t* out, uint64_t content_size) {
  out[0] = (uint8_t)kMagic;
  out[1] = (uint8_t)(kMagic >> 8);
  out[2] = (uint8_t)(kMagic >> 16);
  out[3] = (uint8_t)(kMagic >> 24);
  out[4] = (uint8_t)(3u << 6);                // Frame_Content_Size_flag = 3 (8 bytes)
  out[5] = (uint8_t)((kWindowLog - 10) << 3);  // exponent, mantissa 0
  for (int i = 0; i < 8; i++) out[6 + i] = (uint8_t)(content_size >> (8 * i));
  return kFrameHeader;
}

}  // namespace zstd
}  // namespace cpsz
