// pipeline3d.cu -- the 3D offline (log) compressor / decompressor on one GPU.
//
// Compress (sz_compress_cp_preserve_3d_offline_log<float>,
// src/sz_compress_cp_preserve_3d.cpp:360-581):
//   eb3d (bounds, ids) -> log3d (log2f, signs) -> Lorenzo planes (codes)
//   -> raster compaction (codes, unpredictable triples, final ids, id
//   histogram) + code histogram -> host Huffman trees -> GPU bit packing
//   -> blob assembled in device memory.
// Decompress (sz_decompress_cp_preserve_3d_online_log<float>,
// src/sz_decompress_cp_preserve_3d.cpp:7-110): host header/tree parsing ->
// GPU Huffman decode of ids and codes -> per-point addends / raw values ->
// Lorenzo planes with exp2f and signs fused.
//
// Blob layout (src/sz_compress_cp_preserve_3d.cpp:559-578):
//   int base (2) | int radius (32768) | 3 sign bitmaps of ceil(N/8) bytes
//   | size_t n_unpred | float[n_unpred] | size_t N | HUF(ids, 512 states)
//   | size_t n_codes | HUF(codes, 131072 states)
// For a field without predictable points the code section holds a one-leaf
// tree of symbol 0 and no bits (the reference cannot encode zero symbols).
#include <cstring>
#include <vector>

#include "huffman_host.h"
#include "kernels.h"
#include "transfer.h"
#include "pipeline.h"

namespace cpsz {

namespace {

int read_flag3(cpsz_b200_ctx* ctx, int* out) {
  CPSZ_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *(int*)ctx->pinned;
  return CPSZ_OK;
}

int flag_error3(int flag) {
  if (flag & FLAG_ID_OVERFLOW)
    return set_error(CPSZ_ERR_UNSUPPORTED,
                     "an error-bound id reaches the reference's unpredictable marker 24 (max_pwr_eb >= 3)");
  if (flag & FLAG_RAW_RANGE) return set_error(CPSZ_ERR_FORMAT, "code or unpredictable stream shorter than its ids");
  if (flag & FLAG_HUFF_CORRUPT) return set_error(CPSZ_ERR_FORMAT, "Huffman stream does not decode");
  if (flag & FLAG_OUT_CAPACITY) return set_error(CPSZ_ERR_INVALID, "an output stream exceeded its buffer");
  if (flag & FLAG_TIMEOUT) return set_error(CPSZ_ERR_TIMEOUT, "a bounded device-side wait gave up");
  return set_error(CPSZ_ERR_CUDA, "device flag %d", flag);
}

int check_dims(size_t r1, size_t r2, size_t r3) {
  if (r1 == 0 || r2 == 0 || r3 == 0) return set_error(CPSZ_ERR_INVALID, "empty field (%zu x %zu x %zu)", r1, r2, r3);
  if (r1 > (1u << 30) || r2 > (1u << 30) || r3 > (1u << 30) || r1 * r2 > (size_t)INT32_MAX ||
      r1 * r2 * r3 > ((size_t)1 << 32))
    return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu x %zu x %zu points is beyond 2^32 points", r1, r2, r3);
  return CPSZ_OK;
}

}  // namespace

int compress_3d(cpsz_b200_ctx* ctx, const float* U_in, const float* V_in, const float* W_in, size_t r1s, size_t r2s,
                size_t r3s, double max_pwr_eb, Blob3D* out) {
  if (!U_in || !V_in || !W_in) return set_error(CPSZ_ERR_INVALID, "null input field");
  CPSZ_TRY(check_dims(r1s, r2s, r3s));
  if (max_pwr_eb != max_pwr_eb) return set_error(CPSZ_ERR_INVALID, "max_pwr_eb is NaN");
  const int r1 = (int)r1s, r2 = (int)r2s, r3 = (int)r3s;
  const size_t N = r1s * r2s * r3s;
  const size_t smap = (N - 1) / 8 + 1;
  const size_t sign_words = (N + 31) / 32;
  const size_t nchunks = chunk_count(N);
  const bool dev_in = is_device_ptr(U_in) && is_device_ptr(V_in) && is_device_ptr(W_in);
  const QuantTable& qt = quant_table_3d();
  LibmTables lt;
  CPSZ_TRY(libm_tables_device(ctx, &lt));

  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  if (!dev_in) add(12 * N);
  add(N);              // ids
  add(16 * N);         // pairs
  add(16 * N);         // reconstruction
  add(8 * N);          // codes per point
  add(2 * (nchunks + 1) * 4);
  add(scan_u32_tmp_bytes(nchunks));
  add(6 * N);          // compacted codes
  add(12 * N);         // unpredictable triples
  add(3 * sign_words * 4);
  add(wave3d_scratch_bytes(r1, r2));
  add(256 * 8);
  add(65536 * 8);
  add(QUANT_TAB_MAX * 8);
  add(256 * 9);
  add(65536 * 9);
  add(256 * sizeof(HuffEntry));
  add(std::min<size_t>(65536, 3 * N + 1) * sizeof(HuffEntry));
  add(huff_encode_tmp_bytes(N));
  add(huff_encode_tmp_bytes(3 * N));
  const size_t ids_bits_cap = (N * 8 + 7) / 8 + 64;
  const size_t codes_bits_cap = (3 * N * 17 + 7) / 8 + 64;
  add(ids_bits_cap);
  add(codes_bits_cap);
  add(64);
  const size_t blob_cap = 8 + 3 * smap + 8 + 12 * N + 8 + 8 + 2 * (12 + 13 * 131072 + 8) + ids_bits_cap +
                          codes_bits_cap + 4096;
  add(blob_cap);
  CPSZ_TRY(arena_reserve(ctx, bytes));
  CPSZ_TRY(pinned_reserve(ctx, 65536 * 8 + 256 * 8 + 4096));
  auto A = [&](size_t b) { return arena_alloc(ctx, b); };
  cudaStream_t st = ctx->stream;
  const float *dU, *dV, *dW;
  if (dev_in) {
    dU = U_in;
    dV = V_in;
    dW = W_in;
  } else {
    float* h = (float*)A(12 * N);
    CPSZ_TRY(h2d(ctx, h, U_in, 4 * N, st));
    CPSZ_TRY(h2d(ctx, h + N, V_in, 4 * N, st));
    CPSZ_TRY(h2d(ctx, h + 2 * N, W_in, 4 * N, st));
    dU = h;
    dV = h + N;
    dW = h + 2 * N;
  }
  uint8_t* ids = (uint8_t*)A(N);
  float4* pairs = (float4*)A(16 * N);
  float4* rec = (float4*)A(16 * N);
  ushort4* codes = (ushort4*)A(8 * N);
  unsigned* chunk_cnt = (unsigned*)A((nchunks + 1) * 4);
  unsigned* chunk_off = (unsigned*)A((nchunks + 1) * 4);
  void* scan_tmp = A(scan_u32_tmp_bytes(nchunks));
  uint16_t* codes_out = (uint16_t*)A(6 * N);
  float* unpred = (float*)A(12 * N);
  uint32_t* signs = (uint32_t*)A(3 * sign_words * 4);
  void* wave_sync = A(wave3d_scratch_bytes(r1, r2));
  unsigned long long* hist_ids = (unsigned long long*)A(256 * 8);
  unsigned long long* hist_codes = (unsigned long long*)A(65536 * 8);
  double* thr_tab = (double*)A(QUANT_TAB_MAX * 8);
  unsigned long long* enc_code[2] = {(unsigned long long*)A(256 * 8), (unsigned long long*)A(65536 * 8)};
  uint8_t* enc_len[2] = {(uint8_t*)A(256), (uint8_t*)A(65536)};
  HuffEntry* enc_ent[2] = {(HuffEntry*)A(256 * sizeof(HuffEntry)),
                           (HuffEntry*)A(std::min<size_t>(65536, 3 * N + 1) * sizeof(HuffEntry))};
  void* enc_tmp[2] = {A(huff_encode_tmp_bytes(N)), A(huff_encode_tmp_bytes(3 * N))};
  uint32_t* bits[2] = {(uint32_t*)A(ids_bits_cap), (uint32_t*)A(codes_bits_cap)};
  (void)A(64);
  uint8_t* blob = (uint8_t*)A(blob_cap);
  if (!blob) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");

  reset_marks(ctx);
  mark(ctx, "h2d+setup");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(hist_ids, 0, 256 * 8, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(hist_codes, 0, 65536 * 8, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(thr_tab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice, st));
  mark(ctx, "eb3d");
  CPSZ_TRY(launch_eb3d(ctx, dU, dV, dW, r1, r2, r3, max_pwr_eb, thr_tab, qt.n, ids));
  mark(ctx, "log3d");
  CPSZ_TRY(launch_log3d(ctx, dU, dV, dW, ids, N, lt.log2f, pairs, signs, sign_words));
  mark(ctx, "wave3d_compress");
  CPSZ_TRY(launch_wave3d(ctx, false, pairs, rec, codes, nullptr, 0, &lt, nullptr, nullptr, nullptr, r1, r2, r3,
                          wave_sync));
  mark(ctx, "compact+hist");
  // The code histogram straight from the raster codes, so the host builds
  // the code tree while the GPU compacts: a predictable point's three codes
  // are never 0 (|q| <= 32767 around 32768), an unpredictable point's are,
  // and so is every fourth lane, so the count without symbol 0 is the
  // compacted codes' histogram.
  unsigned* h_npred = (unsigned*)ctx->pinned + 4;  // the flag word lives at offset 0
  unsigned long long* h_hist_ids = (unsigned long long*)ctx->pinned + 8;
  unsigned long long* h_hist_codes = h_hist_ids + 256;
  CPSZ_TRY(launch_hist_u16_nonzero(ctx, reinterpret_cast<const uint16_t*>(codes), 4 * N, hist_codes));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h_hist_codes, hist_codes, 65536 * 8, cudaMemcpyDeviceToHost, st));
  CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));
  CPSZ_TRY(launch_chunk_count_3d(ctx, true, codes, N, chunk_cnt));
  CPSZ_TRY(launch_scan_u32(ctx, chunk_cnt, chunk_off, nchunks, scan_tmp));
  CPSZ_TRY(launch_compact3d(ctx, codes, ids, dU, dV, dW, N, chunk_off, codes_out, unpred, hist_ids));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h_npred, chunk_off + nchunks, 4, cudaMemcpyDeviceToHost, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h_hist_ids, hist_ids, 256 * 8, cudaMemcpyDeviceToHost, st));
  mark(ctx, "host_trees");
  HuffCodebook cb[2];
  CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[1]));
  bool any_code = false;
  for (size_t s = 1; s < 65536 && !any_code; s++) any_code = h_hist_codes[s] != 0;
  if (!any_code) h_hist_codes[0] = 1;  // no predictable point: one-leaf tree of symbol 0, no bits
  if (!huff_build(h_hist_codes, 65536, 131072, &cb[1])) return CPSZ_ERR_INVALID;
  CPSZ_CUDA_TRY(cudaStreamSynchronize(st));
  int flag = 0;
  CPSZ_TRY(read_flag3(ctx, &flag));
  if (flag) return flag_error3(flag);
  const size_t n_pred = *h_npred;
  const size_t n_codes = 3 * n_pred, n_unpred = 3 * (N - n_pred);
  if (!huff_build(h_hist_ids, 256, 512, &cb[0])) return CPSZ_ERR_INVALID;

  mark(ctx, "huffman_encode");
  const size_t sec_bytes[2] = {huff_section_bytes(cb[0]), huff_section_bytes(cb[1])};
  const size_t bits_bytes[2] = {(cb[0].total_bits + 7) / 8, (cb[1].total_bits + 7) / 8};
  if (bits_bytes[0] + 8 > ids_bits_cap || bits_bytes[1] + 8 > codes_bits_cap)
    return set_error(CPSZ_ERR_UNSUPPORTED, "Huffman stream larger than its bound");
  for (int k = 0; k < 2; k++) {
    CPSZ_TRY(huff_upload(ctx, cb[k], nullptr, enc_ent[k], enc_code[k], enc_len[k]));
    CPSZ_CUDA_TRY(cudaMemsetAsync(bits[k], 0, align_up(bits_bytes[k], 4) + 8, st));
  }
  CPSZ_TRY(launch_huff_encode_u8(ctx, ids, N, false, HuffEncTable{enc_code[0], enc_len[0], 256}, bits[0],
                                 ids_bits_cap, nullptr, enc_tmp[0]));
  if (n_codes)
    CPSZ_TRY(launch_huff_encode_u16(ctx, codes_out, n_codes, HuffEncTable{enc_code[1], enc_len[1], 65536}, bits[1],
                                    codes_bits_cap, nullptr, enc_tmp[1]));

  mark(ctx, "blob_assembly");
  const size_t total = 8 + 3 * smap + 8 + 4 * n_unpred + 8 + sec_bytes[0] + 8 + sec_bytes[1];
  if (total > blob_cap) return set_error(CPSZ_ERR_UNSUPPORTED, "blob larger than its bound");
  std::vector<uint8_t> small;
  struct Piece {
    size_t dst, src, n;
  };
  std::vector<Piece> pieces;
  auto stage = [&](size_t dst, const void* p, size_t n) {
    pieces.push_back(Piece{dst, small.size(), n});
    small.insert(small.end(), (const uint8_t*)p, (const uint8_t*)p + n);
  };
  size_t at = 0;
  const int hdr[2] = {2, 32768};
  stage(at, hdr, 8);
  at += 8;
  const size_t sign_at = at;
  at += 3 * smap;
  unsigned long long v64 = n_unpred;
  stage(at, &v64, 8);
  at += 8;
  const size_t unpred_at = at;
  at += 4 * n_unpred;
  v64 = N;
  stage(at, &v64, 8);
  at += 8;
  size_t bit_at[2];
  for (int k = 0; k < 2; k++) {
    if (k == 1) {
      v64 = n_codes;
      stage(at, &v64, 8);
      at += 8;
    }
    stage(at, cb[k].tree_bytes.data(), cb[k].tree_bytes.size());
    at += cb[k].tree_bytes.size();
    unsigned long long nb = bits_bytes[k];
    stage(at, &nb, 8);
    at += 8;
    bit_at[k] = at;
    at += bits_bytes[k];
  }
  if (at != total) return set_error(CPSZ_ERR_INVALID, "internal: blob layout mismatch (%zu != %zu)", at, total);
  uint8_t* d_small = blob + align_up(total, 256);
  if (align_up(total, 256) + small.size() > blob_cap) {
    for (const Piece& p : pieces)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + p.dst, small.data() + p.src, p.n, cudaMemcpyHostToDevice, st));
  } else {
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d_small, small.data(), small.size(), cudaMemcpyHostToDevice, st));
    for (const Piece& p : pieces)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + p.dst, d_small + p.src, p.n, cudaMemcpyDeviceToDevice, st));
  }
  for (int c = 0; c < 3; c++)
    CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + sign_at + c * smap, signs + c * sign_words, smap, cudaMemcpyDeviceToDevice, st));
  if (n_unpred)
    CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + unpred_at, unpred, 4 * n_unpred, cudaMemcpyDeviceToDevice, st));
  for (int k = 0; k < 2; k++)
    if (bits_bytes[k])
      CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + bit_at[k], bits[k], bits_bytes[k], cudaMemcpyDeviceToDevice, st));
  mark(ctx, "end");
  CPSZ_TRY(read_flag3(ctx, &flag));
  if (flag) return flag_error3(flag);
  out->d_blob = blob;
  out->size = total;
  out->n_unpred = n_unpred;
  out->n_codes = n_codes;
  return CPSZ_OK;
}

int decompress_3d(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1s, size_t r2s, size_t r3s,
                  float* U_out, float* V_out, float* W_out) {
  if (!blob || !U_out || !V_out || !W_out) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  CPSZ_TRY(check_dims(r1s, r2s, r3s));
  const int r1 = (int)r1s, r2 = (int)r2s, r3 = (int)r3s;
  const size_t N = r1s * r2s * r3s;
  const size_t smap = (N - 1) / 8 + 1;
  const size_t nchunks = chunk_count(N);
  // ---- header ----
  if (blob_size < 8 + 3 * smap + 8) return set_error(CPSZ_ERR_FORMAT, "blob shorter than its header");
  int base, radius;
  memcpy(&base, blob, 4);
  memcpy(&radius, blob + 4, 4);
  if (base != 2 || radius != 32768)
    return set_error(CPSZ_ERR_UNSUPPORTED, "blob quantizer (base %d, radius %d) is not the offline compressor's", base,
                     radius);
  size_t at = 8 + 3 * smap;
  unsigned long long n_unpred, n_ids, n_codes;
  memcpy(&n_unpred, blob + at, 8);
  at += 8;
  if (n_unpred > 3 * N || (blob_size - at) / 4 < n_unpred)
    return set_error(CPSZ_ERR_FORMAT, "unpredictable count %llu invalid", n_unpred);
  const size_t unpred_at = at;
  at += 4 * n_unpred;
  if (blob_size - at < 8) return set_error(CPSZ_ERR_FORMAT, "blob truncated before the id section");
  memcpy(&n_ids, blob + at, 8);
  at += 8;
  if (n_ids != N) return set_error(CPSZ_ERR_FORMAT, "id count %llu != %zu points", n_ids, N);
  HuffDecoderHost hs[2];
  if (!huff_parse(blob + at, blob_size - at, 511, &hs[0])) return CPSZ_ERR_FORMAT;
  for (uint32_t s : hs[0].sym)
    if (s > (uint32_t)ID_RAW_3D)
      return set_error(CPSZ_ERR_UNSUPPORTED, "error-bound id %u beyond the supported range (<= %d)", s, ID_RAW_3D);
  const size_t ids_at = at;
  at += hs[0].section_bytes;
  if (blob_size - at < 8) return set_error(CPSZ_ERR_FORMAT, "blob truncated before the code section");
  memcpy(&n_codes, blob + at, 8);
  at += 8;
  if (n_codes > 3 * N) return set_error(CPSZ_ERR_FORMAT, "code count %llu invalid", n_codes);
  if (!huff_parse(blob + at, blob_size - at, 65535, &hs[1])) return CPSZ_ERR_FORMAT;
  const size_t codes_at = at;
  const bool dev_out = is_device_ptr(U_out) && is_device_ptr(V_out) && is_device_ptr(W_out);
  LibmTables lt;
  CPSZ_TRY(libm_tables_device(ctx, &lt));

  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  if (!dev_out) add(12 * N);
  add(3 * smap + 16);
  add(4 * n_unpred + 16);
  add(N);
  add(2 * n_codes + 16);
  for (int k = 0; k < 2; k++) {
    add(hs[k].nbytes + 64);
    add((1u << HUFF_LUT_BITS) * 4 + hs[k].child.size() * 4 + hs[k].sym.size() * 4 + hs[k].leaf.size());
    add(huff_decode_tmp_bytes(hs[k].nbytes * 8));
  }
  add(2 * (nchunks + 1) * 4);
  add(scan_u32_tmp_bytes(nchunks));
  add(16 * N);
  add(16 * N);
  add(wave3d_scratch_bytes(r1, r2));
  CPSZ_TRY(arena_reserve(ctx, bytes));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  auto A = [&](size_t b) { return arena_alloc(ctx, b); };
  cudaStream_t st = ctx->stream;
  float* out = dev_out ? nullptr : (float*)A(12 * N);
  float* dU = dev_out ? U_out : out;
  float* dV = dev_out ? V_out : out + N;
  float* dW = dev_out ? W_out : out + 2 * N;
  uint8_t* signs = (uint8_t*)A(3 * smap + 16);
  float* unpred = (float*)A(4 * n_unpred + 16);
  uint8_t* ids = (uint8_t*)A(N);
  uint16_t* codes = (uint16_t*)A(2 * n_codes + 16);
  uint8_t* bits[2];
  HuffDecTable tab[2];
  void* dtmp[2];
  const size_t sec_at[2] = {ids_at, codes_at};
  for (int k = 0; k < 2; k++) {
    const HuffDecoderHost& h = hs[k];
    bits[k] = (uint8_t*)A(h.nbytes + 64);
    const size_t tb = (1u << HUFF_LUT_BITS) * 4 + h.child.size() * 4 + h.sym.size() * 4 + h.leaf.size();
    uint8_t* t = (uint8_t*)A(tb);
    dtmp[k] = A(huff_decode_tmp_bytes(h.nbytes * 8));
    if (!dtmp[k]) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
    CPSZ_CUDA_TRY(cudaMemsetAsync(bits[k], 0, h.nbytes + 64, st));
    if (h.nbytes)
      CPSZ_TRY(h2d(ctx, bits[k], blob + sec_at[k] + h.bits_offset, h.nbytes, st));
    uint32_t* lut = (uint32_t*)t;
    uint32_t* child = lut + (1u << HUFF_LUT_BITS);
    uint32_t* sym = child + h.child.size();
    uint8_t* leaf = (uint8_t*)(sym + h.sym.size());
    CPSZ_CUDA_TRY(cudaMemcpyAsync(lut, h.lut.data(), h.lut.size() * 4, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(child, h.child.data(), h.child.size() * 4, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(sym, h.sym.data(), h.sym.size() * 4, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(leaf, h.leaf.data(), h.leaf.size(), cudaMemcpyHostToDevice, st));
    tab[k] = HuffDecTable{lut, child, sym, leaf, h.node_count, h.root_is_leaf ? 1 : 0, h.root_sym};
  }
  unsigned* chunk_cnt = (unsigned*)A((nchunks + 1) * 4);
  unsigned* chunk_off = (unsigned*)A((nchunks + 1) * 4);
  void* scan_tmp = A(scan_u32_tmp_bytes(nchunks));
  float4* pairs = (float4*)A(16 * N);
  float4* rec = (float4*)A(16 * N);
  void* wave_sync = A(wave3d_scratch_bytes(r1, r2));
  if (!wave_sync) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  CPSZ_TRY(h2d(ctx, signs, blob + 8, 3 * smap, st));
  if (n_unpred) CPSZ_TRY(h2d(ctx, unpred, blob + unpred_at, 4 * n_unpred, st));
  reset_marks(ctx);
  mark(ctx, "huffman_decode");
  CPSZ_TRY(launch_huff_decode(ctx, bits[0], hs[0].nbytes, N, tab[0], ids, 1, dtmp[0]));
  if (n_codes) CPSZ_TRY(launch_huff_decode(ctx, bits[1], hs[1].nbytes, n_codes, tab[1], codes, 2, dtmp[1]));
  mark(ctx, "prep3d");
  CPSZ_TRY(launch_chunk_count_3d(ctx, false, ids, N, chunk_cnt));
  CPSZ_TRY(launch_scan_u32(ctx, chunk_cnt, chunk_off, nchunks, scan_tmp));
  CPSZ_TRY(launch_prep3d(ctx, ids, N, chunk_off, codes, n_codes, unpred, n_unpred, pairs));
  mark(ctx, "wave3d_decompress");
  CPSZ_TRY(launch_wave3d(ctx, true, pairs, rec, nullptr, signs, smap, &lt, dU, dV, dW, r1, r2, r3, wave_sync));
  mark(ctx, "d2h");
  if (!dev_out) {
    CPSZ_TRY(d2h(ctx, U_out, dU, 4 * N, st));
    CPSZ_TRY(d2h(ctx, V_out, dV, 4 * N, st));
    CPSZ_TRY(d2h(ctx, W_out, dW, 4 * N, st));
  }
  mark(ctx, "end");
  int flag = 0;
  CPSZ_TRY(read_flag3(ctx, &flag));
  if (flag) return flag_error3(flag);
  return CPSZ_OK;
}

}  // namespace cpsz
