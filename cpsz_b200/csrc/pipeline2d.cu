// pipeline2d.cu -- the 2D offline compressor / decompressor on one GPU.
//
// Compress (sz_compress_cp_preserve_2d_offline<float>,
// src/sz_compress_cp_preserve_2d.cpp:175-274):
//   eb2d (bounds + ids + id histogram)  ->  wave2d compress of U and V (codes)
//   -> block-order permutation + code histograms, unpredictable gather
//   -> host Huffman trees (reference tie-breaking) -> GPU bit packing
//   -> blob assembled in device memory -> one copy to the caller.
// The id tree is built on the host while the wavefront runs.
//
// Decompress (sz_decompress_cp_preserve_2d_offline<float>,
// src/sz_decompress_cp_preserve_2d.cpp:8-52): host header/tree parsing ->
// GPU Huffman decode of ids and codes -> raster permutation, unpredictable
// scatter -> wave2d decompress of U and V.
//
// Blob layout (src/sz_compress_cp_preserve_2d.cpp:258-269, src/sz_compress_3d.cpp:219-228):
//   int base(4) | double thr(2^-52) | size_t eb_size | size_t u_size | size_t v_size
//   | HUF(ids, 2048 states, 2N) | FIELD(U) | FIELD(V)
//   FIELD = int 12 | char 0 | int 32768 | meanInfo<float>{false,0} (8 B) | size_t 0
//         | size_t n_unpred | float[n_unpred] | ceil(nblocks/8) zero bytes | HUF(codes, 131072 states, N)
#include <cfloat>
#include <cstring>
#include <vector>

#include "huffman_host.h"
#include "kernels.h"
#include "pipeline.h"

namespace cpsz {

namespace {

constexpr int BS = 12;
constexpr size_t FIELD_HDR = 4 + 1 + 4 + 8 + 8 + 8;  // up to and including n_unpred
constexpr size_t BLOB_HDR = 4 + 8 + 8 + 8 + 8;

struct DevBuf {
  // arena sub-allocations of one compress call
  float* U;
  float* V;
  uint8_t* ids;  // 2N: U ids then V ids
  unsigned long long* hist_ids;
  uint16_t* craster[2];
  float2* pairs[2];  // per-point (value, 1/precision) pairs read by the wavefront
  uint16_t* cblocks[2];
  unsigned long long* hist_codes[2];
  unsigned long long* gbnd;
  int* queue;
  WaveField* fields;
  WaveItem* items;
  unsigned int* seg_cnt[2];
  unsigned int* seg_off[2];
  void* scan_tmp[2];
  float* unpred[2];
  double* thr_tab;
  unsigned long long* enc_code[3];
  uint8_t* enc_len[3];
  void* enc_tmp[3];
  uint32_t* bits[3];
  unsigned long long* bits_total;
  uint8_t* blob;
};

int read_flag(cpsz_b200_ctx* ctx, int* out) {
  CPSZ_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *(int*)ctx->pinned;
  return CPSZ_OK;
}

int flag_error(int flag) {
  if (flag & FLAG_TIMEOUT) return set_error(CPSZ_ERR_TIMEOUT, "a bounded device-side wait gave up");
  if (flag & FLAG_ID_OVERFLOW)
    return set_error(CPSZ_ERR_UNSUPPORTED, "an error-bound id does not fit the 8-bit id stream (max_pwr_eb too large)");
  if (flag & FLAG_HUFF_CORRUPT) return set_error(CPSZ_ERR_FORMAT, "Huffman stream does not decode");
  if (flag & FLAG_RAW_RANGE) return set_error(CPSZ_ERR_FORMAT, "unpredictable-value list shorter than its codes");
  if (flag & FLAG_OUT_CAPACITY) return set_error(CPSZ_ERR_INVALID, "an output stream exceeded its buffer");
  return CPSZ_OK;
}

}  // namespace

int build_wave_items(int nfields, const int* r1s, std::vector<WaveItem>& items) {
  int maxg = 0;
  for (int f = 0; f < nfields; f++) maxg = std::max(maxg, (r1s[f] + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS);
  items.clear();
  for (int g = 0; g < maxg; g++)
    for (int f = 0; f < nfields; f++)
      if (g * WAVE_GROUP_ROWS < r1s[f]) items.push_back(WaveItem{f, g});
  return (int)items.size();
}

int compress_2d(cpsz_b200_ctx* ctx, const float* U_in, const float* V_in, size_t r1s, size_t r2s, double max_pwr_eb,
                Blob2D* out, const StageTap* tap) {
  if (!U_in || !V_in) return set_error(CPSZ_ERR_INVALID, "null input field");
  if (r1s == 0 || r2s == 0) return set_error(CPSZ_ERR_INVALID, "empty field (%zu x %zu)", r1s, r2s);
  if (r1s > (1u << 30) || r2s > (1u << 30) || r1s * r2s > (size_t)INT32_MAX)
    return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu x %zu points exceeds 2^31 points", r1s, r2s);
  if (max_pwr_eb != max_pwr_eb) return set_error(CPSZ_ERR_INVALID, "max_pwr_eb is NaN");
  const int r1 = (int)r1s, r2 = (int)r2s;
  const size_t N = r1s * r2s;
  const int ngroups = (r1 + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS;
  const int nby = (r2 - 1) / BS + 1, nbx = (r1 - 1) / BS + 1;
  const size_t nseg = (size_t)r1 * nby;
  const size_t nblocks = (size_t)nbx * nby;
  const bool dev_in = is_device_ptr(U_in) && is_device_ptr(V_in);
  const QuantTable& qt = quant_table_2d();

  // ---- workspace ----
  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  if (!dev_in) add(8 * N);
  add(2 * N);                         // ids
  add(256 * 8);                       // hist ids
  add(4 * N);                         // codes raster
  add(16 * N);                        // wavefront input pairs
  add(4 * N);                         // codes blocks
  add(2 * 65536 * 8);                 // hist codes
  add(2 * (size_t)ngroups * r2 * 8);  // boundary rows (tagged words)
  add(64);                            // work-queue counter
  add(2 * sizeof(WaveField) + 2 * (size_t)ngroups * sizeof(WaveItem));
  add(2 * 2 * (nseg + 1) * 4);
  add(2 * segment_scan_tmp_bytes(r1, r2));
  add(2 * 4 * N);  // unpred
  add(QUANT_TAB_MAX * 8);
  add(256 * 9);
  add(2 * 65536 * 9);
  add(huff_encode_tmp_bytes(2 * N));
  add(2 * huff_encode_tmp_bytes(N));
  // bit streams: Huffman averages < log2(distinct) + 1 bits per symbol
  const size_t ids_bits_cap = (2 * N * 9 + 7) / 8 + 64;
  const size_t codes_bits_cap = (N * 17 + 7) / 8 + 64;
  add(ids_bits_cap);
  add(2 * codes_bits_cap);
  add(64);
  const size_t blob_cap = BLOB_HDR + 2 * FIELD_HDR + 8 * N + 2 * ((nblocks + 7) / 8) + 3 * (12 + 1 + 13 * 131072 + 8) +
                          ids_bits_cap + 2 * codes_bits_cap + 64;
  add(blob_cap);
  CPSZ_TRY(arena_reserve(ctx, bytes));
  CPSZ_TRY(pinned_reserve(ctx, 2 * 65536 * 8 + 256 * 8 + 4096));
  DevBuf d{};
  auto A = [&](size_t b) { return arena_alloc(ctx, b); };
  cudaStream_t st = ctx->stream;
  if (dev_in) {
    d.U = const_cast<float*>(U_in);
    d.V = const_cast<float*>(V_in);
  } else {
    d.U = (float*)A(4 * N);
    d.V = (float*)A(4 * N);
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d.U, U_in, 4 * N, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d.V, V_in, 4 * N, cudaMemcpyHostToDevice, st));
  }
  d.ids = (uint8_t*)A(2 * N);
  d.hist_ids = (unsigned long long*)A(256 * 8);
  for (int f = 0; f < 2; f++) {
    d.craster[f] = (uint16_t*)A(2 * N);
    d.pairs[f] = (float2*)A(8 * N);
    d.cblocks[f] = (uint16_t*)A(2 * N);
    d.hist_codes[f] = (unsigned long long*)A(65536 * 8);
  }
  d.gbnd = (unsigned long long*)A(2 * (size_t)ngroups * r2 * 8);
  d.queue = (int*)A(64);
  d.fields = (WaveField*)A(2 * sizeof(WaveField));
  d.items = (WaveItem*)A(2 * (size_t)ngroups * sizeof(WaveItem));
  for (int f = 0; f < 2; f++) {
    d.seg_cnt[f] = (unsigned int*)A((nseg + 1) * 4);
    d.seg_off[f] = (unsigned int*)A((nseg + 1) * 4);
    d.scan_tmp[f] = A(segment_scan_tmp_bytes(r1, r2));
    d.unpred[f] = (float*)A(4 * N);
  }
  d.thr_tab = (double*)A(QUANT_TAB_MAX * 8);
  d.enc_code[0] = (unsigned long long*)A(256 * 8);
  d.enc_len[0] = (uint8_t*)A(256);
  for (int f = 1; f < 3; f++) {
    d.enc_code[f] = (unsigned long long*)A(65536 * 8);
    d.enc_len[f] = (uint8_t*)A(65536);
  }
  d.enc_tmp[0] = A(huff_encode_tmp_bytes(2 * N));
  d.enc_tmp[1] = A(huff_encode_tmp_bytes(N));
  d.enc_tmp[2] = A(huff_encode_tmp_bytes(N));
  d.bits[0] = (uint32_t*)A(ids_bits_cap);
  d.bits[1] = (uint32_t*)A(codes_bits_cap);
  d.bits[2] = (uint32_t*)A(codes_bits_cap);
  d.bits_total = (unsigned long long*)A(64);
  d.blob = (uint8_t*)A(blob_cap);
  if (!d.blob) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");

  // ---- stage 1: error bounds ----
  reset_marks(ctx);
  mark(ctx, "h2d+setup");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(d.hist_ids, 0, 256 * 8, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d.thr_tab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice, st));
  mark(ctx, "eb2d");
  CPSZ_TRY(launch_eb2d(ctx, d.U, d.V, r1, r2, max_pwr_eb, d.thr_tab, qt.n, d.ids, d.ids + N, d.hist_ids,
                       d.pairs[0], d.pairs[1]));
  mark(ctx, "eb2d_end");
  unsigned long long* h_hist_ids = (unsigned long long*)ctx->pinned;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h_hist_ids, d.hist_ids, 256 * 8, cudaMemcpyDeviceToHost, st));
  CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[0], st));
  if (tap && tap->ids) CPSZ_CUDA_TRY(cudaMemcpyAsync(tap->ids, d.ids, 2 * N, cudaMemcpyDeviceToDevice, st));

  // ---- stage 2: Lorenzo wavefront of U and V ----
  std::vector<WaveField> hf(2);
  for (int f = 0; f < 2; f++) {
    WaveField& F = hf[f];
    F.pair = d.pairs[f];
    F.codes = d.craster[f];
    F.trace = (ctx->d_wave_trace && ctx->wave_trace_len >= 2 * (size_t)ngroups * WAVE_WARPS * 4)
                  ? ctx->d_wave_trace + (size_t)f * ngroups * WAVE_WARPS * 4
                  : nullptr;
    F.out = tap ? tap->recon[f] : nullptr;
    F.gbnd = d.gbnd + (size_t)f * ngroups * r2;
    F.pair_pitch = r2;
    F.code_pitch = r2;
    F.out_pitch = r2;
    F.r1 = r1;
    F.r2 = r2;
  }
  int r1v[2] = {r1, r1};
  std::vector<WaveItem> items;
  int n_items = build_wave_items(2, r1v, items);
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d.fields, hf.data(), 2 * sizeof(WaveField), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d.items, items.data(), n_items * sizeof(WaveItem), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(d.gbnd, 0, 2 * (size_t)ngroups * r2 * 8, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(d.queue, 0, 64, st));
  mark(ctx, "wave2d_compress");
  CPSZ_TRY(launch_wave2d(ctx, false, d.fields, d.items, n_items, d.queue, 0));
  mark(ctx, "blocks+hist+unpred");

  // ---- stage 3: block order, histograms, unpredictables ----
  unsigned long long* h_hist_codes = h_hist_ids + 256;
  unsigned int* h_nunpred = (unsigned int*)(h_hist_codes + 2 * 65536);
  for (int f = 0; f < 2; f++) {
    CPSZ_CUDA_TRY(cudaMemsetAsync(d.hist_codes[f], 0, 65536 * 8, st));
    CPSZ_TRY(launch_raster_to_blocks_u16(ctx, d.craster[f], r2, r1, r2, d.cblocks[f], d.hist_codes[f]));
    CPSZ_TRY(launch_segment_scan(ctx, d.craster[f], r2, r1, r2, d.seg_cnt[f], d.seg_off[f], d.scan_tmp[f]));
    CPSZ_TRY(launch_gather_unpred(ctx, d.craster[f], r2, f ? d.V : d.U, r2, r1, r2, d.seg_off[f], d.unpred[f]));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(h_hist_codes + (size_t)f * 65536, d.hist_codes[f], 65536 * 8,
                                  cudaMemcpyDeviceToHost, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(h_nunpred + f, d.seg_off[f] + nseg, 4, cudaMemcpyDeviceToHost, st));
  }
  mark(ctx, "host_trees");
  CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));

  // host: id tree while the GPU runs the wavefront
  CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[0]));
  HuffCodebook cb[3];
  if (!huff_build(h_hist_ids, 256, 2048, &cb[0])) return CPSZ_ERR_INVALID;
  CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[1]));
  int flag = 0;
  CPSZ_TRY(read_flag(ctx, &flag));
  if (flag) return flag_error(flag);
  for (int f = 0; f < 2; f++)
    if (!huff_build(h_hist_codes + (size_t)f * 65536, 65536, 131072, &cb[1 + f])) return CPSZ_ERR_INVALID;
  const size_t n_unpred[2] = {h_nunpred[0], h_nunpred[1]};

  // ---- stage 4: bit packing ----
  const size_t sec_bytes[3] = {huff_section_bytes(cb[0]), huff_section_bytes(cb[1]), huff_section_bytes(cb[2])};
  const size_t bits_bytes[3] = {(cb[0].total_bits + 7) / 8, (cb[1].total_bits + 7) / 8, (cb[2].total_bits + 7) / 8};
  if (bits_bytes[0] + 8 > ids_bits_cap || bits_bytes[1] + 8 > codes_bits_cap || bits_bytes[2] + 8 > codes_bits_cap)
    return set_error(CPSZ_ERR_UNSUPPORTED, "Huffman stream larger than its bound");
  mark(ctx, "huffman_encode");
  for (int k = 0; k < 3; k++) {
    const size_t bins = k ? 65536 : 256;
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d.enc_code[k], cb[k].code.data(), bins * 8, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d.enc_len[k], cb[k].len.data(), bins, cudaMemcpyHostToDevice, st));
    CPSZ_CUDA_TRY(cudaMemsetAsync(d.bits[k], 0, align_up(bits_bytes[k], 4) + 8, st));
  }
  CPSZ_TRY(launch_huff_encode_u8(ctx, d.ids, 2 * N, true, HuffEncTable{d.enc_code[0], d.enc_len[0], 256}, d.bits[0],
                                 ids_bits_cap, nullptr, d.enc_tmp[0]));
  for (int f = 0; f < 2; f++)
    CPSZ_TRY(launch_huff_encode_u16(ctx, d.cblocks[f], N, HuffEncTable{d.enc_code[1 + f], d.enc_len[1 + f], 65536},
                                    d.bits[1 + f], codes_bits_cap, nullptr, d.enc_tmp[1 + f]));

  mark(ctx, "blob_assembly");
  // ---- stage 5: blob assembly in device memory ----
  const size_t ind_bytes = (nblocks + 7) / 8;
  size_t field_size[2];
  for (int f = 0; f < 2; f++) field_size[f] = FIELD_HDR + 4 * n_unpred[f] + ind_bytes + sec_bytes[1 + f];
  const size_t total = BLOB_HDR + sec_bytes[0] + field_size[0] + field_size[1];
  if (total > blob_cap) return set_error(CPSZ_ERR_UNSUPPORTED, "blob larger than its bound");
  std::vector<uint8_t> hdr(BLOB_HDR + 2 * (FIELD_HDR + 12 + 131072 * 13 + 8), 0);
  // header
  {
    size_t at = 0;
    auto put = [&](const void* p, size_t n) {
      memcpy(hdr.data() + at, p, n);
      at += n;
    };
    const int base = 4;
    const double thr = DBL_EPSILON;
    put(&base, 4);
    put(&thr, 8);
    put(&sec_bytes[0], 8);
    put(&field_size[0], 8);
    put(&field_size[1], 8);
  }
  // host staging of all small pieces: blob header, id tree + size, field headers, code trees + sizes
  std::vector<uint8_t> small;
  struct Piece { size_t dst, src, n; };
  std::vector<Piece> pieces;
  auto stage = [&](size_t dst, const void* p, size_t n) {
    pieces.push_back(Piece{dst, small.size(), n});
    small.insert(small.end(), (const uint8_t*)p, (const uint8_t*)p + n);
  };
  size_t at = 0;
  stage(at, hdr.data(), BLOB_HDR);
  at += BLOB_HDR;
  size_t bit_dst[3], unpred_dst[2];
  auto stage_huff = [&](int k) {
    stage(at, cb[k].tree_bytes.data(), cb[k].tree_bytes.size());
    at += cb[k].tree_bytes.size();
    unsigned long long nb = bits_bytes[k];
    stage(at, &nb, 8);
    at += 8;
    bit_dst[k] = at;
    at += bits_bytes[k];
  };
  stage_huff(0);
  for (int f = 0; f < 2; f++) {
    uint8_t fh[FIELD_HDR];
    memset(fh, 0, sizeof(fh));
    const int bs = BS, radius = 32768;
    memcpy(fh, &bs, 4);
    fh[4] = 0;
    memcpy(fh + 5, &radius, 4);
    // meanInfo<float>{false, 0}: 8 zero bytes; reg_count = 0
    unsigned long long nu = n_unpred[f];
    memcpy(fh + 5 + 4 + 8 + 8, &nu, 8);
    stage(at, fh, FIELD_HDR);
    at += FIELD_HDR;
    unpred_dst[f] = at;
    at += 4 * n_unpred[f];
    std::vector<uint8_t> zeros(ind_bytes, 0);
    stage(at, zeros.data(), ind_bytes);
    at += ind_bytes;
    stage_huff(1 + f);
  }
  if (at != total) return set_error(CPSZ_ERR_INVALID, "internal: blob layout mismatch (%zu != %zu)", at, total);
  // upload the staged small pieces once, then scatter them with D2D copies
  uint8_t* d_small = d.blob + align_up(total, 256);
  if (align_up(total, 256) + small.size() > blob_cap) {
    // fall back: the small pieces go straight from host
    for (const Piece& p : pieces)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(d.blob + p.dst, small.data() + p.src, p.n, cudaMemcpyHostToDevice, st));
  } else {
    CPSZ_CUDA_TRY(cudaMemcpyAsync(d_small, small.data(), small.size(), cudaMemcpyHostToDevice, st));
    for (const Piece& p : pieces)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(d.blob + p.dst, d_small + p.src, p.n, cudaMemcpyDeviceToDevice, st));
  }
  for (int k = 0; k < 3; k++)
    if (bits_bytes[k])
      CPSZ_CUDA_TRY(cudaMemcpyAsync(d.blob + bit_dst[k], d.bits[k], bits_bytes[k], cudaMemcpyDeviceToDevice, st));
  for (int f = 0; f < 2; f++)
    if (n_unpred[f])
      CPSZ_CUDA_TRY(
          cudaMemcpyAsync(d.blob + unpred_dst[f], d.unpred[f], 4 * n_unpred[f], cudaMemcpyDeviceToDevice, st));
  mark(ctx, "end");
  out->d_blob = d.blob;
  out->size = total;
  out->n_unpred[0] = n_unpred[0];
  out->n_unpred[1] = n_unpred[1];
  if (tap) {
    for (int f = 0; f < 2; f++) {
      if (tap->codes_blocks[f])
        CPSZ_CUDA_TRY(cudaMemcpyAsync(tap->codes_blocks[f], d.cblocks[f], 2 * N, cudaMemcpyDeviceToDevice, st));
      if (tap->unpred[f] && n_unpred[f])
        CPSZ_CUDA_TRY(cudaMemcpyAsync(tap->unpred[f], d.unpred[f], 4 * n_unpred[f], cudaMemcpyDeviceToDevice, st));
    }
  }
  // `small` must outlive the async H2D from pageable memory: pageable copies
  // are staged synchronously by the runtime before cudaMemcpyAsync returns.
  return CPSZ_OK;
}

// ---- decompression ---------------------------------------------------------------

namespace {

struct FieldView {
  size_t n_unpred;
  size_t unpred_off;  // from blob start
  HuffDecoderHost huff;
  size_t huff_off;
};

int parse_field(const unsigned char* blob, size_t off, size_t size, size_t N, size_t nblocks, FieldView* fv) {
  if (size < FIELD_HDR) return set_error(CPSZ_ERR_FORMAT, "field blob truncated");
  const unsigned char* p = blob + off;
  int bs, radius;
  memcpy(&bs, p, 4);
  memcpy(&radius, p + 5, 4);
  unsigned char use_mean = p[9];
  unsigned long long reg_count, nu;
  memcpy(&reg_count, p + 17, 8);
  memcpy(&nu, p + 25, 8);
  if (bs != BS || radius != 32768 || use_mean != 0 || reg_count != 0)
    return set_error(CPSZ_ERR_UNSUPPORTED,
                     "field blob parameters (block %d, radius %d, mean %d, regression %llu) are not the offline "
                     "compressor's",
                     bs, radius, (int)use_mean, reg_count);
  if (nu > N || 4 * nu > size - FIELD_HDR) return set_error(CPSZ_ERR_FORMAT, "unpredictable count %llu invalid", nu);
  fv->n_unpred = nu;
  fv->unpred_off = off + FIELD_HDR;
  size_t ind = (nblocks - 1) / 8 + 1;
  size_t hoff = FIELD_HDR + 4 * nu + ind;
  if (hoff > size) return set_error(CPSZ_ERR_FORMAT, "field blob truncated before its Huffman section");
  if (!huff_parse(p + hoff, size - hoff, 65535, &fv->huff)) return CPSZ_ERR_FORMAT;
  fv->huff_off = off + hoff;
  return CPSZ_OK;
}

}  // namespace

int decompress_2d(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1s, size_t r2s, float* U_out,
                  float* V_out) {
  if (!blob || !U_out || !V_out) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  if (r1s == 0 || r2s == 0) return set_error(CPSZ_ERR_INVALID, "empty field");
  if (r1s > (1u << 30) || r2s > (1u << 30) || r1s * r2s > (size_t)INT32_MAX)
    return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu x %zu points exceeds 2^31 points", r1s, r2s);
  if (blob_size < BLOB_HDR) return set_error(CPSZ_ERR_FORMAT, "blob shorter than its header");
  const int r1 = (int)r1s, r2 = (int)r2s;
  const size_t N = r1s * r2s;
  const int nby = (r2 - 1) / BS + 1, nbx = (r1 - 1) / BS + 1;
  const size_t nseg = (size_t)r1 * nby, nblocks = (size_t)nbx * nby;
  const int ngroups = (r1 + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS;
  int base;
  double thr;
  unsigned long long eb_size, u_size, v_size;
  memcpy(&base, blob, 4);
  memcpy(&thr, blob + 4, 8);
  memcpy(&eb_size, blob + 12, 8);
  memcpy(&u_size, blob + 20, 8);
  memcpy(&v_size, blob + 28, 8);
  if (base != 4 || thr != DBL_EPSILON)
    return set_error(CPSZ_ERR_UNSUPPORTED, "blob quantizer (base %d, thr %g) is not the offline compressor's", base, thr);
  const size_t avail = blob_size - BLOB_HDR;
  if (eb_size > avail || u_size > avail - eb_size || v_size > avail - eb_size - u_size)
    return set_error(CPSZ_ERR_FORMAT, "section sizes exceed the blob");
  HuffDecoderHost hid;
  if (!huff_parse(blob + BLOB_HDR, eb_size, 2047, &hid)) return CPSZ_ERR_FORMAT;
  if (hid.section_bytes > eb_size) return set_error(CPSZ_ERR_FORMAT, "id section overruns");
  for (uint32_t s : hid.sym)
    if (s > (uint32_t)ID_MAX_2D)
      return set_error(CPSZ_ERR_UNSUPPORTED, "error-bound id %u beyond the supported range (<= %d)", s, ID_MAX_2D);
  FieldView fv[2];
  CPSZ_TRY(parse_field(blob, BLOB_HDR + eb_size, u_size, N, nblocks, &fv[0]));
  CPSZ_TRY(parse_field(blob, BLOB_HDR + eb_size + u_size, v_size, N, nblocks, &fv[1]));
  const bool dev_out = is_device_ptr(U_out) && is_device_ptr(V_out);

  // ---- workspace ----
  const HuffDecoderHost* hs[3] = {&hid, &fv[0].huff, &fv[1].huff};
  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  if (!dev_out) add(8 * N);
  add(2 * N);  // ids
  for (int k = 0; k < 3; k++) {
    add(hs[k]->nbytes + 64);
    add((1u << HUFF_LUT_BITS) * 4 + hs[k]->child.size() * 4 + hs[k]->sym.size() * 4 + hs[k]->leaf.size());
    add(huff_decode_tmp_bytes(hs[k]->nbytes * 8));
  }
  add(4 * N);  // codes blocks
  add(4 * N);  // codes raster
  add(8 * N);  // (pairs: the raw raster below holds 16 N)
  add(8 * N);  // raw raster
  add(2 * 4 * N);  // unpred lists
  add(2 * 2 * (nseg + 1) * 4);
  add(2 * segment_scan_tmp_bytes(r1, r2));
  add(2 * (size_t)ngroups * r2 * 8);
  add(64);
  add(2 * sizeof(WaveField) + 2 * (size_t)ngroups * sizeof(WaveItem));
  CPSZ_TRY(arena_reserve(ctx, bytes));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  auto A = [&](size_t b) { return arena_alloc(ctx, b); };
  cudaStream_t st = ctx->stream;
  float* dU = dev_out ? U_out : (float*)A(4 * N);
  float* dV = dev_out ? V_out : (float*)A(4 * N);
  uint8_t* ids = (uint8_t*)A(2 * N);
  uint8_t* bits[3];
  HuffDecTable tab[3];
  void* dtmp[3];
  for (int k = 0; k < 3; k++) {
    const HuffDecoderHost& h = *hs[k];
    bits[k] = (uint8_t*)A(h.nbytes + 64);
    size_t tb = (1u << HUFF_LUT_BITS) * 4 + h.child.size() * 4 + h.sym.size() * 4 + h.leaf.size();
    uint8_t* t = (uint8_t*)A(tb);
    dtmp[k] = A(huff_decode_tmp_bytes(h.nbytes * 8));
    const size_t off_bits = (k == 0) ? BLOB_HDR + h.bits_offset : fv[k - 1].huff_off + h.bits_offset;
    CPSZ_CUDA_TRY(cudaMemsetAsync(bits[k], 0, h.nbytes + 64, st));
    if (h.nbytes) CPSZ_CUDA_TRY(cudaMemcpyAsync(bits[k], blob + off_bits, h.nbytes, cudaMemcpyHostToDevice, st));
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
  uint16_t* cblocks[2];
  uint16_t* craster[2];
  float2* raw[2];  // (addend, raw flag) per point; .x holds the raw value where the code is 0
  float* unpred[2];
  unsigned int *seg_cnt[2], *seg_off[2];
  void* scan_tmp[2];
  for (int f = 0; f < 2; f++) {
    cblocks[f] = (uint16_t*)A(2 * N);
    craster[f] = (uint16_t*)A(2 * N);
    raw[f] = (float2*)A(8 * N);
    unpred[f] = (float*)A(4 * fv[f].n_unpred + 4);
    seg_cnt[f] = (unsigned int*)A((nseg + 1) * 4);
    seg_off[f] = (unsigned int*)A((nseg + 1) * 4);
    scan_tmp[f] = A(segment_scan_tmp_bytes(r1, r2));
    if (fv[f].n_unpred)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(unpred[f], blob + fv[f].unpred_off, 4 * fv[f].n_unpred, cudaMemcpyHostToDevice, st));
  }
  unsigned long long* gbnd = (unsigned long long*)A(2 * (size_t)ngroups * r2 * 8);
  int* queue = (int*)A(64);
  WaveField* dfields = (WaveField*)A(2 * sizeof(WaveField));
  WaveItem* ditems = (WaveItem*)A(2 * (size_t)ngroups * sizeof(WaveItem));
  if (!ditems) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  reset_marks(ctx);
  mark(ctx, "huffman_decode");

  // ---- Huffman decode ----
  CPSZ_TRY(launch_huff_decode(ctx, bits[0], hid.nbytes, 2 * N, tab[0], ids, 1, dtmp[0]));
  for (int f = 0; f < 2; f++)
    CPSZ_TRY(launch_huff_decode(ctx, bits[1 + f], fv[f].huff.nbytes, N, tab[1 + f], cblocks[f], 2, dtmp[1 + f]));
  // ---- raster codes, unpredictable scatter ----
  mark(ctx, "raster+scatter");
  unsigned int* h_cnt = (unsigned int*)ctx->pinned + 16;
  for (int f = 0; f < 2; f++) {
    CPSZ_TRY(launch_blocks_to_raster_u16(ctx, cblocks[f], r1, r2, craster[f], r2, ids + (size_t)f * N, raw[f]));
    CPSZ_TRY(launch_segment_scan(ctx, craster[f], r2, r1, r2, seg_cnt[f], seg_off[f], scan_tmp[f]));
    CPSZ_TRY(launch_scatter_unpred(ctx, craster[f], r2, unpred[f], fv[f].n_unpred, r1, r2, seg_off[f], raw[f]));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(h_cnt + f, seg_off[f] + nseg, 4, cudaMemcpyDeviceToHost, st));
  }
  // ---- wavefront ----
  WaveField hf[2];
  for (int f = 0; f < 2; f++) {
    WaveField& F = hf[f];
    F.pair = raw[f];
    F.codes = nullptr;
    F.trace = nullptr;
    F.out = f ? dV : dU;
    F.gbnd = gbnd + (size_t)f * ngroups * r2;
    F.pair_pitch = r2;
    F.code_pitch = r2;
    F.out_pitch = r2;
    F.r1 = r1;
    F.r2 = r2;
  }
  int r1v[2] = {r1, r1};
  std::vector<WaveItem> items;
  int n_items = build_wave_items(2, r1v, items);
  CPSZ_CUDA_TRY(cudaMemcpyAsync(dfields, hf, sizeof(hf), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(ditems, items.data(), n_items * sizeof(WaveItem), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(gbnd, 0, 2 * (size_t)ngroups * r2 * 8, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(queue, 0, 64, st));
  mark(ctx, "wave2d_decompress");
  CPSZ_TRY(launch_wave2d(ctx, true, dfields, ditems, n_items, queue, 0));
  mark(ctx, "d2h");
  if (!dev_out) {
    CPSZ_CUDA_TRY(cudaMemcpyAsync(U_out, dU, 4 * N, cudaMemcpyDeviceToHost, st));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(V_out, dV, 4 * N, cudaMemcpyDeviceToHost, st));
  }
  mark(ctx, "end");
  int flag = 0;
  CPSZ_TRY(read_flag(ctx, &flag));
  if (flag) return flag_error(flag);
  for (int f = 0; f < 2; f++)
    if (h_cnt[f] != fv[f].n_unpred)
      return set_error(CPSZ_ERR_FORMAT, "field %d: %u zero codes but %zu unpredictable values", f, h_cnt[f],
                       fv[f].n_unpred);
  return CPSZ_OK;
}

}  // namespace cpsz
