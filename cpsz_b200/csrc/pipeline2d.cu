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
// Batches (compress_2d_batch) run in passes of up to 32 fields: every stage
// is issued for all fields of the pass, the wavefront is one persistent
// launch over all of them (its work queue interleaves the fields' row
// groups), and the host builds the pass's Huffman trees on all host threads.
// A single-field call is a pass of one field.
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
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

#include "host_pool.h"
#include "huffman_host.h"
#include "kernels.h"
#include "tuning.h"
#include "pipeline.h"
#include "transfer.h"

namespace cpsz {

namespace {

constexpr int BS = 12;
constexpr size_t FIELD_HDR = 4 + 1 + 4 + 8 + 8 + 8;  // up to and including n_unpred
constexpr size_t BLOB_HDR = 4 + 8 + 8 + 8 + 8;
// pinned staging per field: id histogram, two code histograms, unpredictable
// counts, the id codebook's entries
constexpr size_t JOB_PINNED = (256 + 2 * 65536) * 8 + 64 + 256 * sizeof(HuffEntry);
constexpr size_t PINNED_BASE = 4096;  // the flag word and scalars live below
// sub-batch limits: fields per pass (pinned staging) and points per pass (workspace)
constexpr int BATCH_MAX_FIELDS = 32;
constexpr size_t BATCH_MAX_POINTS = (size_t)1 << 27;

struct DevBuf {
  // arena sub-allocations of one field
  float* U;
  float* V;
  uint8_t* ids;  // 2N: U ids then V ids
  unsigned long long* hist_ids;
  uint16_t* craster[2];
  float2* pairs[2];  // per-point (value, 1/precision) pairs read by the wavefront
  uint16_t* cblocks[2];
  unsigned long long* hist_codes[2];
  unsigned long long* gbnd;
  unsigned* gdone;            // per component and row group: the wavefront is done with it; then 2 tickets, gave_up
  unsigned long long* units;  // eb2d progress word, then per-unit counters of finished vertices
  int2* uorder;               // eb2d's unit order (every band's units, band after band)
  void* strip[2];            // strip-pass look-back words and counters
  float* unpred[2];
  unsigned long long* enc_code[3];
  uint8_t* enc_len[3];
  HuffEntry* enc_ent[3];  // codebook entries as uploaded
  void* enc_tmp[3];
  uint32_t* bits[3];
  uint8_t* blob;
  uint8_t* stage;       // the blob's small pieces and their descriptors, as uploaded
  float* logs[2];       // offline_log: log2f |U|, |V| (the unpredictable values it stores)
  uint32_t* signs[2];   // offline_log: sign maps
};

// One field of a compression pass (a pass holds one or more fields).
struct Job2D {
  const float* U_in = nullptr;
  const float* V_in = nullptr;
  int r1 = 0, r2 = 0, ngroups = 0, ncb = 0;
  size_t N = 0, nseg = 0, nblocks = 0;
  double eb = 0;
  const double* eb_ext = nullptr;  // given per-vertex bounds (device), else derived
  bool dev_in = false;
  size_t ids_bits_cap = 0, codes_bits_cap = 0, blob_cap = 0;
  DevBuf d{};
  unsigned long long* h_hist_ids = nullptr;    // pinned
  unsigned long long* h_hist_codes = nullptr;  // pinned, 2 x 65536
  unsigned int* h_nunpred = nullptr;           // pinned, 2
  HuffEntry* h_ids_ent = nullptr;              // pinned, 256
  HuffCodebook cb[3];
  bool tree_ok[3] = {false, false, false};
  size_t n_unpred[2] = {0, 0};
  size_t sec_bytes[3] = {0, 0, 0}, bits_bytes[3] = {0, 0, 0};
  size_t size = 0;  // blob bytes
  // device output: the blob is built in place at blob_base (blob_room bytes
  // there), the caller's buffer when it is a device buffer with room for the
  // blob's bound, else the workspace blob
  unsigned char* dev_out = nullptr;
  size_t dev_cap = 0;
  uint8_t* blob_base = nullptr;
  size_t blob_room = 0;
  // host output: the blob is written straight into host memory (sections
  // copied from their device buffers), not assembled in device memory
  unsigned char* host_out = nullptr;
  size_t host_cap = 0;
  // the offline_log form: base 2, one id stream of N symbols, the two sign
  // maps (device, MSB-first bit streams) between the id section and the fields
  bool log_form = false;
  const uint32_t* d_signs[2] = {nullptr, nullptr};
};

int read_flag(cpsz_b200_ctx* ctx, int* out) {
  CPSZ_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = *(int*)ctx->pinned;
  return CPSZ_OK;
}

// Pinned word receiving the device flag right after the wavefront of a pass
// whose wavefront ran beside the bound kernel.
int* wave_flag_snapshot(cpsz_b200_ctx* ctx) { return (int*)((char*)ctx->pinned + 2048); }
// Pinned word receiving the histogram follower's gave-up flag.
int* follow_flag_snapshot(cpsz_b200_ctx* ctx) { return (int*)((char*)ctx->pinned + 2056); }

int flag_error(int flag) {
  if (flag & FLAG_TIMEOUT) return set_error(CPSZ_ERR_TIMEOUT, "a bounded device-side wait gave up");
  if (flag & FLAG_ID_OVERFLOW)
    return set_error(CPSZ_ERR_UNSUPPORTED, "an error-bound id does not fit the 8-bit id stream (max_pwr_eb too large)");
  if (flag & FLAG_HUFF_CORRUPT) return set_error(CPSZ_ERR_FORMAT, "Huffman stream does not decode");
  if (flag & FLAG_RAW_RANGE) return set_error(CPSZ_ERR_FORMAT, "unpredictable-value list shorter than its codes");
  if (flag & FLAG_OUT_CAPACITY) return set_error(CPSZ_ERR_INVALID, "an output stream exceeded its buffer");
  return CPSZ_OK;
}

// While it lives, the launch wrappers (which all enqueue on ctx->stream) run
// on stream s instead of the context's main stream.
struct OnStream {
  cpsz_b200_ctx* ctx;
  cudaStream_t saved;
  OnStream(cpsz_b200_ctx* c, cudaStream_t s) : ctx(c), saved(c->stream) { c->stream = s; }
  ~OnStream() { ctx->stream = saved; }
};

int job_init(Job2D& j, const float* U, const float* V, size_t r1s, size_t r2s, double eb) {
  if (!U || !V) return set_error(CPSZ_ERR_INVALID, "null input field");
  if (r1s == 0 || r2s == 0) return set_error(CPSZ_ERR_INVALID, "empty field (%zu x %zu)", r1s, r2s);
  if (r1s > (1u << 30) || r2s > (1u << 30) || r1s * r2s > (size_t)INT32_MAX)
    return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu x %zu points exceeds 2^31 points", r1s, r2s);
  if (eb != eb) return set_error(CPSZ_ERR_INVALID, "max_pwr_eb is NaN");
  j.U_in = U;
  j.V_in = V;
  j.r1 = (int)r1s;
  j.r2 = (int)r2s;
  j.N = r1s * r2s;
  j.eb = eb;
  j.ngroups = (j.r1 + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS;
  j.ncb = (j.r2 + UNIT_COLS - 1) / UNIT_COLS;
  const int nby = (j.r2 - 1) / BS + 1, nbx = (j.r1 - 1) / BS + 1;
  j.nseg = (size_t)j.r1 * nby;
  j.nblocks = (size_t)nbx * nby;
  j.dev_in = is_device_ptr(U) && is_device_ptr(V);
  // bit streams: Huffman averages < log2(distinct) + 1 bits per symbol
  j.ids_bits_cap = (2 * j.N * 9 + 7) / 8 + 64;
  j.codes_bits_cap = (j.N * 17 + 7) / 8 + 64;
  j.blob_cap = BLOB_HDR + 2 * FIELD_HDR + 8 * j.N + 2 * ((j.nblocks + 7) / 8) + 2 * (j.N / 8 + 1) +
               3 * (12 + 1 + 13 * 131072 + 8) +
               j.ids_bits_cap + 2 * j.codes_bits_cap + 64;
  return CPSZ_OK;
}

// Bound of the blob's small pieces (header, three trees with their stream
// sizes, field headers, indicators) and their descriptors.
size_t stage_bytes(const Job2D& j) {
  const size_t tree = 12 + 1 + 13 * std::min<size_t>(131072, 2 * j.N + 1) + 8;
  return BLOB_HDR + 2 * FIELD_HDR + 2 * ((j.nblocks + 7) / 8) + (12 + 1 + 13 * 512 + 8) + 2 * tree + 64 + 24 * 32;
}

// Workspace of one field (each piece padded as the arena pads it).
size_t job_bytes(const Job2D& j) {
  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  const size_t N = j.N;
  if (!j.dev_in) add(8 * N);
  add(2 * N);                           // ids
  add(256 * 8);                         // hist ids
  add(4 * N);                           // codes raster
  add(16 * N);                          // wavefront input pairs
  add(4 * N);                           // codes blocks
  add(2 * 65536 * 8);                   // hist codes
  add(2 * (size_t)j.ngroups * j.r2 * 8);  // boundary rows (tagged words)
  add((2 * (size_t)j.ngroups + 4) * 4);   // row-group done flags, follower tickets and flag
  add(((size_t)j.ngroups * j.ncb + 1) * 8);       // eb2d progress word + unit counters
  add((size_t)j.ngroups * j.ncb * sizeof(int2));  // eb2d unit order
  add(2 * strip_scratch_bytes(j.r1, j.r2));
  add(2 * 4 * N);  // unpred
  add(256 * 9);
  add(2 * 65536 * 9);
  add(256 * sizeof(HuffEntry));
  add(std::min<size_t>(65536, N) * sizeof(HuffEntry));
  add(std::min<size_t>(65536, N) * sizeof(HuffEntry));
  add(huff_encode_tmp_bytes(2 * N));
  add(2 * huff_encode_tmp_bytes(N));
  add(j.ids_bits_cap);
  add(2 * j.codes_bits_cap);
  add(j.blob_cap);
  add(stage_bytes(j));
  if (j.log_form) {
    add(2 * 4 * N);                        // log values
    add(2 * 4 * ((N + 31) / 32));          // sign maps
  }
  return bytes;
}

int job_alloc(cpsz_b200_ctx* ctx, Job2D& j) {
  // a request that does not fit fails every later one too (no smaller piece
  // may land behind a failed one): the check of the last piece covers all
  bool failed = false;
  auto A = [&](size_t b) -> void* {
    void* p = failed ? nullptr : arena_alloc(ctx, b);
    failed = failed || !p;
    return p;
  };
  DevBuf& d = j.d;
  const size_t N = j.N;
  if (j.dev_in) {
    d.U = const_cast<float*>(j.U_in);
    d.V = const_cast<float*>(j.V_in);
  } else {
    d.U = (float*)A(4 * N);
    d.V = (float*)A(4 * N);
  }
  d.ids = (uint8_t*)A(2 * N);
  d.hist_ids = (unsigned long long*)A(256 * 8);
  for (int f = 0; f < 2; f++) {
    d.craster[f] = (uint16_t*)A(2 * N);
    d.pairs[f] = (float2*)A(8 * N);
    d.cblocks[f] = (uint16_t*)A(2 * N);
    d.hist_codes[f] = (unsigned long long*)A(65536 * 8);
  }
  d.gbnd = (unsigned long long*)A(2 * (size_t)j.ngroups * j.r2 * 8);
  d.gdone = (unsigned*)A((2 * (size_t)j.ngroups + 4) * 4);
  d.units = (unsigned long long*)A(((size_t)j.ngroups * j.ncb + 1) * 8);
  d.uorder = (int2*)A((size_t)j.ngroups * j.ncb * sizeof(int2));
  for (int f = 0; f < 2; f++) {
    d.strip[f] = A(strip_scratch_bytes(j.r1, j.r2));
    d.unpred[f] = (float*)A(4 * N);
  }
  d.enc_code[0] = (unsigned long long*)A(256 * 8);
  d.enc_len[0] = (uint8_t*)A(256);
  for (int f = 1; f < 3; f++) {
    d.enc_code[f] = (unsigned long long*)A(65536 * 8);
    d.enc_len[f] = (uint8_t*)A(65536);
  }
  d.enc_ent[0] = (HuffEntry*)A(256 * sizeof(HuffEntry));
  d.enc_ent[1] = (HuffEntry*)A(std::min<size_t>(65536, N) * sizeof(HuffEntry));
  d.enc_ent[2] = (HuffEntry*)A(std::min<size_t>(65536, N) * sizeof(HuffEntry));
  d.enc_tmp[0] = A(huff_encode_tmp_bytes(2 * N));
  d.enc_tmp[1] = A(huff_encode_tmp_bytes(N));
  d.enc_tmp[2] = A(huff_encode_tmp_bytes(N));
  d.bits[0] = (uint32_t*)A(j.ids_bits_cap);
  d.bits[1] = (uint32_t*)A(j.codes_bits_cap);
  d.bits[2] = (uint32_t*)A(j.codes_bits_cap);
  d.blob = (uint8_t*)A(j.blob_cap);
  d.stage = (uint8_t*)A(stage_bytes(j));
  if (!d.stage) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
  if (j.dev_out && j.dev_cap >= j.blob_cap + 8) {
    j.blob_base = j.dev_out;
    j.blob_room = j.dev_cap;
  } else {
    j.blob_base = d.blob;
    j.blob_room = align_up(j.blob_cap, 256);
  }
  if (j.log_form) {
    d.logs[0] = (float*)A(4 * N);
    d.logs[1] = (float*)A(4 * N);
    d.signs[0] = (uint32_t*)A(4 * ((N + 31) / 32));
    d.signs[1] = (uint32_t*)A(4 * ((N + 31) / 32));
    if (!d.signs[1]) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
    j.d_signs[0] = d.signs[0];
    j.d_signs[1] = d.signs[1];
  }
  return CPSZ_OK;
}

// Blob assembly of one field in device memory (header, id tree, two field
// blobs); the small host-made pieces go up in one copy and are scattered
// with device-to-device copies.
// The reference's 2D blob (sz_compress_cp_preserve_2d_offline,
// src/sz_compress_cp_preserve_2d.cpp): header, the id stream's Huffman
// section, then per component its header, unpredictable floats, the all-zero
// block indicator and the code stream's Huffman section.  Every small piece is
// staged in `small`; the bit streams and unpredictable floats go to bit_dst /
// unpred_dst.
struct BlobLayout {
  // bytes [dst, dst + n) of the blob: from small[src] (ext null), from ext
  // (host memory that outlives the pass: a code tree), or zeros (zero)
  struct Piece {
    size_t dst, src, n;
    const uint8_t* ext;
    bool zero;
  };
  size_t total = 0, bit_dst[3] = {0, 0, 0}, unpred_dst[2] = {0, 0}, sign_dst = 0, sign_bytes = 0;
  std::vector<uint8_t> small;
  std::vector<Piece> pieces;
};

// offset of the id stream's bits (known once the id tree is)
size_t ids_bits_at(const Job2D& j) { return BLOB_HDR + j.cb[0].tree_bytes.size() + 8; }

int job_layout(const Job2D& j, BlobLayout& L) {
  const size_t ind_bytes = (j.nblocks + 7) / 8;
  size_t field_size[2];
  for (int f = 0; f < 2; f++) field_size[f] = FIELD_HDR + 4 * j.n_unpred[f] + ind_bytes + j.sec_bytes[1 + f];
  const size_t sign_bytes = j.log_form ? (j.N - 1) / 8 + 1 : 0;
  const size_t total = BLOB_HDR + j.sec_bytes[0] + 2 * sign_bytes + field_size[0] + field_size[1];
  L.total = total;
  L.sign_bytes = sign_bytes;
  std::vector<uint8_t>& small = L.small;
  small.reserve(BLOB_HDR + j.cb[0].tree_bytes.size() + 3 * 8 + 2 * FIELD_HDR);
  auto stage = [&](size_t dst, const void* p, size_t n) {
    L.pieces.push_back(BlobLayout::Piece{dst, small.size(), n, nullptr, false});
    small.insert(small.end(), (const uint8_t*)p, (const uint8_t*)p + n);
  };
  // the code trees and the zero indicator bytes are referenced, not copied:
  // the layout precedes the code packing, their bytes go up after it
  auto refer = [&](size_t dst, const uint8_t* p, size_t n) {
    L.pieces.push_back(BlobLayout::Piece{dst, 0, n, p, p == nullptr});
  };
  {
    uint8_t hdr[BLOB_HDR];
    const int base = j.log_form ? 2 : 4;
    const double thr = DBL_EPSILON;
    memcpy(hdr, &base, 4);
    memcpy(hdr + 4, &thr, 8);
    memcpy(hdr + 12, &j.sec_bytes[0], 8);
    memcpy(hdr + 20, &field_size[0], 8);
    memcpy(hdr + 28, &field_size[1], 8);
    stage(0, hdr, BLOB_HDR);
  }
  size_t at = BLOB_HDR;
  size_t* bit_dst = L.bit_dst;
  size_t* unpred_dst = L.unpred_dst;
  auto stage_huff = [&](int k) {
    if (k == 0) stage(at, j.cb[k].tree_bytes.data(), j.cb[k].tree_bytes.size());
    else refer(at, j.cb[k].tree_bytes.data(), j.cb[k].tree_bytes.size());
    at += j.cb[k].tree_bytes.size();
    unsigned long long nb = j.bits_bytes[k];
    stage(at, &nb, 8);
    at += 8;
    bit_dst[k] = at;
    at += j.bits_bytes[k];
  };
  stage_huff(0);
  L.sign_dst = at;  // offline_log: sign maps of U and V (copied from the device)
  at += 2 * sign_bytes;
  for (int f = 0; f < 2; f++) {
    uint8_t fh[FIELD_HDR];
    memset(fh, 0, sizeof(fh));
    const int bs = BS, radius = 32768;
    memcpy(fh, &bs, 4);
    memcpy(fh + 5, &radius, 4);
    // meanInfo<float>{false, 0}: 8 zero bytes; reg_count = 0
    unsigned long long nu = j.n_unpred[f];
    memcpy(fh + 5 + 4 + 8 + 8, &nu, 8);
    stage(at, fh, FIELD_HDR);
    at += FIELD_HDR;
    unpred_dst[f] = at;
    at += 4 * j.n_unpred[f];
    refer(at, nullptr, ind_bytes);
    at += ind_bytes;
    stage_huff(1 + f);
  }
  if (at != total) return set_error(CPSZ_ERR_INVALID, "internal: blob layout mismatch (%zu != %zu)", at, total);
  return CPSZ_OK;
}

// The small pieces of a blob in one launch: CTA (x, y) copies bytes
// [x * 4096, (x + 1) * 4096) of piece y from the staged bytes (byte stores:
// the bytes around a piece belong to other sections, some written before it).
constexpr int PIECE_CHUNK = 4096;
__global__ void __launch_bounds__(256) pieces_kernel(const uint8_t* __restrict__ small,
                                                     const unsigned long long* __restrict__ desc,
                                                     uint8_t* __restrict__ blob) {
  const unsigned long long dst = desc[3 * blockIdx.y], src = desc[3 * blockIdx.y + 1], n = desc[3 * blockIdx.y + 2];
  const unsigned long long c0 = (unsigned long long)blockIdx.x * PIECE_CHUNK;
  const unsigned long long c1 = n < c0 + PIECE_CHUNK ? n : c0 + PIECE_CHUNK;
  if (src == ~0ull) {  // a run of zeros
    for (unsigned long long i = c0 + threadIdx.x; i < c1; i += 256) blob[dst + i] = 0;
    return;
  }
  for (unsigned long long i = c0 + threadIdx.x; i < c1; i += 256) blob[dst + i] = small[src + i];
}

// Bytes job_assemble uploads: the small pieces and the referenced ones, then
// their descriptors.
size_t assemble_payload_bytes(const BlobLayout& L) {
  size_t n = L.small.size();
  for (const BlobLayout::Piece& pc : L.pieces)
    if (pc.ext) n += pc.n;
  return align_up(n, 8);
}
size_t assemble_upload_bytes(const BlobLayout& L) { return assemble_payload_bytes(L) + 24 * L.pieces.size(); }

// The sections of a device blob that the packers do not write: the staged
// small pieces (header, trees, stream sizes, field headers, indicators), the
// unpredictable values and the sign maps.  h_up: page-locked staging of
// assemble_upload_bytes(L), which must stay untouched until the pass ends.
int job_assemble(cpsz_b200_ctx* ctx, Job2D& j, const BlobLayout& L, uint8_t* h_up) {
  cudaStream_t st = ctx->stream;
  uint8_t* blob = j.blob_base;
  // pieces and their descriptors go up in one copy
  const size_t up_size = assemble_upload_bytes(L), payload = assemble_payload_bytes(L);
  memcpy(h_up, L.small.data(), L.small.size());
  size_t ext_at = L.small.size();
  unsigned long long* desc = (unsigned long long*)(h_up + payload);
  for (size_t i = 0; i < L.pieces.size(); i++) {
    const BlobLayout::Piece& pc = L.pieces[i];
    size_t src = pc.src;
    if (pc.ext) {
      memcpy(h_up + ext_at, pc.ext, pc.n);
      src = ext_at;
      ext_at += pc.n;
    }
    desc[3 * i] = pc.dst;
    desc[3 * i + 1] = pc.zero ? ~0ull : src;
    desc[3 * i + 2] = pc.n;
  }
  if (up_size > stage_bytes(j)) return set_error(CPSZ_ERR_INVALID, "internal: blob pieces exceed their bound");
  uint8_t* d_up = j.d.stage;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d_up, h_up, up_size, cudaMemcpyHostToDevice, st));
  if (!L.pieces.empty()) {
    size_t longest = 0;
    for (const BlobLayout::Piece& pc : L.pieces) longest = std::max(longest, pc.n);
    const dim3 grid((unsigned)std::max<size_t>(1, (longest + PIECE_CHUNK - 1) / PIECE_CHUNK), (unsigned)L.pieces.size());
    pieces_kernel<<<grid, 256, 0, st>>>(d_up, (const unsigned long long*)(d_up + payload), blob);
    count_launch(ctx);
    CPSZ_TRY(check_launch("pieces_kernel"));
  }
  for (int f = 0; f < 2; f++)
    if (j.n_unpred[f])
      CPSZ_CUDA_TRY(
          cudaMemcpyAsync(blob + L.unpred_dst[f], j.d.unpred[f], 4 * j.n_unpred[f], cudaMemcpyDeviceToDevice, st));
  for (int f = 0; f < 2 && L.sign_bytes; f++)
    CPSZ_CUDA_TRY(cudaMemcpyAsync(blob + L.sign_dst + f * L.sign_bytes, j.d_signs[f], L.sign_bytes,
                                  cudaMemcpyDeviceToDevice, st));
  j.size = L.total;
  return CPSZ_OK;
}

// One compression pass over `jobs` (workspace reserved by the caller).
int run_pass(cpsz_b200_ctx* ctx, std::vector<Job2D>& jobs, const StageTap* tap) {
  cudaStream_t st = ctx->stream;
  const int nj = (int)jobs.size();
  // the offline_log form runs as a pass of one field
  const bool log_form = nj == 1 && jobs[0].log_form;
  const QuantTable& qt = log_form ? quant_table_2d_log() : quant_table_2d();
  LibmTables libm{};
  if (log_form) CPSZ_TRY(libm_tables_device(ctx, &libm));
  // pass-wide device pieces
  double* thr_tab = (double*)arena_alloc(ctx, QUANT_TAB_MAX * 8);
  int* queue = (int*)arena_alloc(ctx, 64);
  WaveField* d_fields = (WaveField*)arena_alloc(ctx, 2 * nj * sizeof(WaveField));
  int total_groups = 0;
  for (const Job2D& j : jobs) total_groups += j.ngroups;
  WaveItem* d_items = (WaveItem*)arena_alloc(ctx, 2 * (size_t)total_groups * sizeof(WaveItem));
  Eb2dJob* d_ebjobs = (Eb2dJob*)arena_alloc(ctx, nj * sizeof(Eb2dJob));
  if (!d_items || !d_ebjobs) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
  for (Job2D& j : jobs) CPSZ_TRY(job_alloc(ctx, j));
  for (int k = 0; k < nj; k++) {
    uint8_t* base = (uint8_t*)ctx->pinned + PINNED_BASE + (size_t)k * JOB_PINNED;
    jobs[k].h_hist_ids = (unsigned long long*)base;
    jobs[k].h_hist_codes = jobs[k].h_hist_ids + 256;
    jobs[k].h_nunpred = (unsigned int*)(jobs[k].h_hist_codes + 2 * 65536);
    jobs[k].h_ids_ent = (HuffEntry*)(base + (256 + 2 * 65536) * 8 + 64);
  }

  // Derived bounds (eb2d) signal per 128-row group, so for one field the
  // wavefront runs beside them on the high-priority stream and starts on a
  // group as soon as its pairs are written: its items (group-major over the
  // two components) come in the order eb2d finishes them.  A batch's items
  // are group-major across fields while eb2d finishes field after field, so a
  // batch (and given bounds, quant2d, which are not row-ordered) runs the
  // wavefront after the bounds with every CTA slot.
  const bool overlap =
      nj == 1 && jobs[0].eb_ext == nullptr && !log_form && tune_get(TUNE_WAVE2D_OVERLAP, jobs[0].N) != 0;
  // Host input is uploaded and bounded in bands of band_rows(j) rows (a
  // multiple of WAVE_GROUP_ROWS), band c right after its upload.
  auto band_rows = [&](const Job2D& j) -> int {
    const int K = (!j.dev_in && j.N >= ((size_t)1 << 22) && !j.eb_ext) ? tune_get(TUNE_H2D_CHUNKS, j.N) : 1;
    return (int)align_up((size_t)(j.r1 + K - 1) / K, WAVE_GROUP_ROWS);
  };

  // ---- setup: flags, tables, wavefront descriptors ----
  reset_marks(ctx);
  mark(ctx, "h2d+setup");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(thr_tab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice, st));
  for (Job2D& j : jobs) CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.hist_ids, 0, 256 * 8, st));
  std::vector<WaveField> hf(2 * nj);
  std::vector<int> r1v(2 * nj);
  // a pass that quantizes again only some vertices starts the recursion at
  // their first row group: the groups above (and their boundary rows, which
  // the first group run reads) are the previous pass's
  const int g0 = (nj == 1 && tap && tap->recon_only && tap->requant && jobs[0].eb_ext)
                     ? std::min(std::max(tap->first_group, 0), jobs[0].ngroups)
                     : 0;
  // One large field beside its bounds: the code histograms are counted while
  // the wavefront's tail runs (hist_follow on the second stream), as its row
  // groups finish, instead of after it (below 2^22 points the histograms take
  // a few microseconds and the follower's own launch and waits cost more).
  const bool follow = overlap && nj == 1 && !tap && jobs[0].N >= ((size_t)1 << 22);
  for (int k = 0; k < nj; k++) {
    Job2D& j = jobs[k];
    if (follow) CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.gdone, 0, (2 * (size_t)j.ngroups + 4) * 4, st));
    for (int f = 0; f < 2; f++) {
      CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.gbnd + ((size_t)f * j.ngroups + g0) * j.r2, 0,
                                    (size_t)(j.ngroups - g0) * j.r2 * 8, st));
      CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.hist_codes[f], 0, 65536 * 8, st));  // stage 3's histograms
    }
    if (overlap) {
      // eb2d's unit counters and its unit order, band by band (units along
      // diagonals of slope eb2d.skew column blocks per group)
      CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.units, 0, ((size_t)j.ngroups * j.ncb + 1) * 8, st));
      const int R = band_rows(j), skew = tune_get(TUNE_EB2D_SKEW, j.N);
      std::vector<int2> order, part;
      for (int r0 = 0; r0 < j.r1; r0 += R) {
        unit_order(r0 / WAVE_GROUP_ROWS, (std::min(j.r1, r0 + R) + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS, j.ncb, skew,
                   part);
        order.insert(order.end(), part.begin(), part.end());
      }
      // through the page-locked upload staging (no copy from it is in flight
      // yet; the pass's later uploads reuse it after this copy has run)
      CPSZ_TRY(upload_reserve(ctx, order.size() * sizeof(int2)));
      memcpy(ctx->up_pinned, order.data(), order.size() * sizeof(int2));
      CPSZ_CUDA_TRY(
          cudaMemcpyAsync(j.d.uorder, ctx->up_pinned, order.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    }
    for (int f = 0; f < 2; f++) {
      WaveField& F = hf[2 * k + f];
      F.pair = j.d.pairs[f];
      F.codes = j.d.craster[f];
      F.trace = (nj == 1 && ctx->d_wave_trace && ctx->wave_trace_len >= 2 * (size_t)j.ngroups * WAVE_WARPS * 4)
                    ? ctx->d_wave_trace + (size_t)f * j.ngroups * WAVE_WARPS * 4
                    : nullptr;
      F.out = tap ? tap->recon[f] : nullptr;
      F.gbnd = j.d.gbnd + (size_t)f * j.ngroups * j.r2;
      F.pair_pitch = j.r2;
      F.code_pitch = j.r2;
      F.out_pitch = j.r2;
      F.r1 = j.r1;
      F.r2 = j.r2;
      F.unit_done = overlap ? j.d.units + 1 : nullptr;
      F.unit_ncb = j.ncb;
      F.band_wait_ns = ctx->band_wait_ns;
      F.band_extra = ctx->band_unreachable ? 1 : 0;
      F.group_done = follow ? j.d.gdone + (size_t)f * j.ngroups : nullptr;
      r1v[2 * k + f] = j.r1;
    }
  }
  std::vector<WaveItem> items;
  build_wave_items(2 * nj, r1v.data(), items);
  if (g0 > 0) items.erase(std::remove_if(items.begin(), items.end(), [&](const WaveItem& w) { return w.group < g0; }),
                          items.end());
  const int n_items = (int)items.size();
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d_fields, hf.data(), hf.size() * sizeof(WaveField), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), n_items * sizeof(WaveItem), cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(queue, 0, 64, st));
  // A batch of device-resident fields derives its bounds in one bound-kernel
  // launch: every field's tiles in one grid (largest field first, so the
  // small fields' tiles fill the launch's tail), each CTA finding its field in
  // a descriptor table, instead of a launch per field that leaves the SMs
  // idle while a small field's few tiles run.
  bool eb_batched = nj > 1;
  for (const Job2D& j : jobs)
    eb_batched = eb_batched && j.dev_in && !j.eb_ext && !j.log_form && j.eb >= 0 && j.eb <= 1e300;
  int eb_shape = 0, eb_tiles = 0;
  if (eb_batched) {
    size_t largest = 0;
    for (const Job2D& j : jobs) largest = std::max(largest, j.N);
    eb_shape = tune_get(TUNE_EB2D_TILE, largest);
    int tx, ty;
    eb2d_tile_shape(eb_shape, &tx, &ty);
    std::vector<int> by_size(nj);
    for (int k = 0; k < nj; k++) by_size[k] = k;
    std::stable_sort(by_size.begin(), by_size.end(), [&](int a, int b) { return jobs[a].N > jobs[b].N; });
    std::vector<Eb2dJob> ebj;
    for (int k : by_size) {
      const Job2D& j = jobs[k];
      Eb2dJob e;
      e.U = j.d.U;
      e.V = j.d.V;
      e.ids_u = j.d.ids;
      e.ids_v = j.d.ids + j.N;
      e.hist = j.d.hist_ids;
      e.pair_u = j.d.pairs[0];
      e.pair_v = j.d.pairs[1];
      e.max_pwr_eb = j.eb;
      e.r1 = j.r1;
      e.r2 = j.r2;
      e.tiles_x = (j.r2 + tx - 1) / tx;
      e.tile0 = eb_tiles;
      const size_t t = (size_t)e.tiles_x * ((j.r1 + ty - 1) / ty);
      if (eb_tiles + t > (size_t)INT32_MAX) {
        eb_batched = false;  // beyond one grid's tile count: a launch per field
        break;
      }
      eb_tiles += (int)t;
      ebj.push_back(e);
    }
    if (eb_batched)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(d_ebjobs, ebj.data(), nj * sizeof(Eb2dJob), cudaMemcpyHostToDevice, st));
  }
  size_t pass_points = 0;
  for (const Job2D& j : jobs) pass_points += j.N;
  // a wavefront launched beside its producer must be finished before this
  // call returns on any path (its workspace is reused by the next call)
  struct HiDrain {
    cudaStream_t s = nullptr;
    ~HiDrain() {
      if (s) cudaStreamSynchronize(s);
    }
  } hi_drain, follow_drain;
  if (overlap) {
    // The wavefront (high-priority stream, one CTA per SM) is launched before
    // its producer eb2d (stage 1), whose CTAs then fill the rest of every SM:
    // measured at 8192^2, this order takes 7.87 ms a compression against
    // 8.7-9.5 ms with eb2d enqueued first (eb2d itself runs slower behind a
    // late wavefront, which then trails it).  The order is not relied on: a
    // wavefront wait gives up once eb2d shows no progress for a while (a tool
    // that serialises kernels runs the wavefront alone first), and the pass
    // then runs its wavefront again after the bounds (see the code trees
    // below), so serialised execution costs that wait, not a failure.
    CPSZ_TRY(preload_eb2d());
    CPSZ_TRY(preload_wave2d());
    hi_drain.s = ctx->hi;
    CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[3], st));
    CPSZ_CUDA_TRY(cudaStreamWaitEvent(ctx->hi, ctx->ev[3], 0));
    CPSZ_TRY(launch_wave2d(ctx, false, d_fields, d_items, n_items, queue, pass_points, ctx->hi, WAVE_BESIDE));
    CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[4], ctx->hi));
  }

  // Stages 1-3 (bounds, wavefront, code histograms, block order) are the
  // pass's device work before the host builds the code trees.  A batch whose
  // fields are all in device memory captures them once into a CUDA graph,
  // kept on the context and replayed while the pass is the same (fields,
  // shapes, bounds, workspace, tuning table); events the host waits on are
  // recorded as external events of the graph.
  bool all_dev_in = true;
  for (const Job2D& j : jobs) all_dev_in = all_dev_in && j.dev_in;
  bool capturing = false;
  auto record = [&](cudaEvent_t e) {
    return capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
  };
  auto stages_1_2 = [&]() -> int {
    // ---- stage 1: inputs and error bounds ----
    mark(ctx, "eb2d");
    // host-input uploads run on the second stream, after the pass's setup (once
    // per pass: per field it would hold each upload behind the previous field's
    // bound kernels)
    if (!all_dev_in) {
      CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[2], st));
      CPSZ_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->ev[2], 0));
    }
    if (eb_batched)
      CPSZ_TRY(launch_eb2d_batch(ctx, d_ebjobs, nj, eb_tiles, eb_shape, thr_tab, qt.n, qt.float_pow4));
    for (Job2D& j : jobs) {
      // beside the wavefront, eb2d runs unit by unit in the order made in the
      // setup; band_units(g0, g1) is the slice for the rows of groups [g0, g1)
      auto band_units = [&](int g0, int g1) {
        Eb2dUnits u;
        u.order = j.d.uorder + (size_t)g0 * j.ncb;
        u.n = (g1 - g0) * j.ncb;
        u.ncb = j.ncb;
        u.done = j.d.units + 1;  // [-1]: tiles finished
        return u;
      };
      if (j.log_form) {
        // offline_log: the fields whole, one id per vertex, then the logs,
        // wavefront pairs and sign maps
        if (!j.dev_in) {
          CPSZ_TRY(h2d(ctx, j.d.U, j.U_in, 4 * j.N, st));
          CPSZ_TRY(h2d(ctx, j.d.V, j.V_in, 4 * j.N, st));
        }
        CPSZ_TRY(launch_eb2d(ctx, j.d.U, j.d.V, j.r1, j.r2, j.eb, thr_tab, qt.n, j.d.ids, nullptr, j.d.hist_ids,
                             nullptr, nullptr, nullptr, 0, -1, nullptr, true));
        CPSZ_TRY(launch_log2d(ctx, j.d.U, j.d.V, j.d.ids, j.N, libm.log2f, j.d.pairs[0], j.d.pairs[1], j.d.logs[0],
                              j.d.logs[1], j.d.signs[0], j.d.signs[1]));
      } else if (j.dev_in) {
        if (j.eb_ext && nj == 1 && tap && tap->recon_only && tap->requant)
          CPSZ_TRY(launch_requant2d(ctx, j.d.U, j.d.V, j.N, j.eb_ext, thr_tab, qt.n, j.d.ids, j.d.ids + j.N,
                                    j.d.pairs[0], j.d.pairs[1], tap->requant));
        else if (j.eb_ext)
          CPSZ_TRY(launch_quant2d(ctx, j.d.U, j.d.V, j.N, j.eb_ext, thr_tab, qt.n, j.d.ids, j.d.ids + j.N,
                                  j.d.hist_ids, j.d.pairs[0], j.d.pairs[1]));
        else if (!eb_batched) {
          const Eb2dUnits u = band_units(0, j.ngroups);
          CPSZ_TRY(launch_eb2d(ctx, j.d.U, j.d.V, j.r1, j.r2, j.eb, thr_tab, qt.n, j.d.ids, j.d.ids + j.N,
                               j.d.hist_ids, j.d.pairs[0], j.d.pairs[1], nullptr, 0, -1, overlap ? &u : nullptr,
                               false, qt.float_pow4));
        }
      } else {
        // Host input: row chunks go up on the second stream and the bound kernel
        // runs band by band as soon as a band's rows and the row below it are
        // on the device, so the transfer overlaps the bound derivation.  Bands
        // start on wavefront group boundaries.  Chunk c carries its band's rows
        // and the next band's first row (which chunk c + 1 writes again, with
        // the same bytes), so band c waits for chunk c alone and only the last
        // band's bounds follow the end of the transfer.
        const int R = band_rows(j);
        const int nch = (j.r1 + R - 1) / R;
        // band c is enqueued right after chunk c's copy call (a copy from
        // pageable memory returns only once the host has staged it, so
        // enqueueing every copy first would hold the bands back until the whole
        // field was staged)
        auto band_launch = [&](int c) -> int {
          CPSZ_CUDA_TRY(cudaStreamWaitEvent(st, ctx->up_ev[c], 0));
          if (j.eb_ext)
            return launch_quant2d(ctx, j.d.U, j.d.V, j.N, j.eb_ext, thr_tab, qt.n, j.d.ids, j.d.ids + j.N,
                                  j.d.hist_ids, j.d.pairs[0], j.d.pairs[1]);
          const Eb2dUnits u = band_units(c * R / WAVE_GROUP_ROWS, (std::min(j.r1, (c + 1) * R) + WAVE_GROUP_ROWS - 1) /
                                                                     WAVE_GROUP_ROWS);
          return launch_eb2d(ctx, j.d.U, j.d.V, j.r1, j.r2, j.eb, thr_tab, qt.n, j.d.ids, j.d.ids + j.N, j.d.hist_ids,
                             j.d.pairs[0], j.d.pairs[1], nullptr, c * R, std::min(j.r1, (c + 1) * R),
                             overlap ? &u : nullptr, false, qt.float_pow4);
        };
        for (int c = 0; c < nch; c++) {
          const size_t off = (size_t)c * R * j.r2;
          const size_t cnt = (size_t)(std::min(j.r1, (c + 1) * R + 1) - c * R) * j.r2;
          CPSZ_CUDA_TRY(cudaMemcpyAsync(j.d.U + off, j.U_in + off, 4 * cnt, cudaMemcpyHostToDevice, ctx->aux));
          CPSZ_CUDA_TRY(cudaMemcpyAsync(j.d.V + off, j.V_in + off, 4 * cnt, cudaMemcpyHostToDevice, ctx->aux));
          CPSZ_CUDA_TRY(cudaEventRecord(ctx->up_ev[c], ctx->aux));
          CPSZ_TRY(band_launch(c));
        }
      }
      CPSZ_CUDA_TRY(cudaMemcpyAsync(j.h_hist_ids, j.d.hist_ids, 256 * 8, cudaMemcpyDeviceToHost, st));
    }
    CPSZ_CUDA_TRY(record(ctx->ev[0]));
    if (follow) {
      // the code histograms, counted on the second stream as the wavefront
      // finishes its row groups; the flag and the histograms come back there
      Job2D& j = jobs[0];
      follow_drain.s = ctx->aux;
      CPSZ_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->ev[0], 0));
      const uint16_t* codes[2] = {j.d.craster[0], j.d.craster[1]};
      const unsigned* gd[2] = {j.d.gdone, j.d.gdone + j.ngroups};
      unsigned long long* hc[2] = {j.d.hist_codes[0], j.d.hist_codes[1]};
      unsigned* tix = j.d.gdone + 2 * (size_t)j.ngroups;
      CPSZ_TRY(launch_hist_follow(ctx, codes, gd, j.r1, j.r2, hc, tix, (int*)(tix + 2), ctx->aux));
      CPSZ_CUDA_TRY(
          cudaMemcpyAsync(follow_flag_snapshot(ctx), tix + 2, sizeof(int), cudaMemcpyDeviceToHost, ctx->aux));
      for (int f = 0; f < 2; f++) {
        CPSZ_CUDA_TRY(cudaMemcpyAsync(j.h_hist_codes + (size_t)f * 65536, j.d.hist_codes[f], 65536 * 8,
                                      cudaMemcpyDeviceToHost, ctx->aux));
        CPSZ_CUDA_TRY(cudaEventRecord(ctx->job_ev[f], ctx->aux));
      }
    }
    if (tap && tap->ids)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(tap->ids, jobs[0].d.ids, 2 * jobs[0].N, cudaMemcpyDeviceToDevice, st));

    // ---- stage 2: one persistent wavefront over every field of the pass ----
    mark(ctx, "wave2d_compress");
    if (overlap) {
      // the bounds are done: the rest of each SM joins the running wavefront
      CPSZ_TRY(launch_wave2d(ctx, false, d_fields, d_items, n_items, queue, pass_points, st, WAVE_JOIN));
      CPSZ_CUDA_TRY(cudaStreamWaitEvent(st, ctx->ev[4], 0));
      // the flag as the wavefront left it, read by the host once the code
      // histograms (enqueued after it) have arrived
      CPSZ_CUDA_TRY(cudaMemcpyAsync(wave_flag_snapshot(ctx), ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
      CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));
    } else {
      CPSZ_TRY(launch_wave2d(ctx, false, d_fields, d_items, n_items, queue, pass_points));
    }
    return CPSZ_OK;
  };
  auto count_codes = [&]() -> int {
    for (int k = 0; k < nj; k++) {
      Job2D& j = jobs[k];
      CPSZ_TRY(launch_hist_u16_pair(ctx, j.d.craster[0], j.d.craster[1], j.N, j.d.hist_codes[0], j.d.hist_codes[1]));
      for (int f = 0; f < 2; f++) {
        CPSZ_CUDA_TRY(cudaMemcpyAsync(j.h_hist_codes + (size_t)f * 65536, j.d.hist_codes[f], 65536 * 8,
                                      cudaMemcpyDeviceToHost, st));
        CPSZ_CUDA_TRY(record(ctx->job_ev[2 * k + f]));
      }
    }
    return CPSZ_OK;
  };
  bool hist_in_stage3 = !follow;
  auto stage_3 = [&]() -> int {
    mark(ctx, "blocks+hist+unpred");

    // ---- stage 3: code histograms first (the host builds the code trees from
    // them while the GPU converts to block order and gathers unpredictables);
    // a single field beside its bounds has them from the follower ----
    if (hist_in_stage3) CPSZ_TRY(count_codes());
    for (int k = 0; k < nj; k++) {
      Job2D& j = jobs[k];
      const float* x[2] = {j.log_form ? j.d.logs[0] : j.d.U, j.log_form ? j.d.logs[1] : j.d.V};
      CPSZ_TRY(launch_strip_pass(ctx, j.d.craster, j.r2, x, j.r2, j.r1, j.r2, j.d.cblocks, j.d.unpred, j.d.strip));
      for (int f = 0; f < 2; f++)
        CPSZ_CUDA_TRY(cudaMemcpyAsync(j.h_nunpred + f, strip_total(j.d.strip[f], j.r1, j.r2), 4,
                                      cudaMemcpyDeviceToHost, st));
    }
    CPSZ_CUDA_TRY(record(ctx->ev[5]));  // the unpredictable counts are on the host
    return CPSZ_OK;
  };
  const bool use_graph = nj > 1 && all_dev_in && !tap && !ctx->timing && !overlap;
  bool done = false;
  if (use_graph) {
    std::vector<uint64_t> key = {(uint64_t)nj, (uint64_t)(uintptr_t)ctx->arena.base, (uint64_t)(uintptr_t)ctx->pinned,
                                 tune_generation()};
    for (const Job2D& j : jobs) {
      uint64_t ebits;
      memcpy(&ebits, &j.eb, 8);
      key.insert(key.end(), {(uint64_t)(uintptr_t)j.U_in, (uint64_t)(uintptr_t)j.V_in, (uint64_t)j.r1,
                             (uint64_t)j.r2, ebits});
    }
    auto& cache = ctx->pass_graphs;
    auto hit = std::find_if(cache.begin(), cache.end(), [&](const cpsz_b200_ctx::PassGraph& g) { return g.key == key; });
    if (hit != cache.end()) {
      std::rotate(hit, hit + 1, cache.end());  // most recently used last
      CPSZ_CUDA_TRY(cudaGraphLaunch(cache.back().exec, st));
      count_launch(ctx, cache.back().launches);
      ctx->graph_replays++;
      done = true;
    } else {
      if (cache.size() >= cpsz_b200_ctx::kMaxPassGraphs) {
        cudaGraphExecDestroy(cache.front().exec);
        cache.erase(cache.begin());
      }
      const uint64_t launches0 = ctx->launches;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        capturing = true;
        int rc = stages_1_2();
        if (rc == CPSZ_OK) rc = stage_3();
        capturing = false;
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &graph);
        cudaGraphExec_t exec = nullptr;
        if (rc == CPSZ_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
          cache.push_back(cpsz_b200_ctx::PassGraph{key, exec, (int)(ctx->launches - launches0)});
          done = cudaGraphLaunch(exec, st) == cudaSuccess;
          ctx->graph_captures += done;
        }
        if (graph) cudaGraphDestroy(graph);
      }
      if (!done) {
        // capture unavailable or failed: the same work, launched directly
        cudaGetLastError();
        clear_error();
        ctx->launches = launches0;
      }
    }
  }
  if (!done) {
    CPSZ_TRY(stages_1_2());
    if (tap && tap->recon_only) {
      int flag = 0;
      CPSZ_TRY(read_flag(ctx, &flag));
      return flag ? flag_error(flag) : CPSZ_OK;
    }
    CPSZ_TRY(stage_3());
  }
  mark(ctx, "host_trees");
  // Host output (one field): the sections are copied from their device
  // buffers straight into the caller's memory, each right after its producer
  // when that memory is page-locked (the copies then overlap the rest), else
  // once everything is done; no blob is assembled in device memory.
  Job2D* hj = (nj == 1 && jobs[0].host_out) ? &jobs[0] : nullptr;
  const bool h_async = hj && host_kind(hj->host_out) == HOST_PINNED;
  // Page-locked output: each section's copy runs on the aux stream behind its
  // producer, so the next producer does not wait for it.  The main stream
  // joins aux before the pass ends; on an early return the guard drains aux, so
  // no copy out of the workspace outlives the call.
  struct AuxDrain {
    cudaStream_t s = nullptr;
    ~AuxDrain() {
      if (s) cudaStreamSynchronize(s);
    }
  } aux_drain;
  auto d2h_beside = [&](void* dst, const void* src, size_t n) -> int {
    CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[6], st));
    CPSZ_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->ev[6], 0));
    aux_drain.s = ctx->aux;
    return d2h(ctx, dst, src, n, ctx->aux);
  };
  // Bit packing of stream k (0: ids, 1-2: codes of U / V).  A device blob gets
  // the bits in place, at byte `at` (the sections around it are written later
  // byte by byte, and the packer ORs only zero bits into their bytes); host
  // output packs into a buffer of the stream's own that is copied out.
  auto pack = [&](Job2D& j, int k, size_t at, HuffEntry* h_stage) -> int {
    uint8_t* dst = j.host_out ? (uint8_t*)j.d.bits[k] : j.blob_base + at;
    const size_t room = j.host_out ? (k ? j.codes_bits_cap : j.ids_bits_cap) : j.blob_room - at;
    const size_t mis = (uintptr_t)dst & 3;
    CPSZ_CUDA_TRY(cudaMemsetAsync(dst, 0, j.bits_bytes[k], ctx->stream));
    CPSZ_TRY(huff_upload(ctx, j.cb[k], h_stage, j.d.enc_ent[k], j.d.enc_code[k], j.d.enc_len[k]));
    const HuffEncTable tab{j.d.enc_code[k], j.d.enc_len[k], k ? 65536 : 256};
    uint32_t* w = (uint32_t*)(dst - mis);
    if (k == 0)
      return launch_huff_encode_u8(ctx, j.d.ids, j.log_form ? j.N : 2 * j.N, true, tab, w, room + mis, nullptr,
                                   j.d.enc_tmp[0], (int)(8 * mis));
    return launch_huff_encode_u16(ctx, j.d.cblocks[k - 1], j.N, tab, w, room + mis, nullptr, j.d.enc_tmp[k],
                                  (int)(8 * mis));
  };

  // host: the id trees (their histograms arrive with the bounds), and their
  // bit packing on the aux stream as soon as the bounds are done: it runs
  // beside the wavefront's tail, which leaves most SMs idle, and the main
  // stream joins aux before the blob is finished
  auto tree_failure = [&]() {
    int fl = 0;
    CPSZ_TRY(read_flag(ctx, &fl));
    if (fl) return flag_error(fl);
    return set_error(CPSZ_ERR_UNSUPPORTED, "Huffman tree construction failed (code longer than 64 bits)");
  };
  CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[0]));
  host_parallel_for(nj, [&](int k) { jobs[k].tree_ok[0] = huff_build(jobs[k].h_hist_ids, 256, 2048, &jobs[k].cb[0]); });
  CPSZ_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->ev[0], 0));
  aux_drain.s = ctx->aux;
  for (Job2D& j : jobs) {
    if (!j.tree_ok[0]) return tree_failure();
    j.sec_bytes[0] = huff_section_bytes(j.cb[0]);
    j.bits_bytes[0] = (j.cb[0].total_bits + 7) / 8;
    if (j.bits_bytes[0] + 8 > j.ids_bits_cap) return set_error(CPSZ_ERR_UNSUPPORTED, "Huffman stream larger than its bound");
    OnStream on_aux(ctx, ctx->aux);
    CPSZ_TRY(pack(j, 0, ids_bits_at(j), j.h_ids_ent));
  }
  if (h_async) {
    const size_t at = ids_bits_at(*hj);
    if (at + hj->bits_bytes[0] > hj->host_cap)
      return set_error(CPSZ_ERR_INVALID, "output capacity %zu too small for the blob", hj->host_cap);
    CPSZ_TRY(d2h(ctx, hj->host_out + at, hj->d.bits[0], hj->bits_bytes[0], ctx->aux));
  }
  // code trees, each as soon as its histogram is on the host
  auto code_trees = [&]() {
    host_parallel_for(2 * nj, [&](int q) {
      Job2D& j = jobs[q / 2];
      const int f = q % 2;
      j.tree_ok[1 + f] = cudaSetDevice(ctx->device) == cudaSuccess && cudaEventSynchronize(ctx->job_ev[q]) == cudaSuccess &&
                         huff_build(j.h_hist_codes + (size_t)f * 65536, 65536, 131072, &j.cb[1 + f]);
    });
  };
  if (follow) {
    // the follower's histograms; one that gave up (its wavefront was not
    // running beside it) leaves them to be counted here
    CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->job_ev[1]));
    if (*(volatile int*)follow_flag_snapshot(ctx)) {
      for (int f = 0; f < 2; f++) CPSZ_CUDA_TRY(cudaMemsetAsync(jobs[0].d.hist_codes[f], 0, 65536 * 8, st));
      CPSZ_TRY(count_codes());
    }
  }
  code_trees();
  if (overlap) {
    // The histograms are on the host, so is the flag snapshot taken before
    // them.  A wavefront wait that gave up (the bound kernel was held back
    // for seconds: a saturated or time-sliced device) left codes from
    // incomplete inputs; the bounds are complete now, so the wavefront and
    // everything after it runs again, after the bounds, and the pass goes on.
    // The id stream's packing, already enqueued, depends on the bounds only.
    CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[1]));
    const int snap = *(volatile int*)wave_flag_snapshot(ctx);
    if (snap & FLAG_TIMEOUT) {
      if (snap != FLAG_TIMEOUT) return flag_error(snap);
      CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
      for (WaveField& F : hf) {
        F.unit_done = nullptr;
        F.group_done = nullptr;
      }
      CPSZ_CUDA_TRY(cudaMemcpyAsync(d_fields, hf.data(), hf.size() * sizeof(WaveField), cudaMemcpyHostToDevice, st));
      for (Job2D& j : jobs) {
        CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.gbnd, 0, 2 * (size_t)j.ngroups * j.r2 * 8, st));
        for (int f = 0; f < 2; f++) CPSZ_CUDA_TRY(cudaMemsetAsync(j.d.hist_codes[f], 0, 65536 * 8, st));
      }
      CPSZ_CUDA_TRY(cudaMemsetAsync(queue, 0, 64, st));
      CPSZ_TRY(launch_wave2d(ctx, false, d_fields, d_items, n_items, queue, pass_points));
      hist_in_stage3 = true;
      CPSZ_TRY(stage_3());
      code_trees();
      ctx->wave_reruns++;
    }
  }

  // ---- stage 4: blob layout (every section size is known once the
  // unpredictable counts are on the host) and bit packing of the codes ----
  mark(ctx, "huffman_encode");
  for (Job2D& j : jobs) {
    if (!j.tree_ok[1] || !j.tree_ok[2]) return tree_failure();
    for (int k = 1; k < 3; k++) {
      j.sec_bytes[k] = huff_section_bytes(j.cb[k]);
      j.bits_bytes[k] = (j.cb[k].total_bits + 7) / 8;
      if (j.bits_bytes[k] + 8 > j.codes_bits_cap)
        return set_error(CPSZ_ERR_UNSUPPORTED, "Huffman stream larger than its bound");
    }
  }
  CPSZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[5]));
  std::vector<BlobLayout> lay(nj);
  for (int q = 0; q < nj; q++) {
    Job2D& j = jobs[q];
    j.n_unpred[0] = j.h_nunpred[0];
    j.n_unpred[1] = j.h_nunpred[1];
    CPSZ_TRY(job_layout(j, lay[q]));
    if (j.host_out) {
      if (lay[q].total > j.host_cap)
        return set_error(CPSZ_ERR_INVALID, "output capacity %zu < blob size %zu", j.host_cap, lay[q].total);
    } else if (lay[q].total > j.blob_cap) {
      return set_error(CPSZ_ERR_UNSUPPORTED, "blob larger than its bound");
    }
  }
  // page-locked staging of the pass's remaining uploads: code entries, and
  // the device blobs' small pieces (no copy from it is in flight here)
  // (each piece taken at a 16-byte boundary, as counted here)
  size_t up_bytes = 0;
  for (int q = 0; q < nj; q++)
    up_bytes += align_up(jobs[q].cb[1].entries.size() * sizeof(HuffEntry), 16) +
                align_up(jobs[q].cb[2].entries.size() * sizeof(HuffEntry), 16) +
                (jobs[q].host_out ? 0 : align_up(assemble_upload_bytes(lay[q]), 16));
  CPSZ_TRY(upload_reserve(ctx, up_bytes));
  uint8_t* up_at = (uint8_t*)ctx->up_pinned;
  uint8_t* const up_end = up_at + up_bytes;
  auto up_take = [&](size_t n) -> uint8_t* {
    uint8_t* p = up_at;
    up_at += align_up(n, 16);
    return up_at <= up_end ? p : nullptr;
  };
  if (hj) {
    const BlobLayout& hl = lay[0];
    for (const BlobLayout::Piece& pc : hl.pieces) {
      if (pc.zero) memset(hj->host_out + pc.dst, 0, pc.n);
      else memcpy(hj->host_out + pc.dst, pc.ext ? pc.ext : hl.small.data() + pc.src, pc.n);
    }
    if (h_async)
      for (int f = 0; f < 2; f++) {
        CPSZ_TRY(d2h_beside(hj->host_out + hl.unpred_dst[f], hj->d.unpred[f], 4 * hj->n_unpred[f]));
        if (hl.sign_bytes)
          CPSZ_TRY(d2h_beside(hj->host_out + hl.sign_dst + f * hl.sign_bytes, hj->d_signs[f], hl.sign_bytes));
      }
  }
  for (int q = 0; q < nj; q++) {
    Job2D& j = jobs[q];
    for (int k = 1; k < 3; k++) {
      HuffEntry* h_stage = (HuffEntry*)up_take(j.cb[k].entries.size() * sizeof(HuffEntry));
      if (!h_stage) return set_error(CPSZ_ERR_INVALID, "internal: upload staging overrun");
      CPSZ_TRY(pack(j, k, lay[q].bit_dst[k], h_stage));
      if (h_async) CPSZ_TRY(d2h_beside(j.host_out + lay[q].bit_dst[k], j.d.bits[k], j.bits_bytes[k]));
    }
  }
  if (aux_drain.s) {  // the aux stream's work (id packing, section copies) joins the main stream
    CPSZ_CUDA_TRY(cudaEventRecord(ctx->ev[7], ctx->aux));
    CPSZ_CUDA_TRY(cudaStreamWaitEvent(st, ctx->ev[7], 0));
  }
  // ---- stage 5: the rest of a device blob (header, trees, unpredictable
  // values, sign maps), enqueued behind the packers, or, for host output
  // without page-locked memory, the sections not yet copied ----
  mark(ctx, "blob_assembly");
  int assembled = CPSZ_OK;
  if (!hj)
    for (int q = 0; q < nj; q++) {
      uint8_t* h_up = up_take(assemble_upload_bytes(lay[q]));
      if (!h_up) {
        assembled = set_error(CPSZ_ERR_INVALID, "internal: upload staging overrun");
        break;
      }
      if ((assembled = job_assemble(ctx, jobs[q], lay[q], h_up)) != CPSZ_OK) break;
    }
  {
    int flag = 0;
    CPSZ_TRY(read_flag(ctx, &flag));  // synchronizes the stream; a kernel's error outranks the assembly's
    if (flag) return flag_error(flag);
  }
  if (assembled != CPSZ_OK) return assembled;
  if (hj) {
    const BlobLayout& hl = lay[0];
    if (!h_async) {
      CPSZ_TRY(d2h(ctx, hj->host_out + hl.bit_dst[0], hj->d.bits[0], hj->bits_bytes[0], st));
      for (int f = 0; f < 2; f++) {
        CPSZ_TRY(d2h(ctx, hj->host_out + hl.unpred_dst[f], hj->d.unpred[f], 4 * hj->n_unpred[f], st));
        if (hl.sign_bytes)
          CPSZ_TRY(d2h(ctx, hj->host_out + hl.sign_dst + f * hl.sign_bytes, hj->d_signs[f], hl.sign_bytes, st));
      }
      for (int k = 1; k < 3; k++) CPSZ_TRY(d2h(ctx, hj->host_out + hl.bit_dst[k], hj->d.bits[k], hj->bits_bytes[k], st));
    }
    hj->size = hl.total;
  }
  mark(ctx, "end");
  if (tap) {
    Job2D& j = jobs[0];
    for (int f = 0; f < 2; f++) {
      if (tap->codes_blocks[f])
        CPSZ_CUDA_TRY(cudaMemcpyAsync(tap->codes_blocks[f], j.d.cblocks[f], 2 * j.N, cudaMemcpyDeviceToDevice, st));
      if (tap->unpred[f] && j.n_unpred[f])
        CPSZ_CUDA_TRY(
            cudaMemcpyAsync(tap->unpred[f], j.d.unpred[f], 4 * j.n_unpred[f], cudaMemcpyDeviceToDevice, st));
    }
  }
  return CPSZ_OK;
}

size_t pass_bytes(const std::vector<Job2D>& jobs) {
  size_t bytes = 0;
  int total_groups = 0;
  for (const Job2D& j : jobs) {
    bytes += job_bytes(j);
    total_groups += j.ngroups;
  }
  bytes += align_up(QUANT_TAB_MAX * 8, 256) + 256 + 512 + align_up(2 * jobs.size() * sizeof(WaveField), 256) + 256 +
           align_up(2 * (size_t)total_groups * sizeof(WaveItem), 256) + 256 + align_up(jobs.size() * sizeof(Eb2dJob), 256) +
           256;
  return bytes;
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
                Blob2D* out, const StageTap* tap, const double* eb_ext, unsigned char* host_out, size_t host_cap,
                bool log_form) {
  if (log_form && (tap || eb_ext))
    return set_error(CPSZ_ERR_INVALID, "the offline_log form takes neither stage taps nor given bounds");
  std::vector<Job2D> jobs(1);
  CPSZ_TRY(job_init(jobs[0], U_in, V_in, r1s, r2s, max_pwr_eb));
  jobs[0].log_form = log_form;
  jobs[0].eb_ext = eb_ext;
  if (host_out && host_kind(host_out) == HOST_DEVICE) {
    jobs[0].dev_out = host_out;
    jobs[0].dev_cap = host_cap;
  } else {
    jobs[0].host_out = host_out;
    jobs[0].host_cap = host_cap;
  }
  CPSZ_TRY(arena_reserve(ctx, pass_bytes(jobs)));
  CPSZ_TRY(pinned_reserve(ctx, PINNED_BASE + JOB_PINNED));
  CPSZ_TRY(run_pass(ctx, jobs, tap));
  out->d_blob = jobs[0].host_out ? nullptr : jobs[0].blob_base;
  out->size = jobs[0].size;
  out->n_unpred[0] = jobs[0].n_unpred[0];
  out->n_unpred[1] = jobs[0].n_unpred[1];
  return CPSZ_OK;
}

int compress_2d_batch(cpsz_b200_ctx* ctx, int n, const float* const* U, const float* const* V, const size_t* r1,
                      const size_t* r2, const double* ebs, unsigned char* out, size_t out_cap, size_t* offsets) {
  if (n < 0 || (n > 0 && (!U || !V || !r1 || !r2 || !ebs))) return set_error(CPSZ_ERR_INVALID, "null batch argument");
  if (!out || !offsets) return set_error(CPSZ_ERR_INVALID, "null output");
  const bool dev_out = is_device_ptr(out);
  size_t at = 0;
  int k0 = 0;
  offsets[0] = 0;
  while (k0 < n) {
    // greedy pass: up to BATCH_MAX_FIELDS fields and BATCH_MAX_POINTS points (a larger field goes alone)
    std::vector<Job2D> jobs;
    size_t pts = 0;
    int k = k0;
    while (k < n && (int)jobs.size() < BATCH_MAX_FIELDS) {
      Job2D j;
      CPSZ_TRY(job_init(j, U[k], V[k], r1[k], r2[k], ebs[k]));
      if (!jobs.empty() && pts + j.N > BATCH_MAX_POINTS) break;
      pts += j.N;
      jobs.push_back(std::move(j));
      k++;
    }
    CPSZ_TRY(arena_reserve(ctx, pass_bytes(jobs)));
    CPSZ_TRY(pinned_reserve(ctx, PINNED_BASE + jobs.size() * JOB_PINNED));
    CPSZ_TRY(run_pass(ctx, jobs, nullptr));
    for (size_t q = 0; q < jobs.size(); q++) {
      const Job2D& j = jobs[q];
      if (at + j.size > out_cap)
        return set_error(CPSZ_ERR_INVALID, "output capacity %zu < %zu bytes of blobs", out_cap, at + j.size);
      CPSZ_TRY(d2h(ctx, out + at, j.blob_base, j.size, ctx->stream));
      at += j.size;
      offsets[k0 + q + 1] = at;
    }
    // the next pass reuses the workspace
    CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    k0 = k;
  }
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
                  float* V_out, bool log_form) {
  if (!blob || !U_out || !V_out) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  if (r1s == 0 || r2s == 0) return set_error(CPSZ_ERR_INVALID, "empty field");
  if (r1s > (1u << 30) || r2s > (1u << 30) || r1s * r2s > (size_t)INT32_MAX)
    return set_error(CPSZ_ERR_UNSUPPORTED, "field of %zu x %zu points exceeds 2^31 points", r1s, r2s);
  if (blob_size < BLOB_HDR) return set_error(CPSZ_ERR_FORMAT, "blob shorter than its header");
  const int r1 = (int)r1s, r2 = (int)r2s;
  const size_t N = r1s * r2s;
  const int nby = (r2 - 1) / BS + 1, nbx = (r1 - 1) / BS + 1;
  const size_t nblocks = (size_t)nbx * nby;
  const int ngroups = (r1 + WAVE_GROUP_ROWS - 1) / WAVE_GROUP_ROWS;
  int base;
  double thr;
  unsigned long long eb_size, u_size, v_size;
  memcpy(&base, blob, 4);
  memcpy(&thr, blob + 4, 8);
  memcpy(&eb_size, blob + 12, 8);
  memcpy(&u_size, blob + 20, 8);
  memcpy(&v_size, blob + 28, 8);
  if (base != (log_form ? 2 : 4) || thr != DBL_EPSILON)
    return set_error(CPSZ_ERR_UNSUPPORTED, "blob quantizer (base %d, thr %g) is not the offline%s compressor's", base,
                     thr, log_form ? "_log" : "");
  // offline_log: the sign maps of U and V follow the id section
  const size_t sign_bytes = log_form ? (N - 1) / 8 + 1 : 0;
  const size_t avail = blob_size - BLOB_HDR;
  if (eb_size > avail || 2 * sign_bytes > avail - eb_size || u_size > avail - eb_size - 2 * sign_bytes ||
      v_size > avail - eb_size - 2 * sign_bytes - u_size)
    return set_error(CPSZ_ERR_FORMAT, "section sizes exceed the blob");
  const size_t fields_at = BLOB_HDR + eb_size + 2 * sign_bytes;
  const size_t n_ids = log_form ? N : 2 * N;
  HuffDecoderHost hid;
  if (!huff_parse(blob + BLOB_HDR, eb_size, 2047, &hid)) return CPSZ_ERR_FORMAT;
  if (hid.section_bytes > eb_size) return set_error(CPSZ_ERR_FORMAT, "id section overruns");
  for (uint32_t s : hid.sym)
    if (s > (uint32_t)ID_MAX_2D)
      return set_error(CPSZ_ERR_UNSUPPORTED, "error-bound id %u beyond the supported range (<= %d)", s, ID_MAX_2D);
  FieldView fv[2];
  CPSZ_TRY(parse_field(blob, fields_at, u_size, N, nblocks, &fv[0]));
  CPSZ_TRY(parse_field(blob, fields_at + u_size, v_size, N, nblocks, &fv[1]));
  LibmTables libm{};
  if (log_form) CPSZ_TRY(libm_tables_device(ctx, &libm));
  const bool dev_out = is_device_ptr(U_out) && is_device_ptr(V_out);

  // ---- workspace ----
  const HuffDecoderHost* hs[3] = {&hid, &fv[0].huff, &fv[1].huff};
  size_t bytes = 0;
  auto add = [&](size_t b) { bytes += align_up(b, 256) + 256; };
  if (!dev_out) add(8 * N);
  add(n_ids);  // ids
  add(2 * sign_bytes + 16);
  for (int k = 0; k < 3; k++) {
    add(hs[k]->nbytes + 64);
    add((1u << HUFF_LUT_BITS) * 4 + hs[k]->child.size() * 4 + hs[k]->sym.size() * 4 + hs[k]->leaf.size());
    add(huff_decode_tmp_bytes(hs[k]->nbytes * 8));
  }
  add(4 * N);  // codes blocks
  add(8 * N);  // (pairs: the raw raster below holds 16 N)
  add(8 * N);  // raw raster
  add(2 * 4 * N);  // unpred lists
  add(2 * strip_scratch_bytes(r1, r2));
  add(2 * (size_t)ngroups * r2 * 8);
  add(64);
  add(2 * sizeof(WaveField) + 2 * (size_t)ngroups * sizeof(WaveItem));
  CPSZ_TRY(arena_reserve(ctx, bytes));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  auto A = [&](size_t b) { return arena_alloc(ctx, b); };
  cudaStream_t st = ctx->stream;
  float* dU = dev_out ? U_out : (float*)A(4 * N);
  float* dV = dev_out ? V_out : (float*)A(4 * N);
  uint8_t* ids = (uint8_t*)A(n_ids);
  uint8_t* signs = (uint8_t*)A(2 * sign_bytes + 16);
  if (sign_bytes) CPSZ_TRY(h2d(ctx, signs, blob + BLOB_HDR + eb_size, 2 * sign_bytes, st));
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
    if (h.nbytes) CPSZ_TRY(h2d(ctx, bits[k], blob + off_bits, h.nbytes, st));
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
  float2* raw[2];  // (addend, raw flag) per point; .x holds the raw value where the code is 0
  float* unpred[2];
  void* strip[2];
  for (int f = 0; f < 2; f++) {
    cblocks[f] = (uint16_t*)A(2 * N);
    raw[f] = (float2*)A(8 * N);
    unpred[f] = (float*)A(4 * fv[f].n_unpred + 4);
    strip[f] = A(strip_scratch_bytes(r1, r2));
    if (fv[f].n_unpred)
      CPSZ_TRY(h2d(ctx, unpred[f], blob + fv[f].unpred_off, 4 * fv[f].n_unpred, st));
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
  CPSZ_TRY(launch_huff_decode(ctx, bits[0], hid.nbytes, n_ids, tab[0], ids, 1, dtmp[0]));
  for (int f = 0; f < 2; f++)
    CPSZ_TRY(launch_huff_decode(ctx, bits[1 + f], fv[f].huff.nbytes, N, tab[1 + f], cblocks[f], 2, dtmp[1 + f]));
  // ---- raster pairs, unpredictable scatter ----
  mark(ctx, "raster+scatter");
  unsigned int* h_cnt = (unsigned int*)ctx->pinned + 16;
  {
    const uint16_t* cb[2] = {cblocks[0], cblocks[1]};
    // offline_log: one id stream for both components, base 2
    const uint8_t* idf[2] = {ids, log_form ? ids : ids + N};
    const float* un[2] = {unpred[0], unpred[1]};
    const unsigned long long nun[2] = {fv[0].n_unpred, fv[1].n_unpred};
    CPSZ_TRY(launch_strip_unpass(ctx, cb, idf, un, nun, r1, r2, raw, strip, log_form ? 1 : 2));
    for (int f = 0; f < 2; f++)
      CPSZ_CUDA_TRY(cudaMemcpyAsync(h_cnt + f, strip_total(strip[f], r1, r2), 4, cudaMemcpyDeviceToHost, st));
  }
  // ---- wavefront ----
  WaveField hf[2] = {};
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
  CPSZ_TRY(launch_wave2d(ctx, true, dfields, ditems, n_items, queue, (size_t)r1 * r2));
  if (log_form) {
    mark(ctx, "exp2d");
    CPSZ_TRY(launch_exp2d(ctx, dU, dV, signs, signs + sign_bytes, N, libm.exp2f));
  }
  mark(ctx, "d2h");
  if (!dev_out) {
    CPSZ_TRY(d2h(ctx, U_out, dU, 4 * N, st));
    CPSZ_TRY(d2h(ctx, V_out, dV, 4 * N, st));
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
