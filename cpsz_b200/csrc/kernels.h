// kernels.h -- launch wrappers of the device kernels (all on ctx->stream).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "libm.h"
#include "runtime.h"

namespace cpsz {

constexpr int QUANT_TAB_MAX = QuantTable::kMax;
// Byte code of a vertex whose quantized bound is zero (precision 0, Huffman symbol 0).
constexpr uint8_t ID_ZERO = 255;
// Largest supported 2D id: precision 4^id * 2^-52 and its inverse stay normal
// floats (id 88 is a bound of 2^124, far beyond any relative bound <= 1).
constexpr int ID_MAX_2D = 88;

// Device error flag bits (ctx->d_flag[0]).
constexpr int FLAG_ID_OVERFLOW = 1;   // an error-bound id does not fit in a byte
constexpr int FLAG_TIMEOUT = 2;       // a bounded inter-CTA wait gave up
constexpr int FLAG_HUFF_CORRUPT = 4;  // a Huffman stream does not decode to the expected symbols
constexpr int FLAG_RAW_RANGE = 8;     // an unpredictable-value index fell outside the stored list
constexpr int FLAG_OUT_CAPACITY = 16; // an output stream did not fit its buffer

// ---- 2D error bounds ---------------------------------------------------------
// The bound kernel beside the wavefront runs unit by unit: a unit is a
// (WAVE_GROUP_ROWS-row group, UNIT_COLS-column block) of vertices, and the
// units go in `order` (host-made by unit_order), so that the wavefront, which
// waits per unit, meets its inputs along its own diagonal.  Every tile adds
// the vertices it finished to its unit's counter after its outputs are
// visible device-wide; done[-1] counts finished tiles, the waiting
// wavefront's sign that the kernel is running.
constexpr int UNIT_COLS = 256;
struct Eb2dUnits {
  const int2* order = nullptr;         // device: the launch's units, (group, column block)
  int n = 0;                           // units in order
  int ncb = 0;                         // column blocks per group: ceil(r2 / UNIT_COLS)
  unsigned long long* done = nullptr;  // device: one counter per unit (group * ncb + block), zeroed
};
// One field of a batched bound-kernel launch (launch_eb2d_batch): its
// inputs and outputs as launch_eb2d takes them, and its tiles' place in the
// launch (tiles tile0 .. tile0 + tiles of the grid, tiles_x per tile row).
struct Eb2dJob {
  const float* U;
  const float* V;
  uint8_t* ids_u;
  uint8_t* ids_v;
  unsigned long long* hist;
  float2* pair_u;
  float2* pair_v;
  double max_pwr_eb;
  int r1, r2;
  int tile0, tiles_x;
};
// Tile shape (TX, TY) of the batched launch for a launch-shape table value.
void eb2d_tile_shape(int shape, int* tx, int* ty);
// The filtered bounds of several fields in one launch: jobs (device, n,
// ascending tile0, every max_pwr_eb in [0, 1e300]) with their tiles laid
// out for `shape` (eb2d_tile_shape); tiles = the launch's tile count.
int launch_eb2d_batch(cpsz_b200_ctx* ctx, const Eb2dJob* jobs, int n, int tiles, int shape, const double* d_thr_tab,
                      int thr_n, bool pow4_ids);
// The units of groups [g0, g1) in production order: unit (g, b) before
// (g', b') when b * skew + g is smaller (ties: lower group first); skew 0 is
// row order.
void unit_order(int g0, int g1, int ncb, int skew, std::vector<int2>& out);

// Rows [row_begin, row_end) of the vertex outputs (row_end < 0: all rows); the
// kernel reads rows row_begin - 1 .. row_end of U and V.  With `units`
// (row_begin a multiple of WAVE_GROUP_ROWS; the order holds exactly the
// units of the rows' groups), the tiles run in unit order and count.
// log_ids: the offline_log form -- one id per vertex, of the vertex bound
// itself against quant_table_2d_log() (ids_v, pair_u and pair_v null).
// pow4_ids: the table is quant_table_2d() with float_pow4 (the filtered path
// then decides most ids in float).
int launch_eb2d(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, double max_pwr_eb,
                const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, unsigned long long* hist,
                float2* pair_u, float2* pair_v, double* eb_out = nullptr, int row_begin = 0, int row_end = -1,
                const Eb2dUnits* units = nullptr, bool log_ids = false, bool pow4_ids = false);

// Loads every eb2d instantiation (required before a consumer that waits on
// eb2d is launched: a lazily loaded first launch could wait for it).
int preload_eb2d();

// The same quantization for given per-vertex bounds eb_in[n] (learned bounds).
int launch_quant2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t n, const double* eb_in,
                   const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, unsigned long long* hist,
                   float2* pair_u, float2* pair_v);
// launch_quant2d for the vertices whose mask byte is set (clearing it), into
// ids / pairs that hold every other vertex's values already; no histogram.
int launch_requant2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t n, const double* eb_in,
                     const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, float2* pair_u,
                     float2* pair_v, uint8_t* mask);

// ---- 2D Lorenzo wavefront ------------------------------------------------------
// One field of the wavefront.  Raster arrays carry their own row pitch (elements).
struct WaveField {
  // per-point input pair: compress (value, bits of 1/precision; NaN for
  // precision 0), decompress (addend 2(code-32768)*p or the raw value, raw flag)
  const float2* pair;
  uint16_t* codes;     // compress: quantization codes out (raster)
  float* out;          // compress: reconstruction (optional tap); decompress: decoded field
  // last row of every WAVE_GROUP_ROWS-row group, ngroups * r2 tagged words
  // ((column + 1) << 32 | float bits); zeroed before every launch
  unsigned long long* gbnd;
  long long pair_pitch, code_pitch, out_pitch;
  int r1, r2;
  // optional diagnostics: per (group, warp) 4 counters {start clock, end clock,
  // spins waiting for the row above, spins waiting for ring credit}
  long long* trace;
  // optional: per-unit counters of input points written by a concurrently
  // running producer (launch_eb2d's units.done, unit_done[-1] its finished
  // tiles, unit_ncb column blocks per group); a window of the recurrence
  // starts once the counters of the units it reads reach their vertex counts
  // + band_extra.  A wait gives up (FLAG_TIMEOUT) once the producer has shown
  // no progress for band_wait_ns (0: the default).  band_extra is 0 except in
  // the test that makes the wait run out on purpose.
  const unsigned long long* unit_done;
  int unit_ncb;
  long long band_wait_ns;
  unsigned long long band_extra;
  // optional (compression): per row group, set to 1 once the group's codes
  // are stored (the histogram follower's signal); zeroed before the launch
  unsigned* group_done;
};
struct WaveItem {
  int field;
  int group;
};
constexpr int WAVE_WARPS = 4;
constexpr int WAVE_GROUP_ROWS = WAVE_WARPS * 32;
// Items must be ordered so that (field, g-1) precedes (field, g).  `points`
// (all fields of the launch together) keys the launch-shape table.  The launch
// goes to `stream` (default: the context's stream).  Modes:
//   WAVE_ALONE   the only wavefront launch on the queue: the tuned CTAs per SM;
//   WAVE_BESIDE  runs beside its producer (fields with unit_done): one CTA per
//                SM, which leaves every SM room for the producer's CTAs, so
//                the producer always progresses while wavefront CTAs wait;
//   WAVE_JOIN    launched once the producer is done, while a WAVE_BESIDE launch
//                on the same queue still runs: the remaining CTAs per SM pull
//                from the shared queue (no launch when none remain).
// Every dequeued item belongs to a resident CTA, whichever launch it is in, so
// the waits between items of one field end in every mode.
enum WaveMode { WAVE_ALONE = 0, WAVE_BESIDE = 1, WAVE_JOIN = 2 };
// Loads every wavefront kernel (call before a WAVE_BESIDE launch).
int preload_wave2d();
int launch_wave2d(cpsz_b200_ctx* ctx, bool decompress, const WaveField* d_fields, const WaveItem* d_items,
                  int n_items, int* d_queue, size_t points, cudaStream_t stream = nullptr, int mode = WAVE_ALONE);

// ---- block-order plumbing (12 x 12 blocks) ---------------------------------------
// Both directions run as one pass over strips (a 12-row block row cut into
// runs of 32 blocks), one launch for both components of a field, with a
// decoupled look-back for the unpredictable values' offsets.
// scratch[f]: strip_scratch_bytes(r1, r2) bytes (zeroed by the launch); after
// it, *strip_total(scratch[f], ...) holds the component's number of zero codes.
size_t strip_count(int r1, int r2);
size_t strip_scratch_bytes(int r1, int r2);
const unsigned int* strip_total(const void* scratch, int r1, int r2);
// Compression: codes raster -> 12x12-block order, and the values x at zero
// codes (unpredictable) into unpred[f] in block order.
int launch_strip_pass(cpsz_b200_ctx* ctx, const uint16_t* const raster[2], long long pitch, const float* const x[2],
                      long long x_pitch, int r1, int r2, uint16_t* const blocks[2], float* const unpred[2],
                      void* const scratch[2]);
// Decompression: block-order codes -> per raster point (pitch r2) the pair the
// wavefront reads: (addend 2(code - 32768) * 4^id * 2^-52 (0 for id 0), raw
// flag bits 0), or for code 0 (raw value, raw flag bits 1), the raw values
// taken from unpred[f] in block order (an index past n_unpred[f] raises
// FLAG_RAW_RANGE).
// id_shift: 2 for the offline ids (p = 4^id * 2^-52), 1 for the offline_log
// ids (p = 2^id * 2^-52).
int launch_strip_unpass(cpsz_b200_ctx* ctx, const uint16_t* const blocks[2], const uint8_t* const ids[2],
                        const float* const unpred[2], const unsigned long long n_unpred[2], int r1, int r2,
                        float2* const pair[2], void* const scratch[2], int id_shift = 2);

// ---- 2D offline_log (log2d.cu) ------------------------------------------------------
// Compression: per vertex the host library's log2f of |U| and |V| (-100 for 0)
// as wavefront pairs (log, 1/precision = 2^(52 - id), NaN for ID_ZERO) and as
// plain arrays, and the sign maps (value > 0, MSB-first bit streams;
// ceil(n / 32) words each).
int launch_log2d(cpsz_b200_ctx* ctx, const float* U, const float* V, const uint8_t* ids, size_t n, const LibmFn& L,
                 float2* pair_u, float2* pair_v, float* log_u, float* log_v, uint32_t* sign_u, uint32_t* sign_v);
// Decompression, in place: decoded logs below -99 -> 0, others -> +-exp2f(log)
// with the stored sign (the host library's exp2f).
int launch_exp2d(cpsz_b200_ctx* ctx, float* U, float* V, const uint8_t* sign_u, const uint8_t* sign_v, size_t n,
                 const LibmFn& Ex);

// ---- Huffman -------------------------------------------------------------------
// One codebook entry of a symbol that occurs (code right-aligned, bit len-1 = first bit).
struct HuffEntry {
  unsigned long long code;
  uint32_t sym;
  uint32_t len;
};
// Device codebook tables from n entries: code[e.sym] = e.code, len[e.sym] =
// e.len.  Entries of symbols not in the list keep what the tables held: the
// packer looks up only symbols that occur.
int launch_codebook_scatter(cpsz_b200_ctx* ctx, const HuffEntry* d_entries, size_t n, unsigned long long* code,
                            uint8_t* len);
// Codebook for the encoder: per symbol, code right-aligned (bit len-1 = first bit).
struct HuffEncTable {
  const unsigned long long* code;
  const uint8_t* len;
  int nsym;
};
// Symbols: u8 (map 255 -> 0 when map_id_zero) or u16.  Output: MSB-first bit
// stream, zero padded, written as bytes at out (device, zero-initialised for
// ceil(bits/8) bytes rounded up to 4).
size_t huff_encode_tmp_bytes(size_t n);
// Words at or beyond out_cap_bytes / 4 are not written (FLAG_OUT_CAPACITY is raised).
// The stream starts at bit bit0 (0-31, most significant first) of out_words[0];
// the bits before it are left as they are (the first word is ORed), so a
// stream can be written straight after other bytes.  tmp: huff_encode_tmp_bytes(n).
int launch_huff_encode_u8(cpsz_b200_ctx* ctx, const uint8_t* sym, size_t n, bool map_id_zero, HuffEncTable tab,
                          uint32_t* out_words, size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp,
                          int bit0 = 0);
int launch_huff_encode_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, HuffEncTable tab,
                           uint32_t* out_words, size_t out_cap_bytes, unsigned long long* d_total_bits, void* tmp,
                           int bit0 = 0);
// Histograms (global, 64-bit bins).
int launch_hist_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, unsigned long long* hist);
// The same without symbol 0 (its bin stays as it was).
int launch_hist_u16_nonzero(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, unsigned long long* hist);
// Two streams of n symbols each in one launch.
int launch_hist_u16_pair(cpsz_b200_ctx* ctx, const uint16_t* a, const uint16_t* b, size_t n, unsigned long long* ha,
                         unsigned long long* hb);
// The two code histograms of one field (r1 x r2 raster codes, pitch r2)
// while its wavefront runs: row groups are counted as their group_done flags
// (WaveField::group_done) appear.  tickets: 2 words, zeroed.  A wait that
// outlasts its bound sets *gave_up (zeroed by the caller) and leaves the
// histograms incomplete; the caller then counts them with
// launch_hist_u16_pair.  Enqueued on `stream`.
int launch_hist_follow(cpsz_b200_ctx* ctx, const uint16_t* const codes[2], const unsigned* const group_done[2], int r1,
                       int r2, unsigned long long* const hist[2], unsigned* tickets, int* gave_up, cudaStream_t stream);

// Decoder table: first-level lookup of HUFF_LUT_BITS bits; entries
//   leaf:  (sym << 8) | len            (len in 1..HUFF_LUT_BITS)
//   inner: 0x80 | (node << 8)          (walk the tree from `node` bit by bit)
// Tree arrays: child[2*node + bit] (node index; leaves have t = 1 and sym in C).
constexpr int HUFF_LUT_BITS = 12;
struct HuffDecTable {
  const uint32_t* lut;       // 1 << HUFF_LUT_BITS entries
  const uint32_t* child;     // 2 * node_count
  const uint32_t* sym;       // node_count (leaf symbol)
  const uint8_t* leaf;       // node_count
  int node_count;
  int root_is_leaf;          // single-symbol stream (no bits)
  uint32_t root_sym;
};
size_t huff_decode_tmp_bytes(size_t nbits);
// Decodes exactly n symbols from a bit stream of nbits bits (words: big-endian
// byte order, padded with >= 8 zero bytes).  Output u8 or u16.
int launch_huff_decode(cpsz_b200_ctx* ctx, const uint8_t* bytes, size_t nbytes, size_t n, HuffDecTable tab,
                       void* out, int out_bytes_per_sym, void* tmp);

// ---- 3D offline (log) path ----------------------------------------------------------
// Id written for predictable-bound points that still end unpredictable
// (id_max = (int)log2(1/FLT_EPSILON) + 1, src/sz_compress_cp_preserve_3d.cpp:436).
constexpr int ID_RAW_3D = 24;
// Per-vertex bound (24 tets, reference order) -> id byte (ID_ZERO when the
// bound is not positive; ids >= ID_RAW_3D raise FLAG_ID_OVERFLOW).  eb_out
// (optional) receives the bound before quantization.
int launch_eb3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, int r1, int r2, int r3,
                double max_pwr_eb, const double* d_thr, int thr_n, uint8_t* id_q, double* eb_out = nullptr);
// Log transform: pairs[i] = (log2f|U|, log2f|V|, log2f|W| (-100 for 0), 1/precision
// or NaN); sign bitmaps (bit 7-(i%8) of byte i/8 = value > 0) as 3 arrays of
// sign_words 32-bit words.
int launch_log3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, const uint8_t* id_q, size_t n,
                 const LibmFn& L, float4* pairs, uint32_t* signs, size_t sign_words);
// Exhaustive maxima of the operations the filtered bounds rely on
// (selfcheck.cu), FP_COUNT floats as bit patterns in d_out (device).
enum FilterPremise { FP_ACBRT_HI = 0, FP_ACBRT_LO = 1, FP_RCP = 2, FP_EX2 = 3, FP_SQRT = 4, FP_LG2 = 5, FP_COUNT = 132 };
int launch_filter_premises(cpsz_b200_ctx* ctx, unsigned* d_out);
// Host-library log2f (which 0) / exp2f (which 1) of n device floats.
int launch_libm_eval(cpsz_b200_ctx* ctx, int which, const float* in, size_t n, const LibmTables& L, float* out);
// Raster compaction in chunks: chunk_count() chunks; counts of predicted
// points per chunk (compress: codes.x != 0; decompress: id not 0 / ID_RAW_3D).
size_t chunk_count(size_t n);
int launch_chunk_count_3d(cpsz_b200_ctx* ctx, bool compress, const void* src, size_t n, unsigned* cnt);
// Compress: codes_out (3 per predicted point), unpred (U,V,W per other point),
// ids rewritten in place to the reference's final ids, id histogram.
int launch_compact3d(cpsz_b200_ctx* ctx, const ushort4* codes, uint8_t* ids, const float* U, const float* V,
                     const float* W, size_t n, const unsigned* chunk_off, uint16_t* codes_out, float* unpred,
                     unsigned long long* hist_ids);
// Decompress: pairs = (3 addends, 0) for predicted points, (3 raw values, raw
// flag) for the others.  Short streams raise FLAG_RAW_RANGE.
int launch_prep3d(cpsz_b200_ctx* ctx, const uint8_t* ids, size_t n, const unsigned* chunk_off, const uint16_t* codes,
                  size_t n_codes, const float* unpred, size_t n_unpred, float4* pairs);
// Lorenzo recursion in one persistent launch (wave3d.cu).  Compress: in =
// log3d pairs, codes out (0,0,0 for unpredictable points).  Decompress: in =
// prep3d pairs, decoded U, V, W out.  rec: reconstructed log values
// (scratch); scratch: wave3d_scratch_bytes(r1, r2) of device memory.
size_t wave3d_scratch_bytes(int r1, int r2);
int launch_wave3d(cpsz_b200_ctx* ctx, bool decompress, const float4* in, float4* rec, ushort4* codes,
                  const uint8_t* signs, size_t sign_bytes, const LibmTables* L, float* U, float* V, float* W, int r1,
                  int r2, int r3, void* scratch);

// ---- exact critical-point checker -----------------------------------------------------
// Per-cell CP codes of field a (0 none, 1 + type) into `cells` (optional,
// device) and counts[0..3] += {CPs in a, CPs in b, cells with a CP in exactly
// one field, cells whose CP type differs}; b may be null.
int launch_cp_check_2d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Ub, const float* Vb, int r1,
                       int r2, uint8_t* cells, unsigned long long* counts,
                       int row0 = 0);
// Training labels of the learned bound proposer: per vertex idx[s] the largest
// log2 multiplier t in [0, tmax] of its analytic bound (bisection, `steps`
// halvings) under which moving the vertex alone to any corner of its bound box
// keeps the CP codes of its incident triangles.
int launch_labels_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, const double* eb_a,
                     const int* idx, int n, int steps, float tmax, float* out);
int launch_cp_check_3d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Wa, const float* Ub,
                       const float* Vb, const float* Wb, int r1, int r2, int r3, uint8_t* cells,
                       unsigned long long* counts);

// ---- learned-bound MLP (tcgen05) ------------------------------------------------------
// D (128 x 128 fp32, row-major) = A (128 x 128 bf16) * B (128 x 128 bf16)^T on
// one CTA through shared memory and TMEM (device pointers).
int launch_umma_selftest(cpsz_b200_ctx* ctx, const void* A, const void* B, float* D);

// MLP 99 (padded 128) -> 128 -> 128 -> 1 with ReLU.  Flat fp32 parameters:
// W1 [128 x 128] | b1 [128] | W2 [128 x 128] | b2 [128] | w3 [128] | b3.
constexpr int MLP_PARAMS = 2 * 16384 + 3 * 128 + 1;
struct MlpParams {
  float* p;    // master weights
  float* g;    // gradient accumulators
  float* m;    // Adam moments
  float* v;
  void* w1b;   // bf16 copies of W1 and W2 (tensor-core operands)
  void* w2b;
};
// y[M] from features X (bf16 [M x 128], device) or, with X null, from the
// features of every vertex of field (U, V) (r1 x r2 = M) with analytic bounds
// eb_a.  H1 / H2 (optional, bf16 [M x 128]) keep the activations for training.
int launch_mlp_forward(cpsz_b200_ctx* ctx, const MlpParams& w, const void* X, const float* U, const float* V,
                       const double* eb_a, int r1, int r2, int M, float* y, void* H1, void* H2);
// Accumulates the gradients of sum (y - t)^2 * grad_scale / 2 into w.g and the
// squared error into *loss (device).
int launch_mlp_backward(cpsz_b200_ctx* ctx, const MlpParams& w, const void* X, const void* H1, const void* H2,
                        const float* y, const float* t, int M, float grad_scale, float* loss);
int launch_mlp_adam(cpsz_b200_ctx* ctx, const MlpParams& w, float lr, int step);
int launch_mlp_cast(cpsz_b200_ctx* ctx, const MlpParams& w);
// Features (bf16 [n x 128]) of the vertices idx[0..n) of field (U, V).
int launch_mlp_features(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, const double* eb_a,
                        const int* idx, int n, void* X);

// ---- lossless stage: Zstandard frames (zstd_enc.cu) -------------------------------------
// Largest frame for n input bytes; device scratch of a call on n bytes.
size_t zstd_frame_bound(size_t n);
size_t zstd_tmp_bytes(size_t n);
// d_in (n bytes) -> a Zstandard frame at d_out (device, out_cap bytes);
// synchronises the stream once to learn the frame size (*out_size).
int launch_zstd_frame(cpsz_b200_ctx* ctx, const uint8_t* d_in, size_t n, uint8_t* d_out, size_t out_cap,
                      size_t* out_size, void* tmp);

// ---- generic scans ----------------------------------------------------------------
size_t scan_u32_tmp_bytes(size_t n);
// Exclusive scan of n u32 values into out (n+1 entries, out[n] = total).
int launch_scan_u32(cpsz_b200_ctx* ctx, const unsigned int* in, unsigned int* out, size_t n, void* tmp);

}  // namespace cpsz
