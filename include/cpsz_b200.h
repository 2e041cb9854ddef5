/* cpsz_b200.h -- C ABI of the B200-native cpSZ hot path (libcpsz_b200.so).
 *
 * Plain pointers and sizes only.  Every entry point returns a status code
 * (CPSZ_OK = 0); cpsz_b200_last_error() gives the text of the calling thread's
 * last failure.  Pointers documented as "host or device" may be either: the
 * library inspects them with the CUDA runtime and copies host data in/out
 * inside the call.  All GPU work runs on one device (the context's) on one
 * stream per context; a context is not safe for concurrent use from several
 * threads, distinct contexts are.  Passing ctx = NULL uses a per-thread default
 * context on the current device.
 *
 * Blob formats are byte-for-byte those of the reference cpSZ (bzhan166/cpSZ):
 * a blob written here decodes with the reference's decoders and vice versa.
 * The 3 padding bytes of the reference's meanInfo<float> record (written
 * uninitialised by the reference) are written as zero.
 */
#ifndef CPSZ_B200_H
#define CPSZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CPSZ_OK = 0,
  CPSZ_ERR_INVALID = 1,     /* bad argument (null pointer, zero/oversized dimension, ...) */
  CPSZ_ERR_CUDA = 2,        /* CUDA runtime / launch failure */
  CPSZ_ERR_NOMEM = 3,       /* host or device allocation failed */
  CPSZ_ERR_FORMAT = 4,      /* malformed or truncated blob */
  CPSZ_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  CPSZ_ERR_UNSUPPORTED = 6, /* input outside what the format can represent */
  CPSZ_ERR_NO_DEVICE = 7    /* no CUDA device visible */
};

typedef struct cpsz_b200_ctx cpsz_b200_ctx;

/* Text of this thread's last error ("" if none). */
const char* cpsz_b200_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int cpsz_b200_version(void);

/* Context: device workspace (grow-only arena), one CUDA stream, pinned staging. */
int cpsz_b200_ctx_create(int device, cpsz_b200_ctx** ctx);
int cpsz_b200_ctx_destroy(cpsz_b200_ctx* ctx);
/* Number of kernels this context has launched so far (for launch accounting). */
int cpsz_b200_ctx_kernel_launches(cpsz_b200_ctx* ctx, uint64_t* count);
/* Batch passes run from CUDA graphs on this context: graphs captured, and
 * passes replayed from a graph captured earlier. */
int cpsz_b200_ctx_graph_stats(cpsz_b200_ctx* ctx, uint64_t* captures, uint64_t* replays);
/* Single-field compressions run the Lorenzo wavefront beside the bound kernel,
 * each row group waiting (bounded) for its bounds.  If such a wait gives up
 * (the bound kernel did not run beside it: a tool that serialises kernels, a
 * saturated or time-sliced device), the pass runs its wavefront again after
 * the bounds and still returns the same blob; this counts those re-runs on the
 * context. */
int cpsz_b200_ctx_wave_reruns(cpsz_b200_ctx* ctx, uint64_t* reruns);
/* Stream of the context as an opaque handle (a cudaStream_t). */
int cpsz_b200_ctx_stream(cpsz_b200_ctx* ctx, void** stream);
/* Per-stage timing: when on, each call records CUDA events on the context's
 * stream at its stage boundaries; cpsz_b200_ctx_stage_times() returns the
 * last call's stages (name of the stage starting at each mark, duration in ms). */
int cpsz_b200_ctx_set_timing(cpsz_b200_ctx* ctx, int on);
int cpsz_b200_ctx_stage_times(cpsz_b200_ctx* ctx, int max_stages, const char** names, float* ms, int* n_stages);

/* ---- launch-shape tuning table (no reference counterpart) -----------------
 * Parameters that change how kernels are launched and never what they compute
 * (every blob is byte-identical for every value): "eb2d.tile" (0..5: 32x16/256
 * threads, 32x8/128, 64x8/256, 32x32/256, 64x16/256, 32x16/128),
 * "wave2d.ctas_per_sm" (0 = occupancy limit), "eb3d.fill", "eb3d.min_chunk",
 * "h2d.chunks", "wave2d.overlap" (1: the Lorenzo wavefront runs beside the
 * bound kernel; under tools that serialise kernels its waits give up after
 * 50 ms without progress and the pass re-runs it after the bounds; 0: after
 * the bounds on every SM -- also forced by the environment variable
 * CPSZ_B200_OVERLAP=0).  An entry applies to fields of
 * >= min_points points; the
 * largest such threshold wins.  The first cpsz_b200_ctx_create() loads
 * $CPSZ_B200_TUNING (empty or "none": no table) or else tuning_b200.json of the
 * package directory when present; a malformed table fails ctx creation.  Any
 * explicit set / clear / load replaces that automatic load. */
int cpsz_b200_tuning_param_count(void);
int cpsz_b200_tuning_param_info(int index, const char** name, int* def, int* lo, int* hi);
int cpsz_b200_tuning_set(const char* param, size_t min_points, int value);
int cpsz_b200_tuning_get(const char* param, size_t points, int* value);
int cpsz_b200_tuning_clear(void);
/* path NULL: the package's tuning_b200.json. */
int cpsz_b200_tuning_load(const char* path);
/* Path of the table last loaded ("" if none). */
const char* cpsz_b200_tuning_source(void);

/* ---- 2D offline CP-preserving compression -------------------------------
 * Replaces sz_compress_cp_preserve_2d_offline<float>
 * (reference include/sz_compress_cp_preserve_2d.hpp:10,
 *  src/sz_compress_cp_preserve_2d.cpp:175-274).
 * U, V: r1 x r2 row-major float (host or device).  On success *blob is a
 * malloc'd host buffer (caller free()s it) of *blob_size bytes. */
int cpsz_b200_compress_2d_offline_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                      double max_pwr_eb, unsigned char** blob, size_t* blob_size);

/* Same, writing the blob into caller memory out (host or device) of capacity
 * out_cap; *blob_size receives the size (CPSZ_ERR_INVALID if out_cap is too
 * small, with *blob_size set to the size needed). */
int cpsz_b200_compress_2d_offline_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                           double max_pwr_eb, unsigned char* out, size_t out_cap, size_t* blob_size);

/* Replaces sz_decompress_cp_preserve_2d_offline<float>
 * (reference include/sz_decompress_cp_preserve_2d.hpp:11,
 *  src/sz_decompress_cp_preserve_2d.cpp:8-52).
 * blob: host memory of blob_size bytes.  U, V: caller-allocated r1*r2 floats
 * (host or device). */
int cpsz_b200_decompress_2d_offline_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1,
                                        size_t r2, float* U, float* V);

/* ---- 2D offline_log CP-preserving compression ----------------------------
 * Replaces sz_compress_cp_preserve_2d_offline_log<float>
 * (reference include/sz_compress_cp_preserve_2d.hpp:14,
 *  src/sz_compress_cp_preserve_2d.cpp:285-379): the offline per-vertex bound
 * taken to the log domain (log2(1 + eb), base 2, one id stream), U and V
 * compressed as log2f|x| with their sign maps.  Same arguments and output
 * conventions as cpsz_b200_compress_2d_offline_f32 / _into. */
int cpsz_b200_compress_2d_offline_log_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                          double max_pwr_eb, unsigned char** blob, size_t* blob_size);
int cpsz_b200_compress_2d_offline_log_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1,
                                               size_t r2, double max_pwr_eb, unsigned char* out, size_t out_cap,
                                               size_t* blob_size);
/* Replaces sz_decompress_cp_preserve_2d_offline_log<float>
 * (reference include/sz_decompress_cp_preserve_2d.hpp:15,
 *  src/sz_decompress_cp_preserve_2d.cpp:56-99). */
int cpsz_b200_decompress_2d_offline_log_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size,
                                            size_t r1, size_t r2, float* U, float* V);
/* Size of a 2D offline_log blob of an r1 x r2 field from its header. */
size_t cpsz_b200_blob_size_2d_log(const unsigned char* blob, size_t r1, size_t r2);

/* ---- batched 2D compression (many independent fields) ----------------------
 * Compresses n_fields fields in passes of up to 32 fields: every kernel stage
 * runs for all fields of a pass, the Lorenzo wavefront is one persistent
 * launch over all of them, and the Huffman trees are built on all host threads.
 * U[k], V[k]: host or device pointers of r1[k] x r2[k] floats; max_pwr_eb[k]
 * per field.  Blobs are written back to back into `out` (host or device,
 * out_cap bytes): blob k spans [offsets[k], offsets[k+1]), offsets has
 * n_fields + 1 entries.  Each blob is byte-identical to
 * cpsz_b200_compress_2d_offline_f32 of that field alone. */
int cpsz_b200_compress_2d_batch_f32(cpsz_b200_ctx* ctx, int n_fields, const float* const* U, const float* const* V,
                                    const size_t* r1, const size_t* r2, const double* max_pwr_eb, unsigned char* out,
                                    size_t out_cap, size_t* offsets);

/* ---- learned error bounds (2D offline format, decoder unchanged) ----------
 * A small MLP (99 -> 128 -> 128 -> 1, ReLU; BF16 tensor-core kernels with FP32
 * accumulation) proposes per vertex a log2 multiplier t in [0, 16] of the
 * analytic bound from a vertex's 7x7 (u,v) neighbourhood (normalised by its
 * largest |value|) and log2 of its analytic bound.  A proposed bound is
 * eb_analytic * 2^t capped at max_pwr_eb, so every point keeps the plain
 * compressor's point-wise relative bound; only bounds the critical points
 * tighten below max_pwr_eb are loosened.  The fallback loop
 * compresses with the proposals, reconstructs, compares every cell's critical
 * point exactly with the original, reverts the vertices of offending cells to
 * their analytic bounds and repeats until no cell differs.  The result is an
 * ordinary 2D offline blob. */
typedef struct cpsz_b200_mlp cpsz_b200_mlp;
size_t cpsz_b200_mlp_param_count(void);
/* He-initialised MLP on ctx's device (deterministic in seed). */
int cpsz_b200_mlp_create(cpsz_b200_ctx* ctx, uint64_t seed, cpsz_b200_mlp** mlp);
int cpsz_b200_mlp_destroy(cpsz_b200_mlp* mlp);
/* Flat fp32 parameters (host): W1 [128x128] | b1 [128] | W2 [128x128] | b2 [128] | w3 [128] | b3. */
int cpsz_b200_mlp_get_params(cpsz_b200_mlp* mlp, float* params);
int cpsz_b200_mlp_set_params(cpsz_b200_mlp* mlp, const float* params);
/* y[n] for features X (bf16 bits, n x 128, host or device). */
int cpsz_b200_mlp_forward(cpsz_b200_mlp* mlp, const uint16_t* X, size_t n, float* y);
/* Forward + backward of mean (y - t)^2 over n samples, then Adam (lr > 0);
 * grads (optional, host, param_count floats) and loss (mean) out. */
int cpsz_b200_mlp_train_step(cpsz_b200_mlp* mlp, const uint16_t* X, const float* t, size_t n, float lr, float* grads,
                             float* loss);
/* Features (bf16 bits, n x 128) of vertices idx[0..n) of field (U, V) with
 * analytic bounds eb_analytic[r1*r2]. */
int cpsz_b200_mlp_features_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                              const double* eb_analytic, const int32_t* idx, size_t n, uint16_t* X);
/* The proposer's raw outputs (log2 multipliers before clamping) for every
 * vertex of field (U, V) with analytic bounds eb_analytic[r1*r2]: the
 * features computed on the device and both layers on the tensor cores, as
 * the learned compression does.  Host or device buffers; y gets r1*r2 floats. */
int cpsz_b200_mlp_propose_2d(cpsz_b200_mlp* mlp, const float* U, const float* V, size_t r1, size_t r2,
                             const double* eb_analytic, float* y);
/* Diagnostics: the proposer's forward pass over every vertex of a field
 * (features fused, both layers on the tensor cores), timed with CUDA events on
 * the context's stream: *ms = mean of `reps` launches after one warm-up.
 * U, V, eb_analytic: device memory. */
int cpsz_b200_debug_mlp_forward_ms(cpsz_b200_mlp* mlp, const float* U, const float* V, size_t r1, size_t r2,
                                   const double* eb_analytic, int reps, float* ms);
/* Training labels: per vertex the largest log2 multiplier (bisection, `steps`
 * halvings of [0, 16]) that keeps its incident cells' CPs when the vertex
 * alone moves to any corner of its bound box. */
int cpsz_b200_learned_labels_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                const double* eb_analytic, const int32_t* idx, size_t n, int steps, float* t);
/* Compression with learned bounds: proposals from `mlp`, or the given
 * log2_mult[r1*r2] (host or device) when not null.  stats (optional): {compress
 * passes, vertices reverted, 1 if the loop gave up and fell back to the
 * analytic bounds, vertices whose enlarged bound was kept}. */
int cpsz_b200_compress_2d_learned_f32(cpsz_b200_ctx* ctx, cpsz_b200_mlp* mlp, const float* U, const float* V,
                                      size_t r1, size_t r2, double max_pwr_eb, const float* log2_mult,
                                      unsigned char* out, size_t out_cap, size_t* blob_size, uint64_t stats[4]);

/* ---- 3D offline (log) CP-preserving compression -------------------------
 * Replaces sz_compress_cp_preserve_3d_offline_log<float>
 * (reference include/sz_compress_cp_preserve_3d.hpp:8,
 *  src/sz_compress_cp_preserve_3d.cpp:360-581). */
int cpsz_b200_compress_3d_offline_log_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W,
                                          size_t r1, size_t r2, size_t r3, double max_pwr_eb, unsigned char** blob,
                                          size_t* blob_size);
/* Replaces sz_decompress_cp_preserve_3d_online_log<float>
 * (reference include/sz_decompress_cp_preserve_3d.hpp:11,
 *  src/sz_decompress_cp_preserve_3d.cpp:7-110). */
int cpsz_b200_decompress_3d_online_log_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size,
                                           size_t r1, size_t r2, size_t r3, float* U, float* V, float* W);
/* The 3D compressor writing into a caller buffer `out` (host or device) of
 * out_cap bytes; *blob_size receives the blob size (also when it does not fit). */
int cpsz_b200_compress_3d_offline_log_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W,
                                               size_t r1, size_t r2, size_t r3, double max_pwr_eb, unsigned char* out,
                                               size_t out_cap, size_t* blob_size);
/* Size of a 3D blob from its own section headers (the reference's decoder
 * takes no length). */
size_t cpsz_b200_blob_size_3d(const unsigned char* blob, size_t r1, size_t r2, size_t r3);
/* The 3D path reproduces the host C library's log2f / exp2f bit for bit from
 * tables built by scanning every float input once (about a minute on 8 cores)
 * and cached in a file (path; NULL = beside the shared library).  Called by the
 * build; the first 3D call does the same when the cache is missing. */
int cpsz_b200_libm_tables_prepare(const char* path);

/* ---- stage-level entry point (parity tests, profiling) --------------------
 * Runs the 2D offline compressor and copies out its intermediate streams
 * (each output optional, host memory):
 *   ids[2N]      the per-vertex quantized error-bound ids the reference
 *                Huffman-codes (U ids then V ids; src/sz_compress_cp_preserve_2d.cpp:177-244)
 *   codes_u/v[N] Lorenzo quantization codes in 12x12 block order
 *                (include/sz_compress_block_processing.hpp:106-139)
 *   recon_u/v[N] the compressor-side reconstruction (raster)
 *   n_unpred[2]  unpredictable-value counts of U and V. */
int cpsz_b200_compress_2d_stages(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                 double max_pwr_eb, int32_t* ids, int32_t* codes_u, int32_t* codes_v, float* recon_u,
                                 float* recon_v, size_t* n_unpred);

/* ---- SZ-1.x Huffman stage -------------------------------------------------
 * Codebook of the reference's Huffman tree for a histogram over `bins`
 * symbols (Huffman_encode_tree_and_data's tree, reference
 * src/sz_compression_utils.cpp:62-82, src/sz_huffman.cpp:195-215): per symbol
 * the right-aligned code and its length (0 = absent), and the serialized tree
 * section (node_count, tree_size, tree bytes) the blob stores before the bits.
 * Host memory; tree_bytes may be NULL to query *tree_size. */
int cpsz_b200_huffman_codebook(const uint64_t* hist, size_t bins, size_t state_num, uint64_t* code, uint8_t* len,
                               unsigned char* tree_bytes, size_t* tree_size);
/* GPU bit packing of n 16-bit symbols with that codebook (the reference's
 * encode(), src/sz_huffman.cpp:217-320): writes the MSB-first stream, zero
 * padded, as bytes at `out` (device, out_cap bytes, 4-byte aligned) and the
 * stream's bit count to *total_bits (host).  sym, code, len: device memory.
 * Scratch comes from the context's workspace. */
int cpsz_b200_huffman_encode_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, const uint64_t* code,
                                 const uint8_t* len, unsigned char* out, size_t out_cap, uint64_t* total_bits);
/* The same packing for callers that cannot allocate device memory where they
 * encode -- an in-situ hook inside a simulation that reserved the GPU's memory
 * for its own pool, a plugin handed only preallocated buffers, a loop where a
 * possibly synchronising cudaMalloc is not allowed.  This entry point has no
 * counterpart in the reference.  It calls no allocator: its scratch (a tile
 * ticket and per-tile look-back states) is a fixed ~64 KB array inside the
 * library that every GPU loading it keeps until process exit, which limits n
 * to 67,108,864 symbols per call (larger n is rejected with CPSZ_ERR_INVALID).
 * All pointers are device memory: sym (n symbols), code/len (codebook from
 * cpsz_b200_huffman_codebook: every length must be at most 64 bits, which that
 * function guarantees -- the packer appends codes of at most 64 bits),
 * out (out_cap bytes, 4-byte aligned, out_cap a multiple of 4, zeroed by the
 * call), total_bits (one uint64, receives the bit count).  The work is
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) and the
 * call returns without waiting; a stream longer than out_cap is cut off at the
 * capacity, which the caller detects as (*total_bits + 7) / 8 > out_cap.
 * Every call looks up the scratch array's device address
 * (cudaGetSymbolAddress) in the calling thread's current device and context,
 * so the address stays valid after a device reset and in a context the caller
 * made current; the first call on a device also loads the library's kernels
 * there.  All calls on a device share
 * the one array, which keeps the last call's contents (the call clears what
 * must start at zero), so calls whose GPU work overlaps (concurrent streams,
 * threads) race and must be serialised by the caller. */
int cpsz_b200_huffman_encode_u16_noalloc(const uint16_t* sym, size_t n, const uint64_t* code, const uint8_t* len,
                                         unsigned char* out, size_t out_cap, uint64_t* total_bits, void* stream);

/* Size of a 2D offline blob from its header (the reference's decoder takes
 * no length; this lets a caller without one bound the read). */
size_t cpsz_b200_blob_size_2d(const unsigned char* blob);

/* ---- diagnostics (no reference counterpart) ---------------------------------
 * The 2D bound kernel alone: per-vertex bound before quantization (eb_out, N
 * doubles) and id bytes (id_codes, 2N; 255 = precision 0).  Host buffers.
 * With eb_out the kernel evaluates every bound exactly; with eb_out = NULL it
 * takes the compressor's filtered path (ids only), which must give the same
 * ids. */
int cpsz_b200_debug_eb2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                         double max_pwr_eb, double* eb_out, uint8_t* id_codes);
/* The 3D bound kernel alone: per-vertex bound (N doubles) and id bytes (N;
 * 255 = bound not positive).  Host buffers. */
int cpsz_b200_debug_eb3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, size_t r1, size_t r2,
                         size_t r3, double max_pwr_eb, double* eb_out, uint8_t* id_codes);
/* The wavefront's per-group wait for the bound kernel gives up once the bound
 * kernel has finished no tile for wait_ns (0 = the default of 50 ms);
 * unreachable != 0 makes every such wait run out (its target is one point more
 * than the group holds), which exercises the re-run path
 * (cpsz_b200_ctx_wave_reruns) without stalling any kernel beyond the limit. */
int cpsz_b200_debug_band_wait(cpsz_b200_ctx* ctx, long long wait_ns, int unreachable);
/* Tensor-core self-check: D (128x128 fp32) = A (128x128 bf16 bits) * B^T
 * (128x128 bf16 bits), row-major host arrays, through tcgen05 / TMEM. */
int cpsz_b200_debug_umma_gemm(cpsz_b200_ctx* ctx, const uint16_t* A, const uint16_t* B, float* D);
/* The GPU's host-library log2f (which 0) or exp2f (which 1) of n host floats. */
int cpsz_b200_debug_libm(cpsz_b200_ctx* ctx, int which, const float* in, size_t n, float* out);
/* Wavefront trace: with out == NULL, (re)allocates a device trace of len
 * counters (len = 0 disables it); compressions on this context then record,
 * per (field, 256-row group, warp), {start ns, end ns, spins waiting for the
 * row above, spins waiting for ring credit}.  With out != NULL, copies len
 * counters out. */
int cpsz_b200_debug_wave_trace(cpsz_b200_ctx* ctx, size_t len, long long* out);
/* Exhaustive maxima, measured on this device, of the operations whose error
 * bounds the filtered 2D / 3D bound evaluations rely on (no reference
 * counterpart): out[0] / out[1] the largest relative error of the
 * reference's acbrt1 cube root above / below a double cube root over all
 * positive normal floats; out[2] rcp.approx.ftz.f32 (relative, normal floats
 * below 2^126); out[3] ex2.approx.ftz.f32 (relative, [-87, 0]); out[4]
 * sqrt.approx.f32 (relative, positive normal floats); out[5 + e + 126]
 * lg2.approx.ftz.f32 (absolute) on [2^e, 2^(e+1)), e = -126..0.  n >= 132. */
int cpsz_b200_debug_filter_premises(cpsz_b200_ctx* ctx, double* out, size_t n);
/* Host-computed quantization thresholds (which = 2: 2D offline, 1: 2D
 * offline_log, 3: 3D): t[k] is the smallest bound with id >= k under the host
 * libm's log2 (256 doubles); t[0] is the largest bound quantized to precision 0. */
int cpsz_b200_debug_quant_table(int which, double* t, int* n);

/* ---- exact critical-point checker -----------------------------------------
 * Per-cell CP classification with exact predicates (float products compared
 * exactly, expansion arithmetic for Jacobian signs, Simulation of Simplicity
 * on vertex index for ties).  Cell ids follow the reference's evaluation tool
 * (test/cp_extraction_2d.cpp:117-147): cell 2*(i*(r2-1)+j)+k, k=0 triangle
 * {(i,j),(i+1,j),(i+1,j+1)}, k=1 {(i,j),(i,j+1),(i+1,j+1)}.  Types as
 * test/cp_extraction_2d.cpp:34-40 plus 1: 0 = no CP, 1+t for t in
 * {SINGULAR, ATTRACTING, REPELLING, SADDLE, ATTRACTING_FOCUS, REPELLING_FOCUS,
 * CENTER}.  cells_out (optional, host or device): 2*(r1-1)*(r2-1) bytes.
 * counts[0..3] = {CPs in a, CPs in b, lost+spurious, type changed} when b != NULL. */
int cpsz_b200_cp_check_2d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Ub, const float* Vb,
                          size_t r1, size_t r2, uint8_t* cells_out, uint64_t counts[4]);
/* 3D: 6 tets per cube (test/cp_extraction_3d.cpp:39-77 ordering), cell id
 * 6*(cube index)+t; types 1+t for t in test/cp_extraction_3d.cpp:30-38. */
int cpsz_b200_cp_check_3d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Wa, const float* Ub,
                          const float* Vb, const float* Wb, size_t r1, size_t r2, size_t r3, uint8_t* cells_out,
                          uint64_t counts[4]);

/* ---- synthetic workloads (host) -------------------------------------------
 * Seeded Gaussian-windowed linear-flow fields (no reference counterpart: the
 * reference's dataset is not distributed).  Outputs are host arrays. */
int cpsz_b200_generate_field_2d(uint64_t seed, size_t r1, size_t r2, int n_flows, double sigma, double noise_std,
                                float* U, float* V);
int cpsz_b200_generate_field_3d(uint64_t seed, size_t r1, size_t r2, size_t r3, int n_flows, double sigma,
                                double noise_std, float* U, float* V, float* W);
int cpsz_b200_batch_layout(uint64_t base_seed, int n_fields, int lo, int hi, size_t* r1, size_t* r2, uint64_t* seeds,
                           double* ebs);

/* ---- GPU lossless stage ----------------------------------------------------
 * Replaces the reference's host ZSTD stage (sz_lossless_compress,
 * src/sz_lossless.cpp:11-26) on the GPU: `in` (n bytes, host or device) becomes
 * a standard Zstandard frame at `out` (host or device, out_cap bytes; at most
 * cpsz_b200_lossless_bound(n)), which ZSTD_decompress -- and so the
 * reference's sz_lossless_decompress -- reads back.  8 KB blocks encoded
 * independently (greedy matches within the block, raw literals, sequences
 * with the predefined FSE tables); the frame is larger than ZSTD level 3's. */
size_t cpsz_b200_lossless_bound(size_t n);
int cpsz_b200_lossless_compress(cpsz_b200_ctx* ctx, const unsigned char* in, size_t n, unsigned char* out,
                                size_t out_cap, size_t* out_size);

/* ---- host lossless stage (ZSTD level 3, as src/sz_lossless.cpp:11-26) ---- */
int cpsz_b200_zstd_compress(const unsigned char* data, size_t n, int level, unsigned char** out, size_t* out_size);
int cpsz_b200_zstd_decompress(const unsigned char* data, size_t n, unsigned char* out, size_t out_size);

#ifdef __cplusplus
}
#endif
#endif /* CPSZ_B200_H */
