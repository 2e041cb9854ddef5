/* cpsz_oracle.h -- CPU restatement of the cpSZ offline critical-point-preserving
 * compressor / decompressor (reference: bzhan166/cpSZ).
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  It is plain C, single-threaded, and follows the reference's
 * arithmetic operation by operation (float products widened to double, left-to-
 * right sums, glibc log2/pow/log2f/exp2f, no FMA contraction).  Each function
 * cites the reference file:line it restates.  Parity of this restatement with the
 * reference itself is pinned by tests/test_oracle_vs_ref.py (which runs the
 * reference's own sources compiled by oracle/Makefile into oracle/_ref/) and by
 * the committed fixtures under tests/golden/ generated from that build.
 */
#ifndef CPSZ_ORACLE_H
#define CPSZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- 2D offline path ---------------------------------------------------- */

/* Per-vertex maximal relative error bound (before quantization), min over the
 * 6 incident triangles and max_pwr_eb.  src/sz_compress_cp_preserve_2d.cpp:177-218 */
void cpo_eb_2d(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb, double* eb);

/* Exponential quantization of |U|*eb and |V|*eb (base 4, thr = DBL_EPSILON).
 * ids[0..n) = U ids, ids[n..2n) = V ids; eb_u/eb_v = the compressor's precisions.
 * src/sz_compress_cp_preserve_2d.cpp:226-244, include/sz_cp_preserve_utils.hpp:14-22 */
void cpo_quantize_eb_2d(const float* U, const float* V, const double* eb, size_t n, int* ids, double* eb_u,
                        double* eb_v);

/* Lorenzo predict + quantize with per-point precision, codes and unpredictables
 * emitted in 12x12 block order.  recon (optional) receives the compressor's
 * reconstructed field in raster order.  Returns the number of unpredictables.
 * src/sz_compress_3d.cpp:126-193, include/sz_compress_block_processing.hpp:106-139 */
size_t cpo_lorenzo_2d(const float* data, const double* prec, size_t r1, size_t r2, int* type, float* unpred,
                      float* recon);

/* Full field blob of sz_compress_2d_with_eb (src/sz_compress_3d.cpp:196-236).
 * Returns a malloc'd buffer. */
unsigned char* cpo_compress_2d_with_eb(const float* data, const double* prec, size_t r1, size_t r2, size_t* size);

/* sz_compress_cp_preserve_2d_offline<float> (src/sz_compress_cp_preserve_2d.cpp:175-274). */
unsigned char* cpo_compress_2d_offline(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                                       size_t* size);

/* sz_decompress_cp_preserve_2d_offline<float> (src/sz_decompress_cp_preserve_2d.cpp:8-52).
 * Returns 0 on success, nonzero on a malformed blob. */
int cpo_decompress_2d_offline(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, float* U, float* V);

/* sz_compress_cp_preserve_2d_offline_log<float> (src/sz_compress_cp_preserve_2d.cpp:285-379). */
unsigned char* cpo_compress_2d_offline_log(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                                           size_t* size);
/* sz_decompress_cp_preserve_2d_offline_log<float> (src/sz_decompress_cp_preserve_2d.cpp:56-99). */
int cpo_decompress_2d_offline_log(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, float* U,
                                  float* V);

/* ---- Huffman (SZ-1.x codec, src/sz_huffman.cpp) -------------------------- */

/* Huffman_encode_tree_and_data (src/sz_compression_utils.cpp:62-82): writes
 * node_count, tree_size, tree bytes, type_array_size, bits.  Returns bytes written. */
size_t cpo_huffman_encode(size_t state_num, const int* sym, size_t n, unsigned char* out);
/* Upper bound of the bytes cpo_huffman_encode may touch (includes the 8-byte
 * write-ahead of the reference's packer). */
size_t cpo_huffman_encode_bound(size_t state_num, size_t n);
/* Huffman_decode_tree_and_data (src/sz_decompression_utils.cpp:92-108).
 * Returns bytes consumed, or 0 on malformed input. */
size_t cpo_huffman_decode(size_t state_num, size_t n, const unsigned char* in, size_t in_size, int* sym);
/* Code lengths per symbol of the tree the reference would build for this
 * histogram (len[s] = 0 for unused symbols); returns the distinct-symbol count. */
size_t cpo_huffman_code_lengths(size_t state_num, const int* sym, size_t n, unsigned char* len);

/* ---- 3D offline (log) path ----------------------------------------------- */

/* Per-vertex eb over the 24 incident Freudenthal tets.
 * src/sz_compress_cp_preserve_3d.cpp:266-358 (per tet), :362-418 (scatter). */
void cpo_eb_3d(const float* U, const float* V, const float* W, size_t r1, size_t r2, size_t r3, double max_pwr_eb,
               double* eb);
/* sz_compress_cp_preserve_3d_offline_log<float> (src/sz_compress_cp_preserve_3d.cpp:360-581). */
unsigned char* cpo_compress_3d_offline_log(const float* U, const float* V, const float* W, size_t r1, size_t r2,
                                           size_t r3, double max_pwr_eb, size_t* size);
/* sz_decompress_cp_preserve_3d_online_log<float> (src/sz_decompress_cp_preserve_3d.cpp:7-110). */
int cpo_decompress_3d_online_log(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, size_t r3,
                                 float* U, float* V, float* W);

/* The host C library's log2f / exp2f element-wise (what the reference's 3D
 * path calls). */
void cpo_log2f_array(const float* in, size_t n, float* out);
void cpo_exp2f_array(const float* in, size_t n, float* out);

void cpo_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
