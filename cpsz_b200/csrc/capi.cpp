// capi.cpp -- the extern "C" layer of libcpsz_b200.so and the C++ drop-ins
// that keep the reference's template signatures.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cpsz_b200.h"
#include "cpsz_b200.hpp"
#include "huffman_host.h"
#include "pipeline.h"
#include "transfer.h"

// system libzstd.so.1 (linked directly; the image has no zstd.h)
extern "C" {
size_t ZSTD_compress(void* dst, size_t dstCapacity, const void* src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
size_t ZSTD_compressBound(size_t srcSize);
unsigned ZSTD_isError(size_t code);
const char* ZSTD_getErrorName(size_t code);
}

namespace cpsz {

int copy_out(cpsz_b200_ctx* ctx, void* dst, const void* d_src, size_t n) { return d2h(ctx, dst, d_src, n, ctx->stream); }

int copy_in(cpsz_b200_ctx* ctx, void* d_dst, const void* src, size_t n) { return h2d(ctx, d_dst, src, n, ctx->stream); }

}  // namespace cpsz

using namespace cpsz;

#define RESOLVE(ctx)            \
  int _rc = CPSZ_OK;            \
  ctx = resolve_ctx(ctx, &_rc); \
  if (!ctx) return _rc;         \
  clear_error();

extern "C" {

int cpsz_b200_compress_2d_offline_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                      double max_pwr_eb, unsigned char** blob, size_t* blob_size) {
  if (!blob || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  *blob = nullptr;
  *blob_size = 0;
  RESOLVE(ctx);
  Blob2D b;
  CPSZ_TRY(compress_2d(ctx, U, V, r1, r2, max_pwr_eb, &b, nullptr));
  unsigned char* h = (unsigned char*)malloc(b.size ? b.size : 1);
  if (!h) return set_error(CPSZ_ERR_NOMEM, "host blob of %zu bytes", b.size);
  int rc = d2h(ctx, h, b.d_blob, b.size, ctx->stream);
  if (rc == CPSZ_OK) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "blob download: %s", cudaGetErrorString(e));
  }
  if (rc != CPSZ_OK) {
    free(h);
    return rc;
  }
  *blob = h;
  *blob_size = b.size;
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_offline_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                           double max_pwr_eb, unsigned char* out, size_t out_cap, size_t* blob_size) {
  if (!out || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  RESOLVE(ctx);
  Blob2D b;
  // host memory: the sections are written there as they are produced; a
  // device buffer: the blob is built in place when the buffer has room for
  // the blob's bound, else copied there
  CPSZ_TRY(compress_2d(ctx, U, V, r1, r2, max_pwr_eb, &b, nullptr, nullptr, out, out_cap));
  *blob_size = b.size;
  if (b.d_blob && b.d_blob != out) {
    if (b.size > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < blob size %zu", out_cap, b.size);
    CPSZ_TRY(copy_out(ctx, out, b.d_blob, b.size));
  }
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_decompress_2d_offline_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1,
                                        size_t r2, float* U, float* V) {
  RESOLVE(ctx);
  CPSZ_TRY(decompress_2d(ctx, blob, blob_size, r1, r2, U, V));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_offline_log_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                          double max_pwr_eb, unsigned char** blob, size_t* blob_size) {
  if (!blob || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  *blob = nullptr;
  *blob_size = 0;
  RESOLVE(ctx);
  Blob2D b;
  CPSZ_TRY(compress_2d(ctx, U, V, r1, r2, max_pwr_eb, &b, nullptr, nullptr, nullptr, 0, true));
  unsigned char* h = (unsigned char*)malloc(b.size ? b.size : 1);
  if (!h) return set_error(CPSZ_ERR_NOMEM, "host blob of %zu bytes", b.size);
  int rc = d2h(ctx, h, b.d_blob, b.size, ctx->stream);
  if (rc == CPSZ_OK) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "blob download: %s", cudaGetErrorString(e));
  }
  if (rc != CPSZ_OK) {
    free(h);
    return rc;
  }
  *blob = h;
  *blob_size = b.size;
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_offline_log_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1,
                                               size_t r2, double max_pwr_eb, unsigned char* out, size_t out_cap,
                                               size_t* blob_size) {
  if (!out || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  RESOLVE(ctx);
  Blob2D b;
  CPSZ_TRY(compress_2d(ctx, U, V, r1, r2, max_pwr_eb, &b, nullptr, nullptr, out, out_cap, true));
  *blob_size = b.size;
  if (b.d_blob && b.d_blob != out) {
    if (b.size > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < blob size %zu", out_cap, b.size);
    CPSZ_TRY(copy_out(ctx, out, b.d_blob, b.size));
  }
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_decompress_2d_offline_log_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size,
                                            size_t r1, size_t r2, float* U, float* V) {
  RESOLVE(ctx);
  CPSZ_TRY(decompress_2d(ctx, blob, blob_size, r1, r2, U, V, true));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_stages(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                 double max_pwr_eb, int32_t* ids, int32_t* codes_u, int32_t* codes_v, float* recon_u,
                                 float* recon_v, size_t* n_unpred) {
  RESOLVE(ctx);
  const size_t N = r1 * r2;
  if (N == 0) return set_error(CPSZ_ERR_INVALID, "empty field");
  // taps are separate device buffers so the product path's arena layout is untouched
  uint8_t* d_ids = nullptr;
  uint16_t* d_codes = nullptr;
  float* d_recon = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc((void**)&d_ids, 2 * N + 16));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&d_codes, 4 * N + 16));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&d_recon, 8 * N + 16));
  StageTap tap;
  tap.ids = d_ids;
  tap.codes_blocks[0] = d_codes;
  tap.codes_blocks[1] = d_codes + N;
  tap.recon[0] = d_recon;
  tap.recon[1] = d_recon + N;
  Blob2D b;
  int rc = compress_2d(ctx, U, V, r1, r2, max_pwr_eb, &b, &tap);
  if (rc == CPSZ_OK) {
    std::vector<uint8_t> hid(2 * N);
    std::vector<uint16_t> hc(2 * N);
    std::vector<float> hr(2 * N);
    cudaError_t e = cudaMemcpyAsync(hid.data(), d_ids, 2 * N, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), d_codes, 4 * N, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hr.data(), d_recon, 8 * N, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      rc = set_error(CPSZ_ERR_CUDA, "stage download: %s", cudaGetErrorString(e));
    } else {
      if (ids)
        for (size_t i = 0; i < 2 * N; i++) ids[i] = (hid[i] == ID_ZERO) ? 0 : (int32_t)hid[i];
      if (codes_u)
        for (size_t i = 0; i < N; i++) codes_u[i] = hc[i];
      if (codes_v)
        for (size_t i = 0; i < N; i++) codes_v[i] = hc[N + i];
      if (recon_u) memcpy(recon_u, hr.data(), 4 * N);
      if (recon_v) memcpy(recon_v, hr.data() + N, 4 * N);
      if (n_unpred) {
        n_unpred[0] = b.n_unpred[0];
        n_unpred[1] = b.n_unpred[1];
      }
    }
  }
  cudaFree(d_ids);
  cudaFree(d_codes);
  cudaFree(d_recon);
  return rc;
}

int cpsz_b200_debug_eb2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                         double* eb_out, uint8_t* id_codes) {
  RESOLVE(ctx);
  const size_t N = r1 * r2;
  const QuantTable& qt = quant_table_2d();
  float *dU = nullptr, *dV = nullptr;
  double *deb = nullptr, *dtab = nullptr;
  uint8_t* dids = nullptr;
  unsigned long long* dh = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dU, 4 * N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dV, 4 * N));
  if (eb_out) CPSZ_CUDA_TRY(cudaMalloc((void**)&deb, 8 * N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dids, 2 * N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dtab, QUANT_TAB_MAX * 8));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dh, 256 * 8));
  cudaMemcpy(dU, U, 4 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dV, V, 4 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dtab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice);
  cudaMemset(dh, 0, 256 * 8);
  int rc = launch_eb2d(ctx, dU, dV, (int)r1, (int)r2, max_pwr_eb, dtab, qt.n, dids, dids + N, dh, nullptr, nullptr, deb,
                       0, -1, nullptr, false, qt.float_pow4);
  cudaStreamSynchronize(ctx->stream);
  if (rc == CPSZ_OK) {
    if (eb_out) cudaMemcpy(eb_out, deb, 8 * N, cudaMemcpyDeviceToHost);
    if (id_codes) cudaMemcpy(id_codes, dids, 2 * N, cudaMemcpyDeviceToHost);
  }
  cudaFree(dU);
  cudaFree(dV);
  cudaFree(deb);
  cudaFree(dids);
  cudaFree(dtab);
  cudaFree(dh);
  return rc;
}

int cpsz_b200_debug_wave_trace(cpsz_b200_ctx* ctx, size_t len, long long* out) {
  RESOLVE(ctx);
  if (out) {
    if (!ctx->d_wave_trace) return set_error(CPSZ_ERR_INVALID, "wave trace not enabled");
    size_t n = len < ctx->wave_trace_len ? len : ctx->wave_trace_len;
    CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CPSZ_CUDA_TRY(cudaMemcpy(out, ctx->d_wave_trace, n * 8, cudaMemcpyDeviceToHost));
    return CPSZ_OK;
  }
  if (ctx->d_wave_trace) cudaFree(ctx->d_wave_trace);
  ctx->d_wave_trace = nullptr;
  ctx->wave_trace_len = 0;
  if (len) {
    CPSZ_CUDA_TRY(cudaMalloc((void**)&ctx->d_wave_trace, len * 8));
    CPSZ_CUDA_TRY(cudaMemset(ctx->d_wave_trace, 0, len * 8));
    ctx->wave_trace_len = len;
  }
  return CPSZ_OK;
}

int cpsz_b200_debug_quant_table(int which, double* t, int* n) {
  const QuantTable& q = which == 3 ? quant_table_3d() : which == 1 ? quant_table_2d_log() : quant_table_2d();
  if (t) memcpy(t, q.t, sizeof(q.t));
  if (n) *n = q.n;
  return CPSZ_OK;
}

int cpsz_b200_huffman_codebook(const uint64_t* hist, size_t bins, size_t state_num, uint64_t* code, uint8_t* len,
                               unsigned char* tree_bytes, size_t* tree_size) {
  clear_error();
  if (!hist || !bins || !tree_size) return set_error(CPSZ_ERR_INVALID, "null histogram or tree_size");
  HuffCodebook cb;
  if (!huff_build((const unsigned long long*)hist, bins, state_num, &cb)) return CPSZ_ERR_INVALID;
  huff_tables(cb, bins, (unsigned long long*)code, len);
  if (tree_bytes) {
    if (*tree_size < cb.tree_bytes.size())
      return set_error(CPSZ_ERR_INVALID, "tree buffer of %zu bytes < %zu", *tree_size, cb.tree_bytes.size());
    memcpy(tree_bytes, cb.tree_bytes.data(), cb.tree_bytes.size());
  }
  *tree_size = cb.tree_bytes.size();
  return CPSZ_OK;
}

int cpsz_b200_huffman_encode_u16(cpsz_b200_ctx* ctx, const uint16_t* sym, size_t n, const uint64_t* code,
                                 const uint8_t* len, unsigned char* out, size_t out_cap, uint64_t* total_bits) {
  if (!sym || !code || !len || !out || !total_bits) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  if (((uintptr_t)out & 3) != 0) return set_error(CPSZ_ERR_INVALID, "output must be 4-byte aligned");
  RESOLVE(ctx);
  CPSZ_TRY(arena_reserve(ctx, huff_encode_tmp_bytes(n) + 1024));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  void* tmp = arena_alloc(ctx, huff_encode_tmp_bytes(n));
  unsigned long long* d_total = (unsigned long long*)arena_alloc(ctx, 64);
  CPSZ_CUDA_TRY(cudaMemsetAsync(out, 0, out_cap, ctx->stream));
  CPSZ_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, ctx->stream));
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  CPSZ_TRY(launch_huff_encode_u16(ctx, sym, n, HuffEncTable{(const unsigned long long*)code, len, 65536},
                                  (uint32_t*)out, out_cap, d_total, tmp));
  unsigned long long* h = (unsigned long long*)ctx->pinned;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h + 1, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *total_bits = h[0];
  if ((*total_bits + 7) / 8 > out_cap || (*(int*)(h + 1) & FLAG_OUT_CAPACITY))
    return set_error(CPSZ_ERR_INVALID, "output capacity %zu < %llu bytes", out_cap,
                     (unsigned long long)((*total_bits + 7) / 8));
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_batch_f32(cpsz_b200_ctx* ctx, int n_fields, const float* const* U, const float* const* V,
                                    const size_t* r1, const size_t* r2, const double* max_pwr_eb, unsigned char* out,
                                    size_t out_cap, size_t* offsets) {
  RESOLVE(ctx);
  CPSZ_TRY(compress_2d_batch(ctx, n_fields, U, V, r1, r2, max_pwr_eb, out, out_cap, offsets));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

// ---- 3D ----------------------------------------------------------------------------

int cpsz_b200_compress_3d_offline_log_f32(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W,
                                          size_t r1, size_t r2, size_t r3, double max_pwr_eb, unsigned char** blob,
                                          size_t* blob_size) {
  if (!blob || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  *blob = nullptr;
  *blob_size = 0;
  RESOLVE(ctx);
  Blob3D b;
  CPSZ_TRY(compress_3d(ctx, U, V, W, r1, r2, r3, max_pwr_eb, &b));
  unsigned char* h = (unsigned char*)malloc(b.size ? b.size : 1);
  if (!h) return set_error(CPSZ_ERR_NOMEM, "host blob of %zu bytes", b.size);
  int rc = d2h(ctx, h, b.d_blob, b.size, ctx->stream);
  if (rc == CPSZ_OK) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "blob download: %s", cudaGetErrorString(e));
  }
  if (rc != CPSZ_OK) {
    free(h);
    return rc;
  }
  *blob = h;
  *blob_size = b.size;
  return CPSZ_OK;
}

int cpsz_b200_compress_3d_offline_log_f32_into(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W,
                                               size_t r1, size_t r2, size_t r3, double max_pwr_eb, unsigned char* out,
                                               size_t out_cap, size_t* blob_size) {
  if (!out || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output pointer");
  RESOLVE(ctx);
  Blob3D b;
  CPSZ_TRY(compress_3d(ctx, U, V, W, r1, r2, r3, max_pwr_eb, &b));
  *blob_size = b.size;
  if (b.size > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < blob size %zu", out_cap, b.size);
  CPSZ_TRY(copy_out(ctx, out, b.d_blob, b.size));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_decompress_3d_online_log_f32(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size,
                                           size_t r1, size_t r2, size_t r3, float* U, float* V, float* W) {
  RESOLVE(ctx);
  CPSZ_TRY(decompress_3d(ctx, blob, blob_size, r1, r2, r3, U, V, W));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

size_t cpsz_b200_blob_size_3d(const unsigned char* blob, size_t r1, size_t r2, size_t r3) {
  if (!blob || !r1 || !r2 || !r3) return 0;
  const size_t N = r1 * r2 * r3, smap = (N - 1) / 8 + 1;
  size_t at = 8 + 3 * smap;
  unsigned long long n_unpred;
  memcpy(&n_unpred, blob + at, 8);
  at += 8 + 4 * n_unpred + 8;
  for (int k = 0; k < 2; k++) {
    if (k == 1) at += 8;
    unsigned int tree_size;
    unsigned long long nbytes;
    memcpy(&tree_size, blob + at + 8, 4);
    memcpy(&nbytes, blob + at + 12 + tree_size, 8);
    at += 12 + (size_t)tree_size + 8 + nbytes;
  }
  return at;
}

int cpsz_b200_debug_eb3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, size_t r1, size_t r2,
                         size_t r3, double max_pwr_eb, double* eb_out, uint8_t* id_codes) {
  RESOLVE(ctx);
  const size_t N = r1 * r2 * r3;
  if (!N) return set_error(CPSZ_ERR_INVALID, "empty field");
  const QuantTable& qt = quant_table_3d();
  float* dF = nullptr;
  double *deb = nullptr, *dtab = nullptr;
  uint8_t* dids = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dF, 12 * N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&deb, 8 * N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dids, N));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dtab, QUANT_TAB_MAX * 8));
  cudaMemcpy(dF, U, 4 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dF + N, V, 4 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dF + 2 * N, W, 4 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dtab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice);
  cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream);
  int rc = launch_eb3d(ctx, dF, dF + N, dF + 2 * N, (int)r1, (int)r2, (int)r3, max_pwr_eb, dtab, qt.n, dids, deb);
  cudaStreamSynchronize(ctx->stream);
  if (rc == CPSZ_OK) {
    if (eb_out) cudaMemcpy(eb_out, deb, 8 * N, cudaMemcpyDeviceToHost);
    if (id_codes) cudaMemcpy(id_codes, dids, N, cudaMemcpyDeviceToHost);
  }
  cudaFree(dF);
  cudaFree(deb);
  cudaFree(dids);
  cudaFree(dtab);
  return rc;
}

int cpsz_b200_debug_umma_gemm(cpsz_b200_ctx* ctx, const uint16_t* A, const uint16_t* B, float* D) {
  RESOLVE(ctx);
  if (!A || !B || !D) return set_error(CPSZ_ERR_INVALID, "null pointer");
  void *dA = nullptr, *dB = nullptr;
  float* dD = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc(&dA, 128 * 128 * 2));
  CPSZ_CUDA_TRY(cudaMalloc(&dB, 128 * 128 * 2));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dD, 128 * 128 * 4));
  cudaMemcpy(dA, A, 128 * 128 * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, B, 128 * 128 * 2, cudaMemcpyHostToDevice);
  cudaMemset(dD, 0, 128 * 128 * 4);
  cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream);
  int rc = launch_umma_selftest(ctx, dA, dB, dD);
  int flag = 0;
  if (rc == CPSZ_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "tensor-core self-test: %s", cudaGetErrorString(e));
  }
  if (rc == CPSZ_OK) {
    cudaMemcpy(D, dD, 128 * 128 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (flag) rc = set_error(CPSZ_ERR_TIMEOUT, "tensor-core self-test: MMA completion wait gave up");
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  return rc;
}

int cpsz_b200_debug_libm(cpsz_b200_ctx* ctx, int which, const float* in, size_t n, float* out) {
  RESOLVE(ctx);
  if (!in || !out || (which != 0 && which != 1)) return set_error(CPSZ_ERR_INVALID, "invalid argument");
  if (!n) return CPSZ_OK;
  LibmTables lt;
  CPSZ_TRY(libm_tables_device(ctx, &lt));
  float *di = nullptr, *dout = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc((void**)&di, 4 * n));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&dout, 4 * n));
  cudaMemcpy(di, in, 4 * n, cudaMemcpyHostToDevice);
  int rc = launch_libm_eval(ctx, which, di, n, lt, dout);
  cudaStreamSynchronize(ctx->stream);
  if (rc == CPSZ_OK) cudaMemcpy(out, dout, 4 * n, cudaMemcpyDeviceToHost);
  cudaFree(di);
  cudaFree(dout);
  return rc;
}

int cpsz_b200_debug_filter_premises(cpsz_b200_ctx* ctx, double* out, size_t n) {
  RESOLVE(ctx);
  if (!out || n < (size_t)FP_COUNT) return set_error(CPSZ_ERR_INVALID, "need %d output doubles", (int)FP_COUNT);
  unsigned* d = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc((void**)&d, FP_COUNT * sizeof(unsigned)));
  unsigned h[FP_COUNT];
  int rc = launch_filter_premises(ctx, d);
  if (rc == CPSZ_OK) {
    const cudaError_t e = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess || e2 != cudaSuccess)
      rc = set_error(CPSZ_ERR_CUDA, "filter premises: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaFree(d);
  if (rc != CPSZ_OK) return rc;
  for (int i = 0; i < FP_COUNT; i++) {
    float f;
    memcpy(&f, &h[i], 4);
    out[i] = f;
  }
  return CPSZ_OK;
}

// ---- exact critical-point checker ----------------------------------------------------

namespace {

// Device copies of up to six fields (host inputs are uploaded; device ones used in place).
struct CpInputs {
  const float* d[6] = {};
  std::vector<void*> owned;
  ~CpInputs() {
    for (void* p : owned) cudaFree(p);
  }
  int stage(cpsz_b200_ctx* ctx, const float* const* in, int k, size_t n) {
    for (int f = 0; f < k; f++) {
      if (!in[f]) continue;
      if (is_device_ptr(in[f])) {
        d[f] = in[f];
        continue;
      }
      void* p = nullptr;
      CPSZ_CUDA_TRY(cudaMalloc(&p, 4 * n));
      owned.push_back(p);
      CPSZ_CUDA_TRY(cudaMemcpyAsync(p, in[f], 4 * n, cudaMemcpyHostToDevice, ctx->stream));
      d[f] = (const float*)p;
    }
    return CPSZ_OK;
  }
};

int cp_check_run(cpsz_b200_ctx* ctx, int dims, const float* const* in, const size_t* r, uint8_t* cells_out,
                 uint64_t counts[4]) {
  const size_t n = r[0] * r[1] * (dims == 3 ? r[2] : 1);
  if (!n) return set_error(CPSZ_ERR_INVALID, "empty field");
  for (int k = 0; k < dims; k++)
    if (r[k] > (1u << 30)) return set_error(CPSZ_ERR_UNSUPPORTED, "dimension %zu too large", r[k]);
  const int nf = dims;  // fields per set
  for (int f = 0; f < nf; f++)
    if (!in[f]) return set_error(CPSZ_ERR_INVALID, "null field a");
  const bool with_b = in[nf] != nullptr;
  for (int f = 0; f < nf; f++)
    if (with_b != (in[nf + f] != nullptr)) return set_error(CPSZ_ERR_INVALID, "field b given partially");
  size_t ncell = 1;
  for (int k = 0; k < dims; k++) ncell *= (r[k] > 1 ? r[k] - 1 : 0);
  ncell *= (dims == 3 ? 6 : 2);
  CpInputs ci;
  CPSZ_TRY(ci.stage(ctx, in, 2 * nf, n));
  CPSZ_TRY(arena_reserve(ctx, ncell + 4096));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  unsigned long long* d_counts = (unsigned long long*)arena_alloc(ctx, 64);
  uint8_t* d_cells = nullptr;
  const bool cells_dev = cells_out && is_device_ptr(cells_out);
  if (cells_out) d_cells = cells_dev ? cells_out : (uint8_t*)arena_alloc(ctx, ncell + 16);
  CPSZ_CUDA_TRY(cudaMemsetAsync(d_counts, 0, 64, ctx->stream));
  if (dims == 2)
    CPSZ_TRY(launch_cp_check_2d(ctx, ci.d[0], ci.d[1], ci.d[2], ci.d[3], (int)r[0], (int)r[1], d_cells, d_counts));
  else
    CPSZ_TRY(launch_cp_check_3d(ctx, ci.d[0], ci.d[1], ci.d[2], ci.d[3], ci.d[4], ci.d[5], (int)r[0], (int)r[1],
                                (int)r[2], d_cells, d_counts));
  if (cells_out && !cells_dev && ncell)
    CPSZ_CUDA_TRY(cudaMemcpyAsync(cells_out, d_cells, ncell, cudaMemcpyDeviceToHost, ctx->stream));
  unsigned long long* h = (unsigned long long*)ctx->pinned;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(h, d_counts, 32, cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (counts)
    for (int k = 0; k < 4; k++) counts[k] = h[k];
  return CPSZ_OK;
}

}  // namespace

int cpsz_b200_cp_check_2d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Ub, const float* Vb,
                          size_t r1, size_t r2, uint8_t* cells_out, uint64_t counts[4]) {
  RESOLVE(ctx);
  const float* in[4] = {Ua, Va, Ub, Vb};
  const size_t r[2] = {r1, r2};
  return cp_check_run(ctx, 2, in, r, cells_out, counts);
}

int cpsz_b200_cp_check_3d(cpsz_b200_ctx* ctx, const float* Ua, const float* Va, const float* Wa, const float* Ub,
                          const float* Vb, const float* Wb, size_t r1, size_t r2, size_t r3, uint8_t* cells_out,
                          uint64_t counts[4]) {
  RESOLVE(ctx);
  const float* in[6] = {Ua, Va, Wa, Ub, Vb, Wb};
  const size_t r[3] = {r1, r2, r3};
  return cp_check_run(ctx, 3, in, r, cells_out, counts);
}

size_t cpsz_b200_blob_size_2d(const unsigned char* blob) {
  if (!blob) return 0;
  unsigned long long s[3];
  memcpy(s, blob + 12, 24);
  return 36 + (size_t)s[0] + (size_t)s[1] + (size_t)s[2];
}

size_t cpsz_b200_blob_size_2d_log(const unsigned char* blob, size_t r1, size_t r2) {
  if (!blob || !r1 || !r2) return 0;
  unsigned long long s[3];
  memcpy(s, blob + 12, 24);
  return 36 + (size_t)s[0] + 2 * ((r1 * r2 - 1) / 8 + 1) + (size_t)s[1] + (size_t)s[2];
}

size_t cpsz_b200_lossless_bound(size_t n) { return zstd_frame_bound(n); }

int cpsz_b200_lossless_compress(cpsz_b200_ctx* ctx, const unsigned char* in, size_t n, unsigned char* out,
                                size_t out_cap, size_t* out_size) {
  if ((!in && n) || !out || !out_size) return set_error(CPSZ_ERR_INVALID, "null pointer argument");
  RESOLVE(ctx);
  *out_size = 0;
  const bool dev_in = n == 0 || is_device_ptr(in);
  const bool dev_out = is_device_ptr(out);
  const size_t bound = zstd_frame_bound(n);
  size_t bytes = align_up(zstd_tmp_bytes(n), 256) + 256;
  if (!dev_in) bytes += align_up(n, 256) + 256;
  if (!dev_out) bytes += align_up(bound, 256) + 256;
  CPSZ_TRY(arena_reserve(ctx, bytes));
  void* tmp = arena_alloc(ctx, zstd_tmp_bytes(n));
  const uint8_t* d_in = (const uint8_t*)in;
  if (!dev_in) {
    uint8_t* p = (uint8_t*)arena_alloc(ctx, n);
    CPSZ_TRY(h2d(ctx, p, in, n, ctx->stream));
    d_in = p;
  }
  uint8_t* d_out = dev_out ? out : (uint8_t*)arena_alloc(ctx, bound);
  if (!d_out || !tmp) return set_error(CPSZ_ERR_NOMEM, "workspace layout overflow");
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  size_t fsize = 0;
  CPSZ_TRY(launch_zstd_frame(ctx, d_in, n, d_out, dev_out ? out_cap : bound, &fsize, tmp));
  *out_size = fsize;
  if (!dev_out) {
    if (fsize > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < frame size %zu", out_cap, fsize);
    CPSZ_TRY(d2h(ctx, out, d_out, fsize, ctx->stream));
  }
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_zstd_compress(const unsigned char* data, size_t n, int level, unsigned char** out, size_t* out_size) {
  if (!out || !out_size || (!data && n)) return set_error(CPSZ_ERR_INVALID, "null pointer");
  size_t cap = ZSTD_compressBound(n);
  unsigned char* o = (unsigned char*)malloc(cap ? cap : 1);
  if (!o) return set_error(CPSZ_ERR_NOMEM, "zstd output");
  size_t r = ZSTD_compress(o, cap, data, n, level);
  if (ZSTD_isError(r)) {
    free(o);
    return set_error(CPSZ_ERR_INVALID, "ZSTD_compress: %s", ZSTD_getErrorName(r));
  }
  *out = o;
  *out_size = r;
  return CPSZ_OK;
}

int cpsz_b200_zstd_decompress(const unsigned char* data, size_t n, unsigned char* out, size_t out_size) {
  size_t r = ZSTD_decompress(out, out_size, data, n);
  if (ZSTD_isError(r)) return set_error(CPSZ_ERR_FORMAT, "ZSTD_decompress: %s", ZSTD_getErrorName(r));
  if (r != out_size) return set_error(CPSZ_ERR_FORMAT, "ZSTD_decompress: %zu bytes, expected %zu", r, out_size);
  return CPSZ_OK;
}

}  // extern "C"

// ---- C++ drop-ins with the reference's template signatures ---------------------

template <typename T>
unsigned char* sz_compress_cp_preserve_2d_offline(const T* U, const T* V, size_t r1, size_t r2,
                                                  size_t& compressed_size, bool transpose, double max_pwr_eb) {
  (void)transpose;  // ignored by the reference as well
  compressed_size = 0;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return nullptr;
  }
  unsigned char* blob = nullptr;
  size_t size = 0;
  if (cpsz_b200_compress_2d_offline_f32(nullptr, (const float*)U, (const float*)V, r1, r2, max_pwr_eb, &blob, &size) !=
      CPSZ_OK)
    return nullptr;
  compressed_size = size;
  return blob;
}

template <typename T>
void sz_decompress_cp_preserve_2d_offline(const unsigned char* compressed, size_t r1, size_t r2, T*& U, T*& V) {
  if (U) free(U);
  if (V) free(V);
  U = nullptr;
  V = nullptr;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return;
  }
  size_t n = r1 * r2;
  T* u = (T*)malloc(n * sizeof(T));
  T* v = (T*)malloc(n * sizeof(T));
  if (!u || !v) {
    free(u);
    free(v);
    set_error(CPSZ_ERR_NOMEM, "output fields");
    return;
  }
  // The reference reads the blob without a length; the sections it names bound it.
  size_t blob_size = cpsz_b200_blob_size_2d(compressed);
  if (cpsz_b200_decompress_2d_offline_f32(nullptr, compressed, blob_size, r1, r2, (float*)u, (float*)v) != CPSZ_OK) {
    free(u);
    free(v);
    return;
  }
  U = u;
  V = v;
}

template unsigned char* sz_compress_cp_preserve_2d_offline<float>(const float*, const float*, size_t, size_t, size_t&,
                                                                  bool, double);
template unsigned char* sz_compress_cp_preserve_2d_offline<double>(const double*, const double*, size_t, size_t,
                                                                   size_t&, bool, double);
template void sz_decompress_cp_preserve_2d_offline<float>(const unsigned char*, size_t, size_t, float*&, float*&);
template void sz_decompress_cp_preserve_2d_offline<double>(const unsigned char*, size_t, size_t, double*&, double*&);

template <typename T>
unsigned char* sz_compress_cp_preserve_2d_offline_log(const T* U, const T* V, size_t r1, size_t r2,
                                                      size_t& compressed_size, bool transpose, double max_pwr_eb) {
  (void)transpose;  // ignored by the reference as well
  compressed_size = 0;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return nullptr;
  }
  unsigned char* blob = nullptr;
  size_t size = 0;
  if (cpsz_b200_compress_2d_offline_log_f32(nullptr, (const float*)U, (const float*)V, r1, r2, max_pwr_eb, &blob,
                                            &size) != CPSZ_OK)
    return nullptr;
  compressed_size = size;
  return blob;
}

template <typename T>
void sz_decompress_cp_preserve_2d_offline_log(const unsigned char* compressed, size_t r1, size_t r2, T*& U, T*& V) {
  if (U) free(U);
  if (V) free(V);
  U = nullptr;
  V = nullptr;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return;
  }
  size_t n = r1 * r2;
  T* u = (T*)malloc(n * sizeof(T));
  T* v = (T*)malloc(n * sizeof(T));
  if (!u || !v) {
    free(u);
    free(v);
    set_error(CPSZ_ERR_NOMEM, "output fields");
    return;
  }
  size_t blob_size = cpsz_b200_blob_size_2d_log(compressed, r1, r2);
  if (cpsz_b200_decompress_2d_offline_log_f32(nullptr, compressed, blob_size, r1, r2, (float*)u, (float*)v) !=
      CPSZ_OK) {
    free(u);
    free(v);
    return;
  }
  U = u;
  V = v;
}

template unsigned char* sz_compress_cp_preserve_2d_offline_log<float>(const float*, const float*, size_t, size_t,
                                                                      size_t&, bool, double);
template unsigned char* sz_compress_cp_preserve_2d_offline_log<double>(const double*, const double*, size_t, size_t,
                                                                       size_t&, bool, double);
template void sz_decompress_cp_preserve_2d_offline_log<float>(const unsigned char*, size_t, size_t, float*&, float*&);
template void sz_decompress_cp_preserve_2d_offline_log<double>(const unsigned char*, size_t, size_t, double*&,
                                                               double*&);

template <typename T>
unsigned char* sz_compress_cp_preserve_3d_offline_log(const T* U, const T* V, const T* W, size_t r1, size_t r2,
                                                      size_t r3, size_t& compressed_size, bool transpose,
                                                      double max_pwr_eb) {
  (void)transpose;  // ignored by the reference as well
  compressed_size = 0;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return nullptr;
  }
  unsigned char* blob = nullptr;
  size_t size = 0;
  if (cpsz_b200_compress_3d_offline_log_f32(nullptr, (const float*)U, (const float*)V, (const float*)W, r1, r2, r3,
                                            max_pwr_eb, &blob, &size) != CPSZ_OK)
    return nullptr;
  compressed_size = size;
  return blob;
}

template <typename T>
void sz_decompress_cp_preserve_3d_online_log(const unsigned char* compressed, size_t r1, size_t r2, size_t r3, T*& U,
                                             T*& V, T*& W) {
  if (U) free(U);
  if (V) free(V);
  if (W) free(W);
  U = V = W = nullptr;
  if (sizeof(T) != sizeof(float)) {
    set_error(CPSZ_ERR_UNSUPPORTED, "only float fields are supported on the GPU path");
    return;
  }
  const size_t n = r1 * r2 * r3;
  T* u = (T*)malloc(n * sizeof(T));
  T* v = (T*)malloc(n * sizeof(T));
  T* w = (T*)malloc(n * sizeof(T));
  if (!u || !v || !w) {
    free(u);
    free(v);
    free(w);
    set_error(CPSZ_ERR_NOMEM, "output fields");
    return;
  }
  // The reference reads the blob without a length; the sections it names bound it.
  const size_t blob_size = cpsz_b200_blob_size_3d(compressed, r1, r2, r3);
  if (cpsz_b200_decompress_3d_online_log_f32(nullptr, compressed, blob_size, r1, r2, r3, (float*)u, (float*)v,
                                             (float*)w) != CPSZ_OK) {
    free(u);
    free(v);
    free(w);
    return;
  }
  U = u;
  V = v;
  W = w;
}

template unsigned char* sz_compress_cp_preserve_3d_offline_log<float>(const float*, const float*, const float*, size_t,
                                                                      size_t, size_t, size_t&, bool, double);
template unsigned char* sz_compress_cp_preserve_3d_offline_log<double>(const double*, const double*, const double*,
                                                                       size_t, size_t, size_t, size_t&, bool, double);
template void sz_decompress_cp_preserve_3d_online_log<float>(const unsigned char*, size_t, size_t, size_t, float*&,
                                                             float*&, float*&);
template void sz_decompress_cp_preserve_3d_online_log<double>(const unsigned char*, size_t, size_t, size_t, double*&,
                                                              double*&, double*&);
