// C-ABI shim over the reference cpSZ implementation, compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/libcpsz_ref.so.
// TEST INFRASTRUCTURE ONLY: used by tests/ (to pin the restated oracle and the
// CUDA path) and by bench.py's CPU-baseline arm.  Nothing in the product links it.
//
// Wrapped entry points (reference file:line):
//   sz_compress_cp_preserve_2d_offline     include/sz_compress_cp_preserve_2d.hpp:10
//   sz_decompress_cp_preserve_2d_offline   include/sz_decompress_cp_preserve_2d.hpp:11
//   sz_compress_cp_preserve_2d_offline_log include/sz_compress_cp_preserve_2d.hpp:14
//   sz_decompress_cp_preserve_2d_offline_log include/sz_decompress_cp_preserve_2d.hpp:15
//   sz_compress_cp_preserve_3d_offline_log include/sz_compress_cp_preserve_3d.hpp:8
//   sz_decompress_cp_preserve_3d_online_log include/sz_decompress_cp_preserve_3d.hpp:11
//   sz_lossless_compress / _decompress     include/sz_lossless.hpp:13-14
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <fcntl.h>
#include "sz_compress_cp_preserve_2d.hpp"
#include "sz_decompress_cp_preserve_2d.hpp"
#include "sz_compress_cp_preserve_3d.hpp"
#include "sz_decompress_cp_preserve_3d.hpp"
#include "sz_lossless.hpp"

namespace {
// The reference prints progress to stdout on every call; silence it so test
// output stays readable.  Re-entrant use is not needed (tests are serial).
struct Quiet {
  int saved = -1;
  Quiet() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
  }
  ~Quiet() {
    fflush(stdout);
    if (saved >= 0) { dup2(saved, 1); close(saved); }
  }
};
}  // namespace

extern "C" {

unsigned char* cpsz_ref_compress_2d_offline_f32(const float* U, const float* V, size_t r1, size_t r2,
                                                double max_pwr_eb, size_t* out_size) {
  Quiet q;
  size_t sz = 0;
  unsigned char* p = sz_compress_cp_preserve_2d_offline<float>(U, V, r1, r2, sz, false, max_pwr_eb);
  *out_size = sz;
  return p;
}

int cpsz_ref_decompress_2d_offline_f32(const unsigned char* blob, size_t r1, size_t r2, float* U_out,
                                       float* V_out) {
  Quiet q;
  float* U = nullptr;
  float* V = nullptr;
  sz_decompress_cp_preserve_2d_offline<float>(blob, r1, r2, U, V);
  memcpy(U_out, U, r1 * r2 * sizeof(float));
  memcpy(V_out, V, r1 * r2 * sizeof(float));
  free(U);
  free(V);
  return 0;
}

unsigned char* cpsz_ref_compress_2d_offline_log_f32(const float* U, const float* V, size_t r1, size_t r2,
                                                    double max_pwr_eb, size_t* out_size) {
  Quiet q;
  size_t sz = 0;
  unsigned char* p = sz_compress_cp_preserve_2d_offline_log<float>(U, V, r1, r2, sz, false, max_pwr_eb);
  *out_size = sz;
  return p;
}

int cpsz_ref_decompress_2d_offline_log_f32(const unsigned char* blob, size_t r1, size_t r2, float* U_out,
                                           float* V_out) {
  Quiet q;
  float* U = nullptr;
  float* V = nullptr;
  sz_decompress_cp_preserve_2d_offline_log<float>(blob, r1, r2, U, V);
  memcpy(U_out, U, r1 * r2 * sizeof(float));
  memcpy(V_out, V, r1 * r2 * sizeof(float));
  free(U);
  free(V);
  return 0;
}

unsigned char* cpsz_ref_compress_3d_offline_log_f32(const float* U, const float* V, const float* W, size_t r1,
                                                    size_t r2, size_t r3, double max_pwr_eb, size_t* out_size) {
  Quiet q;
  size_t sz = 0;
  unsigned char* p = sz_compress_cp_preserve_3d_offline_log<float>(U, V, W, r1, r2, r3, sz, false, max_pwr_eb);
  *out_size = sz;
  return p;
}

int cpsz_ref_decompress_3d_online_log_f32(const unsigned char* blob, size_t r1, size_t r2, size_t r3,
                                          float* U_out, float* V_out, float* W_out) {
  Quiet q;
  float* U = nullptr;
  float* V = nullptr;
  float* W = nullptr;
  sz_decompress_cp_preserve_3d_online_log<float>(blob, r1, r2, r3, U, V, W);
  size_t n = r1 * r2 * r3;
  memcpy(U_out, U, n * sizeof(float));
  memcpy(V_out, V, n * sizeof(float));
  memcpy(W_out, W, n * sizeof(float));
  free(U);
  free(V);
  free(W);
  return 0;
}

size_t cpsz_ref_zstd_compress(const unsigned char* data, size_t n, unsigned char** out) {
  return sz_lossless_compress(ZSTD_COMPRESSOR, 3, const_cast<unsigned char*>(data), n, out);
}

size_t cpsz_ref_zstd_decompress(const unsigned char* data, size_t n, unsigned char** out, size_t target) {
  return sz_lossless_decompress(ZSTD_COMPRESSOR, const_cast<unsigned char*>(data), n, out, target);
}

void cpsz_ref_free(void* p) { free(p); }

}  // extern "C"
