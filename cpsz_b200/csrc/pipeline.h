// pipeline.h -- host orchestration entry points shared by the C ABI layer.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "kernels.h"
#include "runtime.h"

namespace cpsz {

// Result of a compression call: the blob lives in the context's arena until
// the next call on the same context.
struct Blob2D {
  uint8_t* d_blob = nullptr;
  size_t size = 0;
  size_t n_unpred[2] = {0, 0};
};

// Optional device-side copies of intermediate stages (parity tests).
struct StageTap {
  uint8_t* ids = nullptr;                    // 2N id bytes (ID_ZERO = precision 0)
  uint16_t* codes_blocks[2] = {nullptr, nullptr};
  float* unpred[2] = {nullptr, nullptr};
  float* recon[2] = {nullptr, nullptr};      // compressor-side reconstruction (raster)
  bool recon_only = false;                   // stop after the Lorenzo stage (no blob)
  // With given bounds and recon_only: the vertices (N bytes, 16-byte aligned)
  // whose bound changed since the previous recon_only pass over the same
  // field on this context, whose workspace (ids, wavefront pairs) nothing has
  // touched since.  Only they are quantized again; the mask is cleared.
  uint8_t* requant = nullptr;
  // With requant: the first WAVE_GROUP_ROWS-row group holding one of those
  // vertices.  The groups above keep the previous pass's reconstruction (the
  // recursion reads only rows above and to the left) and are not run again.
  int first_group = 0;
};

int build_wave_items(int nfields, const int* r1s, std::vector<WaveItem>& items);

// eb_ext (optional, device, N doubles): per-vertex bounds to quantize instead
// of the derived ones (the learned-bound path).  host_out (optional, of
// host_cap bytes): host memory gets the blob written there directly
// (out->d_blob is then not set); a device buffer with room for the blob's
// bound gets the blob built in place (out->d_blob == host_out), else the blob
// is built in the workspace (out->d_blob) and the caller copies it.
// log_form: the offline_log blob (src/sz_compress_cp_preserve_2d.cpp:285-379)
// instead of the offline one.
int compress_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                Blob2D* out, const StageTap* tap, const double* eb_ext = nullptr, unsigned char* host_out = nullptr,
                size_t host_cap = 0, bool log_form = false);
int decompress_2d(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, float* U,
                  float* V, bool log_form = false);
// n fields; blobs back to back into `out` (host or device), offsets[0..n].
int compress_2d_batch(cpsz_b200_ctx* ctx, int n, const float* const* U, const float* const* V, const size_t* r1,
                      const size_t* r2, const double* ebs, unsigned char* out, size_t out_cap, size_t* offsets);

struct Blob3D {
  uint8_t* d_blob = nullptr;
  size_t size = 0;
  size_t n_unpred = 0;  // floats (3 per unpredictable point)
  size_t n_codes = 0;   // codes (3 per predicted point)
};
int compress_3d(cpsz_b200_ctx* ctx, const float* U, const float* V, const float* W, size_t r1, size_t r2, size_t r3,
                double max_pwr_eb, Blob3D* out);
int decompress_3d(cpsz_b200_ctx* ctx, const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, size_t r3,
                  float* U, float* V, float* W);

// Copies n bytes from device memory to `dst`, which may be host or device memory.
int copy_out(cpsz_b200_ctx* ctx, void* dst, const void* d_src, size_t n);
// Copies n bytes from `src` (host or device) into device memory `d_dst`.
int copy_in(cpsz_b200_ctx* ctx, void* d_dst, const void* src, size_t n);

}  // namespace cpsz
