// log2d.cu -- the log-domain steps of the 2D offline_log pair.
//
// sz_compress_cp_preserve_2d_offline_log (src/sz_compress_cp_preserve_2d.cpp:285-379)
// compresses log2f|U| and log2f|V| (log_transform, include/sz_cp_preserve_utils.hpp:205-221:
// -100 for a zero, a sign bit x > 0 per value) with one per-vertex precision
// 2^id * 2^-52 taken from log2(1 + eb); the decoder
// (src/sz_decompress_cp_preserve_2d.cpp:56-99) maps decoded logs below -99 to
// 0 and the others to +-exp2f(log).  Both log2f and exp2f are the host C
// library's, reproduced bit for bit through the tables of libm.h.
//
// Sign maps are MSB-first bit streams, 8 values per byte
// (convertIntArray2ByteArray_fast_1b_to_result_sz, src/sz_compression_utils.cpp:31-52),
// built a warp at a time from a ballot: 32 values make one 32-bit word
// whose bytes are in stream order.
#include "kernels.h"
#include "libm_dev.cuh"

namespace cpsz {

namespace {

__global__ void __launch_bounds__(256) log2d_kernel(const float* __restrict__ U, const float* __restrict__ V,
                                                    const uint8_t* __restrict__ ids, size_t n, LibmFn L,
                                                    float2* __restrict__ pair_u, float2* __restrict__ pair_v,
                                                    float* __restrict__ log_u, float* __restrict__ log_v,
                                                    uint32_t* __restrict__ sign_u, uint32_t* __restrict__ sign_v) {
  const int lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t base = (size_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
    const size_t idx = base + lane;
    float x[2] = {0.f, 0.f};
    int id = ID_ZERO;
    if (idx < n) {
      x[0] = __ldg(U + idx);
      x[1] = __ldg(V + idx);
      id = __ldg(ids + idx);
    }
    // 1/precision = 2^(52 - id); NaN marks precision 0
    const float inv = id == ID_ZERO ? __uint_as_float(0x7fc00000u) : __uint_as_float((uint32_t)(127 + 52 - id) << 23);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const unsigned bal = __ballot_sync(0xffffffffu, x[c] > 0.f);
      if (lane == 0) (c ? sign_v : sign_u)[base >> 5] = __byte_perm(__brev(bal), 0, 0x0123);
      const float lg = (x[c] != 0.f) ? dev::host_log2f(fabsf(x[c]), L) : -100.f;
      if (idx < n) {
        (c ? pair_v : pair_u)[idx] = make_float2(lg, inv);
        (c ? log_v : log_u)[idx] = lg;
      }
    }
  }
}

__global__ void __launch_bounds__(256) exp2d_kernel(float* __restrict__ U, float* __restrict__ V,
                                                    const uint8_t* __restrict__ sign_u,
                                                    const uint8_t* __restrict__ sign_v, size_t n, LibmFn Ex) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
    const unsigned byte_bit = 7u - (unsigned)(idx & 7);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      float* X = c ? V : U;
      const float lg = X[idx];
      const bool pos = (__ldg((c ? sign_v : sign_u) + (idx >> 3)) >> byte_bit) & 1u;
      float out = 0.f;
      if (!(lg < -99.f)) {
        const float e = dev::host_exp2f(lg, Ex);
        out = pos ? e : -e;
      }
      X[idx] = out;
    }
  }
}

int grid_of(cpsz_b200_ctx* ctx, size_t n) {
  const size_t blocks = (n + 255) / 256, cap = (size_t)ctx->num_sms * 16;
  return (int)(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

}  // namespace

int launch_log2d(cpsz_b200_ctx* ctx, const float* U, const float* V, const uint8_t* ids, size_t n, const LibmFn& L,
                 float2* pair_u, float2* pair_v, float* log_u, float* log_v, uint32_t* sign_u, uint32_t* sign_v) {
  if (n == 0) return CPSZ_OK;
  log2d_kernel<<<grid_of(ctx, n), 256, 0, ctx->stream>>>(U, V, ids, n, L, pair_u, pair_v, log_u, log_v, sign_u,
                                                         sign_v);
  count_launch(ctx);
  return check_launch("log2d_kernel");
}

int launch_exp2d(cpsz_b200_ctx* ctx, float* U, float* V, const uint8_t* sign_u, const uint8_t* sign_v, size_t n,
                 const LibmFn& Ex) {
  if (n == 0) return CPSZ_OK;
  exp2d_kernel<<<grid_of(ctx, n), 256, 0, ctx->stream>>>(U, V, sign_u, sign_v, n, Ex);
  count_launch(ctx);
  return check_launch("exp2d_kernel");
}

}  // namespace cpsz
