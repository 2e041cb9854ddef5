// mlp.cu -- the learned error-bound proposer's tensor-core kernels (tcgen05,
// BF16 operands, FP32 accumulation in TMEM).
#include <cuda_bf16.h>

#include "kernels.h"
#include "umma.cuh"

namespace cpsz {

namespace {

constexpr uint32_t WAIT_LIMIT = 1u << 22;

// One 128 x 128 x 128 tile product D = A B^T through shared memory and TMEM
// (the building block every MLP kernel uses), for self-checks.
__global__ void __launch_bounds__(128, 1) umma_selftest_kernel(const __nv_bfloat16* __restrict__ A,
                                                               const __nv_bfloat16* __restrict__ B,
                                                               float* __restrict__ D, int* __restrict__ flag) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sa = smem;
  uint8_t* sb = smem + umma::TILE_BYTES;
  uint64_t* mbar = (uint64_t*)(smem + 2 * umma::TILE_BYTES);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < 128 * 128; e += 128) {
    const int r = e >> 7, k = e & 127;
    *(__nv_bfloat16*)(sa + umma::tile_off(r, k)) = A[e];
    *(__nv_bfloat16*)(sb + umma::tile_off(r, k)) = B[e];
  }
  if (tid == 0) umma::mbar_init(mbar, 1);
  if (warp == 0) {
    umma::tmem_alloc(tslot, 128);
    umma::tmem_relinquish();
  }
  umma::fence_async_shared();
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    umma::gemm_tile(tmem, umma::smem_addr(sa), umma::smem_addr(sb), false);
    umma::mma_commit(mbar);
  }
  const bool ok = umma::mbar_wait(mbar, 0, WAIT_LIMIT);
  umma::tc_fence_after();
  if (ok) {
    const int row = warp * 32 + (tid & 31);
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + c, v);
      for (int q = 0; q < 16; q++) D[row * 128 + c + q] = v[q];
    }
  } else if (tid == 0) {
    atomicOr(flag, FLAG_TIMEOUT);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

}  // namespace

int launch_umma_selftest(cpsz_b200_ctx* ctx, const void* A, const void* B, float* D) {
  const int smem = 2 * umma::TILE_BYTES + 64;
  static bool attr = false;
  if (!attr) {
    CPSZ_CUDA_TRY(cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  umma_selftest_kernel<<<1, 128, smem, ctx->stream>>>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, D,
                                                      ctx->d_flag);
  count_launch(ctx);
  return check_launch("umma_selftest_kernel");
}

}  // namespace cpsz
