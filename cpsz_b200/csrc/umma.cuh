// umma.cuh -- minimal sm_100a tensor-core (tcgen05) building blocks for the
// learned-bound MLP: shared-memory matrix descriptors, the BF16 -> FP32
// instruction descriptor, TMEM allocation / loads, MMA issue and completion
// through an mbarrier with a bounded wait.
//
// Operand tiles are 128 (rows, M or N) x 128 (K) BF16 in the no-swizzle
// K-major canonical layout: 8-row x 16-byte core matrices (128 contiguous
// bytes); core matrix (row block rb, K chunk kc) sits at (kc * 16 + rb) * 128.
// One MMA consumes K = 16 (two K chunks): leading-byte offset (next K chunk)
// 2048 B, stride-byte offset (next 8-row block) 128 B.  Bit layouts follow
// the descriptor definitions in CUTLASS (cute/arch/mma_sm100_desc.hpp).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace cpsz {
namespace umma {

constexpr int TILE = 128;                      // rows x K of one operand tile
constexpr int TILE_BYTES = TILE * TILE * 2;    // 32 KB
constexpr uint32_t LBO = 2048, SBO = 128;

// byte offset of element (row, k) inside a canonical tile
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((((k >> 3) * 16 + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// SmemDescriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
// version 1 [46,48), base offset 0, LBO mode 0, layout SWIZZLE_NONE (0) [61,64)
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((LBO >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((SBO >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// InstrDescriptor, kind::f16: D F32 [4,6)=1, A BF16 [7,10)=1, B BF16 [10,13)=1,
// both K-major, N >> 3 at [17,23), M >> 4 at [24,29)
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- TMEM -------------------------------------------------------------------------
// One warp allocates `ncols` columns (power of two >= 32); the address lands in
// shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w of a
// warpgroup reads lanes 32 w .. 32 w + 31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// ---- MMA ----------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The mbarrier receives one arrival when all MMAs issued so far by this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

// D (128 x 128 F32 in TMEM at tmem_d) (+)= A (128 x 128) * B (128 x 128)^T,
// both canonical K-major tiles in shared memory.  One thread issues.
__device__ __forceinline__ void gemm_tile(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, bool accumulate) {
  constexpr uint32_t idesc = idesc_bf16_f32(128, 128);
#pragma unroll
  for (int s = 0; s < TILE / 16; s++) {
    // K step s covers K chunks 2s, 2s+1: start advances by 2 * LBO
    const uint64_t ad = desc_kmajor(a_saddr + s * 2 * LBO);
    const uint64_t bd = desc_kmajor(b_saddr + s * 2 * LBO);
    mma_bf16(tmem_d, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
  }
}

// ---- mbarrier ---------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for phase `parity` to complete, at most `limit` polls; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_addr(mbar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace umma
}  // namespace cpsz
