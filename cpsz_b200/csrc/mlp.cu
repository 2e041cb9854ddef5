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


// ---- the MLP: 99 (padded to 128) -> 128 -> 128 -> 1, ReLU ---------------------------
// Parameters (fp32 master copy, flat): W1 [128 x 128] (row = hidden unit, col =
// input; inputs 99..127 are zero padding), b1 [128], W2 [128 x 128], b2 [128],
// w3 [128], b3.  BF16 copies of W1 / W2 feed the tensor cores.
constexpr int MLP_FEAT = 99;
constexpr int MLP_PATCH = 7;

__device__ __forceinline__ void store_row_chunk(uint8_t* tile, int row, int k0, const float* v8) {
  // 8 consecutive K elements of one row: one 16-byte store in the canonical layout
  __nv_bfloat162 h[4];
#pragma unroll
  for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(v8[2 * q], v8[2 * q + 1]);
  *(uint4*)(tile + umma::tile_off(row, k0)) = *(uint4*)h;
}

// W (row-major [mn][k] bf16, 128 x 128) into a canonical tile (transpose:
// element W[a][b] goes to (mn = b, k = a)).
__device__ void load_weight_tile(uint8_t* tile, const __nv_bfloat16* __restrict__ W, bool transpose) {
  for (int e = threadIdx.x; e < 128 * 16; e += blockDim.x) {
    const int row = e >> 4, c = (e & 15) * 8;
    if (!transpose) {
      *(uint4*)(tile + umma::tile_off(row, c)) = *(const uint4*)(W + row * 128 + c);
    } else {
      const __nv_bfloat16* src = W + row * 128 + c;
      for (int q = 0; q < 8; q++) *(__nv_bfloat16*)(tile + umma::tile_off(c + q, row)) = src[q];
    }
  }
}

// The 99 features of vertex (i, j): its 7 x 7 neighbourhood of (u, v) (zero
// outside the field) divided by the neighbourhood's largest |value| (1 when all
// zero), then log2 of the analytic bound / 32 (bound floored at 1e-30).
__device__ void vertex_features(const float* __restrict__ U, const float* __restrict__ V, int r1, int r2, int i,
                                int j, double eb_a, float* f) {
  float mx = 0.f;
  for (int di = 0; di < MLP_PATCH; di++)
    for (int dj = 0; dj < MLP_PATCH; dj++) {
      const int ii = i + di - 3, jj = j + dj - 3;
      float u = 0.f, v = 0.f;
      if (ii >= 0 && ii < r1 && jj >= 0 && jj < r2) {
        u = __ldg(U + (size_t)ii * r2 + jj);
        v = __ldg(V + (size_t)ii * r2 + jj);
      }
      f[di * MLP_PATCH + dj] = u;
      f[49 + di * MLP_PATCH + dj] = v;
      mx = fmaxf(mx, fmaxf(fabsf(u), fabsf(v)));
    }
  const float s = (mx > 0.f && isfinite(mx)) ? 1.f / mx : 1.f;
  for (int k = 0; k < 98; k++) f[k] *= s;
  f[98] = (float)(log2(fmax(eb_a, 1e-30)) / 32.0);
}

struct FwdArgs {
  // features: either X (global bf16 rows of 128) or computed from a field
  const __nv_bfloat16* X;
  const float* U;
  const float* V;
  const double* eb_a;
  int r1, r2;
  int M;
  const __nv_bfloat16* w1b;
  const __nv_bfloat16* w2b;
  const float* p;
  float* y;
  __nv_bfloat16* H1;  // optional activations (training)
  __nv_bfloat16* H2;
  int* flag;
};

constexpr int FWD_SMEM = 4 * umma::TILE_BYTES + 64;

template <bool kFieldFeatures>
__global__ void __launch_bounds__(128, 1) mlp_fwd_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* W1s = smem;
  uint8_t* W2s = smem + umma::TILE_BYTES;
  uint8_t* Xs = smem + 2 * umma::TILE_BYTES;
  uint8_t* As = smem + 3 * umma::TILE_BYTES;
  uint64_t* mbar = (uint64_t*)(smem + 4 * umma::TILE_BYTES);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const float* b1 = a.p + 16384;
  const float* b2 = a.p + 2 * 16384 + 128;
  const float* w3 = a.p + 2 * 16384 + 256;
  const float b3 = a.p[2 * 16384 + 384];
  load_weight_tile(W1s, a.w1b, false);
  load_weight_tile(W2s, a.w2b, false);
  if (tid == 0) umma::mbar_init(mbar, 1);
  if (warp == 0) {
    umma::tmem_alloc(tslot, 256);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (a.M + 127) / 128;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row = tile * 128 + tid;
    const bool valid = row < a.M;
    if (kFieldFeatures) {
      float f[128];
      if (valid) {
        const int i = row / a.r2, j = row - (row / a.r2) * a.r2;
        vertex_features(a.U, a.V, a.r1, a.r2, i, j, a.eb_a[row], f);
      } else {
        for (int k = 0; k < MLP_FEAT; k++) f[k] = 0.f;
      }
      for (int k = MLP_FEAT; k < 128; k++) f[k] = 0.f;
      for (int c = 0; c < 128; c += 8) store_row_chunk(Xs, tid, c, f + c);
    } else {
      for (int c = 0; c < 128; c += 8) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (valid) v = *(const uint4*)(a.X + (size_t)row * 128 + c);
        *(uint4*)(Xs + umma::tile_off(tid, c)) = v;
      }
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    if (tid == 0) {
      umma::gemm_tile(tmem, umma::smem_addr(Xs), umma::smem_addr(W1s), false);
      umma::mma_commit(mbar);
    }
    // every thread takes the same branch after a bounded wait
    ok = __syncthreads_and(umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    if (!ok) break;
    // epilogue 1: h1 = relu(x W1^T + b1) -> bf16 operand of layer 2
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + c, v);
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = fmaxf(v[q] + b1[c + q], 0.f);
      store_row_chunk(As, tid, c, v);
      store_row_chunk(As, tid, c + 8, v + 8);
      if (a.H1 && valid) {
        *(uint4*)(a.H1 + (size_t)row * 128 + c) = *(const uint4*)(As + umma::tile_off(tid, c));
        *(uint4*)(a.H1 + (size_t)row * 128 + c + 8) = *(const uint4*)(As + umma::tile_off(tid, c + 8));
      }
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    if (tid == 0) {
      umma::gemm_tile(tmem + 128, umma::smem_addr(As), umma::smem_addr(W2s), false);
      umma::mma_commit(mbar);
    }
    // every thread takes the same branch after a bounded wait
    ok = __syncthreads_and(umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    if (!ok) break;
    // epilogue 2: h2 = relu(h1 W2^T + b2); y = h2 . w3 + b3
    float acc = b3;
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + 128 + c, v);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        v[q] = fmaxf(v[q] + b2[c + q], 0.f);
        acc += v[q] * w3[c + q];
      }
      if (a.H2 && valid) {
        __nv_bfloat162 h[8];
#pragma unroll
        for (int q = 0; q < 8; q++) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        *(uint4*)(a.H2 + (size_t)row * 128 + c) = *(uint4*)h;
        *(uint4*)(a.H2 + (size_t)row * 128 + c + 8) = *(uint4*)(h + 4);
      }
    }
    if (valid) a.y[row] = acc;
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
  }
  if (!ok && tid == 0) atomicOr(a.flag, FLAG_TIMEOUT);
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

// The forward pass on field features with two 128-row tiles in flight per
// CTA: warps 0-3 and 4-7 are two independent pipelines (features -> layer 1
// on the tensor cores -> epilogue -> layer 2 -> epilogue), each with its own
// operand tiles, TMEM columns (256 each of the CTA's 512), mbarrier and named
// barrier, so one pipeline's feature gathers overlap the other's MMAs and
// epilogues.  The weights are shared.  Same arithmetic per row as
// mlp_fwd_kernel<true>.
constexpr int FWD2_SMEM = 6 * umma::TILE_BYTES + 64;

__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }
// AND of v over the 128 threads of group g (a named barrier)
__device__ __forceinline__ bool group_and(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + g)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(256, 1) mlp_fwd2_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, g = warp >> 2, gt = tid & 127;
  uint8_t* W1s = smem;
  uint8_t* W2s = smem + umma::TILE_BYTES;
  uint8_t* Xs = smem + (2 + 2 * g) * umma::TILE_BYTES;
  uint8_t* As = smem + (3 + 2 * g) * umma::TILE_BYTES;
  uint64_t* mbars = (uint64_t*)(smem + 6 * umma::TILE_BYTES);
  uint64_t* mbar = mbars + g;
  uint32_t* tslot = (uint32_t*)(mbars + 2);
  const float* b1 = a.p + 16384;
  const float* b2 = a.p + 2 * 16384 + 128;
  const float* w3 = a.p + 2 * 16384 + 256;
  const float b3 = a.p[2 * 16384 + 384];
  load_weight_tile(W1s, a.w1b, false);
  load_weight_tile(W2s, a.w2b, false);
  if (gt == 0) umma::mbar_init(mbar, 1);
  if (warp == 0) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t tmem = tbase + 256 * g;  // this pipeline's columns
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (a.M + 127) / 128;
  for (int tile = 2 * blockIdx.x + g; tile < ntiles && ok; tile += 2 * gridDim.x) {
    const int row = tile * 128 + gt;
    const bool valid = row < a.M;
    {
      float f[128];
      if (valid) {
        const int i = row / a.r2, j = row - (row / a.r2) * a.r2;
        vertex_features(a.U, a.V, a.r1, a.r2, i, j, a.eb_a[row], f);
      } else {
        for (int k = 0; k < MLP_FEAT; k++) f[k] = 0.f;
      }
      for (int k = MLP_FEAT; k < 128; k++) f[k] = 0.f;
      for (int c = 0; c < 128; c += 8) store_row_chunk(Xs, gt, c, f + c);
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    if (gt == 0) {
      umma::gemm_tile(tmem, umma::smem_addr(Xs), umma::smem_addr(W1s), false);
      umma::mma_commit(mbar);
    }
    // every thread of the pipeline takes the same branch after a bounded wait
    ok = group_and(g, umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    if (!ok) break;
    // epilogue 1: h1 = relu(x W1^T + b1) -> bf16 operand of layer 2
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + c, v);
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = fmaxf(v[q] + b1[c + q], 0.f);
      store_row_chunk(As, gt, c, v);
      store_row_chunk(As, gt, c + 8, v + 8);
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
    if (gt == 0) {
      umma::gemm_tile(tmem + 128, umma::smem_addr(As), umma::smem_addr(W2s), false);
      umma::mma_commit(mbar);
    }
    ok = group_and(g, umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    if (!ok) break;
    // epilogue 2: h2 = relu(h1 W2^T + b2); y = h2 . w3 + b3
    float acc = b3;
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + 128 + c, v);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        v[q] = fmaxf(v[q] + b2[c + q], 0.f);
        acc += v[q] * w3[c + q];
      }
    }
    if (valid) a.y[row] = acc;
    umma::tc_fence_before();
    group_sync(g);
    umma::tc_fence_after();
  }
  if (!ok && gt == 0) atomicOr(a.flag, FLAG_TIMEOUT);
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, 512);
}

struct BwdArgs {
  const __nv_bfloat16* X;
  const __nv_bfloat16* H1;
  const __nv_bfloat16* H2;
  const float* y;
  const float* t;
  int M;
  float grad_scale;  // dL/dy = grad_scale * (y - t)
  const __nv_bfloat16* w2b;
  const float* p;
  float* g;     // gradient accumulators (flat, as p)
  float* loss;  // sum of (y - t)^2
  int* flag;
};

constexpr int BWD_SMEM = 4 * umma::TILE_BYTES + 3 * 128 * 4 + 64;

__global__ void __launch_bounds__(128, 1) mlp_bwd_kernel(BwdArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* W2T = smem;                          // (mn = i, k = o) = W2[o][i]
  uint8_t* P = smem + umma::TILE_BYTES;         // dZ2 (mn = r, k = o)
  uint8_t* Q = smem + 2 * umma::TILE_BYTES;     // dZ2^T, later dZ1^T
  uint8_t* R = smem + 3 * umma::TILE_BYTES;     // H1^T, later X^T
  float* red = (float*)(smem + 4 * umma::TILE_BYTES);  // db1 | db2 | dw3
  uint64_t* mbar = (uint64_t*)(red + 3 * 128);
  uint32_t* tslot = (uint32_t*)(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const float* w3 = a.p + 2 * 16384 + 256;
  load_weight_tile(W2T, a.w2b, true);
  for (int k = tid; k < 3 * 128; k += 128) red[k] = 0.f;
  if (tid == 0) umma::mbar_init(mbar, 1);
  if (warp == 0) {
    umma::tmem_alloc(tslot, 512);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true, first = true;
  float loss = 0.f, db3 = 0.f;
  const int ntiles = (a.M + 127) / 128;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row = tile * 128 + tid;
    const bool valid = row < a.M;
    float dy = 0.f;
    if (valid) {
      const float e = a.y[row] - a.t[row];
      loss += e * e;
      dy = a.grad_scale * e;
    }
    db3 += dy;
    // dZ2 = dy w3 (h2 > 0); dw3 += dy h2; db2 += dZ2
    for (int c = 0; c < 128; c += 8) {
      float h2[8], dz[8];
      uint4 raw = make_uint4(0, 0, 0, 0);
      if (valid) raw = *(const uint4*)(a.H2 + (size_t)row * 128 + c);
      const __nv_bfloat16* hb = (const __nv_bfloat16*)&raw;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        h2[q] = __bfloat162float(hb[q]);
        dz[q] = h2[q] > 0.f ? dy * w3[c + q] : 0.f;
        atomicAdd(&red[256 + c + q], dy * h2[q]);
        atomicAdd(&red[128 + c + q], dz[q]);
      }
      store_row_chunk(P, tid, c, dz);
#pragma unroll
      for (int q = 0; q < 8; q++) *(__nv_bfloat16*)(Q + umma::tile_off(c + q, tid)) = __float2bfloat16_rn(dz[q]);
      uint4 h1raw = make_uint4(0, 0, 0, 0);
      if (valid) h1raw = *(const uint4*)(a.H1 + (size_t)row * 128 + c);
      const __nv_bfloat16* h1b = (const __nv_bfloat16*)&h1raw;
#pragma unroll
      for (int q = 0; q < 8; q++) *(__nv_bfloat16*)(R + umma::tile_off(c + q, tid)) = h1b[q];
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    if (tid == 0) {
      umma::gemm_tile(tmem, umma::smem_addr(Q), umma::smem_addr(R), !first);  // dW2 += dZ2^T H1
      umma::gemm_tile(tmem + 128, umma::smem_addr(P), umma::smem_addr(W2T), false);  // dH1 = dZ2 W2
      umma::mma_commit(mbar);
    }
    // every thread takes the same branch after a bounded wait
    ok = __syncthreads_and(umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    if (!ok) break;
    // dZ1 = dH1 (h1 > 0); db1 += dZ1; operands for dW1 = dZ1^T X
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + 128 + c, v);
      for (int half = 0; half < 2; half++) {
        const int cc = c + 8 * half;
        uint4 h1raw = make_uint4(0, 0, 0, 0), xraw = make_uint4(0, 0, 0, 0);
        if (valid) {
          h1raw = *(const uint4*)(a.H1 + (size_t)row * 128 + cc);
          xraw = *(const uint4*)(a.X + (size_t)row * 128 + cc);
        }
        const __nv_bfloat16* h1b = (const __nv_bfloat16*)&h1raw;
        const __nv_bfloat16* xb = (const __nv_bfloat16*)&xraw;
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const float dz = (valid && __bfloat162float(h1b[q]) > 0.f) ? v[8 * half + q] : 0.f;
          atomicAdd(&red[cc + q], dz);
          *(__nv_bfloat16*)(Q + umma::tile_off(cc + q, tid)) = __float2bfloat16_rn(dz);
          *(__nv_bfloat16*)(R + umma::tile_off(cc + q, tid)) = xb[q];
        }
      }
    }
    umma::fence_async_shared();
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    if (tid == 0) {
      umma::gemm_tile(tmem + 256, umma::smem_addr(Q), umma::smem_addr(R), !first);  // dW1 += dZ1^T X
      umma::mma_commit(mbar);
    }
    // every thread takes the same branch after a bounded wait
    ok = __syncthreads_and(umma::mbar_wait(mbar, phase, WAIT_LIMIT));
    phase ^= 1;
    umma::tc_fence_after();
    first = false;
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
  }
  if (!ok && tid == 0) atomicOr(a.flag, FLAG_TIMEOUT);
  if (ok && !first) {
    // this CTA's weight gradients: lane = output unit
    for (int c = 0; c < 128; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_addr + c, v);
      for (int q = 0; q < 16; q++) atomicAdd(&a.g[16384 + 128 + tid * 128 + c + q], v[q]);  // dW2
      umma::tmem_ld16(lane_addr + 256 + c, v);
      for (int q = 0; q < 16; q++) atomicAdd(&a.g[tid * 128 + c + q], v[q]);  // dW1
    }
  }
  __syncthreads();
  atomicAdd(&a.g[16384 + tid], red[tid]);                  // db1
  atomicAdd(&a.g[2 * 16384 + 128 + tid], red[128 + tid]);  // db2
  atomicAdd(&a.g[2 * 16384 + 256 + tid], red[256 + tid]);  // dw3
  for (int o = 16; o; o >>= 1) {
    loss += __shfl_xor_sync(0xffffffffu, loss, o);
    db3 += __shfl_xor_sync(0xffffffffu, db3, o);
  }
  if ((tid & 31) == 0) {
    atomicAdd(a.loss, loss);
    atomicAdd(&a.g[2 * 16384 + 384], db3);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// Adam on the flat parameters; clears the gradients and refreshes the BF16
// weight copies.
__global__ void mlp_adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                                float c2, __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    // padded input columns of W1 stay zero
    if (i < 16384 && (i & 127) >= MLP_FEAT) pi = 0.f;
    p[i] = pi;
    g[i] = 0.f;
    if (i < 16384) w1b[i] = __float2bfloat16_rn(pi);
    else if (i >= 16384 + 128 && i < 2 * 16384 + 128) w2b[i - 16384 - 128] = __float2bfloat16_rn(pi);
  }
}

__global__ void mlp_cast_kernel(const float* __restrict__ p, __nv_bfloat16* __restrict__ w1b,
                                __nv_bfloat16* __restrict__ w2b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 16384; i += gridDim.x * blockDim.x) {
    w1b[i] = __float2bfloat16_rn(p[i]);
    w2b[i] = __float2bfloat16_rn(p[16384 + 128 + i]);
  }
}

__global__ void features_kernel(const float* __restrict__ U, const float* __restrict__ V, int r1, int r2,
                                const double* __restrict__ eb_a, const int* __restrict__ idx, int n,
                                __nv_bfloat16* __restrict__ X) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = idx[s];
    const int i = v / r2, j = v - (v / r2) * r2;
    float f[128];
    vertex_features(U, V, r1, r2, i, j, eb_a[v], f);
    for (int k = MLP_FEAT; k < 128; k++) f[k] = 0.f;
    for (int c = 0; c < 128; c += 8) {
      __nv_bfloat162 h[4];
      for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(f[c + 2 * q], f[c + 2 * q + 1]);
      *(uint4*)(X + (size_t)s * 128 + c) = *(uint4*)h;
    }
  }
}

template <class K>
int set_smem(K kernel, int bytes) {
  CPSZ_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return CPSZ_OK;
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

int launch_mlp_forward(cpsz_b200_ctx* ctx, const MlpParams& w, const void* X, const float* U, const float* V,
                       const double* eb_a, int r1, int r2, int M, float* y, void* H1, void* H2) {
  static bool attr = false;
  if (!attr) {
    CPSZ_TRY(set_smem(mlp_fwd_kernel<false>, FWD_SMEM));
    CPSZ_TRY(set_smem(mlp_fwd_kernel<true>, FWD_SMEM));
    CPSZ_TRY(set_smem(mlp_fwd2_kernel, FWD2_SMEM));
    attr = true;
  }
  if (M <= 0) return CPSZ_OK;
  FwdArgs a{(const __nv_bfloat16*)X, U, V, eb_a, r1, r2, M, (const __nv_bfloat16*)w.w1b, (const __nv_bfloat16*)w.w2b,
            w.p, y, (__nv_bfloat16*)H1, (__nv_bfloat16*)H2, ctx->d_flag};
  const int ntiles = (M + 127) / 128;
  if (!X && !H1 && !H2) {
    // field features, no activations kept: two tiles in flight per CTA
    const int pairs = (ntiles + 1) / 2;
    const int grid2 = pairs < ctx->num_sms ? pairs : ctx->num_sms;
    mlp_fwd2_kernel<<<grid2, 256, FWD2_SMEM, ctx->stream>>>(a);
    count_launch(ctx);
    return check_launch("mlp_fwd2_kernel");
  }
  const int grid = ntiles < ctx->num_sms ? ntiles : ctx->num_sms;
  if (X) mlp_fwd_kernel<false><<<grid, 128, FWD_SMEM, ctx->stream>>>(a);
  else mlp_fwd_kernel<true><<<grid, 128, FWD_SMEM, ctx->stream>>>(a);
  count_launch(ctx);
  return check_launch("mlp_fwd_kernel");
}

int launch_mlp_backward(cpsz_b200_ctx* ctx, const MlpParams& w, const void* X, const void* H1, const void* H2,
                        const float* y, const float* t, int M, float grad_scale, float* loss) {
  static bool attr = false;
  if (!attr) {
    CPSZ_TRY(set_smem(mlp_bwd_kernel, BWD_SMEM));
    attr = true;
  }
  if (M <= 0) return CPSZ_OK;
  BwdArgs a{(const __nv_bfloat16*)X, (const __nv_bfloat16*)H1, (const __nv_bfloat16*)H2, y, t, M, grad_scale,
            (const __nv_bfloat16*)w.w2b, w.p, w.g, loss, ctx->d_flag};
  const int ntiles = (M + 127) / 128;
  const int grid = ntiles < ctx->num_sms ? ntiles : ctx->num_sms;
  mlp_bwd_kernel<<<grid, 128, BWD_SMEM, ctx->stream>>>(a);
  count_launch(ctx);
  return check_launch("mlp_bwd_kernel");
}

int launch_mlp_adam(cpsz_b200_ctx* ctx, const MlpParams& w, float lr, int step) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  mlp_adam_kernel<<<64, 256, 0, ctx->stream>>>(w.p, w.g, w.m, w.v, MLP_PARAMS, lr, b1, b2, eps, c1, c2,
                                               (__nv_bfloat16*)w.w1b, (__nv_bfloat16*)w.w2b);
  count_launch(ctx);
  return check_launch("mlp_adam_kernel");
}

int launch_mlp_cast(cpsz_b200_ctx* ctx, const MlpParams& w) {
  mlp_cast_kernel<<<64, 256, 0, ctx->stream>>>(w.p, (__nv_bfloat16*)w.w1b, (__nv_bfloat16*)w.w2b);
  count_launch(ctx);
  return check_launch("mlp_cast_kernel");
}

int launch_mlp_features(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, const double* eb_a,
                        const int* idx, int n, void* X) {
  if (n <= 0) return CPSZ_OK;
  int grid = (n + 127) / 128;
  if (grid > ctx->num_sms * 8) grid = ctx->num_sms * 8;
  features_kernel<<<grid, 128, 0, ctx->stream>>>(U, V, r1, r2, eb_a, idx, n, (__nv_bfloat16*)X);
  count_launch(ctx);
  return check_launch("features_kernel");
}

}  // namespace cpsz
