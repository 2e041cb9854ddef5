// wave2d.cu -- 2D Lorenzo predict+quantize (compress) and its inverse
// (decompress) as a pipelined wavefront.
//
// The reference predicts every point from *reconstructed* neighbours
// (pred = (L + U) - UL in float, zero outside the field; the 12x12 block
// traversal of src/sz_compress_3d.cpp:126-193 with its rolling (bs+1)x(d2+1)
// buffer is exactly the raster recurrence with zero padding), so the field is
// a serial recurrence whose critical path is r1 + r2 points.  Bit-exactness
// rules out any reformulation; the parallel schedule is a skewed wavefront:
//
//  * a warp owns 32 consecutive rows (lane = row) and at step s lane l
//    processes column s - l; the value above comes from lane l-1's result of
//    the previous step through one __shfl_up_sync, the value up-left is the
//    value above of the previous step, the value to the left is the lane's own
//    previous result;
//  * a CTA owns a 256-row group (8 warps); warp w's lane 0 reads the row above
//    from warp w-1's lane 31 through a shared-memory ring with credit-based
//    flow control;
//  * CTAs are persistent and pull (field, group) items from a device work
//    queue (atomic counter).  An item's predecessor (same field, previous
//    group) was dequeued earlier by a running CTA, so every wait ends; warp 0
//    reads that group's last row from global memory after an acquire load of
//    its progress counter, which the producer advances with release stores.
//    Every wait is bounded; on expiry the kernel sets FLAG_TIMEOUT and
//    finishes without waiting.
//
// Per point (compress, include/sz_compression_utils.hpp:52-65):
//   diff = (float)(x - pred); y = |diff| / p (exact: p is a power of two)
//   y < 65535  <=>  |diff|/p + 1 < 65536 (the reference's capacity test)
//   q = (trunc(y) + 1) >> 1 == (int)((|diff|/p + 1) / 2), signed by diff > 0
//   dec = (float)((double)pred + (double)(2q) * p); kept iff |dec - x| <= p
// and per point (decompress, include/sz_decompression_utils.hpp:65-73):
//   code 0 -> raw value, else (float)((double)pred + (double)(2(code-32768)) * p).
#include "kernels.h"

namespace cpsz {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int RING = 128;
constexpr long long SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ double pow2d(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

struct Shared {
  float ring[WAVE_WARPS][RING];
  volatile int prod[WAVE_WARPS];
  volatile int cons[WAVE_WARPS];
  int item;
};

template <bool DECOMP>
struct Lane {
  // one element of work prefetched into registers
  float x;
  uint8_t id;
  uint16_t code;
};

template <bool DECOMP>
__device__ __forceinline__ void load8(const WaveField& F, bool rowok, long long rowc, int s0, int lane,
                                      Lane<DECOMP> (&b)[8]) {
  const float* xr = F.x + rowc * F.x_pitch;
  const uint8_t* ir = F.ids + rowc * F.id_pitch;
  const uint16_t* cr = F.codes + rowc * F.code_pitch;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int c = s0 + k - lane;
    bool v = rowok && c >= 0 && c < F.r2;
    b[k].x = v ? xr[c] : 0.f;
    b[k].id = v ? ir[c] : (uint8_t)0;
    if (DECOMP) b[k].code = v ? cr[c] : (uint16_t)0;
  }
  // pull the row's next lines into L1 well ahead of use
  int cp = s0 + 64 - lane;
  if (rowok && cp >= 0 && cp < F.r2) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(xr + cp));
    if (DECOMP) asm volatile("prefetch.global.L1 [%0];" ::"l"(cr + cp));
  }
}

template <bool DECOMP>
__device__ __forceinline__ void run_strip(const WaveField& F, int group, int warp, int lane, Shared& sh, int* flag) {
  const int r1 = F.r1, r2 = F.r2;
  const int row0 = group * WAVE_GROUP_ROWS + warp * 32;
  const int row = row0 + lane;
  const bool rowok = row < r1;
  const long long rowc = rowok ? row : 0;
  // who produces for whom
  const bool has_above = row0 > 0;
  const bool above_global = has_above && warp == 0;
  const bool has_below = row0 + 32 < r1;
  const bool below_global = has_below && warp == WAVE_WARPS - 1;
  const float* gb_in = above_global ? F.gbnd + (size_t)(group - 1) * r2 : nullptr;
  const int* gp_in = above_global ? F.gprog + (group - 1) : nullptr;
  float* gb_out = F.gbnd + (size_t)group * r2;
  int* gp_out = F.gprog + group;
  float* orow = F.out ? F.out + rowc * F.out_pitch : nullptr;
  uint16_t* crow = F.codes + rowc * F.code_pitch;

  int avail = 0;       // lane 0: columns of the row above known to be available
  int credit = RING;   // lane 31: columns it may run ahead of its consumer
  bool aborted = false;
  float outPrev = 0.f, upPrev = 0.f;
  const int nsteps = r2 + 31;

  auto step = [&](int s, const Lane<DECOMP>& e) {
    const int c = s - lane;
    float above = __shfl_up_sync(FULL, outPrev, 1);
    if (lane == 0) {
      above = 0.f;
      if (has_above && c >= 0 && c < r2) {
        if (c >= avail && !aborted) {
          long long spins = 0;
          if (above_global) {
            int v = ld_acquire(gp_in);
            while (v <= c) {
              if (++spins > SPIN_LIMIT) { atomicOr(flag, FLAG_TIMEOUT); aborted = true; break; }
              __nanosleep(64);
              v = ld_acquire(gp_in);
            }
            avail = v;
          } else {
            int v = sh.prod[warp - 1];
            while (v <= c) {
              if (++spins > SPIN_LIMIT) { atomicOr(flag, FLAG_TIMEOUT); aborted = true; break; }
              v = sh.prod[warp - 1];
            }
            avail = v;
          }
        }
        if (!aborted) {
          if (above_global) above = __ldcg(gb_in + c);
          else {
            above = sh.ring[warp - 1][c & (RING - 1)];
            if ((c & 15) == 15 || c == r2 - 1) sh.cons[warp] = c + 1;
          }
        }
      }
    }
    const float U = above, UL = upPrev;
    float out = 0.f;
    if (rowok && c >= 0 && c < r2) {
      const float pred = (outPrev + U) - UL;
      if (DECOMP) {
        if (e.code == 0) {
          out = e.x;
        } else {
          const double p = (e.id == 0) ? 0.0 : pow2d(2 * (int)e.id - 52);
          out = (float)((double)pred + (double)(2 * ((int)e.code - 32768)) * p);
        }
        orow[c] = out;
      } else {
        int code = 0;
        out = e.x;
        if (e.id != ID_ZERO) {
          const int ex = 2 * (int)e.id - 52;  // precision = 2^ex
          const float diff = e.x - pred;
          // |diff| * 2^-ex is exact in float for ex in [-52, 126); beyond
          // that range the double path is used.
          bool small;
          int qa;
          if (ex < 100) {
            const float y = fabsf(diff) * pow2f(-ex);
            small = y < 65535.0f;
            qa = small ? (((int)y + 1) >> 1) : 0;
          } else {
            const double qd = fabs((double)diff) * pow2d(-ex) + 1.0;
            small = qd < 65536.0;
            qa = small ? (int)(qd * 0.5) : 0;
          }
          if (small) {
            const int q = (diff > 0) ? qa : -qa;
            const double p = pow2d(ex);
            const float dec = (float)((double)pred + (double)(2 * q) * p);
            if ((double)fabsf(dec - e.x) <= p) {
              out = dec;
              code = q + 32768;
            }
          }
        }
        crow[c] = (uint16_t)code;
        if (orow) orow[c] = out;
      }
      // lane 31 hands the row down
      if (lane == 31) {
        if (below_global) {
          gb_out[c] = out;
          if ((c & 7) == 7 || c == r2 - 1) {
            __threadfence();
            st_release(gp_out, c + 1);
          }
        } else if (has_below && !aborted) {
          if (credit <= c) {
            long long spins = 0;
            int v = sh.cons[warp + 1];
            while (v + RING <= c) {
              if (++spins > SPIN_LIMIT) { atomicOr(flag, FLAG_TIMEOUT); aborted = true; break; }
              v = sh.cons[warp + 1];
            }
            credit = v + RING;
          }
          sh.ring[warp][c & (RING - 1)] = out;
          __threadfence_block();
          sh.prod[warp] = c + 1;
        }
      }
    }
    upPrev = U;
    outPrev = out;
  };

  Lane<DECOMP> A[8], B[8];
  load8<DECOMP>(F, rowok, rowc, 0, lane, A);
  for (int s0 = 0; s0 < nsteps; s0 += 16) {
    load8<DECOMP>(F, rowok, rowc, s0 + 8, lane, B);
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (s0 + k < nsteps) step(s0 + k, A[k]);
    load8<DECOMP>(F, rowok, rowc, s0 + 16, lane, A);
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (s0 + 8 + k < nsteps) step(s0 + 8 + k, B[k]);
  }
  // a producer that aborted still releases its consumers
  if (lane == 31 && below_global && aborted) st_release(gp_out, r2);
  if (lane == 31 && has_below && !below_global) sh.prod[warp] = r2;
}

template <bool DECOMP>
__global__ void __launch_bounds__(WAVE_WARPS * 32) wave2d_kernel(const WaveField* __restrict__ fields,
                                                                 const WaveItem* __restrict__ items, int n_items,
                                                                 int* queue, int* flag) {
  __shared__ Shared sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (;;) {
    if (threadIdx.x == 0) sh.item = atomicAdd(queue, 1);
    if (threadIdx.x < WAVE_WARPS) {
      sh.prod[threadIdx.x] = 0;
      sh.cons[threadIdx.x] = 0;
    }
    __syncthreads();
    const int it = sh.item;
    if (it >= n_items) break;
    const WaveItem item = items[it];
    const WaveField F = fields[item.field];
    if (item.group * WAVE_GROUP_ROWS + warp * 32 < F.r1) run_strip<DECOMP>(F, item.group, warp, lane, sh, flag);
    __syncthreads();
  }
}

}  // namespace

int launch_wave2d(cpsz_b200_ctx* ctx, bool decompress, const WaveField* d_fields, const WaveItem* d_items,
                  int n_items, int* d_queue, int max_ctas) {
  int per_sm = 0;
  if (decompress)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave2d_kernel<true>, WAVE_WARPS * 32, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave2d_kernel<false>, WAVE_WARPS * 32, 0);
  if (per_sm < 1) per_sm = 1;
  int grid = ctx->num_sms * per_sm;
  if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
  if (grid > n_items) grid = n_items;
  if (grid < 1) return CPSZ_OK;
  if (decompress)
    wave2d_kernel<true><<<grid, WAVE_WARPS * 32, 0, ctx->stream>>>(d_fields, d_items, n_items, d_queue, ctx->d_flag);
  else
    wave2d_kernel<false><<<grid, WAVE_WARPS * 32, 0, ctx->stream>>>(d_fields, d_items, n_items, d_queue, ctx->d_flag);
  count_launch(ctx);
  return check_launch("wave2d_kernel");
}

}  // namespace cpsz
