// wave2d.cu -- 2D Lorenzo predict+quantize (compress) and its inverse
// (decompress) as a pipelined wavefront.
//
// The reference predicts every point from *reconstructed* neighbours
// (pred = (L + U) - UL in float, zero outside the field; the 12x12 block
// traversal of src/sz_compress_3d.cpp:126-193 with its rolling (bs+1)x(d2+1)
// buffer is exactly the raster recurrence with zero padding), so the field is
// a serial recurrence whose critical path is r1 + r2 points.  Bit-exactness
// rules out any reformulation; the parallel schedule is a skewed wavefront,
// and the design goal is the fewest issued instructions per step, because a
// warp issues in order and its step time is its instruction stream:
//
//  * a warp owns 32 consecutive rows (lane = row) and at step s lane l
//    processes column s - l; the value above comes from lane l-1's result of
//    the previous step through one __shfl_up_sync, the value up-left is the
//    value above of the previous step, the value to the left is the lane's own
//    previous result;
//  * inputs are one 8-byte pair per point (compress: value and the bits of
//    1/precision, NaN for precision 0; decompress: the precomputed addend or
//    the raw value, and a raw flag), staged per 32-step window k as a
//    "parallelogram" tile -- row l holds columns [32k - l, 32k - l + 32),
//    exactly what lane l touches during steps [32k, 32k + 32) -- filled with
//    coalesced 8-byte cp.async row copies one window ahead (double buffered)
//    and drained with coalesced row stores one window behind.  A 33-element
//    row pitch makes the per-step accesses tile[l][t] bank-conflict free.
//    Points outside the field are staged as pairs that reconstruct to 0, so a
//    step has no bounds branches;
//  * the staging and draining run in a helper warp paired with each compute
//    warp (same scheduler; a named barrier per window), so the compute warp's
//    instruction stream holds only the recurrence, and the helper's
//    instructions issue in the compute warp's dependency stalls;
//  * a step has no branches: the hand-off below and the test tap are single
//    predicated stores, and the tap is a template parameter (a branch in the
//    step splits it into basic blocks the compiler cannot overlap);
//  * a CTA owns a WAVE_GROUP_ROWS-row group (WAVE_WARPS compute warps; 128
//    rows, 4 warps: one per scheduler, plus their helpers).  Warp w takes the
//    row above from warp w-1 through a shared-memory ring of tagged words, 8
//    columns at a time (one warp-uniform tag test per 8 steps); lane 31
//    stores one tagged word per step.  The CTA's first warp takes the previous
//    group's last row from global memory, a whole 32-column window at a time,
//    validated once per window and loaded coalesced one window ahead;
//  * CTAs are persistent and pull (field, group) items from a device work
//    queue (atomic counter).  An item's predecessor (same field, previous
//    group) was dequeued earlier by a running CTA, so every wait ends;
//  * compression runs beside its producer: the bound kernel (eb2d) counts the
//    points it has finished per unit (a 128-row group x 256-column block) and
//    produces the units along diagonals that follow the wavefront's own skew,
//    so a group's recurrence sweeps along as its inputs appear instead of
//    waiting for the whole group; a helper warp stages a window once the
//    units it reads are complete (lane 0 polls with ld.acquire.gpu, every
//    lane then acquires before its loads).  Such a launch keeps to one CTA
//    per SM, so each SM keeps room for the producer's CTAs and the producer
//    cannot be starved by waiting consumers.  A wait ends with FLAG_TIMEOUT
//    when the producer has finished no tile for a while (it is not running
//    beside it), and the host then runs the wavefront again after it.
//
// Tagged words are 64-bit (column + 1) << 32 | float bits, written and read as
// single aligned 64-bit accesses, so a reader that sees the expected tag holds
// that column's value and no memory fence is needed.  Every wait is bounded;
// on expiry the kernel sets FLAG_TIMEOUT and stops waiting.
//
// Arithmetic (bit-identical to include/sz_compression_utils.hpp:52-65 and
// include/sz_decompression_utils.hpp:65-73).  The precision is p = 2^ex, so
//   y = |x - pred| / p = |x - pred| * (1/p) is exact in float, and the
//   reference's capacity test |diff|/p + 1 < 65536 is y < 65535 (y + 1 is
//   exact in double below 2^16);
//   (int)((|diff|/p + 1) / 2) = (trunc(y) + 1) >> 1 = floor(y/2 + 1/2), taken
//   without a conversion: y/2 + 1/2 rounded down keeps its floor, and that
//   plus 2^23 rounded down is 2^23 + floor exactly;
//   the reference's (float)((double)pred + (double)(2q) * p) equals the float
//   sum pred + 2q*p: 2q*p is exact in float (|2q| < 2^17), and whenever the
//   exact sum does not fit a double one addend lies below 2^-5 ulp of the
//   other, where rounding through double and rounding once agree;
//   |dec - x| <= p compares a float against a power of two.
// Decompression adds the precomputed 2(code - 32768) * p (0 when id = 0) or
// takes the stored raw value.
#include "kernels.h"
#include "tuning.h"

namespace cpsz {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int RING = 128;
constexpr int TP = 33;         // tile row pitch (elements)
constexpr int TILE = 32 * TP;  // elements per tile
constexpr long long SPIN_LIMIT = 1ll << 22;
// A wait for the producer gives up after this long without any of its tiles
// finishing (it is not running: a tool serialises kernels, or the device is
// held by other work); the host then runs the wavefront again after it.
constexpr long long BAND_WAIT_NS = 50000000ll;  // 50 ms

__device__ __forceinline__ unsigned long long tagged(int c, float v) {
  return ((unsigned long long)(unsigned)(c + 1) << 32) | (unsigned long long)__float_as_uint(v);
}
__device__ __forceinline__ bool tag_is(unsigned long long w, int c) { return (unsigned)(w >> 32) == (unsigned)(c + 1); }
__device__ __forceinline__ float tag_val(unsigned long long w) { return __uint_as_float((unsigned)w); }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// Named barrier of one compute warp and its helper warp (ids 1..WAVE_WARPS).
__device__ __forceinline__ void pair_sync(int strip) { asm volatile("bar.sync %0, 64;" ::"r"(1 + strip) : "memory"); }
// Stores that only some lanes perform, as single predicated instructions: the
// per-step hand-off then never splits the warp into divergent paths.
__device__ __forceinline__ void st_u64_if(bool p, void* addr, unsigned long long v) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.volatile.u64 [%1], %2;\n\t}" ::"r"((unsigned)p),
               "l"(addr), "l"(v));
}
__device__ __forceinline__ void st_global_f32_if(bool p, void* g, float v) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %0, 0;\n\t@q st.global.f32 [%1], %2;\n\t}" ::"r"((unsigned)p),
               "l"(g), "f"(v)
               : "memory");
}

struct WarpTiles {
  float2 in[2][TILE];
  uint32_t out[2][TILE];
};

struct Shared {
  unsigned long long ring[WAVE_WARPS][RING];
  volatile int cons[WAVE_WARPS];  // ring columns its consumer has finished with
  int item;
};

constexpr size_t kDynSmem = sizeof(WarpTiles) * WAVE_WARPS;
constexpr int WAVE_THREADS = 2 * WAVE_WARPS * 32;  // compute warps, then one helper warp each

// ---- helper warp: stages window k of its strip and writes window k-2's outputs ----
// stage window k: row l, columns [32k - l, 32k - l + 32); lane t takes column t
template <bool DECOMP>
__device__ __forceinline__ void tile_fill(const WaveField& F, WarpTiles& T, long long row0, int nrows, int lane,
                                          int k, int buf) {
  // staged pair of a point outside the field: reconstructs to 0
  const float2 pad = DECOMP ? make_float2(0.f, __int_as_float(1)) : make_float2(0.f, __int_as_float(0x7FC00000));
  const float2* rp = F.pair + row0 * F.pair_pitch;
  int c = 32 * k + lane;
  float2* d = &T.in[buf][lane];
#pragma unroll 4
  for (int l = 0; l < 32; l++, c--, d += TP, rp += F.pair_pitch) {
    if (l < nrows && (unsigned)c < (unsigned)F.r2) cp_async8(d, rp + c);
    else *d = pad;
  }
  cp_commit();
}
// write window k's outputs: row l, columns [32k - l, 32k - l + 32)
template <bool DECOMP>
__device__ __forceinline__ void tile_drain(const WaveField& F, const WarpTiles& T, long long row0, int nrows, int lane,
                                           int k, int buf) {
  int c = 32 * k + lane;
  const uint32_t* s = &T.out[buf][lane];
  long long r = row0;
  for (int l = 0; l < nrows; l++, c--, s += TP, r++) {
    if ((unsigned)c < (unsigned)F.r2) {
      const uint32_t v = *s;
      if (DECOMP) F.out[r * F.out_pitch + c] = __uint_as_float(v);
      else F.codes[r * F.code_pitch + c] = (uint16_t)v;
    }
  }
}

// Compression beside the producer: before window k is staged, wait until the
// producer has finished the units of this group that it reads (columns up to
// 32k + 31).  Lane 0 polls; every lane then acquires.  `ready` is the first
// column block not yet known finished.  A wait gives up (FLAG_TIMEOUT) once
// the producer has finished no tile for the limit, and ends at once when an
// earlier wait gave up.
__device__ __forceinline__ void wait_units(const WaveField& F, int group, int k, int lane, int& ready, int* flag) {
  const int cb_hi = min(32 * k + 31, F.r2 - 1) / UNIT_COLS;
  if (cb_hi < ready) return;
  const unsigned long long* row = F.unit_done + (size_t)group * F.unit_ncb;
  if (lane == 0) {
    const unsigned long long rows = (unsigned long long)min(WAVE_GROUP_ROWS, F.r1 - group * WAVE_GROUP_ROWS);
    const long long limit = F.band_wait_ns > 0 ? F.band_wait_ns : BAND_WAIT_NS;
    for (int cb = ready; cb <= cb_hi; cb++) {
      const unsigned long long target =
          rows * (unsigned long long)min(UNIT_COLS, F.r2 - cb * UNIT_COLS) + F.band_extra;
      if (ld_acquire(row + cb) >= target) continue;
      // progress: the producer's count of finished tiles (unit_done[-1])
      const unsigned long long* tiles = F.unit_done - 1;
      unsigned long long seen = ld_acquire(tiles);
      long long t_seen = globaltimer_ns();
      while (ld_acquire(row + cb) < target) {
        if (*(volatile int*)flag & FLAG_TIMEOUT) break;
        const unsigned long long now_tiles = ld_acquire(tiles);
        const long long now = globaltimer_ns();
        if (now_tiles != seen) {
          seen = now_tiles;
          t_seen = now;
        } else if (now - t_seen > limit) {
          atomicOr(flag, FLAG_TIMEOUT);
          break;
        }
        __nanosleep(500);
      }
    }
  }
  __syncwarp();
  (void)ld_acquire(row + cb_hi);
  ready = cb_hi + 1;
}

template <bool DECOMP>
__device__ __forceinline__ void run_helper(const WaveField& F, int group, int strip, int lane, WarpTiles& T,
                                           int* flag) {
  const long long row0 = (long long)group * WAVE_GROUP_ROWS + strip * 32;
  const int nrows = min(32, F.r1 - (int)row0);
  const int nwin = (F.r2 + 31 + 31) / 32;  // windows that contain any step
  const bool waits = !DECOMP && F.unit_done;
  int ready = 0;
  if (waits) wait_units(F, group, 0, lane, ready, flag);
  tile_fill<DECOMP>(F, T, row0, nrows, lane, 0, 0);
  cp_wait_all();
  for (int k = 0; k < nwin; k++) {
    pair_sync(strip);  // the compute warp starts window k (tiles buf = k & 1)
    if (waits && k + 1 < nwin) wait_units(F, group, k + 1, lane, ready, flag);
    if (k + 1 < nwin) tile_fill<DECOMP>(F, T, row0, nrows, lane, k + 1, (k + 1) & 1);
    if (k >= 1) tile_drain<DECOMP>(F, T, row0, nrows, lane, k - 1, (k - 1) & 1);
    cp_wait_all();
  }
  pair_sync(strip);  // the compute warp has finished the last window
  tile_drain<DECOMP>(F, T, row0, nrows, lane, nwin - 1, (nwin - 1) & 1);
}

// ---- compute warp: the recurrence over its 32 rows ----
template <bool DECOMP, bool TAP>
__device__ __forceinline__ void run_strip(const WaveField& F, int group, int warp, int lane, Shared& sh,
                                          WarpTiles& T, int* flag) {
  const int r1 = F.r1, r2 = F.r2;
  const int row0 = group * WAVE_GROUP_ROWS + warp * 32;
  const int nrows = min(32, r1 - row0);
  const bool has_above = row0 > 0;
  const bool above_global = has_above && warp == 0;
  const bool above_ring = has_above && !above_global;
  const bool has_below = row0 + 32 < r1;
  const bool below_global = has_below && warp == WAVE_WARPS - 1;
  const bool below_ring = has_below && !below_global;
  const unsigned long long* gb_in = above_global ? F.gbnd + (size_t)(group - 1) * r2 : nullptr;
  unsigned long long* gb_out = F.gbnd + (size_t)group * r2;

  int credit = RING;  // ring columns this warp may write before re-reading its consumer's progress
  bool aborted = false;
  long long spin_above = 0, spin_credit = 0;
  const long long t_start = F.trace ? globaltimer_ns() : 0;
  float outPrev = 0.f, upPrev = 0.f;
  const int nwin = (r2 + 31 + 31) / 32;  // windows that contain any step
  auto ring_word = [&](int c) -> unsigned long long {
    return *(volatile unsigned long long*)&sh.ring[warp - 1][c & (RING - 1)];
  };
  // coalesced prefetch of the previous group's last row, one window ahead
  unsigned long long gcur = 0, gnext = 0;
  auto gload = [&](int k) -> unsigned long long {
    const int c = 32 * k + lane;
    return (c < r2) ? __ldcg(gb_in + c) : 0ull;
  };

  if (above_global) gnext = gload(0);
  for (int k = 0; k < nwin; k++) {
    const int buf = k & 1;
    pair_sync(warp);  // window k is staged; window k-1's outputs are handed to the helper
    if (above_global) {
      // the whole window of the row above must be present: one poll per window
      gcur = gnext;
      const int cl = 32 * k + lane;
      bool ok = cl >= r2 || tag_is(gcur, cl);
      long long spins = 0;
      while (!__all_sync(FULL, ok) && !aborted) {
        if (++spins > SPIN_LIMIT) {
          if (lane == 0) atomicOr(flag, FLAG_TIMEOUT);
          aborted = true;
          break;
        }
        __nanosleep(100);
        if (!ok) {
          gcur = __ldcg(gb_in + cl);
          ok = tag_is(gcur, cl);
        }
      }
      spin_above += spins;
      gnext = gload(k + 1);
    }
    const float2* tin = &T.in[buf][lane * TP];
    uint32_t* to = &T.out[buf][lane * TP];
#pragma unroll 1
    for (int tb = 0; tb < 32; tb += 8) {
      const int cb = 32 * k + tb;  // lane 0's column at the block's first step
      // ---- the row above, 8 columns (all lanes hold lane 0's values) ----
      float ab[8];
      if (above_global) {
#pragma unroll
        for (int j = 0; j < 8; j++) ab[j] = tag_val(__shfl_sync(FULL, gcur, tb + j));
      } else if (above_ring) {
        unsigned long long wv[8];
        bool ok = true;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          wv[j] = ring_word(cb + j);
          ok &= (cb + j >= r2) | tag_is(wv[j], cb + j);
        }
        if (!ok && !aborted) {  // warp-uniform: all lanes read the same words
          long long spins = 0;
          do {
            if (++spins > SPIN_LIMIT) {
              if (lane == 0) atomicOr(flag, FLAG_TIMEOUT);
              aborted = true;
              break;
            }
            ok = true;
#pragma unroll
            for (int j = 0; j < 8; j++) {
              wv[j] = ring_word(cb + j);
              ok &= (cb + j >= r2) | tag_is(wv[j], cb + j);
            }
          } while (!ok);
          spin_above += spins;
        }
#pragma unroll
        for (int j = 0; j < 8; j++) ab[j] = tag_val(wv[j]);
        if (lane == 0) sh.cons[warp] = cb;  // columns below cb have been consumed
      } else {
#pragma unroll
        for (int j = 0; j < 8; j++) ab[j] = 0.f;
      }
      if (aborted) {
#pragma unroll
        for (int j = 0; j < 8; j++) ab[j] = 0.f;
      }
      // ---- ring credit for the 8 columns lane 31 writes in this block ----
      if (below_ring) {
        const int cmax = cb - 24;
        if (cmax >= credit && !aborted) {
          long long spins = 0;
          int v = sh.cons[warp + 1];
          while (v + RING <= cmax) {
            if (++spins > SPIN_LIMIT) {
              if (lane == 0) atomicOr(flag, FLAG_TIMEOUT);
              aborted = true;
              break;
            }
            v = sh.cons[warp + 1];
          }
          spin_credit += spins;
          credit = v + RING;
        }
      }
      // ---- 8 steps ----
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int t = tb + j;
        const float shfl = __shfl_up_sync(FULL, outPrev, 1);
        const float U = (lane == 0) ? ab[j] : shfl;
        const float pred = (outPrev + U) - upPrev;
        const float2 e = tin[t];
        float out;
        if (DECOMP) {
          out = (__float_as_int(e.y) != 0) ? e.x : pred + e.x;
          to[t] = __float_as_uint(out);
        } else {
          const float x = e.x, inv = e.y;  // inv = 1/p (NaN for precision 0)
          const float p = __int_as_float(0x7F000000 - __float_as_int(inv));
          const float diff = x - pred;
          // q = (trunc(y) + 1) >> 1 = floor(y/2 + 1/2) for y = |diff|/p >= 0.
          // y/2 = |diff| * (inv/2) is exact; rounding y/2 + 1/2 down keeps
          // its floor, and rounding that plus 2^23 down yields 2^23 + floor
          // exactly (for y >= 2^24 the point is unpredictable anyway).
          const float h = fabsf(diff) * (0.5f * inv);
          const float mq = __fadd_rd(__fadd_rd(h, 0.5f), 8388608.0f);
          const float qf = mq - 8388608.0f;
          // 0 - qf keeps q = 0 a +0 addend (as the decoder's 2(code - 32768) * p is)
          const float dec = pred + ((diff > 0.f) ? qf : 0.f - qf) * (p + p);
          const bool ok = (h < 32767.5f) & (fabsf(dec - x) <= p);
          out = ok ? dec : x;
          const int qa = __float_as_int(mq) - 0x4B000000;
          to[t] = ok ? (uint32_t)(((diff > 0.f) ? qa : -qa) + 32768) : 0u;
          if (TAP) {  // optional reconstruction tap (tests)
            const int c = cb + j - lane;
            st_global_f32_if((lane < nrows) & ((unsigned)c < (unsigned)r2),
                             F.out + (long long)(row0 + lane) * F.out_pitch + c, out);
          }
        }
        // lane 31 hands its row down (column cb + j - 31)
        const int c31 = cb + j - 31;
        const bool w31 = (lane == 31) & ((unsigned)c31 < (unsigned)r2) & has_below;
        st_u64_if(w31, below_ring ? (void*)&sh.ring[warp][c31 & (RING - 1)] : (void*)(gb_out + c31), tagged(c31, out));
        upPrev = U;
        outPrev = out;
      }
    }
  }
  pair_sync(warp);  // the last window's outputs go to the helper
  if (lane == 0 && above_ring) sh.cons[warp] = r2 + RING;
  if (F.trace && lane == 0) {
    long long* tr = F.trace + ((long long)group * WAVE_WARPS + warp) * 4;
    tr[0] = t_start;
    tr[1] = globaltimer_ns();
    tr[2] = spin_above;
    tr[3] = spin_credit;
  }
}

template <bool DECOMP>
__device__ __forceinline__ void wave2d_body(const WaveField* __restrict__ fields, const WaveItem* __restrict__ items,
                                            int n_items, int* queue, int* flag) {
  __shared__ Shared sh;
  extern __shared__ __align__(16) unsigned char dyn[];
  WarpTiles* tiles = reinterpret_cast<WarpTiles*>(dyn);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int strip = warp % WAVE_WARPS;  // the strip a compute warp runs, or its helper serves
  for (;;) {
    if (threadIdx.x == 0) sh.item = atomicAdd(queue, 1);
    for (int k = threadIdx.x; k < WAVE_WARPS * RING; k += blockDim.x) (&sh.ring[0][0])[k] = 0ull;
    if (threadIdx.x < WAVE_WARPS) sh.cons[threadIdx.x] = 0;
    __syncthreads();
    const int it = sh.item;
    if (it >= n_items) break;
    const WaveItem item = items[it];
    const WaveField F = fields[item.field];
    if (item.group * WAVE_GROUP_ROWS + strip * 32 < F.r1) {
      if (warp < WAVE_WARPS) {
        if (!DECOMP && F.out) run_strip<DECOMP, true>(F, item.group, strip, lane, sh, tiles[strip], flag);
        else run_strip<DECOMP, false>(F, item.group, strip, lane, sh, tiles[strip], flag);
      }
      else run_helper<DECOMP>(F, item.group, strip, lane, tiles[strip], flag);
    }
    if (!DECOMP && F.group_done) {
      // every thread's code stores are visible device-wide before the flag
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) *(volatile unsigned*)(F.group_done + item.group) = 1u;
    }
    __syncthreads();
  }
}

template <bool DECOMP>
__global__ void __launch_bounds__(WAVE_THREADS, 1) wave2d_kernel(const WaveField* __restrict__ fields,
                                                                 const WaveItem* __restrict__ items, int n_items,
                                                                 int* queue, int* flag) {
  wave2d_body<DECOMP>(fields, items, n_items, queue, flag);
}

// The compression launch that runs beside the bound kernel, held to 64
// registers a thread: it then leaves an SM room for three bound-kernel CTAs
// instead of two, for a slightly slower recurrence step.
__global__ void __launch_bounds__(WAVE_THREADS, 4) wave2d_beside_kernel(const WaveField* __restrict__ fields,
                                                                        const WaveItem* __restrict__ items,
                                                                        int n_items, int* queue, int* flag) {
  wave2d_body<false>(fields, items, n_items, queue, flag);
}

}  // namespace

int preload_wave2d() {
  // every wavefront kernel loaded (and its shared-memory limit set) before
  // any of them runs beside a producer: a later first launch of another one
  // would otherwise load its module while the running launch waits
  const void* fns[] = {(const void*)wave2d_kernel<false>, (const void*)wave2d_kernel<true>,
                       (const void*)wave2d_beside_kernel};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDynSmem);
    if (e != cudaSuccess) return set_error(CPSZ_ERR_CUDA, "loading wave2d kernels: %s", cudaGetErrorString(e));
  }
  return CPSZ_OK;
}

int launch_wave2d(cpsz_b200_ctx* ctx, bool decompress, const WaveField* d_fields, const WaveItem* d_items,
                  int n_items, int* d_queue, size_t points, cudaStream_t stream, int mode) {
  if (n_items <= 0) return CPSZ_OK;
  if (!stream) stream = ctx->stream;
  static bool attr_set[3] = {false, false, false};
  const bool beside = mode == WAVE_BESIDE && !decompress;
  const void* fn = decompress ? (const void*)wave2d_kernel<true>
                              : beside ? (const void*)wave2d_beside_kernel : (const void*)wave2d_kernel<false>;
  const int which = decompress ? 1 : beside ? 2 : 0;
  if (!attr_set[which]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDynSmem);
    if (e != cudaSuccess) return set_error(CPSZ_ERR_CUDA, "wave2d smem attribute: %s", cudaGetErrorString(e));
    attr_set[which] = true;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, WAVE_THREADS, kDynSmem);
  if (per_sm < 1) return set_error(CPSZ_ERR_CUDA, "wave2d kernel does not fit on an SM");
  const int cap = tune_get(TUNE_WAVE2D_CTAS_PER_SM, points);
  if (cap > 0 && per_sm > cap) per_sm = cap;
  if (mode == WAVE_BESIDE) per_sm = 1;
  if (mode == WAVE_JOIN) per_sm -= 1;
  if (per_sm < 1) return CPSZ_OK;
  int grid = ctx->num_sms * per_sm;
  if (grid > n_items) grid = n_items;
  if (grid < 1) return CPSZ_OK;
  if (decompress)
    wave2d_kernel<true><<<grid, WAVE_THREADS, kDynSmem, stream>>>(d_fields, d_items, n_items, d_queue, ctx->d_flag);
  else if (beside)
    wave2d_beside_kernel<<<grid, WAVE_THREADS, kDynSmem, stream>>>(d_fields, d_items, n_items, d_queue, ctx->d_flag);
  else
    wave2d_kernel<false><<<grid, WAVE_THREADS, kDynSmem, stream>>>(d_fields, d_items, n_items, d_queue, ctx->d_flag);
  count_launch(ctx);
  return check_launch("wave2d_kernel");
}

}  // namespace cpsz
