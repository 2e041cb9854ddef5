// wave3d.cu -- the 3D Lorenzo recursion of the offline (log) path on
// reconstructed log values (src/sz_compress_cp_preserve_3d.cpp:441-520,
// src/sz_decompress_cp_preserve_3d.cpp:52-104).
//
// A point's predictor reads its seven lower neighbours (i-1 / j-1 / k-1
// combinations).  One persistent kernel runs the whole recursion:
//  * a unit is W3_P planes i0 .. i0+P-1 of 32 rows j0 .. j0+31, run by one
//    CTA: warp p owns plane i0 + p, lane l row j0 + l, and at step t the
//    thread handles column k = t - l - p (lanes skewed by one column, planes
//    by one step), so all seven neighbours were produced at steps t-1 .. t-3;
//    one barrier per step;
//  * each plane keeps its last results in a ring in shared memory: slot
//    t % W3_SR, entry l+1 = lane l's value of step t, entry 0 = row j0-1 at
//    column t+1-p (as if from a lane -1), loaded from the unit of the rows
//    below.  A point reads (i,j,k-1), (i,j-1,k), (i,j-1,k-1) from its own
//    plane's ring and the four (i-1, ., .) values from plane p-1's; plane
//    i0-1 is a ring loaded from the unit of the planes below.  Lane 0 needs
//    no special case;
//  * units are dequeued in ticket order u = (i0 / P) * slabs + s from an
//    atomic counter, so a unit's producers (the planes below, the rows
//    below) hold smaller tickets, taken by CTAs that are already running:
//    every wait ends;
//  * a unit publishes its progress (steps done by all its planes) every
//    W3_PUB steps: after the step barrier one thread fences and stores it.  Step t's loads need the unit of the planes
//    below at >= t + P + 1 and the unit of the rows below at >= t + 33; the
//    latter covers the unit below and behind, which that unit waited for;
//  * loads go through L2 (cp.async.cg: another SM's writes must not meet a
//    stale L1 line): the unit's input W3_DIN steps ahead (no dependency),
//    the loaded ring entries W3_DD steps ahead.
// Every wait is bounded: on expiry (or once any wait has expired) the kernel
// sets FLAG_TIMEOUT and stops waiting; the host then fails the call.
//
// Step arithmetic (all float; equal to the reference's float/double mix, see
// the wavefront notes in wave2d.cu): with p = 2^(id-23) and y = |x - pred| / p
// exact, the reference's capacity test is y < 65535, the code is
// 32768 +- ((int)y + 1) >> 1, and (float)(pred + 2 q p) equals the float sum
// pred + (2q) p.  The decoder's (float)(pred + 2 (code - 32768) p) is likewise
// pred + addend with the addend precomputed exactly in float; its exp2f and
// signs are applied afterwards, point by point, off the recursion.
#include "kernels.h"
#include "libm_dev.cuh"

namespace cpsz {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int W3_P = 8;                 // planes per unit = warps per CTA
constexpr int W3_THREADS = 32 * W3_P;
constexpr int W3_DIN = 8;               // input prefetch distance (steps)
constexpr int W3_DD = 3;                // loaded ring entries: prefetch distance (steps)
constexpr int W3_SIN = W3_DIN + 1;      // input ring slots
constexpr int W3_SR = W3_DD + 4;        // result ring slots: three read back, one written, the rest in flight
constexpr int W3_PUB = 8;               // steps between progress publications
constexpr long long W3_WAIT_NS = 4000000000ll;

struct W3Args {
  const float4* in;  // compress: (log u, log v, log w, 1/p); decompress: addends or raw values (w != 0)
  float4* rec;       // reconstructed log values
  ushort4* codes;    // compress: codes (0,0,0 for unpredictable points)
  LibmFn Lg;         // decompress: the host library's log2f (raw points)
  int r1, r2, r3, slabs;
  int* sync;  // [0] the work queue, [1 + u] unit u's published progress
  int* flag;
};

struct W3Smem {
  float4 in[W3_P][W3_SIN][32];
  float4 ring[W3_P + 1][W3_SR][33];  // ring[0]: plane i0-1 (loaded); ring[p+1]: plane i0+p
  int unit;
};
constexpr size_t kW3Smem = sizeof(W3Smem);

__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s32(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// 16-byte cp.async through L2; zero-fills the slot when !valid (src unread)
__device__ __forceinline__ void cp16(void* smem, const void* g, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(g), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Lane 0: waits until *p >= need (bounded), polling with relaxed loads and a
// growing pause, then acquires once; `have` caches the last value seen.
__device__ __noinline__ void w3_wait(const int* p, int need, int& have, int* flag, bool& aborted) {
  have = ld_relaxed_s32(p);
  if (have < need) {
    const long long t0 = globaltimer_ns();
    unsigned pause = 32;
    while (have < need) {
      if ((*(volatile int*)flag & FLAG_TIMEOUT) || globaltimer_ns() - t0 > W3_WAIT_NS) {
        atomicOr(flag, FLAG_TIMEOUT);
        aborted = true;
        return;
      }
      __nanosleep(pause);
      if (pause < 1024) pause *= 2;
      have = ld_relaxed_s32(p);
    }
  }
  have = ld_acquire_s32(p);
}

__device__ __forceinline__ float4 shfl_up3(const float4& v) {
  return make_float4(__shfl_up_sync(FULL, v.x, 1), __shfl_up_sync(FULL, v.y, 1), __shfl_up_sync(FULL, v.z, 1), 0.f);
}
__device__ __forceinline__ float comp(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

__device__ __forceinline__ float small_int_to_float(int v) { return __int_as_float(0x4B400000 + v) - 12582912.0f; }

template <bool DECOMP>
__global__ void __launch_bounds__(W3_THREADS, 1) wave3d_kernel(const W3Args a) {
  extern __shared__ __align__(16) unsigned char w3_smem[];
  W3Smem& M = *reinterpret_cast<W3Smem*>(w3_smem);
  const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
  const int r1 = a.r1, r2 = a.r2, r3 = a.r3, slabs = a.slabs;
  const size_t d1 = (size_t)r3, d0 = (size_t)r2 * r3;
  const int units = ((r1 + W3_P - 1) / W3_P) * slabs;
  int* const prog = a.sync + 1;
  const float4 Z = make_float4(0.f, 0.f, 0.f, 0.f);
  bool aborted = false;  // thread 0: a wait has expired; no more waiting
  for (;;) {
    __syncthreads();  // the previous unit's last reads of the rings are done
    if (threadIdx.x == 0) M.unit = atomicAdd(a.sync, 1);
    __syncthreads();
    const int u = M.unit;
    if (u >= units) break;
    const int g = u / slabs, s = u - g * slabs;
    const int i0 = g * W3_P, np = min(W3_P, r1 - i0);
    const int j0 = 32 * s, nrows = min(32, r2 - j0);
    const int t_end = r3 + nrows - 1 + np - 1;
    const bool jin = lane < nrows, pin = p < np;
    const size_t row = (size_t)(j0 + (jin ? lane : 0)) * d1;  // this lane's row within a plane
    const size_t brow = s > 0 ? (size_t)(j0 - 1) * d1 : 0;     // row j0-1
    const size_t plane = (size_t)(i0 + (pin ? p : 0)) * d0;
    int have_prev = 0, have_below = 0;

    // thread 0: the producers have reached what the loads of slot tp read.
    // Plane i0-1's row j0+l at column tp-l+1 is the planes-below unit's step
    // tp+P; row j0-1 of plane i0+p at column tp+1-p is the rows-below unit's
    // step tp+32.  Targets are capped at the producers' step counts (the
    // planes-below unit has P planes and these rows, the rows-below unit 32
    // rows and these planes): a step beyond them loads only zero fill.
    const int end_prev = r3 + nrows - 1 + W3_P - 1, end_below = r3 + 31 + np - 1;
    auto wait_for = [&](int tp) {
      if (threadIdx.x != 0 || aborted) return;
      const int need_prev = min(tp + W3_P + 1, end_prev), need_below = min(tp + 33, end_below);
      if (i0 > 0 && have_prev < need_prev) w3_wait(prog + u - slabs, need_prev, have_prev, a.flag, aborted);
      if (s > 0 && have_below < need_below) w3_wait(prog + u - 1, need_below, have_below, a.flag, aborted);
    };
    // this plane's input for step tp
    auto issue_in = [&](int tp) {
      const int k = tp - lane - p;
      const bool act = tp < t_end && pin && jin && k >= 0 && k < r3;
      cp16(&M.in[p][tp % W3_SIN][lane], act ? a.in + plane + row + k : a.in, act);
    };
    // the loaded ring entries of slot tp (tp >= -3): entry 0 of every plane
    // (row j0-1), and all of plane i0-1's
    auto issue_dep = [&](int tp) {
      const int slot = (tp + W3_SR) % W3_SR;
      if (lane == 0) {
        const int kq = tp + 1 - p;
        const bool bb = s > 0 && pin && kq >= 0 && kq < r3;
        cp16(&M.ring[p + 1][slot][0], bb ? a.rec + plane + brow + kq : a.rec, bb);
      }
      if (p == 0) {
        // plane i0-1, entry l+1 = row j0+l at column tp-l+1, entry 0 = row j0-1 at column tp+2
        const int k = tp - lane + 1;
        const bool act = i0 > 0 && jin && k >= 0 && k < r3;
        cp16(&M.ring[0][slot][lane + 1], act ? a.rec + (size_t)(i0 - 1) * d0 + row + k : a.rec, act);
        if (lane == 0) {
          const int kb = tp + 2;
          const bool b0 = i0 > 0 && s > 0 && kb >= 0 && kb < r3;
          cp16(&M.ring[0][slot][0], b0 ? a.rec + (size_t)(i0 - 1) * d0 + brow + kb : a.rec, b0);
        }
      }
    };

    // prologue: the input of steps 0 .. W3_DIN-1 and the loaded entries of
    // slots -3 .. W3_DD-1; the computed entries of slots -3 .. -1 are zero
    for (int e = threadIdx.x; e < W3_P * 3 * 32; e += W3_THREADS) {
      const int r = e / (3 * 32), rest = e - r * 3 * 32, sl = rest / 32, en = rest - sl * 32;
      M.ring[r + 1][W3_SR - 3 + sl][en + 1] = Z;
    }
    wait_for(W3_DD - 1);
    __syncthreads();
    for (int tp = 0; tp < W3_DIN; tp++) issue_in(tp);
    for (int tp = -3; tp < W3_DD; tp++) issue_dep(tp);
    cp_commit();
    // W3_DD empty groups stand for steps -W3_DD .. -1, so that the wait of
    // step t (all but the newest W3_DD groups) covers the prologue's group
    // from step 0 on
#pragma unroll
    for (int e = 0; e < W3_DD; e++) cp_commit();
#pragma unroll 1
    for (int t = 0; t < t_end; t++) {
      // step t reads slots t-1 .. t-3 and input slot t: slot t-1 came with the
      // group issued at step t-1-W3_DD, so the newest W3_DD groups may still
      // be in flight
      wait_for(t + W3_DD);
      cp_wait<W3_DD>();
      __syncthreads();
      // every plane has finished step t-1 (the barrier above): thread 0's fence
      // makes the CTA's writes visible before its progress
      if (threadIdx.x == 0 && t > 0 && (t % W3_PUB == 0)) {
        __threadfence();
        st_release_s32(prog + u, t);
      }
      issue_in(t + W3_DIN);
      issue_dep(t + W3_DD);
      cp_commit();
      const float4* R1 = M.ring[p + 1][(t - 1 + W3_SR) % W3_SR];
      const float4* R2 = M.ring[p + 1][(t - 2 + W3_SR) % W3_SR];
      const float4* B1 = M.ring[p][(t - 1 + W3_SR) % W3_SR];
      const float4* B2 = M.ring[p][(t - 2 + W3_SR) % W3_SR];
      const float4* B3 = M.ring[p][(t - 3 + W3_SR) % W3_SR];
      // q0 = (i-1,j-1,k-1), q1 = (i-1,j-1,k), q2 = (i-1,j,k-1), q3 = (i-1,j,k),
      // q4 = (i,j-1,k-1), q5 = (i,j-1,k), q6 = (i,j,k-1)
      const float4 q0 = B3[lane], q1 = B2[lane], q2 = B2[lane + 1], q3 = B1[lane + 1];
      const float4 q4 = R2[lane], q5 = R1[lane], q6 = R1[lane + 1];
      const int k = t - lane - p;
      const bool act = pin && jin && k >= 0 && k < r3;
      const size_t idx = plane + row + (size_t)(act ? k : 0);
      // pred = q0 + q3 + q5 + q6 - q1 - q2 - q4, left to right
      float pred[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float v = comp(q0, c) + comp(q3, c);
        v = v + comp(q5, c);
        v = v + comp(q6, c);
        v = v - comp(q1, c);
        v = v - comp(q2, c);
        v = v - comp(q4, c);
        pred[c] = v;
      }
      const float4 x = M.in[p][t % W3_SIN][lane];
      float4 res;
      if (!DECOMP) {
        const float inv = x.w;  // NaN: precision 0 (unpredictable)
        const float pw = __int_as_float(0x7F000000 - __float_as_int(inv));
        bool ok = true;
        float dec[3];
        int q[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float xc = comp(x, c);
          const float diff = xc - pred[c];
          const float y = fabsf(diff) * inv;
          const int qa = ((int)fminf(y, 65536.0f) + 1) >> 1;
          q[c] = (diff > 0.f) ? qa : -qa;
          dec[c] = pred[c] + small_int_to_float(2 * q[c]) * pw;
          ok = ok & (y < 65535.0f) & (fabsf(dec[c] - xc) < pw);
        }
        res = ok ? make_float4(dec[0], dec[1], dec[2], 0.f) : make_float4(x.x, x.y, x.z, 0.f);
        if (act) {
          a.rec[idx] = res;
          a.codes[idx] = ok ? make_ushort4((unsigned short)(q[0] + 32768), (unsigned short)(q[1] + 32768),
                                           (unsigned short)(q[2] + 32768), 0)
                            : make_ushort4(0, 0, 0, 0);
        }
      } else {
        if (__float_as_int(x.w) != 0) {
          // raw point: its log feeds the neighbours' predictors
          float lg[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const float r = comp(x, c);
            lg[c] = (r == 0.f) ? -100.f : dev::host_log2f(fabsf(r), a.Lg);
          }
          res = make_float4(lg[0], lg[1], lg[2], 0.f);
        } else {
          res = make_float4(pred[0] + x.x, pred[1] + x.y, pred[2] + x.z, 0.f);
        }
        if (act) a.rec[idx] = res;
      }
      M.ring[p + 1][t % W3_SR][lane + 1] = act ? res : Z;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy into the rings is left in flight
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_s32(prog + u, t_end);
    }
  }
}

// Decoded values from the reconstructed logs: raw points keep their stored
// float; others are 0 below log -99 and +-exp2f(log) (the host library's)
// with the stored sign.
__global__ void __launch_bounds__(256) exp3d_kernel(const float4* __restrict__ in, const float4* __restrict__ rec,
                                                    const uint8_t* __restrict__ signs, size_t sign_bytes, LibmFn Ex,
                                                    float* __restrict__ U, float* __restrict__ V,
                                                    float* __restrict__ W, size_t n) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
    const float4 x = in[idx];
    float out[3];
    if (__float_as_int(x.w) != 0) {
      out[0] = x.x;
      out[1] = x.y;
      out[2] = x.z;
    } else {
      const float4 l = rec[idx];
      const unsigned byte = (unsigned)(idx >> 3), bit = 7u - (unsigned)(idx & 7);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float lg = comp(l, c);
        const bool pos = (__ldg(signs + (size_t)c * sign_bytes + byte) >> bit) & 1u;
        if (lg < -99.f) {
          out[c] = 0.f;
        } else {
          const float e = dev::host_exp2f(lg, Ex);
          out[c] = pos ? e : -e;
        }
      }
    }
    U[idx] = out[0];
    V[idx] = out[1];
    W[idx] = out[2];
  }
}

}  // namespace

size_t wave3d_scratch_bytes(int r1, int r2) {
  return ((size_t)((r1 + W3_P - 1) / W3_P) * ((r2 + 31) / 32) + 1) * sizeof(int);
}

int launch_wave3d(cpsz_b200_ctx* ctx, bool decompress, const float4* in, float4* rec, ushort4* codes,
                  const uint8_t* signs, size_t sign_bytes, const LibmTables* L, float* U, float* V, float* W, int r1,
                  int r2, int r3, void* scratch) {
  W3Args a{};
  a.in = in;
  a.rec = rec;
  a.codes = codes;
  if (decompress) a.Lg = L->log2f;
  a.r1 = r1;
  a.r2 = r2;
  a.r3 = r3;
  a.slabs = (r2 + 31) / 32;
  a.sync = (int*)scratch;
  a.flag = ctx->d_flag;
  CPSZ_CUDA_TRY(cudaMemsetAsync(scratch, 0, wave3d_scratch_bytes(r1, r2), ctx->stream));
  const long long units = (long long)((r1 + W3_P - 1) / W3_P) * a.slabs;
  auto kern = decompress ? wave3d_kernel<true> : wave3d_kernel<false>;
  CPSZ_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kW3Smem));
  int per_sm = 0;
  CPSZ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W3_THREADS, kW3Smem));
  long long ctas = (long long)ctx->num_sms * (per_sm > 0 ? per_sm : 1);
  if (ctas > units) ctas = units;
  kern<<<(int)ctas, W3_THREADS, kW3Smem, ctx->stream>>>(a);
  count_launch(ctx);
  CPSZ_TRY(check_launch("wave3d_kernel"));
  if (!decompress) return CPSZ_OK;
  const size_t n = (size_t)r1 * r2 * r3;
  const size_t blocks = (n + 255) / 256, cap = (size_t)ctx->num_sms * 8;
  exp3d_kernel<<<(int)(blocks < cap ? blocks : cap), 256, 0, ctx->stream>>>(in, rec, signs, sign_bytes, L->exp2f, U,
                                                                            V, W, n);
  count_launch(ctx);
  return check_launch("exp3d_kernel");
}

}  // namespace cpsz
