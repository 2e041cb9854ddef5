// selfcheck.cu -- exhaustive checks of the premises behind the filtered bounds.
//
// The filtered 2D and 3D bound evaluations (eb_math.cuh) prove that their
// float approximations enclose the reference's values, from the maximum
// errors of a few operations over the inputs those operations receive.  This
// kernel measures every such maximum over every float of its range on the
// device at hand (about 9e9 evaluations, well under a second), so a test can
// recompute the error budget from measured values:
//   acbrt1 (the reference's cube root, bit for bit the product path's) against
//     a double cube root, relative, over all positive normal floats (above
//     and below 1 separately);
//   rcp.approx.ftz.f32, relative, over the normal floats below 2^126;
//   ex2.approx.ftz.f32, relative, over [-87, 0];
//   sqrt.approx.f32, relative, over all positive normal floats;
//   lg2.approx.ftz.f32, absolute, per binade [2^e, 2^(e+1)), e = -126..0.
#include "eb_math.cuh"
#include "kernels.h"

namespace cpsz {

namespace {

__device__ __forceinline__ float sqrt_approx_f(float x) {
  float y;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// out[] holds non-negative floats as bit patterns (their integer order is
// their value order), raised with atomicMax
__device__ __forceinline__ void raise_max(unsigned* out, int slot, double e) {
  atomicMax(out + slot, __float_as_uint((float)e));
}

__global__ void filter_premises_kernel(unsigned* __restrict__ out) {
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  const unsigned long long nt = (unsigned long long)gridDim.x * blockDim.x;
  double hi = 0, lo = 0, rc = 0, ex = 0, sq = 0, lg = 0;
  int lg_slot = -1;  // the binade lg accumulates (a thread's b rises, so binades come in order)
  for (unsigned long long b = 0x00800000ull + tid; b < 0x7f800000ull; b += nt) {
    const float x = __uint_as_float((unsigned)b);
    const double xd = (double)x;
    const double e = (double)dev::acbrt1_nonneg(x) / cbrt(xd) - 1.0;
    hi = fmax(hi, e);
    lo = fmax(lo, -e);
    sq = fmax(sq, fabs((double)sqrt_approx_f(x) / sqrt(xd) - 1.0));
    if (b < 0x7e800000ull) rc = fmax(rc, fabs((double)dev::rcp_approx(x) * xd - 1.0));
    if (b < 0x40000000ull) {
      const int slot = FP_LG2 + (int)(b >> 23) - 1;  // exponent field 1..127: binade -126..0
      if (slot != lg_slot) {
        if (lg_slot >= 0) raise_max(out, lg_slot, lg);
        lg_slot = slot;
        lg = 0;
      }
      lg = fmax(lg, fabs((double)dev::lg2_approx(x) - log2(xd)));
    }
  }
  if (lg_slot >= 0) raise_max(out, lg_slot, lg);
  // ex2 over [-87, 0]: the bit patterns of -0 .. -87
  for (unsigned long long b = 0x80000000ull + tid; b <= 0xC2AE0000ull; b += nt) {
    const float a = __uint_as_float((unsigned)b);
    ex = fmax(ex, fabs((double)dev::ex2_approx(a) / exp2((double)a) - 1.0));
  }
  raise_max(out, FP_ACBRT_HI, hi);
  raise_max(out, FP_ACBRT_LO, lo);
  raise_max(out, FP_RCP, rc);
  raise_max(out, FP_EX2, ex);
  raise_max(out, FP_SQRT, sq);
}

}  // namespace

int launch_filter_premises(cpsz_b200_ctx* ctx, unsigned* d_out) {
  CPSZ_CUDA_TRY(cudaMemsetAsync(d_out, 0, FP_COUNT * sizeof(unsigned), ctx->stream));
  filter_premises_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(d_out);
  count_launch(ctx);
  return check_launch("filter_premises_kernel");
}

}  // namespace cpsz
