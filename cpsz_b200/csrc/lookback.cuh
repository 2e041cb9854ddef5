// lookback.cuh -- decoupled look-back (Merrill & Garland, "Single-pass
// Parallel Prefix Scan with Decoupled Look-back", 2016) for kernels that hand
// out work items in ticket order: an item publishes its own count, then finds
// the sum over all earlier items by reading their status words backwards
// until one that already knows its inclusive prefix.
#pragma once

#include "kernels.h"

namespace cpsz {

// Status word of an item: 2-bit state (0 = not yet, LB_AGG = the item's own
// count, LB_PRE = its inclusive prefix) over a 62-bit count.  A word carries
// its count itself and nothing else is read on its strength, so relaxed loads
// and stores suffice.
constexpr unsigned long long LB_AGG = 1ull << 62, LB_PRE = 2ull << 62, LB_VAL = (1ull << 62) - 1;
constexpr int LB_DEPTH = 4;  // 32-item windows read per round trip

__device__ __forceinline__ unsigned long long lb_ld(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void lb_st(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Publishes item s's own count (one thread; item 0's count is its prefix).
__device__ __forceinline__ void lookback_publish(unsigned long long* status, unsigned long long s,
                                                 unsigned long long tot) {
  lb_st(&status[s], (s == 0 ? LB_PRE : LB_AGG) | tot);
}

// Called by one full warp for item s with count tot (same in every lane),
// after lookback_publish(status, s, tot) by a thread of the same CTA: returns
// the sum of the counts of items 0..s-1 (in every lane) and publishes the
// inclusive prefix.  Items must be handed out in ticket order (every earlier
// item then belongs to a running or finished CTA).  Every lane keeps
// LB_DEPTH loads in flight, so one L2 round trip covers 32 * LB_DEPTH items.
// A wait past spin_limit polls sets FLAG_TIMEOUT in *flag and returns what
// was summed.
__device__ __forceinline__ unsigned long long lookback_warp(unsigned long long* status, unsigned long long s,
                                                            unsigned long long tot, int lane, long long spin_limit,
                                                            int* flag) {
  constexpr unsigned FULL = 0xffffffffu;
  unsigned long long excl = 0;
  if (s == 0) return 0;
  long long p = (long long)s - 1;  // the nearest item not yet summed
  long long spins = 0;
  bool done = false;
  while (!done) {
    unsigned long long w[LB_DEPTH];
#pragma unroll
    for (int m = 0; m < LB_DEPTH; m++) {
      const long long q = p - 32 * m - lane;
      w[m] = q >= 0 ? lb_ld(&status[q]) : LB_PRE;  // before item 0: prefix 0
    }
    // the windows in order, nearest first; a window with an unpublished item
    // before its nearest prefix is read again from there
    bool wait = false;
#pragma unroll
    for (int m = 0; m < LB_DEPTH; m++) {
      if (done || wait) continue;
      const unsigned int pre_m = __ballot_sync(FULL, (w[m] & ~LB_VAL) == LB_PRE);
      const unsigned int none_m = __ballot_sync(FULL, (w[m] & ~LB_VAL) == 0);
      const int last = pre_m ? __ffs(pre_m) - 1 : 31;  // the nearest prefix, or the whole window
      const unsigned int upto = last == 31 ? FULL : ((1u << (last + 1)) - 1u);
      if (none_m & upto) {
        wait = true;
        continue;
      }
      unsigned long long add = lane <= last ? (w[m] & LB_VAL) : 0ull;
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) add += __shfl_xor_sync(FULL, add, d);
      excl += add;
      p -= 32;
      done = pre_m != 0;
    }
    if (wait) {
      if (++spins > spin_limit) {
        if (lane == 0) atomicOr(flag, FLAG_TIMEOUT);
        break;
      }
      __nanosleep(64);
    }
  }
  if (lane == 0) lb_st(&status[s], LB_PRE | ((excl + tot) & LB_VAL));
  return excl;
}

}  // namespace cpsz
