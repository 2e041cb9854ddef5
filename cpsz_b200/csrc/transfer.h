// transfer.h -- host <-> device copies of bulk data.
//
// Device and page-locked host memory are copied directly (enqueued on `st`).
// Pageable host memory of 1 MiB or more moves through the context's pinned
// ring (kStageSlots slots of kStageBytes) with the host copies spread over a
// small thread pool, chunk by chunk, each chunk's host copy overlapping the
// previous chunks' DMA.  For pageable memory both calls return once the host
// side is complete: after h2d the source may be reused, after d2h the
// destination holds the data.  Device-side ordering is that of `st`.
#pragma once

#include "runtime.h"

namespace cpsz {

enum HostKind { HOST_PAGEABLE = 0, HOST_PINNED = 1, HOST_DEVICE = 2 };
HostKind host_kind(const void* p);

int h2d(cpsz_b200_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st);
int d2h(cpsz_b200_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st);

}  // namespace cpsz
