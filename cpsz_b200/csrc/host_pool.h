// host_pool.h -- a process-wide pool of host worker threads for the
// per-pass host work (Huffman trees of a pass's streams).
#pragma once

#include <functional>

namespace cpsz {

// Runs f(0..n-1) on the calling thread and the pool's workers (up to
// hardware_concurrency - 1 of them, started on first use and kept for the
// life of the process, so per-thread scratch such as the tree builder's stays
// warm from call to call).  Returns when every f(i) has returned.  Calls from
// several threads take turns; f must not call host_parallel_for itself.
void host_parallel_for(int n, const std::function<void(int)>& f);

}  // namespace cpsz
