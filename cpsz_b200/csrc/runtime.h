// runtime.h -- host-side runtime of libcpsz_b200: error reporting, per-call
// device arena, pinned staging, launch accounting, and the host-computed
// quantization tables shared by the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "cpsz_b200.h"

namespace cpsz {

// ---- errors ---------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
void clear_error();

struct Status {
  int code = CPSZ_OK;
  bool ok() const { return code == CPSZ_OK; }
};

#define CPSZ_CUDA_TRY(expr)                                                                         \
  do {                                                                                              \
    cudaError_t _e = (expr);                                                                        \
    if (_e != cudaSuccess)                                                                          \
      return ::cpsz::set_error(CPSZ_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                               __FILE__, __LINE__);                                                 \
  } while (0)

#define CPSZ_TRY(expr)           \
  do {                           \
    int _rc = (expr);            \
    if (_rc != CPSZ_OK) return _rc; \
  } while (0)

// ---- quantization tables (computed on the host with glibc's log2) ----------
// The reference quantizes an error bound e with
//   id = (int)(log2(e / thr) / log2(base)),   e <= thr -> id 0 (precision 0)
// (include/sz_cp_preserve_utils.hpp:14-22).  Because glibc's log2 is not
// CUDA's, the kernels never call log2: for every id k >= 1 the host finds
// the smallest double e with id(e) >= k by bisection over the ordered bit
// patterns, calling the host log2 itself, and the kernels count thresholds.
struct QuantTable {
  static constexpr int kMax = 256;
  double thr = 0;       // quantization threshold
  int base = 0;         // 4 (2D) or 2 (3D)
  int n = 0;            // thresholds t[1..n) valid; t[0] = thr (id >= 0 region starts above thr)
  double t[kMax] = {};  // t[k] = smallest e with id(e) >= k
  // 2D table only: every t[k] (k >= 0) lies in (the float below 2^(2k-52),
  // 2^(2k-52)], so a float x has id >= k exactly when x >= 2^(2k-52): the
  // float id of x > thr is (exponent(x) + 52) >> 1 (eb2d's float vertex path)
  bool float_pow4 = false;
};
// 2D: base 4, thr = DBL_EPSILON, applied to e = |U| * eb.
const QuantTable& quant_table_2d();
// 2D offline_log: id of log2(1 + eb) with base 2, thr = DBL_EPSILON, over the
// relative bound eb directly; t[0] is the largest eb with precision 0.
const QuantTable& quant_table_2d_log();
// 3D: id of abs_eb = log2(1 + required_eb) with base 2, thr = FLT_EPSILON;
// thresholds are over required_eb directly (log2(1+x) folded in).
const QuantTable& quant_table_3d();

// ---- context ----------------------------------------------------------------
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t used = 0;
};

}  // namespace cpsz

struct cpsz_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;  // second stream for overlapping independent stages
  cudaStream_t hi = nullptr;   // highest-priority stream: consumers that run beside their producer
  cudaEvent_t ev[8] = {};
  // batch passes' device work captured as CUDA graphs (pipeline2d.cu), each
  // replayed while its pass recurs; least recently used first
  struct PassGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
  };
  static constexpr size_t kMaxPassGraphs = 64;
  std::vector<PassGraph> pass_graphs;
  uint64_t graph_captures = 0, graph_replays = 0;
  // chunked host-to-device uploads (one event per chunk, recorded on `aux`)
  static constexpr int kUploadChunks = 32;
  cudaEvent_t up_ev[kUploadChunks] = {};
  // per (field, component) "histogram on the host" events of a compression pass
  static constexpr int kJobEvents = 64;
  cudaEvent_t job_ev[kJobEvents] = {};
  cpsz::Arena arena;
  // pinned ring for bulk copies of pageable host memory (transfer.h)
  static constexpr int kStageSlots = 4;
  static constexpr size_t kStageBytes = (size_t)16 << 20;
  void* stage = nullptr;
  cudaEvent_t stage_ev[kStageSlots] = {};
  void* pinned = nullptr;
  size_t pinned_cap = 0;
  // pinned staging of a pass's small uploads made once the pass's trees are
  // known (codebook entries, blob pieces): page-locked, so the copies are
  // asynchronous and never wait on the streams' earlier work
  void* up_pinned = nullptr;
  size_t up_cap = 0;
  uint64_t launches = 0;
  int num_sms = 0;
  int* d_flag = nullptr;  // device error / timeout flag (persistent)
  // optional per-stage timing of the last call (CUDA events on `stream`)
  bool timing = false;
  static constexpr int kMaxMarks = 24;
  cudaEvent_t tev[kMaxMarks] = {};
  const char* tname[kMaxMarks] = {};
  int nmarks = 0;
  // optional wavefront trace (diagnostics): 4 counters per (field, group, warp)
  long long* d_wave_trace = nullptr;
  size_t wave_trace_len = 0;
  // The wavefront that runs beside the bound kernel waits per row group for
  // the bounds (limit band_wait_ns, 0 = the kernel's default).  When a wait
  // gives up, the pass runs its wavefront again after the bounds
  // (wave_reruns counts these).  band_unreachable (diagnostics only) makes
  // every such wait run out, to exercise that path.
  long long band_wait_ns = 0;
  bool band_unreachable = false;
  uint64_t wave_reruns = 0;
  // device copy of the host log2f / exp2f tables (libm.h), uploaded on first use
  void* libm_mem = nullptr;
  void* libm_view = nullptr;  // cpsz::LibmTables*
};

namespace cpsz {

cpsz_b200_ctx* resolve_ctx(cpsz_b200_ctx* ctx, int* rc);
// Ensures the arena holds at least `bytes` and resets it for a new call.
int arena_reserve(cpsz_b200_ctx* ctx, size_t bytes);
// Bump allocation (256-byte aligned) from the reserved arena.
void* arena_alloc(cpsz_b200_ctx* ctx, size_t bytes);
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
int pinned_reserve(cpsz_b200_ctx* ctx, size_t bytes);
// Grows ctx->up_pinned to at least `bytes` (its old contents are dropped:
// call it only when no copy from it is in flight).
int upload_reserve(cpsz_b200_ctx* ctx, size_t bytes);

// Pointer kind: true if `p` is device (or managed) memory usable by kernels.
bool is_device_ptr(const void* p);

inline void count_launch(cpsz_b200_ctx* ctx, int n = 1) { ctx->launches += (uint64_t)n; }
// Stage marks: when timing is on, records an event named `name` on the stream;
// stage i spans marks i..i+1.  reset_marks() starts a new call.
void reset_marks(cpsz_b200_ctx* ctx);
void mark(cpsz_b200_ctx* ctx, const char* name);
int check_launch(const char* what);

}  // namespace cpsz
