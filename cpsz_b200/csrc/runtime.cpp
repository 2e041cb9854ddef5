// runtime.cpp -- errors, contexts, arenas and host-computed quantization tables.
#include "runtime.h"

#include "libm.h"
#include "tuning.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace cpsz {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(CPSZ_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return CPSZ_OK;
}

// ---- quantization tables ----------------------------------------------------

static inline uint64_t dbits(double x) {
  uint64_t b;
  memcpy(&b, &x, 8);
  return b;
}
static inline double bitsd(uint64_t b) {
  double x;
  memcpy(&x, &b, 8);
  return x;
}

// id of the 2D offline quantizer (include/sz_cp_preserve_utils.hpp:14-22 with
// base 4, log_of_base = log2(4), thr = DBL_EPSILON), evaluated with the host libm.
static int id_2d(double e) {
  const double thr = DBL_EPSILON;
  if (e <= thr) return 0;
  return (int)(log2(e / thr) / log2(4.0));
}

// id of the 3D offline_log quantizer for a required relative bound r
// (src/sz_compress_cp_preserve_3d.cpp:455-458: abs_eb = log2(1 + r), base 2,
// thr = FLT_EPSILON).  Valid for r > 0.
static int id_3d(double r) {
  const double thr = FLT_EPSILON;
  double abs_eb = log2(1 + r);
  if (abs_eb <= thr) return 0;
  return (int)(log2(abs_eb / thr) / log2(2.0));
}

// id of the 2D offline_log quantizer for a relative bound r
// (src/sz_compress_cp_preserve_2d.cpp:345-350: log2(1 + r), base 2, thr =
// DBL_EPSILON); 0 at or below the threshold.
static int id_2d_log(double r) {
  const double thr = DBL_EPSILON;
  const double e = log2(1 + r);
  if (e <= thr) return 0;
  return (int)(log2(e / thr) / log2(2.0));
}

// Smallest positive double x in [lo, hi] with f(x) >= k, by bisection on the
// (monotone) bit patterns of positive doubles.
template <class F>
static double first_at_least(F f, int k, double lo, double hi) {
  uint64_t a = dbits(lo), b = dbits(hi);
  if (f(bitsd(a)) >= k) return bitsd(a);
  while (b - a > 1) {
    uint64_t m = a + (b - a) / 2;
    if (f(bitsd(m)) >= k) b = m;
    else a = m;
  }
  return bitsd(b);
}

// Builds t[k] and checks monotonicity of the host function around each
// threshold (a window of 256 neighbouring doubles on each side).
template <class F>
static void build_table(QuantTable& T, F f, double lo, double hi) {
  int kmax = f(hi);
  if (kmax >= QuantTable::kMax) kmax = QuantTable::kMax - 1;
  if (kmax < 1) {
    fprintf(stderr, "cpsz_b200: quantization table bound invalid\n");
    kmax = 1;
  }
  T.n = kmax + 1;
  T.t[0] = lo;
  for (int k = 1; k <= kmax; k++) {
    T.t[k] = first_at_least(f, k, lo, hi);
    uint64_t b = dbits(T.t[k]);
    for (uint64_t d = 1; d <= 256; d++) {
      if (f(bitsd(b - d)) >= k || f(bitsd(b + d - 1)) < k) {
        fprintf(stderr, "cpsz_b200: host log2 is not monotone near quantization threshold %d\n", k);
        break;
      }
    }
  }
}

const QuantTable& quant_table_2d() {
  static QuantTable T;
  static std::once_flag once;
  std::call_once(once, [] {
    T.thr = DBL_EPSILON;
    T.base = 4;
    // e ranges over |U| * eb; the upper end keeps e / thr finite (ids beyond
    // the table's 255 are rejected by the kernel anyway).
    build_table(T, id_2d, DBL_EPSILON, 1e280);
    bool ok = T.n > 1;
    for (int k = 0; k < T.n && ok; k++) {
      const double p = ldexp(1.0, 2 * k - 52);
      ok = T.t[k] <= p && T.t[k] > (double)nextafterf((float)p, 0.f);
    }
    T.float_pow4 = ok;
  });
  return T;
}

const QuantTable& quant_table_2d_log() {
  static QuantTable T;
  static std::once_flag once;
  std::call_once(once, [] {
    T.thr = DBL_EPSILON;
    T.base = 2;
    // t[0]: the largest r whose log-domain bound log2(1 + r) is still <= thr
    // (precision 0); ids count thresholds above it
    const double first = first_at_least([](double r) { return log2(1 + r) > DBL_EPSILON ? 1 : 0; }, 1, DBL_MIN, 1.0);
    build_table(T, id_2d_log, bitsd(dbits(first) - 1), 1e300);
  });
  return T;
}

const QuantTable& quant_table_3d() {
  static QuantTable T;
  static std::once_flag once;
  std::call_once(once, [] {
    T.thr = FLT_EPSILON;
    T.base = 2;
    build_table(T, id_3d, DBL_MIN, 1e300);
  });
  return T;
}

// ---- contexts -----------------------------------------------------------------

static thread_local cpsz_b200_ctx* g_default_ctx[64] = {};

cpsz_b200_ctx* resolve_ctx(cpsz_b200_ctx* ctx, int* rc) {
  *rc = CPSZ_OK;
  if (ctx) {
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
      *rc = set_error(CPSZ_ERR_CUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
      return nullptr;
    }
    return ctx;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    *rc = set_error(CPSZ_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    return nullptr;
  }
  if (dev < 0 || dev >= 64) {
    *rc = set_error(CPSZ_ERR_INVALID, "device %d out of range", dev);
    return nullptr;
  }
  if (!g_default_ctx[dev]) {
    cpsz_b200_ctx* c = nullptr;
    int r = cpsz_b200_ctx_create(dev, &c);
    if (r != CPSZ_OK) {
      *rc = r;
      return nullptr;
    }
    g_default_ctx[dev] = c;
  }
  return g_default_ctx[dev];
}

// Cached pass graphs hold the workspace's and the page-locked staging's
// addresses (kernel arguments, memset and copy nodes); once either is
// reallocated they are destroyed, even if the new allocation happens to
// return the same address (the copy nodes refer to the old allocation).
static void drop_pass_graphs(cpsz_b200_ctx* ctx) {
  if (ctx->pass_graphs.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto& g : ctx->pass_graphs) cudaGraphExecDestroy(g.exec);
  ctx->pass_graphs.clear();
}

int arena_reserve(cpsz_b200_ctx* ctx, size_t bytes) {
  bytes = align_up(bytes + 4096, 1 << 20);
  ctx->arena.used = 0;
  if (ctx->arena.cap >= bytes) return CPSZ_OK;
  drop_pass_graphs(ctx);
  if (ctx->arena.base) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->arena.base);
    ctx->arena.base = nullptr;
    ctx->arena.cap = 0;
  }
  cudaError_t e = cudaMalloc((void**)&ctx->arena.base, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(CPSZ_ERR_NOMEM, "device workspace of %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  ctx->arena.cap = bytes;
  return CPSZ_OK;
}

void* arena_alloc(cpsz_b200_ctx* ctx, size_t bytes) {
  size_t off = align_up(ctx->arena.used, 256);
  if (off + bytes > ctx->arena.cap) return nullptr;
  ctx->arena.used = off + bytes;
  return ctx->arena.base + off;
}

int pinned_reserve(cpsz_b200_ctx* ctx, size_t bytes) {
  if (ctx->pinned_cap >= bytes) return CPSZ_OK;
  drop_pass_graphs(ctx);
  if (ctx->pinned) {
    cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_cap = 0;
  }
  bytes = align_up(bytes, 1 << 20);
  cudaError_t e = cudaMallocHost(&ctx->pinned, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(CPSZ_ERR_NOMEM, "pinned staging of %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  ctx->pinned_cap = bytes;
  return CPSZ_OK;
}

int upload_reserve(cpsz_b200_ctx* ctx, size_t bytes) {
  if (ctx->up_cap >= bytes) return CPSZ_OK;
  if (ctx->up_pinned) cudaFreeHost(ctx->up_pinned);
  ctx->up_pinned = nullptr;
  ctx->up_cap = 0;
  bytes = align_up(bytes, 1 << 20);
  cudaError_t e = cudaMallocHost(&ctx->up_pinned, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->up_pinned = nullptr;
    return set_error(CPSZ_ERR_NOMEM, "pinned upload staging of %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  ctx->up_cap = bytes;
  return CPSZ_OK;
}

void reset_marks(cpsz_b200_ctx* ctx) { ctx->nmarks = 0; }

void mark(cpsz_b200_ctx* ctx, const char* name) {
  if (!ctx->timing || ctx->nmarks >= cpsz_b200_ctx::kMaxMarks) return;
  int i = ctx->nmarks++;
  if (!ctx->tev[i]) cudaEventCreate(&ctx->tev[i]);
  ctx->tname[i] = name;
  cudaEventRecord(ctx->tev[i], ctx->stream);
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace cpsz

using namespace cpsz;

extern "C" {

const char* cpsz_b200_last_error(void) { return g_last_error.c_str(); }

int cpsz_b200_version(void) { return 10000; }

int cpsz_b200_ctx_create(int device, cpsz_b200_ctx** out) {
  if (!out) return set_error(CPSZ_ERR_INVALID, "ctx_create: null output");
  CPSZ_TRY(tune_autoload());
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_error(CPSZ_ERR_NO_DEVICE, "no CUDA device visible (%s)", cudaGetErrorString(e));
  }
  if (device < 0 || device >= n) return set_error(CPSZ_ERR_INVALID, "device %d out of range [0,%d)", device, n);
  CPSZ_CUDA_TRY(cudaSetDevice(device));
  cpsz_b200_ctx* c = new cpsz_b200_ctx();
  c->device = device;
  CPSZ_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CPSZ_CUDA_TRY(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
  {
    // the block scheduler dispatches a higher-priority stream's CTAs first as
    // SMs free up, so a consumer launched beside its producer starts early
    int lo_pri = 0, hi_pri = 0;
    CPSZ_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
    CPSZ_CUDA_TRY(cudaStreamCreateWithPriority(&c->hi, cudaStreamNonBlocking, hi_pri));
  }
  for (auto& ev : c->ev) CPSZ_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  for (auto& ev : c->up_ev) CPSZ_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  for (auto& ev : c->job_ev) CPSZ_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  for (auto& ev : c->stage_ev) CPSZ_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CPSZ_CUDA_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
  CPSZ_CUDA_TRY(cudaMalloc((void**)&c->d_flag, 64));
  CPSZ_CUDA_TRY(cudaMemset(c->d_flag, 0, 64));
  // Tables are built once per process, before any stream capture.
  (void)quant_table_2d();
  (void)quant_table_2d_log();
  (void)quant_table_3d();
  *out = c;
  return CPSZ_OK;
}

int cpsz_b200_ctx_destroy(cpsz_b200_ctx* c) {
  if (!c) return CPSZ_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->aux);
  if (c->hi) cudaStreamSynchronize(c->hi);
  for (auto& g : c->pass_graphs) cudaGraphExecDestroy(g.exec);
  if (c->arena.base) cudaFree(c->arena.base);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->up_pinned) cudaFreeHost(c->up_pinned);
  if (c->stage) cudaFreeHost(c->stage);
  if (c->d_flag) cudaFree(c->d_flag);
  if (c->libm_mem) cudaFree(c->libm_mem);
  delete (cpsz::LibmTables*)c->libm_view;
  for (auto& ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->up_ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->job_ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->stage_ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->tev)
    if (ev) cudaEventDestroy(ev);
  cudaStreamDestroy(c->stream);
  cudaStreamDestroy(c->aux);
  if (c->hi) cudaStreamDestroy(c->hi);
  for (auto& d : g_default_ctx)
    if (d == c) d = nullptr;
  delete c;
  return CPSZ_OK;
}

int cpsz_b200_ctx_kernel_launches(cpsz_b200_ctx* ctx, uint64_t* count) {
  int rc;
  ctx = resolve_ctx(ctx, &rc);
  if (!ctx) return rc;
  if (!count) return set_error(CPSZ_ERR_INVALID, "null count");
  *count = ctx->launches;
  return CPSZ_OK;
}

int cpsz_b200_ctx_graph_stats(cpsz_b200_ctx* ctx, uint64_t* captures, uint64_t* replays) {
  if (!ctx || !captures || !replays) return set_error(CPSZ_ERR_INVALID, "null argument");
  *captures = ctx->graph_captures;
  *replays = ctx->graph_replays;
  return CPSZ_OK;
}

int cpsz_b200_ctx_wave_reruns(cpsz_b200_ctx* ctx, uint64_t* reruns) {
  if (!ctx || !reruns) return set_error(CPSZ_ERR_INVALID, "null argument");
  *reruns = ctx->wave_reruns;
  return CPSZ_OK;
}

int cpsz_b200_debug_band_wait(cpsz_b200_ctx* ctx, long long wait_ns, int unreachable) {
  if (!ctx) return set_error(CPSZ_ERR_INVALID, "null argument");
  if (wait_ns < 0) return set_error(CPSZ_ERR_INVALID, "negative wait limit");
  ctx->band_wait_ns = wait_ns;
  ctx->band_unreachable = unreachable != 0;
  return CPSZ_OK;
}

int cpsz_b200_ctx_set_timing(cpsz_b200_ctx* ctx, int on) {
  int rc;
  ctx = resolve_ctx(ctx, &rc);
  if (!ctx) return rc;
  ctx->timing = on != 0;
  ctx->nmarks = 0;
  return CPSZ_OK;
}

int cpsz_b200_ctx_stage_times(cpsz_b200_ctx* ctx, int max_stages, const char** names, float* ms, int* n_stages) {
  int rc;
  ctx = resolve_ctx(ctx, &rc);
  if (!ctx) return rc;
  if (!n_stages) return set_error(CPSZ_ERR_INVALID, "null n_stages");
  int n = ctx->nmarks > 0 ? ctx->nmarks - 1 : 0;
  if (n > max_stages) n = max_stages;
  for (int i = 0; i < n; i++) {
    cudaError_t e = cudaEventSynchronize(ctx->tev[i + 1]);
    if (e != cudaSuccess) return set_error(CPSZ_ERR_CUDA, "stage timing: %s", cudaGetErrorString(e));
    float t = 0;
    cudaEventElapsedTime(&t, ctx->tev[i], ctx->tev[i + 1]);
    if (names) names[i] = ctx->tname[i];
    if (ms) ms[i] = t;
  }
  *n_stages = n;
  return CPSZ_OK;
}

int cpsz_b200_ctx_stream(cpsz_b200_ctx* ctx, void** stream) {
  int rc;
  ctx = resolve_ctx(ctx, &rc);
  if (!ctx) return rc;
  if (!stream) return set_error(CPSZ_ERR_INVALID, "null stream output");
  *stream = (void*)ctx->stream;
  return CPSZ_OK;
}

}  // extern "C"
