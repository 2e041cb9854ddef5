// learned.cu -- the learned error-bound path (2D offline format, decoder
// unchanged): an MLP proposes a log2 multiplier of every vertex's analytic
// bound; the fallback loop compresses with the proposed bounds, reconstructs,
// checks every cell's critical point exactly against the original field, and
// reverts the vertices of offending cells to their analytic bounds until no
// cell differs.  Only the stored bound ids change, so the blob stays readable
// by sz_decompress_cp_preserve_2d_offline.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "cpsz_b200.h"
#include "kernels.h"
#include "transfer.h"
#include "pipeline.h"

struct cpsz_b200_mlp {
  cpsz_b200_ctx* ctx = nullptr;
  cpsz::MlpParams w{};
  void* mem = nullptr;
  int step = 0;
  // training scratch (grown on demand)
  void* scratch = nullptr;
  size_t scratch_cap = 0;
};

namespace cpsz {

namespace {

constexpr float TMAX = 16.f;  // largest log2 multiplier proposed

// Proposed bound eb_a * 2^m, m clamped to [0, TMAX], and never above the
// caller's point-wise relative bound max_pwr_eb: a vertex's relative error
// stays within what the plain compressor promises (its analytic bound is
// min(max_pwr_eb, bounds of its triangles), src/sz_compress_cp_preserve_2d.cpp:195-218),
// so the learned form only loosens bounds the critical points constrain.
__global__ void scale_bounds_kernel(const double* __restrict__ eb_a, const float* __restrict__ mult, size_t n,
                                    double max_pwr_eb, double* __restrict__ eb,
                                    unsigned long long* __restrict__ enlarged) {
  unsigned long long c = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float m = mult[i];
    m = (m == m) ? fminf(fmaxf(m, 0.f), TMAX) : 0.f;
    const double a = eb_a[i];
    const double e = a * exp2((double)m);
    eb[i] = e > max_pwr_eb ? (a > max_pwr_eb ? a : max_pwr_eb) : e;
    c += eb[i] != a;
  }
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(enlarged, c);
}

// Cell c's CP code differs between the original (cells_a) and the
// reconstruction (cells_b): revert its vertices whose
// bound was enlarged (counts[0] cells differing, counts[1] of them with no
// enlarged vertex left).
__device__ __forceinline__ void mark_cell(long long c, int r2, const double* __restrict__ eb,
                                          const double* __restrict__ eb_a, uint8_t* __restrict__ revert,
                                          unsigned long long& stuck) {
  const long long q = c >> 1;
  const int k = (int)(c & 1);
  const int i = (int)(q / (r2 - 1)), j = (int)(q - (long long)i * (r2 - 1));
  const size_t p[3] = {(size_t)i * r2 + j, (size_t)(i + (k == 0)) * r2 + j + (k == 1), (size_t)(i + 1) * r2 + j + 1};
  bool any = false;
  for (int t = 0; t < 3; t++)
    if (eb[p[t]] != eb_a[p[t]]) {
      revert[p[t]] = 1;
      any = true;
    }
  stuck += !any;
}

// Differing cells are rare: 16 cells per load, a byte loop only where a
// 16-byte word differs (ca and cb are 16-byte aligned).
__global__ void mark_kernel(const uint8_t* __restrict__ ca, const uint8_t* __restrict__ cb, int r1, int r2,
                            const double* __restrict__ eb, const double* __restrict__ eb_a, uint8_t* __restrict__ revert,
                            unsigned long long* __restrict__ counts) {
  const long long ncell = 2LL * (r1 - 1) * (r2 - 1);
  const long long nvec = ncell / 16;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long long)gridDim.x * blockDim.x;
  unsigned long long diff = 0, stuck = 0;
  for (long long v = tid; v < nvec; v += nt) {
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(ca) + v), y = __ldg(reinterpret_cast<const uint4*>(cb) + v);
    if (x.x == y.x && x.y == y.y && x.z == y.z && x.w == y.w) continue;
    for (int e = 0; e < 16; e++) {
      const long long c = 16 * v + e;
      if (ca[c] == cb[c]) continue;
      diff++;
      mark_cell(c, r2, eb, eb_a, revert, stuck);
    }
  }
  for (long long c = 16 * nvec + tid; c < ncell; c += nt) {
    if (ca[c] == cb[c]) continue;
    diff++;
    mark_cell(c, r2, eb, eb_a, revert, stuck);
  }
  for (int o = 16; o; o >>= 1) {
    diff += __shfl_xor_sync(0xffffffffu, diff, o);
    stuck += __shfl_xor_sync(0xffffffffu, stuck, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (diff) atomicAdd(&counts[0], diff);
    if (stuck) atomicAdd(&counts[1], stuck);
  }
}

__device__ __forceinline__ void revert_one(size_t i, uint8_t* __restrict__ revert, uint8_t* __restrict__ requant,
                                           const double* __restrict__ eb_a, double* __restrict__ eb,
                                           unsigned long long& c, size_t& first) {
  revert[i] = 0;
  requant[i] = 1;
  c += eb[i] != eb_a[i];
  eb[i] = eb_a[i];
  first = i < first ? i : first;
}

// Marked vertices get their analytic bound back and are flagged for
// quantization in the next pass (16 flags per load; revert is 16-byte
// aligned); first gets the lowest flagged vertex index (atomic min).
__global__ void revert_kernel(uint8_t* __restrict__ revert, uint8_t* __restrict__ requant,
                              const double* __restrict__ eb_a, double* __restrict__ eb, size_t n,
                              unsigned long long* __restrict__ count, unsigned long long* __restrict__ first_out) {
  unsigned long long c = 0;
  size_t first = ~(size_t)0;
  const size_t nvec = n / 16;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (size_t)gridDim.x * blockDim.x;
  for (size_t v = tid; v < nvec; v += nt) {
    const uint4 x = reinterpret_cast<const uint4*>(revert)[v];
    if ((x.x | x.y | x.z | x.w) == 0) continue;
    for (int e = 0; e < 16; e++)
      if (revert[16 * v + e]) revert_one(16 * v + e, revert, requant, eb_a, eb, c, first);
  }
  for (size_t i = 16 * nvec + tid; i < n; i += nt)
    if (revert[i]) revert_one(i, revert, requant, eb_a, eb, c, first);
  for (int o = 16; o; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    const size_t f = __shfl_xor_sync(0xffffffffu, first, o);
    first = f < first ? f : first;
  }
  if ((threadIdx.x & 31) == 0) {
    if (c) atomicAdd(count, c);
    if (first != ~(size_t)0) atomicMin(first_out, (unsigned long long)first);
  }
}

int grid_of(cpsz_b200_ctx* ctx, size_t n) {
  size_t g = (n + 255) / 256;
  const size_t cap = (size_t)ctx->num_sms * 8;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// A device allocation freed when the holder goes out of scope.
struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    CPSZ_CUDA_TRY(cudaMalloc(&p, bytes));
    return CPSZ_OK;
  }
};

int ensure_scratch(cpsz_b200_mlp* m, size_t bytes) {
  if (m->scratch_cap >= bytes) return CPSZ_OK;
  if (m->scratch) {
    cudaStreamSynchronize(m->ctx->stream);
    cudaFree(m->scratch);
    m->scratch = nullptr;
    m->scratch_cap = 0;
  }
  CPSZ_CUDA_TRY(cudaMalloc(&m->scratch, bytes));
  m->scratch_cap = bytes;
  return CPSZ_OK;
}

}  // namespace

// The fallback loop (see the file comment).  stats: {passes (reconstruction
// passes + the final compression),
// vertices reverted, 1 if the loop gave up and the analytic bounds were used
// everywhere, vertices whose enlarged bound was kept}.
int compress_2d_learned(cpsz_b200_ctx* ctx, cpsz_b200_mlp* mlp, const float* U_in, const float* V_in, size_t r1s,
                        size_t r2s, double max_pwr_eb, const float* mult_in, Blob2D* out, uint64_t stats[4]) {
  if (!U_in || !V_in) return set_error(CPSZ_ERR_INVALID, "null input field");
  if (!mlp && !mult_in) return set_error(CPSZ_ERR_INVALID, "neither a proposer MLP nor multipliers given");
  if (r1s < 2 || r2s < 2 || r1s * r2s > (size_t)INT32_MAX)
    return set_error(CPSZ_ERR_UNSUPPORTED, "learned bounds need a field of at least 2 x 2 and below 2^31 points");
  const int r1 = (int)r1s, r2 = (int)r2s;
  const size_t N = r1s * r2s, ncell = 2 * (r1s - 1) * (r2s - 1);
  cudaStream_t st = ctx->stream;
  const bool dev_in = is_device_ptr(U_in) && is_device_ptr(V_in);
  // workspace of the loop (the compressor's own arena is reused by every pass)
  DevMem mem;
  const size_t bytes = align_up(8 * N, 256) * 2 + align_up(QUANT_TAB_MAX * 8, 256) + align_up(4 * N, 256) * 3 +
                       align_up(2 * N, 256) +
                       align_up(ncell, 256) * 2 + align_up(N, 256) * 2 + 4096 + (dev_in ? 0 : align_up(8 * N, 256));
  CPSZ_TRY(mem.alloc(bytes));
  uint8_t* w = (uint8_t*)mem.p;
  auto take = [&](size_t b) {
    void* p = w;
    w += align_up(b, 256);
    return p;
  };
  double* eb_a = (double*)take(8 * N);
  double* eb = (double*)take(8 * N);
  double* thr_tab = (double*)take(QUANT_TAB_MAX * 8);
  float* mult = (float*)take(4 * N);
  float* rec_u = (float*)take(4 * N);
  float* rec_v = (float*)take(4 * N);
  uint8_t* ids = (uint8_t*)take(2 * N);
  uint8_t* cells_a = (uint8_t*)take(ncell);
  uint8_t* cells_b = (uint8_t*)take(ncell);
  uint8_t* revert = (uint8_t*)take(N);
  uint8_t* requant = (uint8_t*)take(N);  // vertices reverted since the last pass (quantized again)
  unsigned long long* counts = (unsigned long long*)take(4096);
  const float* dU = U_in;
  const float* dV = V_in;
  if (!dev_in) {
    float* h = (float*)take(8 * N);
    CPSZ_TRY(h2d(ctx, h, U_in, 4 * N, st));
    CPSZ_TRY(h2d(ctx, h + N, V_in, 4 * N, st));
    dU = h;
    dV = h + N;
  }
  const QuantTable& qt = quant_table_2d();
  CPSZ_CUDA_TRY(cudaMemcpyAsync(thr_tab, qt.t, QUANT_TAB_MAX * 8, cudaMemcpyHostToDevice, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(counts, 0, 4096, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(revert, 0, N, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(requant, 0, N, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  // analytic bounds (the hist / pair outputs are not needed here)
  CPSZ_TRY(launch_eb2d(ctx, dU, dV, r1, r2, max_pwr_eb, thr_tab, qt.n, ids, ids + N, counts + 64, nullptr, nullptr,
                       eb_a));
  // proposals
  if (mult_in) {
    CPSZ_CUDA_TRY(cudaMemcpyAsync(mult, mult_in, 4 * N, is_device_ptr(mult_in) ? cudaMemcpyDeviceToDevice
                                                                                : cudaMemcpyHostToDevice,
                                  st));
  } else {
    CPSZ_TRY(launch_mlp_forward(ctx, mlp->w, nullptr, dU, dV, eb_a, r1, r2, (int)N, mult, nullptr, nullptr));
  }
  scale_bounds_kernel<<<grid_of(ctx, N), 256, 0, st>>>(eb_a, mult, N, max_pwr_eb, eb, counts + 4);
  count_launch(ctx);
  CPSZ_TRY(check_launch("scale_bounds_kernel"));
  CPSZ_TRY(launch_cp_check_2d(ctx, dU, dV, nullptr, nullptr, r1, r2, cells_a, counts + 8));
  // the loop's passes stop after the Lorenzo stage (the reconstruction is all
  // the check needs); one full compression follows with the final bounds
  StageTap tap;
  tap.recon[0] = rec_u;
  tap.recon[1] = rec_v;
  tap.recon_only = true;
  uint64_t reverted = 0;
  int it = 0;
  unsigned long long h[7] = {0, 0, 0, 0, 0, 0, 0};
  for (;; it++) {
    // After the first pass only the vertices reverted since are quantized
    // again (the rest of the quantization stays in the compressor's
    // workspace), and the recursion and the check start at the row group of
    // the first of them: rows above it reconstruct as before.
    int first_group = 0;
    if (it > 0) {
      first_group = (int)(h[6] / (unsigned long long)r2) / WAVE_GROUP_ROWS;
      tap.requant = requant;
      tap.first_group = first_group;
    }
    CPSZ_TRY(compress_2d(ctx, dU, dV, r1s, r2s, max_pwr_eb, out, &tap, eb));
    CPSZ_CUDA_TRY(cudaMemsetAsync(counts, 0, 32, st));
    CPSZ_CUDA_TRY(cudaMemsetAsync(counts + 6, 0xff, 8, st));
    // cells of row first_group * WAVE_GROUP_ROWS - 1 on touch the changed rows
    CPSZ_TRY(launch_cp_check_2d(ctx, rec_u, rec_v, nullptr, nullptr, r1, r2, cells_b, counts + 8,
                                first_group * WAVE_GROUP_ROWS - 1));
    mark_kernel<<<grid_of(ctx, ncell), 256, 0, st>>>(cells_a, cells_b, r1, r2, eb, eb_a, revert, counts);
    count_launch(ctx);
    CPSZ_TRY(check_launch("mark_kernel"));
    revert_kernel<<<grid_of(ctx, N), 256, 0, st>>>(revert, requant, eb_a, eb, N, counts + 2, counts + 6);
    count_launch(ctx);
    CPSZ_TRY(check_launch("revert_kernel"));
    CPSZ_CUDA_TRY(cudaMemcpyAsync(h, counts, 56, cudaMemcpyDeviceToHost, st));
    CPSZ_CUDA_TRY(cudaStreamSynchronize(st));
    reverted += h[2];
    // clean, or nothing left to revert (every offending cell already analytic)
    if (h[0] == 0 || h[2] == 0 || it >= 63) break;
  }
  const bool fallback = h[0] != 0;
  if (fallback) {
    // not converged: the analytic bounds everywhere (the plain compressor)
    CPSZ_TRY(compress_2d(ctx, dU, dV, r1s, r2s, max_pwr_eb, out, nullptr, nullptr));
  } else {
    CPSZ_TRY(compress_2d(ctx, dU, dV, r1s, r2s, max_pwr_eb, out, nullptr, eb));
  }
  unsigned long long enlarged = 0;
  CPSZ_CUDA_TRY(cudaMemcpy(&enlarged, counts + 4, 8, cudaMemcpyDeviceToHost));
  if (stats) {
    stats[0] = (uint64_t)it + 2;
    stats[1] = reverted;
    stats[2] = fallback ? 1 : 0;
    stats[3] = fallback ? 0 : enlarged - reverted;
  }
  return CPSZ_OK;
}

}  // namespace cpsz

using namespace cpsz;

namespace {

int resolve(cpsz_b200_ctx*& ctx) {
  int rc = CPSZ_OK;
  ctx = resolve_ctx(ctx, &rc);
  if (!ctx) return rc;
  clear_error();
  return CPSZ_OK;
}

// Host or device source -> device destination.
int upload(cpsz_b200_ctx* ctx, void* dst, const void* src, size_t n) { return h2d(ctx, dst, src, n, ctx->stream); }
int download(cpsz_b200_ctx* ctx, void* dst, const void* src, size_t n) { return d2h(ctx, dst, src, n, ctx->stream); }

// training scratch layout for n samples: X | H1 | H2 (bf16 n x 128) | y | t (f32) | loss
struct TrainBufs {
  void* X;
  void* H1;
  void* H2;
  float* y;
  float* t;
  float* loss;
};
int train_bufs(cpsz_b200_mlp* m, size_t n, TrainBufs* b) {
  const size_t act = align_up(n * 256, 256);
  const size_t vec = align_up(n * 4, 256);
  CPSZ_TRY(ensure_scratch(m, 3 * act + 2 * vec + 256));
  uint8_t* p = (uint8_t*)m->scratch;
  b->X = p;
  b->H1 = p + act;
  b->H2 = p + 2 * act;
  b->y = (float*)(p + 3 * act);
  b->t = (float*)(p + 3 * act + vec);
  b->loss = (float*)(p + 3 * act + 2 * vec);
  return CPSZ_OK;
}

}  // namespace

extern "C" {

size_t cpsz_b200_mlp_param_count(void) { return (size_t)MLP_PARAMS; }

int cpsz_b200_mlp_create(cpsz_b200_ctx* ctx, uint64_t seed, cpsz_b200_mlp** out) {
  if (!out) return set_error(CPSZ_ERR_INVALID, "null output");
  CPSZ_TRY(resolve(ctx));
  cpsz_b200_mlp* m = new cpsz_b200_mlp();
  m->ctx = ctx;
  const size_t P = MLP_PARAMS;
  const size_t fbytes = align_up(P * 4, 256);
  if (cudaMalloc(&m->mem, 4 * fbytes + 2 * 16384 * 2) != cudaSuccess) {
    delete m;
    return set_error(CPSZ_ERR_NOMEM, "MLP parameters");
  }
  uint8_t* p = (uint8_t*)m->mem;
  m->w.p = (float*)p;
  m->w.g = (float*)(p + fbytes);
  m->w.m = (float*)(p + 2 * fbytes);
  m->w.v = (float*)(p + 3 * fbytes);
  m->w.w1b = p + 4 * fbytes;
  m->w.w2b = p + 4 * fbytes + 16384 * 2;
  // He initialisation (deterministic), padded inputs zero
  std::vector<float> h(P, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> nd(0.0, 1.0);
  for (int o = 0; o < 128; o++)
    for (int i = 0; i < 99; i++) h[o * 128 + i] = (float)(nd(rng) * std::sqrt(2.0 / 99.0));
  for (int k = 0; k < 16384; k++) h[16384 + 128 + k] = (float)(nd(rng) * std::sqrt(2.0 / 128.0));
  for (int k = 0; k < 128; k++) h[2 * 16384 + 256 + k] = (float)(nd(rng) * std::sqrt(1.0 / 128.0));
  cudaMemcpy(m->w.p, h.data(), P * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->w.g, 0, 3 * fbytes);
  int rc = launch_mlp_cast(ctx, m->w);
  if (rc == CPSZ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "MLP init");
  if (rc != CPSZ_OK) {
    cudaFree(m->mem);
    delete m;
    return rc;
  }
  *out = m;
  return CPSZ_OK;
}

int cpsz_b200_mlp_destroy(cpsz_b200_mlp* m) {
  if (!m) return CPSZ_OK;
  cudaStreamSynchronize(m->ctx->stream);
  if (m->scratch) cudaFree(m->scratch);
  if (m->mem) cudaFree(m->mem);
  delete m;
  return CPSZ_OK;
}

int cpsz_b200_mlp_get_params(cpsz_b200_mlp* m, float* out) {
  if (!m || !out) return set_error(CPSZ_ERR_INVALID, "null argument");
  CPSZ_CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  CPSZ_CUDA_TRY(cudaMemcpy(out, m->w.p, (size_t)MLP_PARAMS * 4, cudaMemcpyDeviceToHost));
  return CPSZ_OK;
}

int cpsz_b200_mlp_set_params(cpsz_b200_mlp* m, const float* in) {
  if (!m || !in) return set_error(CPSZ_ERR_INVALID, "null argument");
  CPSZ_CUDA_TRY(cudaMemcpy(m->w.p, in, (size_t)MLP_PARAMS * 4, cudaMemcpyHostToDevice));
  CPSZ_CUDA_TRY(cudaMemset(m->w.m, 0, (size_t)MLP_PARAMS * 4));
  CPSZ_CUDA_TRY(cudaMemset(m->w.v, 0, (size_t)MLP_PARAMS * 4));
  m->step = 0;
  CPSZ_TRY(launch_mlp_cast(m->ctx, m->w));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_mlp_forward(cpsz_b200_mlp* m, const uint16_t* X, size_t n, float* y) {
  if (!m || !X || !y) return set_error(CPSZ_ERR_INVALID, "null argument");
  if (n > (size_t)INT32_MAX / 2) return set_error(CPSZ_ERR_UNSUPPORTED, "too many rows");
  cpsz_b200_ctx* ctx = m->ctx;
  TrainBufs b;
  CPSZ_TRY(train_bufs(m, n, &b));
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  CPSZ_TRY(upload(ctx, b.X, X, n * 256));
  CPSZ_TRY(launch_mlp_forward(ctx, m->w, b.X, nullptr, nullptr, nullptr, 0, 0, (int)n, b.y, nullptr, nullptr));
  CPSZ_TRY(download(ctx, y, b.y, n * 4));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  int flag = 0;
  CPSZ_CUDA_TRY(cudaMemcpy(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return set_error(CPSZ_ERR_TIMEOUT, "MLP forward: an MMA completion wait gave up");
  return CPSZ_OK;
}

// One training step on n samples (features X, targets t): forward, backward,
// and (when lr > 0) an Adam update; grads_out (optional, host) receives the
// gradients of mean (y - t)^2, loss_out the mean squared error.
int cpsz_b200_mlp_train_step(cpsz_b200_mlp* m, const uint16_t* X, const float* t, size_t n, float lr,
                             float* grads_out, float* loss_out) {
  if (!m || !X || !t || !n) return set_error(CPSZ_ERR_INVALID, "null argument");
  if (n > (size_t)INT32_MAX / 2) return set_error(CPSZ_ERR_UNSUPPORTED, "too many rows");
  cpsz_b200_ctx* ctx = m->ctx;
  TrainBufs b;
  CPSZ_TRY(train_bufs(m, n, &b));
  cudaStream_t st = ctx->stream;
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), st));
  CPSZ_TRY(upload(ctx, b.X, X, n * 256));
  CPSZ_TRY(upload(ctx, b.t, t, n * 4));
  CPSZ_CUDA_TRY(cudaMemsetAsync(b.loss, 0, 4, st));
  CPSZ_CUDA_TRY(cudaMemsetAsync(m->w.g, 0, (size_t)MLP_PARAMS * 4, st));
  CPSZ_TRY(launch_mlp_forward(ctx, m->w, b.X, nullptr, nullptr, nullptr, 0, 0, (int)n, b.y, b.H1, b.H2));
  CPSZ_TRY(launch_mlp_backward(ctx, m->w, b.X, b.H1, b.H2, b.y, b.t, (int)n, 2.f / (float)n, b.loss));
  if (grads_out) CPSZ_TRY(download(ctx, grads_out, m->w.g, (size_t)MLP_PARAMS * 4));
  if (lr > 0) CPSZ_TRY(launch_mlp_adam(ctx, m->w, lr, ++m->step));
  float loss = 0;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(&loss, b.loss, 4, cudaMemcpyDeviceToHost, st));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(st));
  int flag = 0;
  CPSZ_CUDA_TRY(cudaMemcpy(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return set_error(CPSZ_ERR_TIMEOUT, "MLP training step: an MMA completion wait gave up");
  if (loss_out) *loss_out = loss / (float)n;
  return CPSZ_OK;
}

int cpsz_b200_mlp_features_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                              const double* eb_analytic, const int32_t* idx, size_t n, uint16_t* X) {
  CPSZ_TRY(resolve(ctx));
  if (!U || !V || !eb_analytic || !idx || !X) return set_error(CPSZ_ERR_INVALID, "null argument");
  const size_t N = r1 * r2;
  DevMem mem;
  CPSZ_TRY(mem.alloc(8 * N + 8 * N + 4 * n + 256 * n + 4096));
  uint8_t* p = (uint8_t*)mem.p;
  float* dU = (float*)p;
  float* dV = dU + N;
  double* deb = (double*)(p + 8 * N);
  int* didx = (int*)(p + 16 * N);
  void* dX = p + 16 * N + align_up(4 * n, 256);
  CPSZ_TRY(upload(ctx, dU, U, 4 * N));
  CPSZ_TRY(upload(ctx, dV, V, 4 * N));
  CPSZ_TRY(upload(ctx, deb, eb_analytic, 8 * N));
  CPSZ_TRY(upload(ctx, didx, idx, 4 * n));
  CPSZ_TRY(launch_mlp_features(ctx, dU, dV, (int)r1, (int)r2, deb, didx, (int)n, dX));
  CPSZ_TRY(download(ctx, X, dX, 256 * n));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_mlp_propose_2d(cpsz_b200_mlp* mlp, const float* U, const float* V, size_t r1, size_t r2,
                             const double* eb_analytic, float* y) {
  if (!mlp) return set_error(CPSZ_ERR_INVALID, "null MLP");
  cpsz_b200_ctx* ctx = mlp->ctx;
  CPSZ_TRY(resolve(ctx));
  if (!U || !V || !eb_analytic || !y) return set_error(CPSZ_ERR_INVALID, "null argument");
  if (r1 * r2 == 0 || r1 * r2 > (size_t)INT32_MAX) return set_error(CPSZ_ERR_UNSUPPORTED, "field size out of range");
  const size_t N = r1 * r2;
  DevMem mem;
  CPSZ_TRY(mem.alloc(8 * N + 8 * N + 4 * N + 4096));
  uint8_t* p = (uint8_t*)mem.p;
  float* dU = (float*)p;
  float* dV = dU + N;
  double* deb = (double*)(p + 8 * N);
  float* dy = (float*)(p + 16 * N);
  CPSZ_TRY(upload(ctx, dU, U, 4 * N));
  CPSZ_TRY(upload(ctx, dV, V, 4 * N));
  CPSZ_TRY(upload(ctx, deb, eb_analytic, 8 * N));
  CPSZ_TRY(pinned_reserve(ctx, 4096));
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  CPSZ_TRY(launch_mlp_forward(ctx, mlp->w, nullptr, dU, dV, deb, (int)r1, (int)r2, (int)N, dy, nullptr, nullptr));
  CPSZ_TRY(download(ctx, y, dy, 4 * N));
  int flag = 0;
  CPSZ_CUDA_TRY(cudaMemcpyAsync(ctx->pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  flag = *(int*)ctx->pinned;
  if (flag & FLAG_TIMEOUT) return set_error(CPSZ_ERR_TIMEOUT, "a bounded device-side wait gave up");
  return CPSZ_OK;
}

int cpsz_b200_debug_mlp_forward_ms(cpsz_b200_mlp* mlp, const float* U, const float* V, size_t r1, size_t r2,
                                   const double* eb_analytic, int reps, float* ms) {
  if (!mlp || !ms || reps < 1) return set_error(CPSZ_ERR_INVALID, "null argument or no repetition");
  cpsz_b200_ctx* ctx = mlp->ctx;
  CPSZ_TRY(resolve(ctx));
  if (!U || !V || !eb_analytic || !is_device_ptr(U) || !is_device_ptr(V) || !is_device_ptr(eb_analytic))
    return set_error(CPSZ_ERR_INVALID, "U, V and the analytic bounds must be device memory");
  const size_t N = r1 * r2;
  if (N == 0 || N > (size_t)INT32_MAX) return set_error(CPSZ_ERR_UNSUPPORTED, "field size out of range");
  CPSZ_TRY(ensure_scratch(mlp, 4 * N + 256));
  float* dy = (float*)mlp->scratch;
  cudaEvent_t a, b;
  CPSZ_CUDA_TRY(cudaEventCreate(&a));
  CPSZ_CUDA_TRY(cudaEventCreate(&b));
  CPSZ_CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  int rc = launch_mlp_forward(ctx, mlp->w, nullptr, U, V, eb_analytic, (int)r1, (int)r2, (int)N, dy, nullptr, nullptr);
  if (rc == CPSZ_OK && cudaEventRecord(a, ctx->stream) != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "event");
  for (int k = 0; k < reps && rc == CPSZ_OK; k++)
    rc = launch_mlp_forward(ctx, mlp->w, nullptr, U, V, eb_analytic, (int)r1, (int)r2, (int)N, dy, nullptr, nullptr);
  if (rc == CPSZ_OK && cudaEventRecord(b, ctx->stream) != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "event");
  if (rc == CPSZ_OK && cudaEventSynchronize(b) != cudaSuccess) rc = set_error(CPSZ_ERR_CUDA, "event sync");
  float total = 0;
  if (rc == CPSZ_OK) cudaEventElapsedTime(&total, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CPSZ_TRY(rc);
  int flag = 0;
  CPSZ_CUDA_TRY(cudaMemcpy(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag & FLAG_TIMEOUT) return set_error(CPSZ_ERR_TIMEOUT, "a bounded device-side wait gave up");
  *ms = total / (float)reps;
  return CPSZ_OK;
}

int cpsz_b200_learned_labels_2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t r1, size_t r2,
                                const double* eb_analytic, const int32_t* idx, size_t n, int steps, float* t_out) {
  CPSZ_TRY(resolve(ctx));
  if (!U || !V || !eb_analytic || !idx || !t_out) return set_error(CPSZ_ERR_INVALID, "null argument");
  const size_t N = r1 * r2;
  DevMem mem;
  CPSZ_TRY(mem.alloc(16 * N + 8 * n + 4096));
  uint8_t* p = (uint8_t*)mem.p;
  float* dU = (float*)p;
  float* dV = dU + N;
  double* deb = (double*)(p + 8 * N);
  int* didx = (int*)(p + 16 * N);
  float* dt = (float*)(p + 16 * N + align_up(4 * n, 256));
  CPSZ_TRY(upload(ctx, dU, U, 4 * N));
  CPSZ_TRY(upload(ctx, dV, V, 4 * N));
  CPSZ_TRY(upload(ctx, deb, eb_analytic, 8 * N));
  CPSZ_TRY(upload(ctx, didx, idx, 4 * n));
  CPSZ_TRY(launch_labels_2d(ctx, dU, dV, (int)r1, (int)r2, deb, didx, (int)n, steps, TMAX, dt));
  CPSZ_TRY(download(ctx, t_out, dt, 4 * n));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

int cpsz_b200_compress_2d_learned_f32(cpsz_b200_ctx* ctx, cpsz_b200_mlp* mlp, const float* U, const float* V,
                                      size_t r1, size_t r2, double max_pwr_eb, const float* log2_mult,
                                      unsigned char* out, size_t out_cap, size_t* blob_size, uint64_t stats[4]) {
  if (!out || !blob_size) return set_error(CPSZ_ERR_INVALID, "null output");
  if (mlp && !ctx) ctx = mlp->ctx;
  CPSZ_TRY(resolve(ctx));
  Blob2D b;
  CPSZ_TRY(compress_2d_learned(ctx, mlp, U, V, r1, r2, max_pwr_eb, log2_mult, &b, stats));
  *blob_size = b.size;
  if (b.size > out_cap) return set_error(CPSZ_ERR_INVALID, "output capacity %zu < blob size %zu", out_cap, b.size);
  CPSZ_TRY(copy_out(ctx, out, b.d_blob, b.size));
  CPSZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CPSZ_OK;
}

}  // extern "C"
