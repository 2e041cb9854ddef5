// eb2d.cu -- 2D offline error-bound derivation fused with its exponential
// quantization and the id histogram.
//
// One CTA owns a TY x TX tile of vertices.  It stages the (TY+2) x (TX+2)
// vertex halo of U and V in shared memory (coalesced row loads), evaluates
// both triangles of every one of the (TY+1) x (TX+1) cells that touch the tile
// once (FP64, bit-exact to src/sz_compress_cp_preserve_2d.cpp:125-172), keeps
// the per-triangle bounds in shared memory, and then reduces the six incident
// triangles of each vertex in the reference's traversal order (:195-218).
// The vertex bound is quantized for U and V against host-computed thresholds
// (base 4, thr = 2^-52; include/sz_cp_preserve_utils.hpp:14-22, applied at
// src/sz_compress_cp_preserve_2d.cpp:226-244) and written as one byte per
// component: the id, or 255 when the bound is <= thr (precision 0, Huffman
// symbol 0).  A shared-memory histogram of the Huffman symbols is folded into
// a global one.
//
// The tile shape and block size are template parameters; the launch-shape
// table ("eb2d.tile", tuning.h) picks one of six instantiations per field
// size.  Every shape computes the same bytes: each vertex's bound is the same
// minimum over the same six triangles, whichever tile evaluates them.
//
// One CTA per tile (a 2D grid in row-major tile order, so row groups complete
// roughly in order): measured faster than a persistent grid that takes tiles
// with a stride or from a counter (3.75 against 4.27 ms at 8192^2 alone, and
// the wavefront beside it keeps pace only with the per-tile grid).
#include <algorithm>

#include "eb_math.cuh"
#include "kernels.h"
#include "tuning.h"

namespace cpsz {

// 64 registers a thread at most (2048 threads an SM): with the wavefront
// beside it, three 256-thread CTAs of this kernel still fit on an SM.
template <int TX, int TY, int NT, bool FAST, bool BATCH = false>
__global__ void __launch_bounds__(NT, 2048 / 64 / (NT / 32)) eb2d_kernel(const float* __restrict__ U, const float* __restrict__ V, int r1,
                                                  int r2, double max_pwr_eb, const double* __restrict__ thr_tab,
                                                  int thr_n, uint8_t* __restrict__ ids_u, uint8_t* __restrict__ ids_v,
                                                  unsigned long long* __restrict__ hist, int* __restrict__ flag,
                                                  float2* __restrict__ pair_u, float2* __restrict__ pair_v,
                                                  double* __restrict__ eb_out, int row_begin, int row_end,
                                                  const int2* __restrict__ unit_order, int unit_ncb,
                                                  unsigned long long* __restrict__ unit_done, int log_ids,
                                                  int pow4_ids, const Eb2dJob* __restrict__ bjobs, int bn) {
  constexpr int CX = TX + 1;  // cells per tile row
  constexpr int CY = TY + 1;
  static_assert(WAVE_GROUP_ROWS % TY == 0, "a tile's rows must lie in one wavefront group");
  static_assert(UNIT_COLS % TX == 0, "a tile's columns must lie in one unit");
  __shared__ float su[TY + 2][TX + 3];
  __shared__ float sv[TY + 2][TX + 3];
  // compression (FAST): the float bound of an ordinary triangle, or +inf when
  // the triangle took the exact path (its bound is in tri) or does not exist;
  // exact mode: tri alone
  __shared__ float trf[2][CY][CX];
  __shared__ double tri[2][CY][CX];
  __shared__ double tab[QUANT_TAB_MAX];
  __shared__ unsigned int shist[256];

  const int tid = threadIdx.x;
  int i0, j0;
  if constexpr (BATCH) {
    __shared__ int s_job;
    // a batched launch: the CTA's field (the last one whose tiles start at or
    // before it) takes the place of the single field's arguments
    if (tid == 0) {
      int lo = 0, hi = bn - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bjobs[mid].tile0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
      }
      s_job = lo;
    }
    __syncthreads();
    const Eb2dJob& d = bjobs[s_job];
    U = d.U;
    V = d.V;
    r1 = d.r1;
    r2 = d.r2;
    max_pwr_eb = d.max_pwr_eb;
    ids_u = d.ids_u;
    ids_v = d.ids_v;
    hist = d.hist;
    pair_u = d.pair_u;
    pair_v = d.pair_v;
    row_begin = 0;
    row_end = d.r1;
    const int t = (int)blockIdx.x - d.tile0;
    i0 = (t / d.tiles_x) * TY;
    j0 = (t % d.tiles_x) * TX;
  } else if (unit_order) {
    // tile t of unit blockIdx.x / tiles-per-unit, row-major inside the unit
    constexpr int TPR = UNIT_COLS / TX;  // tiles per unit row
    const int2 u = unit_order[blockIdx.x / (TPR * (WAVE_GROUP_ROWS / TY))];
    const int t = blockIdx.x % (TPR * (WAVE_GROUP_ROWS / TY));
    i0 = u.x * WAVE_GROUP_ROWS + (t / TPR) * TY;
    j0 = u.y * UNIT_COLS + (t % TPR) * TX;
    if (i0 >= row_end || j0 >= r2) return;  // beyond the field's last rows / columns (uniform)
  } else {
    i0 = row_begin + blockIdx.y * TY;
    j0 = blockIdx.x * TX;
  }
  for (int k = tid; k < 256; k += NT) shist[k] = 0;
  for (int k = tid; k < thr_n; k += NT) tab[k] = thr_tab[k];
  // vertex halo: rows i0-1 .. i0+TY, cols j0-1 .. j0+TX
  for (int k = tid; k < (TY + 2) * (TX + 2); k += NT) {
    int a = k / (TX + 2), b = k % (TX + 2);
    int gi = i0 - 1 + a, gj = j0 - 1 + b;
    float u = 0.f, v = 0.f;
    if (gi >= 0 && gi < r1 && gj >= 0 && gj < r2) {
      size_t g = (size_t)gi * r2 + gj;
      u = U[g];
      v = V[g];
    }
    su[a][b] = u;
    sv[a][b] = v;
  }
  __syncthreads();
  // cells (ci, cj) = (i0-1+a, j0-1+b), a in [0, CY), b in [0, CX).
  // Compression (FAST): both triangles of a cell per thread and round
  // (1089 cells over 256 threads at 32x32), the float bound in trf, or +inf
  // there and the exact bound in tri for a triangle that takes the exact
  // path; a cell outside the field holds +inf in both (it has no triangles,
  // and +inf leaves every vertex minimum unchanged).  Exact mode: one
  // triangle per thread and round, every exact bound in tri.  The exact
  // bound is a call (tri_eb_exact is not inlined), so its code is in the
  // instruction cache once.
  bool any_exact = false;
  if (FAST) {
    for (int c = tid; c < CY * CX; c += NT) {
      const int a = c / CX, b = c - (c / CX) * CX;
      const int ci = i0 - 1 + a, cj = j0 - 1 + b;
      const bool in = ci >= 0 && ci < r1 - 1 && cj >= 0 && cj < r2 - 1;
      float t[2] = {INFINITY, INFINITY};
      bool ok[2] = {false, false};
      if (in)
        dev::cell_eb_float(su[a][b], su[a + 1][b], su[a][b + 1], su[a + 1][b + 1], sv[a][b], sv[a + 1][b],
                           sv[a][b + 1], sv[a + 1][b + 1], t[0], t[1], ok[0], ok[1]);
#pragma unroll
      for (int kind = 0; kind < 2; kind++) {
        if (!ok[kind]) {
          double e = INFINITY;
          if (in) {
            // upper: (a,b), (a+1,b), (a+1,b+1); lower: (a,b), (a,b+1), (a+1,b+1)
            const int a1 = a + (kind == 0), b1 = b + (kind == 1);
            e = dev::tri_eb_exact(su[a][b], su[a1][b1], su[a + 1][b + 1], sv[a][b], sv[a1][b1], sv[a + 1][b + 1],
                                  kind);
            t[kind] = INFINITY;
            any_exact = true;
          }
          tri[kind][a][b] = e;
        }
        trf[kind][a][b] = t[kind];
      }
    }
  } else {
    for (int k = tid; k < 2 * CY * CX; k += NT) {
      const int kind = k >= CY * CX;
      const int c = k - kind * CY * CX;
      const int a = c / CX, b = c % CX;
      const int ci = i0 - 1 + a, cj = j0 - 1 + b;
      double e = 0;
      if (ci >= 0 && ci < r1 - 1 && cj >= 0 && cj < r2 - 1) {
        const int a1 = a + (kind == 0), b1 = b + (kind == 1);
        e = dev::tri_eb_exact(su[a][b], su[a1][b1], su[a + 1][b + 1], sv[a][b], sv[a1][b1], sv[a + 1][b + 1], kind);
      }
      tri[kind][a][b] = e;
    }
  }
  // whether any triangle of the tile took the exact path (uniform over the CTA)
  const bool tile_exact = __syncthreads_or(any_exact);
  const double thr = tab[0];
  const float eb_dn = __double2float_rd(max_pwr_eb), eb_up = __double2float_ru(max_pwr_eb);
  // id of a quantized bound e (-1 for precision 0), before the range check
  auto quant = [&](double e) -> int {
    if (e <= thr) return -1;
    const int ex = (int)((__double_as_longlong(e) >> 52) & 0x7ff) - 1023;
    return dev::count_thresholds(tab, thr_n, e, (ex + 52) >> (log_ids ? 0 : 1));
  };
  for (int k = tid; k < TY * TX; k += NT) {
    int a = k / TX, b = k % TX;
    int gi = i0 + a, gj = j0 + b;
    if (gi >= row_end || gj >= r2) continue;
    // vertex (gi, gj) is local (a+1, b+1); cell (gi-1+x, gj-1+y) is tri[.][a+x][b+y]
    bool up = gi >= 1, left = gj >= 1, down = gi < r1 - 1, right = gj < r2 - 1;
    const float uu = su[a + 1][b + 1], vv = sv[a + 1][b + 1];
    // Offline: one id per component, of |x| * eb (base 4).  offline_log: one
    // id of the vertex bound itself (the log2(1 + eb) quantizer's table).
    const double s0 = log_ids ? 1.0 : (double)fabsf(uu), s1 = (double)fabsf(vv);
    // the reference's chain eb = MINF(eb, triangle bound) over the six triangles
    auto vertex_eb = [&](auto&& tri_at) {
      double eb = max_pwr_eb;
      if (up && left) {
        eb = dev::minf_d(eb, tri_at(0, a, b));
        eb = dev::minf_d(eb, tri_at(1, a, b));
      }
      if (up && right) eb = dev::minf_d(eb, tri_at(0, a, b + 1));
      if (down && left) eb = dev::minf_d(eb, tri_at(1, a + 1, b));
      if (down && right) {
        eb = dev::minf_d(eb, tri_at(0, a + 1, b + 1));
        eb = dev::minf_d(eb, tri_at(1, a + 1, b + 1));
      }
      return eb;
    };
    int code[2];
    double eb = 0;
    if (FAST) {
      // enclosure of the vertex bound: the float bounds of its ordinary
      // triangles (min mf, each within FFILT_REL and FFILT_ABS of the
      // reference's value) and the exact ones (min md).  The six incident
      // triangles are read unconditionally: a missing one (a cell outside the
      // field) holds +inf.
      const float mf = fminf(fminf(fminf(trf[0][a][b], trf[1][a][b]), fminf(trf[0][a][b + 1], trf[1][a + 1][b])),
                             fminf(trf[0][a + 1][b + 1], trf[1][a + 1][b + 1]));
      double md = INFINITY;
      bool nan = false;
      if (tile_exact) {
        auto take = [&](int kind, int ca, int cb) {
          if (trf[kind][ca][cb] == INFINITY) {
            const double e = tri[kind][ca][cb];
            nan |= isnan(e);
            md = fmin(md, e);
          }
        };
        take(0, a, b);
        take(1, a, b);
        take(0, a, b + 1);
        take(1, a + 1, b);
        take(0, a + 1, b + 1);
        take(1, a + 1, b + 1);
      }
      // The float route: the same enclosure rounded outwards in float, each
      // component's |x| * bound with directed products, and the id of a float
      // read off its exponent (exact for this table: quant_table_2d's
      // float_pow4).  Ends with different ids, an id past the table's range
      // or an overflow take the double route below.
      bool decided = false;
      if (pow4_ids && !nan) {
        float lo_f = fminf(__fmaf_rd(mf, 1.0f - dev::FFILT_REL, -dev::FFILT_ABS), eb_dn);
        float hi_f = fminf(__fmaf_ru(mf, 1.0f + dev::FFILT_REL, dev::FFILT_ABS), eb_up);
        if (md < INFINITY) {
          lo_f = fminf(lo_f, __double2float_rd(md));
          hi_f = fminf(hi_f, __double2float_ru(md));
        }
        const float su = fabsf(uu), sv = fabsf(vv);
        const int c0 = dev::pow4_id(__fmul_rd(su, lo_f)), c0h = dev::pow4_id(__fmul_ru(su, hi_f));
        const int c1 = dev::pow4_id(__fmul_rd(sv, lo_f)), c1h = dev::pow4_id(__fmul_ru(sv, hi_f));
        if (c0 == c0h && c1 == c1h && c0h <= ID_MAX_2D && c1h <= ID_MAX_2D) {
          code[0] = c0;
          code[1] = c1;
          decided = true;
        }
      }
      if (!decided) {
        const double m = (double)mf;
        const double lo = fmin(max_pwr_eb, fmin(m * (1.0 - dev::FFILT_REL) - dev::FFILT_ABS, md));
        const double hi = fmin(max_pwr_eb, fmin(m * (1.0 + dev::FFILT_REL) + dev::FFILT_ABS, md));
        // the upper end has the same id iff it stays below the next threshold
        auto stays = [&](int c, double e) { return c < 0 ? e <= thr : (c + 1 >= thr_n || e < tab[c + 1]); };
        code[0] = quant(s0 * lo);
        code[1] = log_ids ? -1 : quant(s1 * lo);
        if (nan || !stays(code[0], s0 * hi) || (!log_ids && !stays(code[1], s1 * hi))) {
          // the enclosure straddles a threshold (or a bound is NaN): exact bounds
          eb = vertex_eb([&](int kind, int ca, int cb) {
            const int a1 = ca + (kind == 0), b1 = cb + (kind == 1);
            return dev::tri_eb_exact(su[ca][cb], su[a1][b1], su[ca + 1][cb + 1], sv[ca][cb], sv[a1][b1],
                                     sv[ca + 1][cb + 1], kind);
          });
          code[0] = quant(s0 * eb);
          code[1] = log_ids ? -1 : quant(s1 * eb);
        }
      }
    } else {
      eb = vertex_eb([&](int kind, int ca, int cb) { return tri[kind][ca][cb]; });
      code[0] = quant(s0 * eb);
      code[1] = log_ids ? -1 : quant(s1 * eb);
    }
    int sym[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
      if (code[c] > ID_MAX_2D) {
        atomicOr(flag, FLAG_ID_OVERFLOW);
        code[c] = ID_MAX_2D;
      }
      sym[c] = code[c] < 0 ? 0 : code[c];
      if (code[c] < 0) code[c] = ID_ZERO;
    }
    size_t g = (size_t)gi * r2 + gj;
    if (!FAST && eb_out) eb_out[g] = eb;
    ids_u[g] = (uint8_t)code[0];
    if (!log_ids) ids_v[g] = (uint8_t)code[1];
    if (pair_u) {
      // the wavefront's input: value and 1/precision = 2^(52 - 2 id) (NaN for precision 0)
      pair_u[g] = make_float2(uu, code[0] == ID_ZERO ? __int_as_float(0x7FC00000)
                                                     : __int_as_float((127 + 52 - 2 * (int)code[0]) << 23));
      pair_v[g] = make_float2(vv, code[1] == ID_ZERO ? __int_as_float(0x7FC00000)
                                                     : __int_as_float((127 + 52 - 2 * (int)code[1]) << 23));
    }
    atomicAdd(&shist[sym[0]], 1u);
    if (!log_ids) atomicAdd(&shist[sym[1]], 1u);
  }
  __syncthreads();
  for (int k = tid; k < 256; k += NT)
    if (shist[k]) atomicAdd(&hist[k], (unsigned long long)shist[k]);
  if (unit_done) {
    // every thread's outputs are visible device-wide before the tile counts;
    // unit_done[-1] counts finished tiles (the wavefront's sign of progress)
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      const int rows = min(TY, row_end - i0), cols = min(TX, r2 - j0);
      atomicAdd(&unit_done[(i0 / WAVE_GROUP_ROWS) * unit_ncb + j0 / UNIT_COLS], (unsigned long long)rows * cols);
      atomicAdd(&unit_done[-1], 1ull);
    }
  }
}

void unit_order(int g0, int g1, int ncb, int skew, std::vector<int2>& out) {
  out.clear();
  for (int g = g0; g < g1; g++)
    for (int b = 0; b < ncb; b++) out.push_back(make_int2(g, b));
  std::stable_sort(out.begin(), out.end(), [&](const int2& a, const int2& c) {
    const long long ka = (long long)a.y * skew + a.x, kc = (long long)c.y * skew + c.x;
    return ka < kc;
  });
}

int preload_eb2d() {
  // With lazy module loading a kernel's first launch loads its module, and a
  // load may wait for running kernels; a wavefront already waiting on eb2d
  // would then never see it start.  Querying the attributes loads each
  // instantiation up front.
  cudaFuncAttributes a;
  const void* fns[] = {(const void*)eb2d_kernel<32, 16, 256, true>,  (const void*)eb2d_kernel<32, 8, 128, true>,
                       (const void*)eb2d_kernel<64, 8, 256, true>,   (const void*)eb2d_kernel<32, 32, 256, true>,
                       (const void*)eb2d_kernel<64, 16, 256, true>,  (const void*)eb2d_kernel<32, 16, 128, true>,
                       (const void*)eb2d_kernel<32, 16, 256, false>, (const void*)eb2d_kernel<32, 8, 128, false>,
                       (const void*)eb2d_kernel<64, 8, 256, false>,  (const void*)eb2d_kernel<32, 32, 256, false>,
                       (const void*)eb2d_kernel<64, 16, 256, false>, (const void*)eb2d_kernel<32, 16, 128, false>};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return set_error(CPSZ_ERR_CUDA, "loading eb2d_kernel: %s", cudaGetErrorString(e));
  }
  return CPSZ_OK;
}

int launch_eb2d(cpsz_b200_ctx* ctx, const float* U, const float* V, int r1, int r2, double max_pwr_eb,
                const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, unsigned long long* hist,
                float2* pair_u, float2* pair_v, double* eb_out, int row_begin, int row_end,
                const Eb2dUnits* units, bool log_ids, bool pow4_ids) {
  if (row_end < 0) row_end = r1;
  if (log_ids && (pair_u || pair_v || ids_v))
    return set_error(CPSZ_ERR_INVALID, "eb2d: the log-domain ids have no wavefront pairs and one stream");
  if (row_end <= row_begin) return CPSZ_OK;
  if (units && row_begin % WAVE_GROUP_ROWS)
    return set_error(CPSZ_ERR_INVALID, "eb2d band start %d is not a multiple of %d", row_begin, WAVE_GROUP_ROWS);
  auto go = [&](auto kernel, int tx, int ty, int nt) {
    if (units) {
      const long long tiles = (long long)units->n * (UNIT_COLS / tx) * (WAVE_GROUP_ROWS / ty);
      kernel<<<(unsigned)tiles, nt, 0, ctx->stream>>>(U, V, r1, r2, max_pwr_eb, d_thr_tab, thr_n, ids_u, ids_v, hist,
                                                      ctx->d_flag, pair_u, pair_v, eb_out, row_begin, row_end,
                                                      units->order, units->ncb, units->done, log_ids ? 1 : 0,
                                                      pow4_ids && !log_ids ? 1 : 0, nullptr, 0);
      return;
    }
    dim3 grid((r2 + tx - 1) / tx, (row_end - row_begin + ty - 1) / ty);
    kernel<<<grid, nt, 0, ctx->stream>>>(U, V, r1, r2, max_pwr_eb, d_thr_tab, thr_n, ids_u, ids_v, hist, ctx->d_flag,
                                         pair_u, pair_v, eb_out, row_begin, row_end, nullptr, 0, nullptr,
                                         log_ids ? 1 : 0, pow4_ids && !log_ids ? 1 : 0, nullptr, 0);
  };
  // filtered bounds unless the caller wants the bounds themselves (or an
  // unusual max_pwr_eb takes the reference's NaN paths)
  const bool fast = eb_out == nullptr && max_pwr_eb >= 0 && max_pwr_eb <= 1e300;
  switch (tune_get(TUNE_EB2D_TILE, (size_t)r1 * r2) + (fast ? 0 : 6)) {
    case 1: go(eb2d_kernel<32, 8, 128, true>, 32, 8, 128); break;
    case 2: go(eb2d_kernel<64, 8, 256, true>, 64, 8, 256); break;
    case 3: go(eb2d_kernel<32, 32, 256, true>, 32, 32, 256); break;
    case 4: go(eb2d_kernel<64, 16, 256, true>, 64, 16, 256); break;
    case 5: go(eb2d_kernel<32, 16, 128, true>, 32, 16, 128); break;
    case 0: go(eb2d_kernel<32, 16, 256, true>, 32, 16, 256); break;
    case 7: go(eb2d_kernel<32, 8, 128, false>, 32, 8, 128); break;
    case 8: go(eb2d_kernel<64, 8, 256, false>, 64, 8, 256); break;
    case 9: go(eb2d_kernel<32, 32, 256, false>, 32, 32, 256); break;
    case 10: go(eb2d_kernel<64, 16, 256, false>, 64, 16, 256); break;
    case 11: go(eb2d_kernel<32, 16, 128, false>, 32, 16, 128); break;
    default: go(eb2d_kernel<32, 16, 256, false>, 32, 16, 256); break;
  }
  count_launch(ctx);
  return check_launch("eb2d_kernel");
}

void eb2d_tile_shape(int shape, int* tx, int* ty) {
  static const int shapes[6][2] = {{32, 16}, {32, 8}, {64, 8}, {32, 32}, {64, 16}, {32, 16}};
  const int s = shape >= 0 && shape < 6 ? shape : 0;
  *tx = shapes[s][0];
  *ty = shapes[s][1];
}

int launch_eb2d_batch(cpsz_b200_ctx* ctx, const Eb2dJob* jobs, int n, int tiles, int shape, const double* d_thr_tab,
                      int thr_n, bool pow4_ids) {
  if (n <= 0 || tiles <= 0) return CPSZ_OK;
  auto go = [&](auto kernel, int nt) {
    kernel<<<(unsigned)tiles, nt, 0, ctx->stream>>>(nullptr, nullptr, 0, 0, 0.0, d_thr_tab, thr_n, nullptr, nullptr,
                                                    nullptr, ctx->d_flag, nullptr, nullptr, nullptr, 0, 0, nullptr, 0,
                                                    nullptr, 0, pow4_ids ? 1 : 0, jobs, n);
  };
  switch (shape) {
    case 1: go(eb2d_kernel<32, 8, 128, true, true>, 128); break;
    case 2: go(eb2d_kernel<64, 8, 256, true, true>, 256); break;
    case 3: go(eb2d_kernel<32, 32, 256, true, true>, 256); break;
    case 4: go(eb2d_kernel<64, 16, 256, true, true>, 256); break;
    case 5: go(eb2d_kernel<32, 16, 128, true, true>, 128); break;
    default: go(eb2d_kernel<32, 16, 256, true, true>, 256); break;
  }
  count_launch(ctx);
  return check_launch("eb2d_kernel (batched)");
}

}  // namespace cpsz

namespace cpsz {

namespace {

// Quantization of given per-vertex bounds (the learned-bound path): the same
// id arithmetic, symbols and wavefront pairs as eb2d_kernel, with the bound
// read from eb_in instead of derived from the triangles.
// One vertex of the given-bound quantization: ids and wavefront pairs of
// U and V (the id of |x| * eb against the threshold table, ID_ZERO at or
// below thr); sym[] gets the histogram symbols.
__device__ __forceinline__ void quant2d_vertex(size_t g, const float* __restrict__ U, const float* __restrict__ V,
                                               const double* __restrict__ eb_in, const double* tab, int thr_n,
                                               uint8_t* __restrict__ ids_u, uint8_t* __restrict__ ids_v,
                                               int* __restrict__ flag, float2* __restrict__ pair_u,
                                               float2* __restrict__ pair_v, int sym[2]) {
  const double thr = tab[0];
  const double eb = eb_in[g];
  const float uu = U[g], vv = V[g];
  uint8_t code[2];
  const double ev[2] = {(double)fabsf(uu) * eb, (double)fabsf(vv) * eb};
#pragma unroll
  for (int c = 0; c < 2; c++) {
    const double e = ev[c];
    if (e <= thr) {
      code[c] = ID_ZERO;
      sym[c] = 0;
    } else {
      int ex = (int)((__double_as_longlong(e) >> 52) & 0x7ff) - 1023;
      int id = dev::count_thresholds(tab, thr_n, e, (ex + 52) >> 1);
      if (id > ID_MAX_2D) {
        atomicOr(flag, FLAG_ID_OVERFLOW);
        id = ID_MAX_2D;
      }
      code[c] = (uint8_t)id;
      sym[c] = id;
    }
  }
  ids_u[g] = code[0];
  ids_v[g] = code[1];
  pair_u[g] = make_float2(uu, code[0] == ID_ZERO ? __int_as_float(0x7FC00000)
                                                 : __int_as_float((127 + 52 - 2 * (int)code[0]) << 23));
  pair_v[g] = make_float2(vv, code[1] == ID_ZERO ? __int_as_float(0x7FC00000)
                                                 : __int_as_float((127 + 52 - 2 * (int)code[1]) << 23));
}

__global__ void __launch_bounds__(256) quant2d_kernel(const float* __restrict__ U, const float* __restrict__ V,
                                                      size_t n, const double* __restrict__ eb_in,
                                                      const double* __restrict__ thr_tab, int thr_n,
                                                      uint8_t* __restrict__ ids_u, uint8_t* __restrict__ ids_v,
                                                      unsigned long long* __restrict__ hist, int* __restrict__ flag,
                                                      float2* __restrict__ pair_u, float2* __restrict__ pair_v) {
  __shared__ double tab[QUANT_TAB_MAX];
  __shared__ unsigned int shist[256];
  for (int k = threadIdx.x; k < 256; k += blockDim.x) shist[k] = 0;
  for (int k = threadIdx.x; k < thr_n; k += blockDim.x) tab[k] = thr_tab[k];
  __syncthreads();
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
    int sym[2];
    quant2d_vertex(g, U, V, eb_in, tab, thr_n, ids_u, ids_v, flag, pair_u, pair_v, sym);
    atomicAdd(&shist[sym[0]], 1u);
    atomicAdd(&shist[sym[1]], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 256; k += blockDim.x)
    if (shist[k]) atomicAdd(&hist[k], (unsigned long long)shist[k]);
}

// The same for the vertices whose mask byte is set (16 mask bytes per load;
// mask is 16-byte aligned), clearing it; no histogram.
__global__ void __launch_bounds__(256) requant2d_kernel(const float* __restrict__ U, const float* __restrict__ V,
                                                        size_t n, const double* __restrict__ eb_in,
                                                        const double* __restrict__ thr_tab, int thr_n,
                                                        uint8_t* __restrict__ ids_u, uint8_t* __restrict__ ids_v,
                                                        int* __restrict__ flag, float2* __restrict__ pair_u,
                                                        float2* __restrict__ pair_v, uint8_t* __restrict__ mask) {
  __shared__ double tab[QUANT_TAB_MAX];
  for (int k = threadIdx.x; k < thr_n; k += blockDim.x) tab[k] = thr_tab[k];
  __syncthreads();
  const size_t nvec = n / 16, tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nt = (size_t)gridDim.x * blockDim.x;
  int sym[2];
  for (size_t v = tid; v < nvec; v += nt) {
    const uint4 x = reinterpret_cast<const uint4*>(mask)[v];
    if ((x.x | x.y | x.z | x.w) == 0) continue;
    for (int e = 0; e < 16; e++) {
      const size_t g = 16 * v + e;
      if (!mask[g]) continue;
      quant2d_vertex(g, U, V, eb_in, tab, thr_n, ids_u, ids_v, flag, pair_u, pair_v, sym);
      mask[g] = 0;
    }
  }
  for (size_t g = 16 * nvec + tid; g < n; g += nt)
    if (mask[g]) {
      quant2d_vertex(g, U, V, eb_in, tab, thr_n, ids_u, ids_v, flag, pair_u, pair_v, sym);
      mask[g] = 0;
    }
}

}  // namespace

int launch_quant2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t n, const double* eb_in,
                   const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, unsigned long long* hist,
                   float2* pair_u, float2* pair_v) {
  size_t g = (n + 255) / 256;
  if (g > (size_t)ctx->num_sms * 8) g = (size_t)ctx->num_sms * 8;
  quant2d_kernel<<<(int)(g ? g : 1), 256, 0, ctx->stream>>>(U, V, n, eb_in, d_thr_tab, thr_n, ids_u, ids_v, hist,
                                                            ctx->d_flag, pair_u, pair_v);
  count_launch(ctx);
  return check_launch("quant2d_kernel");
}

int launch_requant2d(cpsz_b200_ctx* ctx, const float* U, const float* V, size_t n, const double* eb_in,
                     const double* d_thr_tab, int thr_n, uint8_t* ids_u, uint8_t* ids_v, float2* pair_u,
                     float2* pair_v, uint8_t* mask) {
  size_t g = (n / 16 + 255) / 256;
  if (g > (size_t)ctx->num_sms * 8) g = (size_t)ctx->num_sms * 8;
  requant2d_kernel<<<(int)(g ? g : 1), 256, 0, ctx->stream>>>(U, V, n, eb_in, d_thr_tab, thr_n, ids_u, ids_v,
                                                              ctx->d_flag, pair_u, pair_v, mask);
  count_launch(ctx);
  return check_launch("requant2d_kernel");
}

}  // namespace cpsz
