// Seeded synthetic vector-field generators (host C++, multithreaded).
//
// The reference's own dataset (ocean u/v .dat files) is not distributed, so
// every workload is generated from a seed:
//   field(x) = sum_k A_k (x - c_k) * exp(-|x - c_k|^2 / (2 sigma^2))   (+ noise)
// with centres c_k uniform over the grid, A_k entries N(0,1), the Gaussian
// window truncated at 4 sigma (radius ceil(4 sigma) cells per axis), additive
// N(0, noise_std^2) noise per component and per vertex, and finally a joint
// rescale of all components by their common max |value| so the field lies in
// [-1, 1] with its zero set unchanged.
//
// Determinism: flow parameters come from a splitmix64 stream seeded with
// `seed`; the per-vertex noise is a counter-based hash of (seed, vertex index,
// component), so the result does not depend on the number of threads.  The
// Gaussian window is evaluated separably (g(di) * g(dj) [* g(dk)]) in double.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

#include "cpsz_b200.h"

namespace {

inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t hash3(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t s = a * 0xD1B54A32D192ED03ull ^ (b + 0x8CB92BA72F3D8DD7ull) * 0xABC98388FB8FAC03ull ^ c;
  return splitmix64(s);
}

inline double u01(uint64_t x) { return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed ^ 0x5DEECE66Dull) {}
  double uniform() { return u01(splitmix64(s)); }
  double normal() {
    double a = uniform(), b = uniform();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }
};

inline double noise_normal(uint64_t seed, uint64_t idx, uint64_t comp) {
  uint64_t h1 = hash3(seed, idx, 2 * comp);
  uint64_t h2 = hash3(seed, idx, 2 * comp + 1);
  return std::sqrt(-2.0 * std::log(u01(h1))) * std::cos(6.283185307179586 * u01(h2));
}

unsigned worker_count(size_t rows) {
  unsigned hc = std::thread::hardware_concurrency();
  if (hc == 0) hc = 4;
  return (unsigned)std::max<size_t>(1, std::min<size_t>(hc, rows));
}

template <class F>
void parallel_rows(size_t rows, F f) {
  unsigned nt = worker_count(rows);
  std::vector<std::thread> th;
  size_t per = (rows + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    size_t lo = t * per, hi = std::min(rows, lo + per);
    if (lo >= hi) break;
    th.emplace_back([=]() { f(lo, hi); });
  }
  for (auto& x : th) x.join();
}

}  // namespace

extern "C" int cpsz_b200_generate_field_2d(uint64_t seed, size_t r1, size_t r2, int n_flows, double sigma,
                                           double noise_std, float* U, float* V) {
  if (!U || !V || r1 == 0 || r2 == 0 || n_flows < 0 || !(sigma > 0)) return CPSZ_ERR_INVALID;
  struct Flow { double ci, cj, a00, a01, a10, a11; };
  Rng rng(seed);
  std::vector<Flow> flows(n_flows);
  for (auto& f : flows) {
    f.ci = rng.uniform() * (double)r1;
    f.cj = rng.uniform() * (double)r2;
    f.a00 = rng.normal(); f.a01 = rng.normal(); f.a10 = rng.normal(); f.a11 = rng.normal();
  }
  const long R = (long)std::ceil(4.0 * sigma);
  const double inv2s2 = 1.0 / (2.0 * sigma * sigma);
  std::vector<double> du(r1 * r2, 0.0), dv(r1 * r2, 0.0);
  parallel_rows(r1, [&](size_t lo, size_t hi) {
    std::vector<double> gj;
    for (const Flow& f : flows) {
      long i0 = std::max<long>((long)lo, (long)std::floor(f.ci) - R);
      long i1 = std::min<long>((long)hi - 1, (long)std::floor(f.ci) + R);
      if (i0 > i1) continue;
      long j0 = std::max<long>(0, (long)std::floor(f.cj) - R);
      long j1 = std::min<long>((long)r2 - 1, (long)std::floor(f.cj) + R);
      gj.resize(j1 - j0 + 1);
      for (long j = j0; j <= j1; j++) { double d = j - f.cj; gj[j - j0] = std::exp(-d * d * inv2s2); }
      for (long i = i0; i <= i1; i++) {
        double di = i - f.ci;
        double gi = std::exp(-di * di * inv2s2);
        double* pu = &du[(size_t)i * r2];
        double* pv = &dv[(size_t)i * r2];
        for (long j = j0; j <= j1; j++) {
          double dj = j - f.cj;
          double w = gi * gj[j - j0];
          pu[j] += (f.a00 * di + f.a01 * dj) * w;
          pv[j] += (f.a10 * di + f.a11 * dj) * w;
        }
      }
    }
    for (size_t i = lo; i < hi; i++)
      for (size_t j = 0; j < r2; j++) {
        size_t idx = i * r2 + j;
        du[idx] += noise_std * noise_normal(seed, idx, 0);
        dv[idx] += noise_std * noise_normal(seed, idx, 1);
      }
  });
  double m = 0;
  for (size_t i = 0; i < r1 * r2; i++) m = std::max(m, std::max(std::fabs(du[i]), std::fabs(dv[i])));
  double s = m > 0 ? 1.0 / m : 1.0;
  parallel_rows(r1, [&](size_t lo, size_t hi) {
    for (size_t i = lo * r2; i < hi * r2; i++) { U[i] = (float)(du[i] * s); V[i] = (float)(dv[i] * s); }
  });
  return CPSZ_OK;
}

extern "C" int cpsz_b200_generate_field_3d(uint64_t seed, size_t r1, size_t r2, size_t r3, int n_flows,
                                           double sigma, double noise_std, float* U, float* V, float* W) {
  if (!U || !V || !W || r1 == 0 || r2 == 0 || r3 == 0 || n_flows < 0 || !(sigma > 0)) return CPSZ_ERR_INVALID;
  struct Flow { double c[3]; double a[3][3]; };
  Rng rng(seed);
  std::vector<Flow> flows(n_flows);
  for (auto& f : flows) {
    f.c[0] = rng.uniform() * (double)r1;
    f.c[1] = rng.uniform() * (double)r2;
    f.c[2] = rng.uniform() * (double)r3;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) f.a[a][b] = rng.normal();
  }
  const long R = (long)std::ceil(4.0 * sigma);
  const double inv2s2 = 1.0 / (2.0 * sigma * sigma);
  const size_t n = r1 * r2 * r3, plane = r2 * r3;
  std::vector<double> acc[3] = {std::vector<double>(n, 0.0), std::vector<double>(n, 0.0), std::vector<double>(n, 0.0)};
  parallel_rows(r1, [&](size_t lo, size_t hi) {
    std::vector<double> gj, gk;
    for (const Flow& f : flows) {
      long i0 = std::max<long>((long)lo, (long)std::floor(f.c[0]) - R);
      long i1 = std::min<long>((long)hi - 1, (long)std::floor(f.c[0]) + R);
      if (i0 > i1) continue;
      long j0 = std::max<long>(0, (long)std::floor(f.c[1]) - R), j1 = std::min<long>((long)r2 - 1, (long)std::floor(f.c[1]) + R);
      long k0 = std::max<long>(0, (long)std::floor(f.c[2]) - R), k1 = std::min<long>((long)r3 - 1, (long)std::floor(f.c[2]) + R);
      gj.resize(j1 - j0 + 1);
      gk.resize(k1 - k0 + 1);
      for (long j = j0; j <= j1; j++) { double d = j - f.c[1]; gj[j - j0] = std::exp(-d * d * inv2s2); }
      for (long k = k0; k <= k1; k++) { double d = k - f.c[2]; gk[k - k0] = std::exp(-d * d * inv2s2); }
      for (long i = i0; i <= i1; i++) {
        double di = i - f.c[0];
        double gi = std::exp(-di * di * inv2s2);
        for (long j = j0; j <= j1; j++) {
          double dj = j - f.c[1];
          double gij = gi * gj[j - j0];
          size_t base = (size_t)i * plane + (size_t)j * r3;
          for (long k = k0; k <= k1; k++) {
            double dk = k - f.c[2];
            double w = gij * gk[k - k0];
            for (int a = 0; a < 3; a++) acc[a][base + k] += (f.a[a][0] * di + f.a[a][1] * dj + f.a[a][2] * dk) * w;
          }
        }
      }
    }
    for (size_t idx = lo * plane; idx < hi * plane; idx++)
      for (int a = 0; a < 3; a++) acc[a][idx] += noise_std * noise_normal(seed, idx, a);
  });
  double m = 0;
  for (int a = 0; a < 3; a++)
    for (size_t i = 0; i < n; i++) m = std::max(m, std::fabs(acc[a][i]));
  double s = m > 0 ? 1.0 / m : 1.0;
  float* out[3] = {U, V, W};
  parallel_rows(r1, [&](size_t lo, size_t hi) {
    for (int a = 0; a < 3; a++)
      for (size_t i = lo * plane; i < hi * plane; i++) out[a][i] = (float)(acc[a][i] * s);
  });
  return CPSZ_OK;
}

// Field sizes, seeds and error bounds of the batched workload: 256 fields whose
// two side lengths are drawn independently and uniformly from [lo, hi], each
// with its own seed (base_seed + 1 + k), and a relative bound drawn uniformly
// from {0.01, 0.05, 0.1}.
extern "C" int cpsz_b200_batch_layout(uint64_t base_seed, int n_fields, int lo, int hi, size_t* r1, size_t* r2,
                                      uint64_t* seeds, double* ebs) {
  if (n_fields < 0 || lo < 2 || hi < lo) return CPSZ_ERR_INVALID;
  Rng rng(base_seed);
  static const double eb_choices[3] = {0.01, 0.05, 0.1};
  for (int k = 0; k < n_fields; k++) {
    r1[k] = (size_t)lo + (size_t)std::min<double>(hi - lo, std::floor(rng.uniform() * (hi - lo + 1)));
    r2[k] = (size_t)lo + (size_t)std::min<double>(hi - lo, std::floor(rng.uniform() * (hi - lo + 1)));
    seeds[k] = base_seed + 1 + (uint64_t)k;
    ebs[k] = eb_choices[std::min(2, (int)std::floor(rng.uniform() * 3))];
  }
  return CPSZ_OK;
}
