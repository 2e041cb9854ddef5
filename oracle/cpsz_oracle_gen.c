/* cpsz_oracle_gen.c -- TEST INFRASTRUCTURE: the seeded synthetic workloads in
 * plain C, so the reference's CPU arm (bench.py --impl reference) and the CPU
 * parity checks can build their inputs without loading the product library.
 *
 * It restates the workload definition the product uses (Gaussian-windowed
 * linear flows, cpsz_b200/csrc/gen.cpp): centres uniform over the grid, matrix
 * entries N(0,1) from a splitmix64 stream seeded with `seed`, the window
 * exp(-|x-c|^2 / 2 sigma^2) truncated at ceil(4 sigma) cells per axis and
 * evaluated separably in double, per-vertex N(0, noise^2) noise from a
 * counter-based hash of (seed, vertex, component), and a joint rescale by the
 * common max |value|.  Every vertex sums its flows in flow order, so the
 * result does not depend on the thread count; tests/test_oracle_gen.py checks
 * it against the product's generator bit for bit.  The reference itself has no
 * generator: its dataset (data/uf.dat, data/vf.dat) is not distributed. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

static uint64_t sm64(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t hash3(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t s = a * 0xD1B54A32D192ED03ull ^ (b + 0x8CB92BA72F3D8DD7ull) * 0xABC98388FB8FAC03ull ^ c;
  return sm64(&s);
}

static double u01(uint64_t x) { return ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

typedef struct {
  uint64_t s;
} rng_t;

static void rng_init(rng_t* r, uint64_t seed) { r->s = seed ^ 0x5DEECE66Dull; }
static double rng_uniform(rng_t* r) { return u01(sm64(&r->s)); }
static double rng_normal(rng_t* r) {
  double a = rng_uniform(r), b = rng_uniform(r);
  return sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b);
}

static double noise_normal(uint64_t seed, uint64_t idx, uint64_t comp) {
  uint64_t h1 = hash3(seed, idx, 2 * comp);
  uint64_t h2 = hash3(seed, idx, 2 * comp + 1);
  return sqrt(-2.0 * log(u01(h1))) * cos(6.283185307179586 * u01(h2));
}

static long lmax(long a, long b) { return a > b ? a : b; }
static long lmin(long a, long b) { return a < b ? a : b; }

/* ---- rows split over threads ---- */
typedef struct {
  void (*fn)(void* arg, size_t lo, size_t hi);
  void* arg;
  size_t lo, hi;
} job_t;

static void* job_run(void* p) {
  job_t* j = (job_t*)p;
  j->fn(j->arg, j->lo, j->hi);
  return NULL;
}

static void parallel_rows(size_t rows, void (*fn)(void*, size_t, size_t), void* arg) {
  long nt = sysconf(_SC_NPROCESSORS_ONLN);
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if ((size_t)nt > rows) nt = (long)rows;
  pthread_t th[64];
  job_t jobs[64];
  size_t per = (rows + (size_t)nt - 1) / (size_t)nt;
  int started = 0;
  for (long t = 0; t < nt; t++) {
    size_t lo = (size_t)t * per, hi = lo + per < rows ? lo + per : rows;
    if (lo >= hi) break;
    jobs[t].fn = fn;
    jobs[t].arg = arg;
    jobs[t].lo = lo;
    jobs[t].hi = hi;
    if (pthread_create(&th[t], NULL, job_run, &jobs[t]) != 0) {
      job_run(&jobs[t]);
      th[t] = 0;
    }
    started = (int)t + 1;
  }
  for (int t = 0; t < started; t++)
    if (th[t]) pthread_join(th[t], NULL);
}

/* ---- 2D ---- */
typedef struct {
  double ci, cj, a00, a01, a10, a11;
} flow2_t;

typedef struct {
  const flow2_t* flows;
  int n_flows;
  size_t r1, r2;
  long R;
  double inv2s2, noise;
  uint64_t seed;
  double *du, *dv;
  float *U, *V;
  double scale;
} gen2_t;

static void gen2_rows(void* p, size_t lo, size_t hi) {
  gen2_t* g = (gen2_t*)p;
  double* gj = (double*)malloc(sizeof(double) * (size_t)(2 * g->R + 3));
  for (int k = 0; k < g->n_flows; k++) {
    const flow2_t* f = &g->flows[k];
    long i0 = lmax((long)lo, (long)floor(f->ci) - g->R);
    long i1 = lmin((long)hi - 1, (long)floor(f->ci) + g->R);
    if (i0 > i1) continue;
    long j0 = lmax(0, (long)floor(f->cj) - g->R);
    long j1 = lmin((long)g->r2 - 1, (long)floor(f->cj) + g->R);
    for (long j = j0; j <= j1; j++) {
      double d = j - f->cj;
      gj[j - j0] = exp(-d * d * g->inv2s2);
    }
    for (long i = i0; i <= i1; i++) {
      double di = i - f->ci;
      double gi = exp(-di * di * g->inv2s2);
      double* pu = &g->du[(size_t)i * g->r2];
      double* pv = &g->dv[(size_t)i * g->r2];
      for (long j = j0; j <= j1; j++) {
        double dj = j - f->cj;
        double w = gi * gj[j - j0];
        pu[j] += (f->a00 * di + f->a01 * dj) * w;
        pv[j] += (f->a10 * di + f->a11 * dj) * w;
      }
    }
  }
  free(gj);
  for (size_t i = lo; i < hi; i++)
    for (size_t j = 0; j < g->r2; j++) {
      size_t idx = i * g->r2 + j;
      g->du[idx] += g->noise * noise_normal(g->seed, idx, 0);
      g->dv[idx] += g->noise * noise_normal(g->seed, idx, 1);
    }
}

static void gen2_scale(void* p, size_t lo, size_t hi) {
  gen2_t* g = (gen2_t*)p;
  for (size_t i = lo * g->r2; i < hi * g->r2; i++) {
    g->U[i] = (float)(g->du[i] * g->scale);
    g->V[i] = (float)(g->dv[i] * g->scale);
  }
}

int cpo_generate_field_2d(uint64_t seed, size_t r1, size_t r2, int n_flows, double sigma, double noise, float* U,
                          float* V) {
  if (!U || !V || r1 == 0 || r2 == 0 || n_flows < 0 || !(sigma > 0)) return 1;
  flow2_t* flows = (flow2_t*)malloc(sizeof(flow2_t) * (size_t)(n_flows > 0 ? n_flows : 1));
  rng_t rng;
  rng_init(&rng, seed);
  for (int k = 0; k < n_flows; k++) {
    flows[k].ci = rng_uniform(&rng) * (double)r1;
    flows[k].cj = rng_uniform(&rng) * (double)r2;
    flows[k].a00 = rng_normal(&rng);
    flows[k].a01 = rng_normal(&rng);
    flows[k].a10 = rng_normal(&rng);
    flows[k].a11 = rng_normal(&rng);
  }
  gen2_t g;
  g.flows = flows;
  g.n_flows = n_flows;
  g.r1 = r1;
  g.r2 = r2;
  g.R = (long)ceil(4.0 * sigma);
  g.inv2s2 = 1.0 / (2.0 * sigma * sigma);
  g.noise = noise;
  g.seed = seed;
  g.du = (double*)calloc(r1 * r2, sizeof(double));
  g.dv = (double*)calloc(r1 * r2, sizeof(double));
  g.U = U;
  g.V = V;
  if (!g.du || !g.dv) {
    free(g.du);
    free(g.dv);
    free(flows);
    return 3;
  }
  parallel_rows(r1, gen2_rows, &g);
  double m = 0;
  for (size_t i = 0; i < r1 * r2; i++) {
    double a = fabs(g.du[i]), b = fabs(g.dv[i]);
    double x = a > b ? a : b;
    if (x > m) m = x;
  }
  g.scale = m > 0 ? 1.0 / m : 1.0;
  parallel_rows(r1, gen2_scale, &g);
  free(g.du);
  free(g.dv);
  free(flows);
  return 0;
}

/* ---- 3D ---- */
typedef struct {
  double c[3];
  double a[3][3];
} flow3_t;

typedef struct {
  const flow3_t* flows;
  int n_flows;
  size_t r1, r2, r3;
  long R;
  double inv2s2, noise;
  uint64_t seed;
  double* acc[3];
  float* out[3];
  double scale;
} gen3_t;

static void gen3_rows(void* p, size_t lo, size_t hi) {
  gen3_t* g = (gen3_t*)p;
  const size_t plane = g->r2 * g->r3;
  double* gj = (double*)malloc(sizeof(double) * (size_t)(2 * g->R + 3));
  double* gk = (double*)malloc(sizeof(double) * (size_t)(2 * g->R + 3));
  for (int q = 0; q < g->n_flows; q++) {
    const flow3_t* f = &g->flows[q];
    long i0 = lmax((long)lo, (long)floor(f->c[0]) - g->R);
    long i1 = lmin((long)hi - 1, (long)floor(f->c[0]) + g->R);
    if (i0 > i1) continue;
    long j0 = lmax(0, (long)floor(f->c[1]) - g->R), j1 = lmin((long)g->r2 - 1, (long)floor(f->c[1]) + g->R);
    long k0 = lmax(0, (long)floor(f->c[2]) - g->R), k1 = lmin((long)g->r3 - 1, (long)floor(f->c[2]) + g->R);
    for (long j = j0; j <= j1; j++) {
      double d = j - f->c[1];
      gj[j - j0] = exp(-d * d * g->inv2s2);
    }
    for (long k = k0; k <= k1; k++) {
      double d = k - f->c[2];
      gk[k - k0] = exp(-d * d * g->inv2s2);
    }
    for (long i = i0; i <= i1; i++) {
      double di = i - f->c[0];
      double gi = exp(-di * di * g->inv2s2);
      for (long j = j0; j <= j1; j++) {
        double dj = j - f->c[1];
        double gij = gi * gj[j - j0];
        size_t base = (size_t)i * plane + (size_t)j * g->r3;
        for (long k = k0; k <= k1; k++) {
          double dk = k - f->c[2];
          double w = gij * gk[k - k0];
          for (int a = 0; a < 3; a++)
            g->acc[a][base + k] += (f->a[a][0] * di + f->a[a][1] * dj + f->a[a][2] * dk) * w;
        }
      }
    }
  }
  free(gj);
  free(gk);
  for (size_t idx = lo * plane; idx < hi * plane; idx++)
    for (int a = 0; a < 3; a++) g->acc[a][idx] += g->noise * noise_normal(g->seed, idx, a);
}

static void gen3_scale(void* p, size_t lo, size_t hi) {
  gen3_t* g = (gen3_t*)p;
  const size_t plane = g->r2 * g->r3;
  for (int a = 0; a < 3; a++)
    for (size_t i = lo * plane; i < hi * plane; i++) g->out[a][i] = (float)(g->acc[a][i] * g->scale);
}

int cpo_generate_field_3d(uint64_t seed, size_t r1, size_t r2, size_t r3, int n_flows, double sigma, double noise,
                          float* U, float* V, float* W) {
  if (!U || !V || !W || r1 == 0 || r2 == 0 || r3 == 0 || n_flows < 0 || !(sigma > 0)) return 1;
  flow3_t* flows = (flow3_t*)malloc(sizeof(flow3_t) * (size_t)(n_flows > 0 ? n_flows : 1));
  rng_t rng;
  rng_init(&rng, seed);
  for (int q = 0; q < n_flows; q++) {
    flows[q].c[0] = rng_uniform(&rng) * (double)r1;
    flows[q].c[1] = rng_uniform(&rng) * (double)r2;
    flows[q].c[2] = rng_uniform(&rng) * (double)r3;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) flows[q].a[a][b] = rng_normal(&rng);
  }
  const size_t n = r1 * r2 * r3;
  gen3_t g;
  g.flows = flows;
  g.n_flows = n_flows;
  g.r1 = r1;
  g.r2 = r2;
  g.r3 = r3;
  g.R = (long)ceil(4.0 * sigma);
  g.inv2s2 = 1.0 / (2.0 * sigma * sigma);
  g.noise = noise;
  g.seed = seed;
  g.out[0] = U;
  g.out[1] = V;
  g.out[2] = W;
  int ok = 1;
  for (int a = 0; a < 3; a++) {
    g.acc[a] = (double*)calloc(n, sizeof(double));
    ok = ok && g.acc[a];
  }
  if (!ok) {
    for (int a = 0; a < 3; a++) free(g.acc[a]);
    free(flows);
    return 3;
  }
  parallel_rows(r1, gen3_rows, &g);
  double m = 0;
  for (int a = 0; a < 3; a++)
    for (size_t i = 0; i < n; i++) {
      double x = fabs(g.acc[a][i]);
      if (x > m) m = x;
    }
  g.scale = m > 0 ? 1.0 / m : 1.0;
  parallel_rows(r1, gen3_scale, &g);
  for (int a = 0; a < 3; a++) free(g.acc[a]);
  free(flows);
  return 0;
}

/* Sizes, seeds and bounds of the batched workload: side lengths drawn
 * independently and uniformly from [lo, hi], seed base_seed + 1 + k, bound
 * drawn uniformly from {0.01, 0.05, 0.1}. */
int cpo_batch_layout(uint64_t base_seed, int n_fields, int lo, int hi, size_t* r1, size_t* r2, uint64_t* seeds,
                     double* ebs) {
  static const double choices[3] = {0.01, 0.05, 0.1};
  if (n_fields < 0 || lo < 2 || hi < lo) return 1;
  rng_t rng;
  rng_init(&rng, base_seed);
  for (int k = 0; k < n_fields; k++) {
    double a = floor(rng_uniform(&rng) * (hi - lo + 1));
    r1[k] = (size_t)lo + (size_t)(a < (double)(hi - lo) ? a : (double)(hi - lo));
    double b = floor(rng_uniform(&rng) * (hi - lo + 1));
    r2[k] = (size_t)lo + (size_t)(b < (double)(hi - lo) ? b : (double)(hi - lo));
    seeds[k] = base_seed + 1 + (uint64_t)k;
    int c = (int)floor(rng_uniform(&rng) * 3);
    ebs[k] = choices[c < 2 ? c : 2];
  }
  return 0;
}
