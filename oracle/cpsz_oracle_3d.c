/* cpsz_oracle_3d.c -- 3D offline (log-domain) path of the CPU oracle (test
 * infrastructure only; see cpsz_oracle.h).  Restates
 *   sz_compress_cp_preserve_3d_offline_log<float>  src/sz_compress_cp_preserve_3d.cpp:360-581
 *   max_eb_to_keep_position_and_type_3d_offline   src/sz_compress_cp_preserve_3d.cpp:266-358
 *   sz_decompress_cp_preserve_3d_online_log<float> src/sz_decompress_cp_preserve_3d.cpp:7-110
 * with the same operand types (float triple products widened to double, float
 * sums of the per-minor magnitudes, the reference's acbrt1 bit-hack cube root),
 * glibc log2 / log2f / pow / exp2f where the reference calls them.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cpsz_oracle.h"

static inline void acc(double value, double* pos, double* neg) {
  if (value >= 0) *pos += value;
  else *neg += -value;
}

/* acbrt1: include/sz_cp_preserve_utils.hpp:173-184 (bit-level initial guess and
 * two Newton steps in float). */
static float acbrt1(float x0) {
  union { int ix; float x; } u;
  u.x = x0;
  u.ix = u.ix / 4 + u.ix / 16;
  u.ix = u.ix + u.ix / 16;
  u.ix = u.ix + u.ix / 256;
  u.ix = 0x2a5137a0 + u.ix;
  u.x = 0.33333333f * (2.0f * u.x + x0 / (u.x * u.x));
  u.x = 0.33333333f * (2.0f * u.x + x0 / (u.x * u.x));
  return u.x;
}

/* max_eb_to_keep_sign_3d_offline: include/sz_cp_preserve_utils.hpp:186-191 */
static float keep_sign_3d(float positive, float negative) {
  if (positive == 0 && negative == 0) return 0;
  float P = acbrt1(positive);
  float N = acbrt1(negative);
  return fabsf(P - N) / (P + N);
}

static inline int sgnf(float v) { return (0.0f < v) - (v < 0.0f); }
/* same_direction: include/sz_cp_preserve_utils.hpp:52-57 */
static int same_direction(float a, float b, float c, float d) {
  int s = sgnf(a);
  if (s == 0) return 0;
  return (s == sgnf(b)) && (s == sgnf(c)) && (s == sgnf(d));
}

static inline float maxf_(float a, float b) { return (a > b) ? a : b; }
static inline float minf_(float a, float b) { return (a < b) ? a : b; }

static double tet_eb(float u0, float u1, float u2, float u3, float v0, float v1, float v2, float v3, float w0,
                     float w1, float w2, float w3) {
  double u3v1w2 = u3 * v1 * w2, u3v2w1 = u3 * v2 * w1, u3v2w0 = u3 * v2 * w0, u3v0w2 = u3 * v0 * w2,
         u3v0w1 = u3 * v0 * w1, u3v1w0 = u3 * v1 * w0;
  double u1v3w2 = u1 * v3 * w2, u2v3w1 = u2 * v3 * w1, u2v3w0 = u2 * v3 * w0, u0v3w2 = u0 * v3 * w2,
         u0v3w1 = u0 * v3 * w1, u1v3w0 = u1 * v3 * w0;
  double u1v2w3 = u1 * v2 * w3, u2v1w3 = u2 * v1 * w3, u0v2w3 = u0 * v2 * w3, u2v0w3 = u2 * v0 * w3,
         u0v1w3 = u0 * v1 * w3, u1v0w3 = u1 * v0 * w3;
  double u0v1w2 = u0 * v1 * w2, u0v2w1 = u0 * v2 * w1, u1v2w0 = u1 * v2 * w0, u1v0w2 = u1 * v0 * w2,
         u2v0w1 = u2 * v0 * w1, u2v1w0 = u2 * v1 * w0;
  double u3_0 = -u3v1w2 + u3v2w1, u3_1 = -u3v2w0 + u3v0w2, u3_2 = -u3v0w1 + u3v1w0;
  double v3_0 = u1v3w2 - u2v3w1, v3_1 = u2v3w0 - u0v3w2, v3_2 = u0v3w1 - u1v3w0;
  double w3_0 = -u1v2w3 + u2v1w3, w3_1 = u0v2w3 - u2v0w3, w3_2 = -u0v1w3 + u1v0w3;
  double c_4 = u0v1w2 - u0v2w1 + u1v2w0 - u1v0w2 + u2v0w1 - u2v1w0;
  double M0 = u3_0 + v3_0 + w3_0;
  double M1 = u3_1 + v3_1 + w3_1;
  double M2 = u3_2 + v3_2 + w3_2;
  double M3 = c_4;
  double M = M0 + M1 + M2 + M3;
  if (M == 0) return 0;
  int flag0 = (M0 == 0) || (M / M0 > 1);
  int flag1 = (M1 == 0) || (M / M1 > 1);
  int flag2 = (M2 == 0) || (M / M2 > 1);
  int flag3 = (M3 == 0) || (M / M3 > 1);
  if (flag0 && flag1 && flag2 && flag3) {
    if (same_direction(u0, u1, u2, u3) || same_direction(v0, v1, v2, v3) || same_direction(w0, w1, w2, w3)) return 1;
    return 0;
  }
  float eb = 0;
  double pm0 = 0, nm0 = 0, pm1 = 0, nm1 = 0, pm2 = 0, nm2 = 0, pm3 = 0, nm3 = 0;
  acc(-u3v1w2, &pm0, &nm0); acc(u3v2w1, &pm0, &nm0); acc(u1v3w2, &pm0, &nm0);
  acc(-u2v3w1, &pm0, &nm0); acc(-u1v2w3, &pm0, &nm0); acc(u2v1w3, &pm0, &nm0);
  acc(-u3v2w0, &pm1, &nm1); acc(u3v0w2, &pm1, &nm1); acc(u2v3w0, &pm1, &nm1);
  acc(-u0v3w2, &pm1, &nm1); acc(u0v2w3, &pm1, &nm1); acc(-u2v0w3, &pm1, &nm1);
  acc(-u3v0w1, &pm2, &nm2); acc(u3v1w0, &pm2, &nm2); acc(u0v3w1, &pm2, &nm2);
  acc(-u1v3w0, &pm2, &nm2); acc(-u0v1w3, &pm2, &nm2); acc(u1v0w3, &pm2, &nm2);
  acc(u0v1w2, &pm3, &nm3); acc(-u0v2w1, &pm3, &nm3); acc(u1v2w0, &pm3, &nm3);
  acc(-u1v0w2, &pm3, &nm3); acc(u2v0w1, &pm3, &nm3); acc(-u2v1w0, &pm3, &nm3);
  float p_m0 = (float)pm0, p_m1 = (float)pm1, p_m2 = (float)pm2, p_m3 = (float)pm3;
  float n_m0 = (float)nm0, n_m1 = (float)nm1, n_m2 = (float)nm2, n_m3 = (float)nm3;
  if (!flag0) {
    float eb1 = keep_sign_3d(p_m0, n_m0);
    float eb2 = keep_sign_3d(p_m1 + p_m2 + p_m3, n_m1 + n_m2 + n_m3);
    eb = maxf_(eb, minf_(eb1, eb2));
  }
  if (!flag1) {
    float eb1 = keep_sign_3d(p_m1, n_m1);
    float eb2 = keep_sign_3d(p_m0 + p_m2 + p_m3, n_m0 + n_m2 + n_m3);
    eb = maxf_(eb, minf_(eb1, eb2));
  }
  if (!flag2) {
    float eb1 = keep_sign_3d(p_m2, n_m2);
    float eb2 = keep_sign_3d(p_m0 + p_m1 + p_m3, n_m0 + n_m1 + n_m3);
    eb = maxf_(eb, minf_(eb1, eb2));
  }
  if (!flag3) {
    float eb1 = keep_sign_3d(p_m3, n_m3);
    float eb2 = keep_sign_3d(p_m0 + p_m1 + p_m2, n_m0 + n_m1 + n_m2);
    eb = maxf_(eb, minf_(eb1, eb2));
  }
  return eb;
}

/* Tet vertex offsets within a cube, (dx, dy, dz) = (fastest, middle, slowest)
 * axis; the 4th vertex of every tet is the cube corner (0,0,0).
 * src/sz_compress_cp_preserve_3d.cpp:9-46 (first six entries of `coordinates`). */
static const int tet_coords[6][3][3] = {
    {{0, 0, 1}, {0, 1, 1}, {1, 1, 1}}, {{0, 1, 0}, {0, 1, 1}, {1, 1, 1}}, {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}},
    {{1, 0, 0}, {1, 0, 1}, {1, 1, 1}}, {{0, 1, 0}, {1, 1, 0}, {1, 1, 1}}, {{1, 0, 0}, {1, 1, 0}, {1, 1, 1}}};

static inline double mind(double a, double b) { return (a < b) ? a : b; }

/* src/sz_compress_cp_preserve_3d.cpp:366-418 */
void cpo_eb_3d(const float* U, const float* V, const float* W, size_t r1, size_t r2, size_t r3, double max_pwr_eb,
               double* eb) {
  size_t n = r1 * r2 * r3, d0 = r2 * r3, d1 = r3;
  for (size_t i = 0; i < n; i++) eb[i] = max_pwr_eb;
  if (r1 < 2 || r2 < 2 || r3 < 2) return;
  ptrdiff_t off[6][3];
  for (int t = 0; t < 6; t++)
    for (int x = 0; x < 3; x++)
      off[t][x] = tet_coords[t][x][0] + tet_coords[t][x][1] * (ptrdiff_t)d1 + tet_coords[t][x][2] * (ptrdiff_t)d0;
  for (size_t i = 0; i + 1 < r1; i++)
    for (size_t j = 0; j + 1 < r2; j++)
      for (size_t k = 0; k + 1 < r3; k++) {
        size_t c = i * d0 + j * d1 + k;
        for (int t = 0; t < 6; t++) {
          double cur = tet_eb(U[c + off[t][0]], U[c + off[t][1]], U[c + off[t][2]], U[c], V[c + off[t][0]],
                              V[c + off[t][1]], V[c + off[t][2]], V[c], W[c + off[t][0]], W[c + off[t][1]],
                              W[c + off[t][2]], W[c]);
          eb[c] = mind(eb[c], cur);
          for (int x = 0; x < 3; x++) eb[c + off[t][x]] = mind(eb[c + off[t][x]], cur);
        }
      }
}

static int eb_exp_quantize(double* eb, int base, double log_of_base, double threshold) {
  if (*eb <= threshold) {
    *eb = 0;
    return 0;
  }
  int id = (int)(log2(*eb / threshold) / log_of_base);
  *eb = pow(base, id) * threshold;
  return id;
}

static void pack_bits(const unsigned char* bits, size_t n, unsigned char* out) {
  size_t nb = (n % 8 == 0) ? n / 8 : n / 8 + 1;
  for (size_t b = 0; b < nb; b++) {
    int tmp = 0;
    for (size_t j = 0; j < 8 && b * 8 + j < n; j++)
      if (bits[b * 8 + j] == 1) tmp |= 1 << (7 - j);
    out[b] = (unsigned char)tmp;
  }
}

static void put(unsigned char** p, const void* v, size_t n) {
  memcpy(*p, v, n);
  *p += n;
}

/* Encodes a Huffman section; for zero symbols (which the reference cannot
 * encode: its heap root would be NULL) a one-leaf tree of symbol 0 with an empty
 * bit stream is written, which the reference's decoder reads back as no symbols. */
static size_t huffman_section(size_t state_num, const int* sym, size_t n, unsigned char* out) {
  if (n > 0) return cpo_huffman_encode(state_num, sym, n, out);
  int zero = 0;
  return cpo_huffman_encode(state_num, &zero, 1, out);
}

/* src/sz_compress_cp_preserve_3d.cpp:360-581 */
unsigned char* cpo_compress_3d_offline_log(const float* U, const float* V, const float* W, size_t r1, size_t r2,
                                           size_t r3, double max_pwr_eb, size_t* size) {
  size_t n = r1 * r2 * r3, d0 = r2 * r3, d1 = r3;
  double* eb = (double*)malloc(n * sizeof(double));
  cpo_eb_3d(U, V, W, r1, r2, r3, max_pwr_eb, eb);
  size_t smap = (n - 1) / 8 + 1;
  unsigned char* signs = (unsigned char*)malloc(3 * smap);
  unsigned char* sign = (unsigned char*)malloc(n);
  const float* src[3] = {U, V, W};
  float* lg[3];
  for (int a = 0; a < 3; a++) {
    lg[a] = (float*)malloc(n * sizeof(float));
    for (size_t i = 0; i < n; i++) { /* log_transform, include/sz_cp_preserve_utils.hpp:201-216 */
      float x = src[a][i];
      sign[i] = 0;
      if (x != 0) {
        sign[i] = (x > 0);
        lg[a][i] = (x > 0) ? log2f(x) : log2f(-x);
      } else {
        lg[a][i] = -100;
      }
    }
    pack_bits(sign, n, signs + a * smap);
  }
  free(sign);
  const int capacity = 65536, radius = capacity >> 1, base = 2;
  const double log_of_base = log2(base);
  const double threshold = FLT_EPSILON;
  const int id_max = (int)(log2(1.0 / threshold) / log_of_base) + 1;
  int* ids = (int*)malloc(n * sizeof(int));
  int* codes = (int*)malloc(3 * n * sizeof(int));
  float* unpred = (float*)malloc(3 * n * sizeof(float));
  size_t n_codes = 0, n_unpred = 0;
  for (size_t i = 0; i < r1; i++)
    for (size_t j = 0; j < r2; j++)
      for (size_t k = 0; k < r3; k++) {
        size_t idx = i * d0 + j * d1 + k;
        double required_eb = eb[idx];
        int unpred_flag = 0;
        if (required_eb > 0) {
          float dec[3];
          double abs_eb = log2(1 + required_eb);
          ids[idx] = eb_exp_quantize(&abs_eb, base, log_of_base, threshold);
          if (ids[idx] > 0) {
            for (int p = 0; p < 3; p++) {
              float* L = lg[p];
              float cur = L[idx];
              float q0 = (i && j && k) ? L[idx - d0 - d1 - 1] : 0;
              float q1 = (i && j) ? L[idx - d0 - d1] : 0;
              float q2 = (i && k) ? L[idx - d0 - 1] : 0;
              float q3 = i ? L[idx - d0] : 0;
              float q4 = (j && k) ? L[idx - d1 - 1] : 0;
              float q5 = j ? L[idx - d1] : 0;
              float q6 = k ? L[idx - 1] : 0;
              float pred = q0 + q3 + q5 + q6 - q1 - q2 - q4;
              double diff = (float)(cur - pred);
              double qd = fabs(diff) / abs_eb + 1;
              if (qd < capacity) {
                qd = (diff > 0) ? qd : -qd;
                int qi = (int)(qd / 2) + radius;
                codes[n_codes + p] = qi;
                dec[p] = (float)(pred + 2 * (qi - radius) * abs_eb);
                if (fabsf(dec[p] - cur) >= abs_eb) { unpred_flag = 1; break; }
              } else { unpred_flag = 1; break; }
            }
          } else unpred_flag = 1;
          if (unpred_flag) {
            ids[idx] = id_max;
          } else {
            n_codes += 3;
            lg[0][idx] = dec[0];
            lg[1][idx] = dec[1];
            lg[2][idx] = dec[2];
          }
        } else {
          ids[idx] = 0;
          unpred_flag = 1;
        }
        if (unpred_flag) {
          unpred[n_unpred++] = U[idx];
          unpred[n_unpred++] = V[idx];
          unpred[n_unpred++] = W[idx];
        }
      }
  free(eb);
  for (int a = 0; a < 3; a++) free(lg[a]);
  size_t cap = 8 + 3 * smap + 8 + n_unpred * 4 + 8 + cpo_huffman_encode_bound(2 * 256, n) + 8 +
               cpo_huffman_encode_bound(2 * capacity, n_codes ? n_codes : 1);
  unsigned char* out = (unsigned char*)calloc(cap, 1);
  unsigned char* p = out;
  put(&p, &base, sizeof(int));
  put(&p, &radius, sizeof(int));
  put(&p, signs, 3 * smap);
  put(&p, &n_unpred, sizeof(size_t));
  put(&p, unpred, n_unpred * sizeof(float));
  put(&p, &n, sizeof(size_t));
  p += huffman_section(2 * 256, ids, n, p);
  put(&p, &n_codes, sizeof(size_t));
  p += huffman_section(2 * capacity, codes, n_codes, p);
  *size = (size_t)(p - out);
  free(signs);
  free(ids);
  free(codes);
  free(unpred);
  return out;
}

static void unpack_bits(const unsigned char* in, size_t n, unsigned char* bits) {
  for (size_t i = 0; i < n; i++) bits[i] = (in[i >> 3] >> (7 - (i & 7))) & 1;
}

/* src/sz_decompress_cp_preserve_3d.cpp:7-110 */
int cpo_decompress_3d_online_log(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, size_t r3,
                                 float* U, float* V, float* W) {
  size_t n = r1 * r2 * r3, d0 = r2 * r3, d1 = r3;
  const unsigned char* p = blob;
  const unsigned char* end = blob + blob_size;
  size_t smap = (n - 1) / 8 + 1;
  if (blob_size < 8 + 3 * smap + 8) return 1;
  int base, radius;
  memcpy(&base, p, 4); p += 4;
  memcpy(&radius, p, 4); p += 4;
  unsigned char* sgn[3];
  for (int a = 0; a < 3; a++) {
    sgn[a] = (unsigned char*)malloc(n);
    unpack_bits(p, n, sgn[a]);
    p += smap;
  }
  int rc = 0;
  size_t n_unpred, n_ids, n_codes;
  int *ids = NULL, *codes = NULL;
  unsigned char* is_raw = NULL;
  memcpy(&n_unpred, p, 8); p += 8;
  if (n_unpred > 3 * n || (size_t)(end - p) < n_unpred * 4 + 8) { rc = 2; goto out; }
  const float* unpred = (const float*)p;
  p += n_unpred * 4;
  memcpy(&n_ids, p, 8); p += 8;
  if (n_ids != n) { rc = 3; goto out; }
  ids = (int*)malloc(n * sizeof(int));
  size_t used = cpo_huffman_decode(2 * 256, n, p, (size_t)(end - p), ids);
  if (!used) { rc = 4; goto out; }
  p += used;
  if ((size_t)(end - p) < 8) { rc = 5; goto out; }
  memcpy(&n_codes, p, 8); p += 8;
  if (n_codes > 3 * n) { rc = 5; goto out; }
  codes = (int*)malloc((n_codes ? n_codes : 1) * sizeof(int));
  used = cpo_huffman_decode(2 * 2 * (size_t)radius, n_codes, p, (size_t)(end - p), codes);
  if (!used) { rc = 6; goto out; }
  {
    const double threshold = FLT_EPSILON;
    const double log_of_base = log2(base);
    const int id_max = (int)(log2(1.0 / threshold) / log_of_base) + 1;
    float* out[3] = {U, V, W};
    is_raw = (unsigned char*)calloc(n, 1);
    const float* up = unpred;
    const int* cp = codes;
    const int* cp_end = codes + n_codes;
    for (size_t i = 0; i < r1; i++)
      for (size_t j = 0; j < r2; j++)
        for (size_t k = 0; k < r3; k++) {
          size_t idx = i * d0 + j * d1 + k;
          int id = ids[idx];
          if (id == 0 || id == id_max) {
            is_raw[idx] = 1;
            if (up + 3 > unpred + n_unpred) { rc = 7; goto out; }
            for (int a = 0; a < 3; a++) {
              float x = *up++;
              out[a][idx] = (x == 0) ? -100 : log2f(fabsf(x));
            }
          } else {
            double e = pow(base, id) * threshold;
            if (cp + 3 > cp_end) { rc = 8; goto out; }
            for (int a = 0; a < 3; a++) {
              float* L = out[a];
              float q0 = (i && j && k) ? L[idx - d0 - d1 - 1] : 0;
              float q1 = (i && j) ? L[idx - d0 - d1] : 0;
              float q2 = (i && k) ? L[idx - d0 - 1] : 0;
              float q3 = i ? L[idx - d0] : 0;
              float q4 = (j && k) ? L[idx - d1 - 1] : 0;
              float q5 = j ? L[idx - d1] : 0;
              float q6 = k ? L[idx - 1] : 0;
              float pred = q0 + q3 + q5 + q6 - q1 - q2 - q4;
              L[idx] = (float)(pred + 2 * (cp[a] - radius) * e);
            }
            cp += 3;
          }
        }
    up = unpred;
    for (size_t i = 0; i < n; i++) {
      if (is_raw[i]) {
        U[i] = *up++;
        V[i] = *up++;
        W[i] = *up++;
      } else {
        for (int a = 0; a < 3; a++) {
          float x = out[a][i];
          if (x < -99) out[a][i] = 0;
          else out[a][i] = sgn[a][i] ? exp2f(x) : -exp2f(x);
        }
      }
    }
  }
out:
  for (int a = 0; a < 3; a++) free(sgn[a]);
  free(ids);
  free(codes);
  free(is_raw);
  return rc;
}
