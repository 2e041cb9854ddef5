/* cpsz_oracle.c -- 2D offline path of the CPU oracle (test infrastructure only;
 * see cpsz_oracle.h).  Every function restates the cited reference code with the
 * same operand types and evaluation order:
 *   - `float * float` products stay float and are widened afterwards,
 *   - sums are evaluated left to right in the type the reference declares,
 *   - MINF(a,b) = (a<b)?a:b and MAX(a,b) = (a>b)?a:b keep their NaN behaviour,
 *   - glibc log2 / pow / sqrt are called exactly where the reference calls them.
 */
#include "cpsz_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline double minf_d(double a, double b) { return (a < b) ? a : b; }  /* include/sz_def.hpp:157-160 */
static inline double max_d(double a, double b) { return (a > b) ? a : b; }   /* include/sz_def.hpp:154 */
static inline float minf_f(float a, float b) { return (a < b) ? a : b; }

/* accumulate<T>(value, positive, negative): include/sz_cp_preserve_utils.hpp:194-198 */
static inline void acc(double value, double* pos, double* neg) {
  if (value >= 0) *pos += value;
  else *neg += -value;
}

/* max_eb_to_keep_sign (degree 1 or 2): include/sz_cp_preserve_utils.hpp:61-92.
 * The negative-input exit(0) branch cannot trigger (sums of magnitudes). */
static double keep_sign(double positive, double negative, int degree) {
  if ((negative == 0) || (positive == 0)) return 1;
  double P, N;
  if (degree == 1) { P = positive; N = negative; }
  else { P = sqrt(positive); N = sqrt(negative); }
  return fabs(P - N) / (P + N);
}

/* max_eb_to_keep_sign_2d_offline_2 / _4 with T = double:
 * src/sz_compress_cp_preserve_2d.cpp:31-49 */
static double keep_sign_off2(double a, double b) {
  double p = 0, n = 0;
  acc(a, &p, &n);
  acc(b, &p, &n);
  return keep_sign(p, n, 2);
}
static double keep_sign_off4(double a, double b, double c, double d) {
  double p = 0, n = 0;
  acc(a, &p, &n);
  acc(b, &p, &n);
  acc(c, &p, &n);
  acc(d, &p, &n);
  return keep_sign(p, n, 2);
}

/* max_eb_to_keep_sign_det2x2<float>: src/sz_compress_cp_preserve_2d.cpp:18-29 */
static double keep_sign_det2x2(float u0, float u1, float u2, float v0, float v1, float v2) {
  double p = 0, n = 0;
  acc((float)(u0 * v1), &p, &n);
  acc((float)(-u0 * v2), &p, &n);
  acc((float)(u1 * v2), &p, &n);
  acc((float)(-u1 * v0), &p, &n);
  acc((float)(u2 * v0), &p, &n);
  acc((float)(-u2 * v1), &p, &n);
  return keep_sign(p, n, 2);
}

/* max_eb_to_keep_sign_eigen_delta_2<float>: src/sz_compress_cp_preserve_2d.cpp:79-123
 * (with get_adjugate_matrix_for_position :55-63 and accumulate_in_square :67-73). */
static double keep_sign_eigen(float u0, float u1, float u2, float v0, float v1, float v2, float x0, float x1,
                              float x2, float y0, float y1, float y2) {
  double eb = 1;
  float c[4];
  {
    float det = (x0 - x2) * (y1 - y2) - (x1 - x2) * (y0 - y2);
    c[0] = (y1 - y2) / det;
    c[1] = -(y0 - y2) / det;
    c[2] = -(x1 - x2) / det;
    c[3] = (x0 - x2) / det;
    double p = 0, n = 0;
    acc((float)(c[0] * u0), &p, &n);
    acc((float)(c[1] * u1), &p, &n);
    acc((float)(-(c[0] + c[1]) * u2), &p, &n);
    acc((float)(c[2] * v0), &p, &n);
    acc((float)(c[3] * v1), &p, &n);
    acc((float)(-(c[2] + c[3]) * v2), &p, &n);
    eb = keep_sign(p, n, 1);
    eb = minf_d(eb, keep_sign_det2x2(u0, u1, u2, v0, v1, v2));
  }
  float m = c[1] * c[2] - c[0] * c[3];
  float C = (-m) * (u0 * v1 - u0 * v2 + u1 * v2 - u1 * v0 + u2 * v0 - u2 * v1);
  if (C == 0) return 0;
  if (C < 0) return eb;
  {
    float coeff[6];
    coeff[0] = c[0] * u0;
    coeff[1] = c[1] * u1;
    coeff[2] = -(c[1] + c[0]) * u2;
    coeff[3] = c[2] * v0;
    coeff[4] = c[3] * v1;
    coeff[5] = -(c[3] + c[2]) * v2;
    double p = 0, n = 0;
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) acc((float)(coeff[i] * coeff[j]), &p, &n);
    acc((float)(-4 * m * u1 * v0), &p, &n);
    acc((float)(4 * m * u2 * v0), &p, &n);
    acc((float)(4 * m * u0 * v1), &p, &n);
    acc((float)(-4 * m * u2 * v1), &p, &n);
    acc((float)(-4 * m * u0 * v2), &p, &n);
    acc((float)(4 * m * u1 * v2), &p, &n);
    eb = minf_d(eb, keep_sign(p, n, 2));
  }
  return eb;
}

/* max_eb_to_keep_position_and_type<float>: src/sz_compress_cp_preserve_2d.cpp:125-172 */
static double tri_eb(float u0, float u1, float u2, float v0, float v1, float v2, float x0, float x1, float x2,
                     float y0, float y1, float y2) {
  double u0v1 = (float)(u0 * v1);
  double u1v0 = (float)(u1 * v0);
  double u0v2 = (float)(u0 * v2);
  double u2v0 = (float)(u2 * v0);
  double u1v2 = (float)(u1 * v2);
  double u2v1 = (float)(u2 * v1);
  double det = u0v1 - u1v0 + u1v2 - u2v1 + u2v0 - u0v2;
  double eb = 0;
  if (det != 0) {
    int f1 = (det / (u2v0 - u0v2) >= 1);
    int f2 = (det / (u1v2 - u2v1) >= 1);
    int f3 = (det / (u0v1 - u1v0) >= 1);
    if (f1 && f2 && f3) {
      eb = 1;
      double eb1 = minf_d(keep_sign_off2(u2v0, -u0v2), keep_sign_off4(u0v1, -u1v0, u1v2, -u2v1));
      double eb2 = minf_d(keep_sign_off2(u1v2, -u2v1), keep_sign_off4(u0v1, -u1v0, u2v0, -u0v2));
      double eb3 = minf_d(keep_sign_off2(u0v1, -u1v0), keep_sign_off4(u1v2, -u2v1, u2v0, -u0v2));
      double eb4 = minf_d(eb3, keep_sign_eigen(u0, u1, u2, v0, v1, v2, x0, x1, x2, y0, y1, y2));
      eb = minf_d(eb1, eb2);
      eb = minf_d(eb, eb4);
    } else {
      eb = 0;
      if (!f1) {
        double cur = minf_d(keep_sign_off2(u2v0, -u0v2), keep_sign_off4(u0v1, -u1v0, u1v2, -u2v1));
        eb = max_d(eb, cur);
      }
      if (!f2) {
        double cur = minf_d(keep_sign_off2(u1v2, -u2v1), keep_sign_off4(u0v1, -u1v0, u2v0, -u0v2));
        eb = max_d(eb, cur);
      }
      if (!f3) {
        double cur = minf_d(keep_sign_off2(u0v1, -u1v0), keep_sign_off4(u1v2, -u2v1, u2v0, -u0v2));
        eb = max_d(eb, cur);
      }
    }
  }
  return eb;
}

/* Offline eb loop: src/sz_compress_cp_preserve_2d.cpp:177-218.  Triangle k=0
 * ("upper") = offsets {0, r2, r2+1} with X = {{0,0},{1,0},{1,1}}, k=1 ("lower")
 * = {0, 1, r2+1} with X = {{0,0},{0,1},{1,1}}; X is passed "reversed"
 * (x = column 1 of X, y = column 0). */
void cpo_eb_2d(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb, double* eb) {
  size_t n = r1 * r2;
  for (size_t i = 0; i < n; i++) eb[i] = max_pwr_eb;
  if (r1 < 2 || r2 < 2) return;
  static const float Xu[3][2] = {{0, 0}, {1, 0}, {1, 1}};
  static const float Xl[3][2] = {{0, 0}, {0, 1}, {1, 1}};
  const size_t ou[3] = {0, r2, r2 + 1};
  const size_t ol[3] = {0, 1, r2 + 1};
  for (size_t i = 0; i + 1 < r1; i++) {
    for (size_t j = 0; j + 1 < r2; j++) {
      size_t b = i * r2 + j;
      for (int k = 0; k < 2; k++) {
        const float(*X)[2] = (k == 0) ? Xu : Xl;
        const size_t* o = (k == 0) ? ou : ol;
        double cur = tri_eb(U[b + o[0]], U[b + o[1]], U[b + o[2]], V[b + o[0]], V[b + o[1]], V[b + o[2]], X[0][1],
                            X[1][1], X[2][1], X[0][0], X[1][0], X[2][0]);
        eb[b + o[0]] = minf_d(eb[b + o[0]], cur);
        eb[b + o[1]] = minf_d(eb[b + o[1]], cur);
        eb[b + o[2]] = minf_d(eb[b + o[2]], cur);
      }
    }
  }
}

/* eb_exponential_quantize: include/sz_cp_preserve_utils.hpp:14-22 */
static int eb_exp_quantize(double* eb, int base, double log_of_base, double threshold) {
  if (*eb <= threshold) {
    *eb = 0;
    return 0;
  }
  int id = (int)(log2(*eb / threshold) / log_of_base);
  *eb = pow(base, id) * threshold;
  return id;
}

/* src/sz_compress_cp_preserve_2d.cpp:226-244 */
void cpo_quantize_eb_2d(const float* U, const float* V, const double* eb, size_t n, int* ids, double* eb_u,
                        double* eb_v) {
  const int base = 4;
  const double log2_of_base = log2(base);
  const double threshold = DBL_EPSILON;
  for (size_t i = 0; i < n; i++) {
    eb_u[i] = fabsf(U[i]) * eb[i];
    ids[i] = eb_exp_quantize(&eb_u[i], base, log2_of_base, threshold);
    if (eb_u[i] < threshold) eb_u[i] = 0;
  }
  for (size_t i = 0; i < n; i++) {
    eb_v[i] = fabsf(V[i]) * eb[i];
    ids[n + i] = eb_exp_quantize(&eb_v[i], base, log2_of_base, threshold);
    if (eb_v[i] < threshold) eb_v[i] = 0;
  }
}

/* quantize() with reconstruction: include/sz_compression_utils.hpp:52-65
 * (T = float, capacity 65536, radius 32768). */
static int quantize_f(float pred, float cur, double precision, int capacity, int radius, float** unpred_pos,
                      float* decompressed) {
  double diff = (float)(cur - pred);
  double quant_diff = fabs(diff) / precision + 1;
  if (quant_diff < capacity) {
    quant_diff = (diff > 0) ? quant_diff : -quant_diff;
    int qi = (int)(quant_diff / 2) + radius;
    float dec = (float)(pred + 2 * (qi - radius) * precision);
    *decompressed = dec;
    if (fabsf(dec - cur) <= precision) return qi;
  }
  *decompressed = cur;
  *((*unpred_pos)++) = cur;
  return 0;
}

/* Block traversal of prediction_and_quantization_2d_with_border_prediction_with_eb
 * (src/sz_compress_3d.cpp:126-193) and block_pred_and_quant_lorenzo_2d_with_eb
 * (include/sz_compress_block_processing.hpp:106-139), block size 12.  The
 * reference's (bs+1) x (d2+1) rolling buffer with a zero first row/column is the
 * raster reconstruction with zero padding, kept here as a full array. */
size_t cpo_lorenzo_2d(const float* data, const double* prec, size_t r1, size_t r2, int* type, float* unpred,
                      float* recon_out) {
  const int bs = 12, capacity = 65536, radius = 32768;
  float* rec = recon_out ? recon_out : (float*)malloc(r1 * r2 * sizeof(float));
  float* up = unpred;
  int* tp = type;
  size_t nbx = (r1 - 1) / bs + 1, nby = (r2 - 1) / bs + 1;
  for (size_t bi = 0; bi < nbx; bi++) {
    for (size_t bj = 0; bj < nby; bj++) {
      size_t sx = ((bi + 1) * bs < r1) ? bs : r1 - bi * bs;
      size_t sy = ((bj + 1) * bs < r2) ? bs : r2 - bj * bs;
      for (size_t li = 0; li < sx; li++) {
        size_t i = bi * bs + li;
        for (size_t lj = 0; lj < sy; lj++) {
          size_t j = bj * bs + lj;
          size_t idx = i * r2 + j;
          double precision = prec[idx];
          if (precision == 0) {
            *tp++ = 0;
            *up++ = data[idx];
            rec[idx] = data[idx];
          } else {
            float L = j ? rec[idx - 1] : 0.0f;
            float Up = i ? rec[idx - r2] : 0.0f;
            float UL = (i && j) ? rec[idx - r2 - 1] : 0.0f;
            float pred = L + Up - UL; /* include/sz_prediction.hpp:12-14 */
            *tp++ = quantize_f(pred, data[idx], precision, capacity, radius, &up, &rec[idx]);
          }
        }
      }
    }
  }
  size_t count = (size_t)(up - unpred);
  if (!recon_out) free(rec);
  return count;
}

static inline void put_bytes(unsigned char** p, const void* v, size_t n) {
  memcpy(*p, v, n);
  *p += n;
}

/* sz_compress_2d_with_eb<float>: src/sz_compress_3d.cpp:196-236.  The 3 padding
 * bytes of meanInfo<float> (uninitialised in the reference) are written as 0. */
unsigned char* cpo_compress_2d_with_eb(const float* data, const double* prec, size_t r1, size_t r2, size_t* size) {
  const int bs = 12, capacity = 65536, radius = capacity >> 1;
  size_t n = r1 * r2;
  size_t nblocks = ((r1 - 1) / bs + 1) * ((r2 - 1) / bs + 1);
  int* type = (int*)malloc(n * sizeof(int));
  float* unpred = (float*)malloc(n * sizeof(float));
  size_t n_unpred = cpo_lorenzo_2d(data, prec, r1, r2, type, unpred, NULL);
  size_t cap = 64 + n_unpred * 4 + nblocks / 8 + 1 + cpo_huffman_encode_bound(2 * capacity, n);
  unsigned char* out = (unsigned char*)calloc(cap, 1);
  unsigned char* p = out;
  put_bytes(&p, &bs, sizeof(int));
  char bi = 0;
  put_bytes(&p, &bi, 1);
  put_bytes(&p, &radius, sizeof(int));
  unsigned char mean_info[8] = {0, 0, 0, 0, 0, 0, 0, 0}; /* {bool use_mean=false; float mean=0} */
  put_bytes(&p, mean_info, 8);
  size_t reg_count = 0;
  put_bytes(&p, &reg_count, sizeof(size_t));
  put_bytes(&p, &n_unpred, sizeof(size_t));
  put_bytes(&p, unpred, n_unpred * sizeof(float));
  /* indicator: all blocks Lorenzo (0), packed 8 per byte (src/sz_compression_utils.cpp:31-52) */
  size_t ind_bytes = (nblocks % 8 == 0) ? nblocks / 8 : nblocks / 8 + 1;
  memset(p, 0, ind_bytes);
  p += ind_bytes;
  p += cpo_huffman_encode(2 * capacity, type, n, p);
  *size = (size_t)(p - out);
  free(type);
  free(unpred);
  return out;
}

/* sz_compress_cp_preserve_2d_offline<float>: src/sz_compress_cp_preserve_2d.cpp:175-274 */
unsigned char* cpo_compress_2d_offline(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                                       size_t* size) {
  size_t n = r1 * r2;
  double* eb = (double*)malloc(n * sizeof(double));
  cpo_eb_2d(U, V, r1, r2, max_pwr_eb, eb);
  double* eb_u = (double*)malloc(n * sizeof(double));
  double* eb_v = (double*)malloc(n * sizeof(double));
  int* ids = (int*)malloc(2 * n * sizeof(int));
  cpo_quantize_eb_2d(U, V, eb, n, ids, eb_u, eb_v);
  free(eb);
  unsigned char* ceb = (unsigned char*)calloc(cpo_huffman_encode_bound(2 * 1024, 2 * n), 1);
  size_t ceb_size = cpo_huffman_encode(2 * 1024, ids, 2 * n, ceb);
  free(ids);
  if (!ceb_size) { /* bound ids out of range (NaN bounds): unsupported */
    free(ceb);
    free(eb_u);
    free(eb_v);
    *size = 0;
    return NULL;
  }
  size_t cu_size = 0, cv_size = 0;
  unsigned char* cu = cpo_compress_2d_with_eb(U, eb_u, r1, r2, &cu_size);
  unsigned char* cv = cpo_compress_2d_with_eb(V, eb_v, r1, r2, &cv_size);
  free(eb_u);
  free(eb_v);
  size_t total = sizeof(int) + sizeof(size_t) + ceb_size + sizeof(size_t) + cu_size + sizeof(size_t) + cv_size +
                 sizeof(size_t);
  unsigned char* out = (unsigned char*)malloc(total);
  unsigned char* p = out;
  const int base = 4;
  const double threshold = DBL_EPSILON;
  put_bytes(&p, &base, sizeof(int));
  put_bytes(&p, &threshold, sizeof(double));
  put_bytes(&p, &ceb_size, sizeof(size_t));
  put_bytes(&p, &cu_size, sizeof(size_t));
  put_bytes(&p, &cv_size, sizeof(size_t));
  put_bytes(&p, ceb, ceb_size);
  put_bytes(&p, cu, cu_size);
  put_bytes(&p, cv, cv_size);
  free(ceb);
  free(cu);
  free(cv);
  *size = total;
  return out;
}

/* sz_decompress_2d_with_eb<float> (src/sz_decompress_3d.cpp:124-155) with
 * prediction_and_decompression_2d_with_border_prediction_with_eb (:85-122),
 * block_pred_and_decompress_lorenzo_2d_with_eb
 * (include/sz_decompress_block_processing.hpp:68-83) and recover
 * (include/sz_decompression_utils.hpp:65-73).  Returns bytes consumed or 0. */
static size_t decompress_2d_with_eb(const unsigned char* in, size_t in_size, const double* prec, size_t r1,
                                    size_t r2, float* out) {
  const unsigned char* p = in;
  const unsigned char* end = in + in_size;
  if (in_size < 4 + 1 + 4 + 8 + 8 + 8) return 0;
  int bs;
  memcpy(&bs, p, 4); p += 4;
  p += 1; /* block_independant */
  int radius;
  memcpy(&radius, p, 4); p += 4;
  unsigned char mean_info[8];
  memcpy(mean_info, p, 8); p += 8;
  size_t reg_count, n_unpred;
  memcpy(&reg_count, p, 8); p += 8;
  memcpy(&n_unpred, p, 8); p += 8;
  if (bs <= 0 || reg_count != 0 || mean_info[0] != 0) return 0; /* only the format the offline compressor emits */
  if (n_unpred > r1 * r2 || (size_t)(end - p) < n_unpred * 4) return 0;
  const float* unpred = (const float*)p;
  p += n_unpred * 4;
  size_t nblocks = ((r1 - 1) / bs + 1) * ((r2 - 1) / bs + 1);
  p += (nblocks - 1) / 8 + 1;
  if (p > end) return 0;
  size_t n = r1 * r2;
  int* type = (int*)malloc(n * sizeof(int));
  size_t used = cpo_huffman_decode(4 * (size_t)radius, n, p, (size_t)(end - p), type);
  if (!used) { free(type); return 0; }
  p += used;
  size_t nbx = (r1 - 1) / bs + 1, nby = (r2 - 1) / bs + 1;
  const int* tp = type;
  const float* up = unpred;
  const float* up_end = unpred + n_unpred;
  for (size_t bi = 0; bi < nbx; bi++) {
    for (size_t bj = 0; bj < nby; bj++) {
      size_t sx = ((bi + 1) * bs < r1) ? bs : r1 - bi * bs;
      size_t sy = ((bj + 1) * bs < r2) ? bs : r2 - bj * bs;
      for (size_t li = 0; li < sx; li++) {
        size_t i = bi * bs + li;
        for (size_t lj = 0; lj < sy; lj++) {
          size_t j = bj * bs + lj;
          size_t idx = i * r2 + j;
          float L = j ? out[idx - 1] : 0.0f;
          float Up = i ? out[idx - r2] : 0.0f;
          float UL = (i && j) ? out[idx - r2 - 1] : 0.0f;
          float pred = L + Up - UL;
          int t = *tp++;
          if (t == 0) {
            if (up >= up_end) { free(type); return 0; }
            out[idx] = *up++;
          } else {
            out[idx] = (float)(pred + 2 * (t - radius) * prec[idx]);
          }
        }
      }
    }
  }
  free(type);
  return (size_t)(p - in);
}

/* sz_decompress_cp_preserve_2d_offline<float>: src/sz_decompress_cp_preserve_2d.cpp:8-52 */
int cpo_decompress_2d_offline(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, float* U,
                              float* V) {
  const unsigned char* p = blob;
  if (blob_size < 4 + 8 + 24) return 1;
  int base;
  double threshold;
  size_t eb_size, u_size, v_size;
  memcpy(&base, p, 4); p += 4;
  memcpy(&threshold, p, 8); p += 8;
  memcpy(&eb_size, p, 8); p += 8;
  memcpy(&u_size, p, 8); p += 8;
  memcpy(&v_size, p, 8); p += 8;
  size_t hdr = (size_t)(p - blob);
  if (eb_size > blob_size - hdr || u_size > blob_size - hdr - eb_size ||
      v_size > blob_size - hdr - eb_size - u_size)
    return 2;
  size_t n = r1 * r2;
  int* type = (int*)malloc(2 * n * sizeof(int));
  if (!cpo_huffman_decode(2 * 1024, 2 * n, p, eb_size, type)) { free(type); return 3; }
  p += eb_size;
  double* eb = (double*)malloc(n * sizeof(double));
  for (size_t i = 0; i < n; i++) eb[i] = (type[i] == 0) ? 0 : pow(base, type[i]) * threshold;
  int rc = 0;
  if (!decompress_2d_with_eb(p, u_size, eb, r1, r2, U)) rc = 4;
  p += u_size;
  for (size_t i = 0; i < n; i++) eb[i] = (type[n + i] == 0) ? 0 : pow(base, type[n + i]) * threshold;
  if (!rc && !decompress_2d_with_eb(p, v_size, eb, r1, r2, V)) rc = 5;
  free(eb);
  free(type);
  return rc;
}

/* ---- 2D offline_log pair ---------------------------------------------------- */

/* convertIntArray2ByteArray_fast_1b_to_result_sz: src/sz_compression_utils.cpp:31-52
 * (bit 7 - j of byte b holds element 8b + j). */
static void pack_bits_2d(const unsigned char* bits, size_t n, unsigned char* out) {
  size_t nb = (n % 8 == 0) ? n / 8 : n / 8 + 1;
  for (size_t b = 0; b < nb; b++) {
    int tmp = 0;
    for (size_t j = 0; j < 8 && b * 8 + j < n; j++)
      if (bits[b * 8 + j] == 1) tmp |= 1 << (7 - j);
    out[b] = (unsigned char)tmp;
  }
}

/* log_transform: include/sz_cp_preserve_utils.hpp:205-221 (log2f of |x|, -100 for 0,
 * sign = x > 0). */
static float* log_transform_2d(const float* data, unsigned char* sign, size_t n) {
  float* out = (float*)malloc(n * sizeof(float));
  for (size_t i = 0; i < n; i++) {
    sign[i] = 0;
    if (data[i] != 0) {
      sign[i] = (data[i] > 0);
      out[i] = (data[i] > 0) ? log2f(data[i]) : log2f(-data[i]);
    } else {
      out[i] = -100;
    }
  }
  return out;
}

/* sz_compress_cp_preserve_2d_offline_log<float>: src/sz_compress_cp_preserve_2d.cpp:285-379.
 * The per-vertex bound is the offline one; it is taken to the log domain as
 * log2(1 + eb) and quantized with base 2 and threshold DBL_EPSILON (one id
 * stream for both components); U and V are compressed as log2f values. */
unsigned char* cpo_compress_2d_offline_log(const float* U, const float* V, size_t r1, size_t r2, double max_pwr_eb,
                                           size_t* size) {
  size_t n = r1 * r2;
  double* eb = (double*)malloc(n * sizeof(double));
  cpo_eb_2d(U, V, r1, r2, max_pwr_eb, eb);
  size_t smap = (n - 1) / 8 + 1;
  unsigned char* signs = (unsigned char*)malloc(2 * smap);
  unsigned char* sign = (unsigned char*)malloc(n);
  float* log_u = log_transform_2d(U, sign, n);
  pack_bits_2d(sign, n, signs);
  float* log_v = log_transform_2d(V, sign, n);
  pack_bits_2d(sign, n, signs + smap);
  free(sign);
  int* ids = (int*)malloc(n * sizeof(int));
  const int base = 2;
  const double log2_of_base = log2(base);
  const double threshold = DBL_EPSILON;
  for (size_t i = 0; i < n; i++) {
    eb[i] = log2(1 + eb[i]);
    ids[i] = eb_exp_quantize(&eb[i], base, log2_of_base, threshold);
  }
  unsigned char* ceb = (unsigned char*)calloc(cpo_huffman_encode_bound(2 * 1024, n), 1);
  size_t ceb_size = cpo_huffman_encode(2 * 1024, ids, n, ceb);
  free(ids);
  if (!ceb_size) { /* bound ids out of range (NaN bounds): unsupported */
    free(ceb);
    free(log_u);
    free(log_v);
    free(eb);
    free(signs);
    *size = 0;
    return NULL;
  }
  size_t cu_size = 0, cv_size = 0;
  unsigned char* cu = cpo_compress_2d_with_eb(log_u, eb, r1, r2, &cu_size);
  free(log_u);
  unsigned char* cv = cpo_compress_2d_with_eb(log_v, eb, r1, r2, &cv_size);
  free(log_v);
  free(eb);
  size_t total = sizeof(int) + sizeof(double) + 3 * sizeof(size_t) + ceb_size + 2 * smap + cu_size + cv_size;
  unsigned char* out = (unsigned char*)malloc(total);
  unsigned char* p = out;
  put_bytes(&p, &base, sizeof(int));
  put_bytes(&p, &threshold, sizeof(double));
  put_bytes(&p, &ceb_size, sizeof(size_t));
  put_bytes(&p, &cu_size, sizeof(size_t));
  put_bytes(&p, &cv_size, sizeof(size_t));
  put_bytes(&p, ceb, ceb_size);
  put_bytes(&p, signs, 2 * smap);
  put_bytes(&p, cu, cu_size);
  put_bytes(&p, cv, cv_size);
  free(ceb);
  free(signs);
  free(cu);
  free(cv);
  *size = total;
  return out;
}

/* sz_decompress_cp_preserve_2d_offline_log<float>: src/sz_decompress_cp_preserve_2d.cpp:56-99
 * (exp2f of the decoded log values, -99 and below decode to 0). */
int cpo_decompress_2d_offline_log(const unsigned char* blob, size_t blob_size, size_t r1, size_t r2, float* U,
                                  float* V) {
  const unsigned char* p = blob;
  size_t n = r1 * r2, smap = (n - 1) / 8 + 1;
  if (blob_size < 4 + 8 + 24) return 1;
  int base;
  double threshold;
  size_t eb_size, u_size, v_size;
  memcpy(&base, p, 4); p += 4;
  memcpy(&threshold, p, 8); p += 8;
  memcpy(&eb_size, p, 8); p += 8;
  memcpy(&u_size, p, 8); p += 8;
  memcpy(&v_size, p, 8); p += 8;
  size_t hdr = (size_t)(p - blob);
  if (eb_size > blob_size - hdr || 2 * smap > blob_size - hdr - eb_size ||
      u_size > blob_size - hdr - eb_size - 2 * smap || v_size > blob_size - hdr - eb_size - 2 * smap - u_size)
    return 2;
  int* type = (int*)malloc(n * sizeof(int));
  if (!cpo_huffman_decode(2 * 1024, n, p, eb_size, type)) { free(type); return 3; }
  p += eb_size;
  double* eb = (double*)malloc(n * sizeof(double));
  for (size_t i = 0; i < n; i++) eb[i] = (type[i] == 0) ? 0 : pow(base, type[i]) * threshold;
  free(type);
  const unsigned char* su = p;
  const unsigned char* sv = p + smap;
  p += 2 * smap;
  int rc = 0;
  if (!decompress_2d_with_eb(p, u_size, eb, r1, r2, U)) rc = 4;
  p += u_size;
  if (!rc && !decompress_2d_with_eb(p, v_size, eb, r1, r2, V)) rc = 5;
  free(eb);
  if (rc) return rc;
  for (size_t i = 0; i < n; i++) {
    int bu = (su[i / 8] >> (7 - i % 8)) & 1, bv = (sv[i / 8] >> (7 - i % 8)) & 1;
    U[i] = (U[i] < -99) ? 0 : (bu ? exp2f(U[i]) : -exp2f(U[i]));
    V[i] = (V[i] < -99) ? 0 : (bv ? exp2f(V[i]) : -exp2f(V[i]));
  }
  return 0;
}

void cpo_free(void* p) { free(p); }

/* The host C library's single-precision log2f / exp2f over arrays: the
 * functions the reference's 3D path calls (include/sz_cp_preserve_utils.hpp:
 * 201-216, src/sz_decompress_cp_preserve_3d.cpp:95-104), exposed so the GPU's
 * reproduction can be checked element by element. */
void cpo_log2f_array(const float* in, size_t n, float* out) {
  for (size_t i = 0; i < n; i++) out[i] = log2f(in[i]);
}

void cpo_exp2f_array(const float* in, size_t n, float* out) {
  for (size_t i = 0; i < n; i++) out[i] = exp2f(in[i]);
}
