/* cpsz_oracle_huffman.c -- restatement of the SZ-1.x Huffman codec used by the
 * reference (src/sz_huffman.cpp, src/sz_compression_utils.cpp:54-82,
 * src/sz_decompression_utils.cpp:92-108).  Test infrastructure only.
 *
 * Tree construction follows the reference's binary heap exactly:
 *   - leaves are inserted in increasing symbol order (init, sz_huffman.cpp:195-215),
 *   - qinsert sifts up while parent.freq > n.freq (stops on <=, :119-129),
 *   - qremove takes the root and sifts the last element down choosing the right
 *     child only if strictly smaller (:131-144),
 *   - each merge is new_node(0, 0, qremove(), qremove()).  The order in which the
 *     two qremove() calls run is unspecified C++; the reference's g++ -O2 x86-64
 *     build evaluates the arguments right to left, so the FIRST removed node
 *     becomes the RIGHT child.  tests/test_oracle_vs_ref.py pins this against
 *     the compiled reference.
 * Codes: left = 0, right = 1, MSB-first (build_code, :152-187); the bit stream is
 * the MSB-first concatenation of the codes, zero padded to a byte (encode, :217-320).
 * Tree bytes: endian byte 0, then L, R (u8 / u16 / u32 by node count <=256 /
 * <=65536 / more), C (u32), t (u8) in pre-order numbering (pad_tree_*, :357-499).
 */
#include <stdlib.h>
#include <string.h>

#include "cpsz_oracle.h"

typedef struct {
  size_t freq;
  int left, right; /* node indices, -1 = none */
  unsigned int c;
  unsigned char t;
} HNode;

typedef struct {
  HNode* pool;
  int n_nodes;
  int* heap; /* 1-based */
  int qend;
} HTree;

static void qinsert(HTree* h, int n) {
  int j, i = h->qend++;
  while ((j = (i >> 1))) {
    if (h->pool[h->heap[j]].freq <= h->pool[n].freq) break;
    h->heap[i] = h->heap[j];
    i = j;
  }
  h->heap[i] = n;
}

static int qremove(HTree* h) {
  int i = 1, l;
  int n = h->heap[i];
  if (h->qend < 2) return -1;
  h->qend--;
  while ((l = (i << 1)) < h->qend) {
    if (l + 1 < h->qend && h->pool[h->heap[l + 1]].freq < h->pool[h->heap[l]].freq) l++;
    h->heap[i] = h->heap[l];
    i = l;
  }
  h->heap[i] = h->heap[h->qend];
  return n;
}

/* Builds the reference's tree from a histogram over `bins` symbols.
 * Returns the root index (or -1 for an empty histogram). */
static int build_tree(HTree* h, const size_t* freq, size_t bins) {
  h->pool = (HNode*)calloc(2 * bins + 2, sizeof(HNode));
  h->heap = (int*)calloc(2 * bins + 2, sizeof(int));
  h->n_nodes = 0;
  h->qend = 1;
  for (size_t i = 0; i < bins; i++) {
    if (freq[i]) {
      int n = h->n_nodes++;
      h->pool[n].freq = freq[i];
      h->pool[n].c = (unsigned int)i;
      h->pool[n].t = 1;
      h->pool[n].left = h->pool[n].right = -1;
      qinsert(h, n);
    }
  }
  if (h->qend == 1) return -1;
  while (h->qend > 2) {
    int first = qremove(h);  /* evaluated first (rightmost argument) */
    int second = qremove(h);
    int n = h->n_nodes++;
    h->pool[n].left = second;
    h->pool[n].right = first;
    h->pool[n].freq = h->pool[second].freq + h->pool[first].freq;
    h->pool[n].t = 0;
    h->pool[n].c = 0;
    qinsert(h, n);
  }
  return h->heap[1];
}

static void free_tree(HTree* h) {
  free(h->pool);
  free(h->heap);
}

typedef struct {
  unsigned long long* code; /* left-aligned in 64 bits */
  unsigned char* len;
} Codebook;

static void build_codes(const HTree* h, int n, int len, unsigned long long bits, Codebook* cb) {
  const HNode* nd = &h->pool[n];
  if (nd->t) {
    cb->code[nd->c] = len ? (bits << (64 - len)) : 0;
    cb->len[nd->c] = (unsigned char)len;
    return;
  }
  build_codes(h, nd->left, len + 1, bits << 1, cb);
  build_codes(h, nd->right, len + 1, (bits << 1) | 1, cb);
}

static int tree_depth(const HTree* h, int n) {
  const HNode* nd = &h->pool[n];
  if (nd->t) return 0;
  int a = tree_depth(h, nd->left), b = tree_depth(h, nd->right);
  return 1 + (a > b ? a : b);
}

/* pre-order numbering of pad_tree_* */
static void pad_tree(const HTree* h, int n, unsigned int i, unsigned int* n_inode, unsigned int* L, unsigned int* R,
                     unsigned int* C, unsigned char* t) {
  const HNode* nd = &h->pool[n];
  C[i] = nd->c;
  t[i] = nd->t;
  if (nd->left >= 0) {
    (*n_inode)++;
    L[i] = *n_inode;
    pad_tree(h, nd->left, *n_inode, n_inode, L, R, C, t);
  }
  if (nd->right >= 0) {
    (*n_inode)++;
    R[i] = *n_inode;
    pad_tree(h, nd->right, *n_inode, n_inode, L, R, C, t);
  }
}

static size_t tree_bytes_size(size_t node_count) {
  if (node_count <= 256) return 1 + 3 * node_count + 4 * node_count;
  if (node_count <= 65536) return 1 + 2 * 2 * node_count + node_count + 4 * node_count;
  return 1 + 3 * 4 * node_count + node_count;
}

size_t cpo_huffman_encode_bound(size_t state_num, size_t n) {
  size_t nodes = 2 * (2 * state_num) + 1;
  return 8 + 4 + tree_bytes_size(nodes) + 8 + n * 8 + 16;
}

/* 0, or -1 when a symbol lies outside [0, bins) (the reference indexes its
 * histogram out of range there: NaN bounds give such ids). */
static int histogram(const int* sym, size_t n, size_t bins, size_t* freq) {
  memset(freq, 0, bins * sizeof(size_t));
  for (size_t i = 0; i < n; i++) {
    if (sym[i] < 0 || (size_t)sym[i] >= bins) return -1;
    freq[sym[i]]++;
  }
  return 0;
}

size_t cpo_huffman_code_lengths(size_t state_num, const int* sym, size_t n, unsigned char* len) {
  size_t bins = 2 * state_num;
  size_t* freq = (size_t*)malloc(bins * sizeof(size_t));
  memset(len, 0, bins);
  if (histogram(sym, n, bins, freq) != 0) {
    free(freq);
    return 0;
  }
  HTree h;
  int root = build_tree(&h, freq, bins);
  size_t distinct = 0;
  for (size_t i = 0; i < bins; i++) distinct += freq[i] != 0;
  if (root >= 0 && tree_depth(&h, root) <= 64) {
    Codebook cb;
    cb.code = (unsigned long long*)calloc(bins, sizeof(unsigned long long));
    cb.len = len;
    build_codes(&h, root, 0, 0, &cb);
    free(cb.code);
  }
  free_tree(&h);
  free(freq);
  return distinct;
}

static void put(unsigned char** p, const void* v, size_t n) {
  memcpy(*p, v, n);
  *p += n;
}

size_t cpo_huffman_encode(size_t state_num, const int* sym, size_t n, unsigned char* out) {
  size_t bins = 2 * state_num; /* allNodes */
  size_t* freq = (size_t*)malloc(bins * sizeof(size_t));
  if (histogram(sym, n, bins, freq) != 0) { /* symbols out of range: unsupported */
    free(freq);
    return 0;
  }
  HTree h;
  int root = build_tree(&h, freq, bins);
  if (root < 0 || tree_depth(&h, root) > 64) { /* empty input / >64-bit codes: unsupported */
    free_tree(&h);
    free(freq);
    return 0;
  }
  Codebook cb;
  cb.code = (unsigned long long*)calloc(bins, sizeof(unsigned long long));
  cb.len = (unsigned char*)calloc(bins, 1);
  build_codes(&h, root, 0, 0, &cb);
  size_t node_count = 0;
  for (size_t i = 0; i < state_num; i++)
    if (freq[i]) node_count++;
  if (node_count == 0) { /* every symbol at or above state_num: unsupported */
    free(cb.code);
    free(cb.len);
    free_tree(&h);
    free(freq);
    return 0;
  }
  node_count = node_count * 2 - 1;
  /* tree serialization */
  unsigned int* L = (unsigned int*)calloc(node_count, sizeof(unsigned int));
  unsigned int* R = (unsigned int*)calloc(node_count, sizeof(unsigned int));
  unsigned int* C = (unsigned int*)calloc(node_count, sizeof(unsigned int));
  unsigned char* t = (unsigned char*)calloc(node_count, 1);
  unsigned int n_inode = 0;
  pad_tree(&h, root, 0, &n_inode, L, R, C, t);
  unsigned int tree_size = (unsigned int)tree_bytes_size(node_count);
  unsigned char* p = out;
  put(&p, &node_count, sizeof(size_t));
  put(&p, &tree_size, sizeof(unsigned int));
  *p++ = 0; /* sysEndianType (static 0 in sz_huffman.cpp:13) */
  for (size_t i = 0; i < node_count; i++) {
    if (node_count <= 256) { unsigned char v = (unsigned char)L[i]; put(&p, &v, 1); }
    else if (node_count <= 65536) { unsigned short v = (unsigned short)L[i]; put(&p, &v, 2); }
    else put(&p, &L[i], 4);
  }
  for (size_t i = 0; i < node_count; i++) {
    if (node_count <= 256) { unsigned char v = (unsigned char)R[i]; put(&p, &v, 1); }
    else if (node_count <= 65536) { unsigned short v = (unsigned short)R[i]; put(&p, &v, 2); }
    else put(&p, &R[i], 4);
  }
  put(&p, C, node_count * 4);
  put(&p, t, node_count);
  /* bit stream */
  unsigned char* size_pos = p;
  p += sizeof(size_t);
  unsigned long long acc = 0;
  int nacc = 0; /* bits pending in acc (MSB-aligned) */
  unsigned char* q = p;
  for (size_t i = 0; i < n; i++) {
    int s = sym[i];
    int l = cb.len[s];
    unsigned long long c = cb.code[s];
    while (l > 0) {
      int take = (64 - nacc) < l ? (64 - nacc) : l;
      unsigned long long part = c >> (64 - take);
      acc |= (take == 64) ? part : (part << (64 - nacc - take));
      nacc += take;
      c = (take == 64) ? 0 : (c << take);
      l -= take;
      while (nacc >= 8) {
        *q++ = (unsigned char)(acc >> 56);
        acc <<= 8;
        nacc -= 8;
      }
    }
  }
  if (nacc > 0) *q++ = (unsigned char)(acc >> 56);
  size_t nbytes = (size_t)(q - p);
  memcpy(size_pos, &nbytes, sizeof(size_t));
  p = q;
  free(L); free(R); free(C); free(t);
  free(cb.code); free(cb.len);
  free_tree(&h);
  free(freq);
  return (size_t)(p - out);
}

/* Huffman_decode_tree_and_data + reconstruct_HuffTree_from_bytes_anyStates +
 * decode (sz_huffman.cpp:322-355, :570-667).  The decoder walks the serialized
 * L/R arrays directly; node 0 is the root.  Returns bytes consumed, 0 on error. */
size_t cpo_huffman_decode(size_t state_num, size_t n, const unsigned char* in, size_t in_size, int* sym) {
  (void)state_num;
  if (in_size < 12) return 0;
  const unsigned char* p = in;
  size_t node_count;
  unsigned int tree_size;
  memcpy(&node_count, p, 8); p += 8;
  memcpy(&tree_size, p, 4); p += 4;
  if (node_count == 0 || node_count > (1u << 30) || tree_size != tree_bytes_size(node_count) ||
      (size_t)(in + in_size - p) < (size_t)tree_size + 8)
    return 0;
  const unsigned char* tb = p + 1;
  unsigned int* L = (unsigned int*)malloc(node_count * 4);
  unsigned int* R = (unsigned int*)malloc(node_count * 4);
  unsigned int* C = (unsigned int*)malloc(node_count * 4);
  unsigned char* t = (unsigned char*)malloc(node_count);
  int w = node_count <= 256 ? 1 : (node_count <= 65536 ? 2 : 4);
  for (size_t i = 0; i < node_count; i++) {
    L[i] = R[i] = 0;
    memcpy(&L[i], tb + i * w, w);
    memcpy(&R[i], tb + node_count * w + i * w, w);
  }
  memcpy(C, tb + 2 * node_count * w, node_count * 4);
  memcpy(t, tb + 2 * node_count * w + node_count * 4, node_count);
  p += tree_size;
  size_t nbytes;
  memcpy(&nbytes, p, 8); p += 8;
  size_t rc = 0;
  if ((size_t)(in + in_size - p) < nbytes) goto done;
  /* for node_count > 256 the reference rebuilds the root with t = 0 (new_node2(0,0)) */
  int root_leaf = (node_count <= 256) ? t[0] : 0;
  if (root_leaf) {
    for (size_t k = 0; k < n; k++) sym[k] = (int)C[0];
  } else {
    size_t bit = 0, count = 0, nbits = nbytes * 8;
    unsigned int cur = 0;
    while (count < n) {
      if (bit >= nbits) goto done;
      int b = (p[bit >> 3] >> (7 - (bit & 7))) & 1;
      bit++;
      cur = b ? R[cur] : L[cur];
      if (cur == 0 || cur >= node_count) goto done;
      if (t[cur]) {
        sym[count++] = (int)C[cur];
        cur = 0;
      }
    }
  }
  rc = (size_t)(p - in) + nbytes;
done:
  free(L); free(R); free(C); free(t);
  return rc;
}
