// huffman_host.cpp -- tree construction, serialization and decoder tables.
//
// Tree construction reproduces the reference's binary-heap Huffman
// (src/sz_huffman.cpp:103-215): leaves are inserted in symbol order; the
// sift-up stops at a parent with freq <= the new node's; the sift-down of a
// removal takes the right child only when strictly smaller; each merge creates
// new_node(0, 0, qremove(), qremove()), whose arguments the reference's g++
// x86-64 build evaluates right to left, so the node removed first becomes the
// right child.  Codes: left 0 / right 1 (build_code, :152-187).  Serialization:
// pre-order numbering into L/R (u8/u16/u32 for <=256 / <=65536 / more nodes),
// C (u32), t (u8), after a zero endianness byte (pad_tree_*,
// convert_HuffTree_to_bytes_anyStates, :357-499).
#include "huffman_host.h"

#include <cstring>

#include "kernels.h"
#include "runtime.h"

namespace cpsz {

namespace {

struct Node {
  unsigned long long freq;
  int left, right;
  uint32_t c;
  bool leaf;
};

class Heap {
 public:
  Heap(std::vector<Node>& pool, size_t cap) : pool_(pool), q_(cap + 2, -1) {}
  void insert(int n) {
    int i = end_++, j;
    while ((j = i >> 1)) {
      if (pool_[q_[j]].freq <= pool_[n].freq) break;
      q_[i] = q_[j];
      i = j;
    }
    q_[i] = n;
  }
  int remove() {
    int i = 1, l;
    int n = q_[1];
    end_--;
    while ((l = i << 1) < end_) {
      if (l + 1 < end_ && pool_[q_[l + 1]].freq < pool_[q_[l]].freq) l++;
      q_[i] = q_[l];
      i = l;
    }
    q_[i] = q_[end_];
    return n;
  }
  int size() const { return end_ - 1; }
  int top() const { return q_[1]; }

 private:
  std::vector<Node>& pool_;
  std::vector<int> q_;
  int end_ = 1;
};

size_t tree_size_for(size_t nodes) {
  if (nodes <= 256) return 1 + 3 * nodes + 4 * nodes;
  if (nodes <= 65536) return 1 + 4 * nodes + nodes + 4 * nodes;
  return 1 + 12 * nodes + nodes;
}

struct Walker {
  const std::vector<Node>& pool;
  const unsigned long long* hist;
  HuffCodebook* out;
  std::vector<uint32_t> L, R, C;
  std::vector<uint8_t> T;
  uint32_t n_inode = 0;
  bool too_long = false;

  void codes(int n, int depth, unsigned long long bits) {
    const Node& nd = pool[n];
    if (nd.leaf) {
      if (depth > 64) {
        too_long = true;
        return;
      }
      out->code[nd.c] = bits;
      out->len[nd.c] = (uint8_t)depth;
      if (depth > out->max_len) out->max_len = depth;
      out->total_bits += hist[nd.c] * (unsigned long long)depth;
      return;
    }
    if (depth >= 64) {
      too_long = true;
      return;
    }
    codes(nd.left, depth + 1, bits << 1);
    codes(nd.right, depth + 1, (bits << 1) | 1ull);
  }
  void pad(int n, uint32_t i) {
    const Node& nd = pool[n];
    C[i] = nd.c;
    T[i] = nd.leaf ? 1 : 0;
    if (nd.left >= 0) {
      L[i] = ++n_inode;
      pad(nd.left, n_inode);
    }
    if (nd.right >= 0) {
      R[i] = ++n_inode;
      pad(nd.right, n_inode);
    }
  }
};

template <class T>
void put(std::vector<uint8_t>& v, size_t& at, T x) {
  memcpy(v.data() + at, &x, sizeof(T));
  at += sizeof(T);
}

}  // namespace

bool huff_build(const unsigned long long* hist, size_t bins, size_t state_num, HuffCodebook* out) {
  size_t distinct = 0;
  for (size_t s = 0; s < bins; s++)
    if (hist[s]) distinct++;
  if (distinct == 0) {
    set_error(CPSZ_ERR_INVALID, "Huffman: empty histogram");
    return false;
  }
  std::vector<Node> pool;
  pool.reserve(2 * distinct);
  Heap heap(pool, 2 * distinct);
  for (size_t s = 0; s < bins; s++) {
    if (!hist[s]) continue;
    pool.push_back(Node{hist[s], -1, -1, (uint32_t)s, true});
    heap.insert((int)pool.size() - 1);
  }
  while (heap.size() > 1) {
    int first = heap.remove();
    int second = heap.remove();
    pool.push_back(Node{pool[second].freq + pool[first].freq, second, first, 0u, false});
    heap.insert((int)pool.size() - 1);
  }
  const int root = heap.top();
  out->code.assign(bins, 0);
  out->len.assign(bins, 0);
  out->distinct = distinct;
  out->max_len = 0;
  out->total_bits = 0;
  Walker w{pool, hist, out, {}, {}, {}, {}};
  w.codes(root, 0, 0);
  if (w.too_long) {
    set_error(CPSZ_ERR_UNSUPPORTED, "Huffman code longer than 64 bits");
    return false;
  }
  size_t node_count = 0;
  for (size_t s = 0; s < state_num && s < bins; s++)
    if (hist[s]) node_count++;
  node_count = node_count * 2 - 1;
  const size_t nn = pool.size();
  if (node_count != nn) {
    set_error(CPSZ_ERR_UNSUPPORTED, "Huffman: symbols beyond state_num");
    return false;
  }
  w.L.assign(nn, 0);
  w.R.assign(nn, 0);
  w.C.assign(nn, 0);
  w.T.assign(nn, 0);
  w.pad(root, 0);
  const size_t tsz = tree_size_for(node_count);
  out->tree_bytes.assign(8 + 4 + tsz, 0);
  size_t at = 0;
  put<unsigned long long>(out->tree_bytes, at, (unsigned long long)node_count);
  put<uint32_t>(out->tree_bytes, at, (uint32_t)tsz);
  put<uint8_t>(out->tree_bytes, at, 0);  // sysEndianType
  const int wdt = node_count <= 256 ? 1 : (node_count <= 65536 ? 2 : 4);
  for (int side = 0; side < 2; side++) {
    const std::vector<uint32_t>& A = side ? w.R : w.L;
    for (size_t i = 0; i < node_count; i++) {
      if (wdt == 1) put<uint8_t>(out->tree_bytes, at, (uint8_t)A[i]);
      else if (wdt == 2) put<uint16_t>(out->tree_bytes, at, (uint16_t)A[i]);
      else put<uint32_t>(out->tree_bytes, at, A[i]);
    }
  }
  for (size_t i = 0; i < node_count; i++) put<uint32_t>(out->tree_bytes, at, w.C[i]);
  for (size_t i = 0; i < node_count; i++) put<uint8_t>(out->tree_bytes, at, w.T[i]);
  return true;
}

bool huff_parse(const unsigned char* p, size_t avail, size_t max_symbol, HuffDecoderHost* out) {
  if (avail < 12) {
    set_error(CPSZ_ERR_FORMAT, "Huffman section truncated (%zu bytes)", avail);
    return false;
  }
  unsigned long long node_count;
  uint32_t tree_size;
  memcpy(&node_count, p, 8);
  memcpy(&tree_size, p + 8, 4);
  if (node_count == 0 || node_count > (1ull << 28) || tree_size != tree_size_for(node_count) ||
      avail < 12 + (size_t)tree_size + 8) {
    set_error(CPSZ_ERR_FORMAT, "Huffman tree header invalid (nodes %llu, size %u, avail %zu)", node_count, tree_size,
              avail);
    return false;
  }
  const unsigned char* tb = p + 12 + 1;
  const size_t nc = (size_t)node_count;
  const int wdt = nc <= 256 ? 1 : (nc <= 65536 ? 2 : 4);
  auto rd = [&](const unsigned char* base, size_t i) -> uint32_t {
    uint32_t v = 0;
    memcpy(&v, base + i * wdt, wdt);
    return v;
  };
  out->node_count = (int)nc;
  out->child.assign(2 * nc, 0);
  out->sym.assign(nc, 0);
  out->leaf.assign(nc, 0);
  for (size_t i = 0; i < nc; i++) {
    out->child[2 * i] = rd(tb, i);
    out->child[2 * i + 1] = rd(tb + nc * wdt, i);
    memcpy(&out->sym[i], tb + 2 * nc * wdt + 4 * i, 4);
    out->leaf[i] = tb[2 * nc * wdt + 4 * nc + i];
  }
  // The reference rebuilds the root with t = C[0]/t[0] only for <= 256 nodes
  // (reconstruct_HuffTree_from_bytes_anyStates, src/sz_huffman.cpp:570-596);
  // larger trees get an inner root.
  out->root_is_leaf = (nc <= 256) && out->leaf[0];
  out->root_sym = out->sym[0];
  if (!out->root_is_leaf) out->leaf[0] = 0;
  // validate: inner nodes have two children with larger indices; leaves carry
  // an in-range symbol.
  for (size_t i = 0; i < nc; i++) {
    if (out->leaf[i] || (i == 0 && out->root_is_leaf)) {
      if (out->sym[i] > max_symbol) {
        set_error(CPSZ_ERR_FORMAT, "Huffman leaf symbol %u out of range", out->sym[i]);
        return false;
      }
      continue;
    }
    uint32_t l = out->child[2 * i], r = out->child[2 * i + 1];
    if (l <= i || r <= i || l >= nc || r >= nc) {
      set_error(CPSZ_ERR_FORMAT, "Huffman tree node %zu has invalid children", i);
      return false;
    }
  }
  // first-level table
  out->lut.assign(1u << HUFF_LUT_BITS, 0);
  if (!out->root_is_leaf) {
    for (uint32_t pat = 0; pat < (1u << HUFF_LUT_BITS); pat++) {
      uint32_t node = 0;
      uint32_t e = 0;
      bool done = false;
      for (int k = 0; k < HUFF_LUT_BITS; k++) {
        uint32_t bit = (pat >> (HUFF_LUT_BITS - 1 - k)) & 1u;
        node = out->child[2 * node + bit];
        if (out->leaf[node]) {
          e = (out->sym[node] << 8) | (uint32_t)(k + 1);
          done = true;
          break;
        }
      }
      if (!done) e = 0x80u | (node << 8);
      out->lut[pat] = e;
    }
  }
  out->tree_size = tree_size;
  memcpy(&out->nbytes, p + 12 + tree_size, 8);
  out->bits_offset = 12 + (size_t)tree_size + 8;
  if (out->nbytes > avail - out->bits_offset) {
    set_error(CPSZ_ERR_FORMAT, "Huffman bit stream truncated (%zu > %zu)", out->nbytes, avail - out->bits_offset);
    return false;
  }
  out->section_bytes = out->bits_offset + out->nbytes;
  return true;
}

}  // namespace cpsz
