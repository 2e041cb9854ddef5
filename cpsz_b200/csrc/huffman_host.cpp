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

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "kernels.h"
#include "runtime.h"

namespace cpsz {

namespace {

// The heap stores freq << 20 | node in one word (the comparisons look at the
// frequency only): the reference's exact insertion / removal semantics with
// one 8-byte load per visited slot.
class Heap {
 public:
  // `storage` keeps its capacity across calls (fresh pages cost a fault each);
  // slot 0 of the heap sits on a 64-byte boundary, so the 8 great-grandchildren
  // 8i..8i+7 of slot i share one cache line.
  Heap(std::vector<unsigned long long>& storage, size_t cap) {
    if (storage.size() < cap + 2 + 8) storage.resize(cap + 2 + 8);
    q_ = (unsigned long long*)(((uintptr_t)storage.data() + 63) & ~(uintptr_t)63);
  }
  void insert(unsigned long long f, int n) {
    const unsigned long long e = (f << kShift) | (unsigned long long)n;
    int i = end_++, j;
    while ((j = i >> 1)) {
      if ((q_[j] >> kShift) <= f) break;
      q_[i] = q_[j];
      i = j;
    }
    q_[i] = e;
  }
  // Removes the top entry and returns its key (freq << kShift | node).  The
  // hole at the top moves down to a leaf, each step taking the right child
  // only when its frequency is strictly smaller; the last entry then fills it.
  unsigned long long remove_key() {
    unsigned long long* q = q_;
    const unsigned long long n = q[1];
    end_--;
    const size_t end = (size_t)end_;
    size_t i = 1;
    // Three levels per step while all 8 great-grandchildren are in the heap:
    // the children and grandchildren load together, the choices are
    // register selects (they are data-dependent and would mispredict), and
    // one load of the chosen grandchild's pair completes the step.
    while (8 * i + 7 < end) {
      const unsigned long long* c = q + 2 * i;
      const unsigned long long* g = q + 4 * i;
      const unsigned long long c0 = c[0], c1 = c[1], g0 = g[0], g1 = g[1], g2 = g[2], g3 = g[3];
      const size_t s1 = (c1 >> kShift) < (c0 >> kShift);
      const unsigned long long cv = s1 ? c1 : c0, ga = s1 ? g2 : g0, gb = s1 ? g3 : g1;
      const size_t s2 = (gb >> kShift) < (ga >> kShift);
      const unsigned long long gv = s2 ? gb : ga;
      const size_t k = 2 * s1 + s2;  // the chosen grandchild is 4i + k
      const unsigned long long ha = q[8 * i + 2 * k], hb = q[8 * i + 2 * k + 1];
      const size_t s3 = (hb >> kShift) < (ha >> kShift);
      q[i] = cv;
      q[2 * i + s1] = gv;
      q[4 * i + k] = s3 ? hb : ha;
      i = 8 * i + 2 * k + s3;
    }
    size_t l;
    while ((l = 2 * i) < end) {
      l += (size_t)((l + 1 < end) & ((q[l + 1] >> kShift) < (q[l] >> kShift)));
      q[i] = q[l];
      i = l;
    }
    q[i] = q[end];
    return n;
  }
  int size() const { return end_ - 1; }
  int top() const { return (int)(q_[1] & kMask); }
  static constexpr int kShift = 20;
  static constexpr unsigned long long kMask = (1ull << kShift) - 1;

 private:
  unsigned long long* q_;
  int end_ = 1;
};

// Per node of a built tree: its code (right-aligned), pre-order number and depth.
struct NodeInfo {
  unsigned long long code;
  uint32_t pre, depth;
};

// Per-thread scratch reused by every build on the thread.
struct Scratch {
  std::vector<uint32_t> leaf_sym, size;
  std::vector<int> kids;
  std::vector<unsigned long long> heap, leaf_freq;
  std::vector<NodeInfo> info;
};
Scratch& scratch() {
  static thread_local Scratch s;
  return s;
}

size_t tree_size_for(size_t nodes) {
  if (nodes <= 256) return 1 + 3 * nodes + 4 * nodes;
  if (nodes <= 65536) return 1 + 4 * nodes + nodes + 4 * nodes;
  return 1 + 12 * nodes + nodes;
}

}  // namespace

bool huff_build(const unsigned long long* hist, size_t bins, size_t state_num, HuffCodebook* out) {
  // Leaves are nodes 0..distinct-1 in symbol order (the reference inserts them
  // that way); merged nodes follow.  Node data lives in two small arrays so
  // the merge loop and the walk stay cache-resident.
  Scratch& sc = scratch();
  std::vector<uint32_t>& leaf_sym = sc.leaf_sym;
  std::vector<unsigned long long>& leaf_freq = sc.leaf_freq;
  leaf_sym.clear();
  leaf_freq.clear();
  for (size_t s = 0; s < bins; s++)
    if (hist[s]) {
      leaf_sym.push_back((uint32_t)s);
      leaf_freq.push_back(hist[s]);
    }
  const size_t distinct = leaf_sym.size();
  if (distinct == 0) {
    set_error(CPSZ_ERR_INVALID, "Huffman: empty histogram");
    return false;
  }
  std::vector<int>& kids = sc.kids;  // (left, right) of merged node distinct + m
  if (kids.size() < 2 * distinct) kids.resize(2 * distinct);
  Heap heap(sc.heap, 2 * distinct);
  for (size_t d = 0; d < distinct; d++) heap.insert(leaf_freq[d], (int)d);
  int next_node = (int)distinct;
  while (heap.size() > 1) {
    // new_node(0, 0, qremove(), qremove()): the first removal becomes the
    // right child
    const unsigned long long first = heap.remove_key();
    const unsigned long long second = heap.remove_key();
    const int m = next_node - (int)distinct;
    kids[2 * m] = (int)(second & Heap::kMask);
    kids[2 * m + 1] = (int)(first & Heap::kMask);
    heap.insert((second >> Heap::kShift) + (first >> Heap::kShift), next_node++);
  }
  const int root = heap.top();
  out->distinct = distinct;
  out->max_len = 0;
  out->total_bits = 0;
  // leaves are in symbol order: those below state_num are a prefix
  const size_t below = (size_t)(std::lower_bound(leaf_sym.begin(), leaf_sym.end(), (uint32_t)std::min(state_num, bins)) -
                                leaf_sym.begin());
  const size_t node_count = below * 2 - 1;
  const size_t nn = (size_t)next_node;
  if (node_count != nn) {
    set_error(CPSZ_ERR_UNSUPPORTED, "Huffman: symbols beyond state_num");
    return false;
  }
  // Codes (left 0 / right 1, build_code) and the serialization's node
  // numbering (pad_tree_*: a node's number is its pre-order position; L/R
  // hold the children's numbers), without walking the tree: a merged node is
  // created after both its children, so subtree sizes follow in creation
  // order, and pre-order numbers, depths and codes in reverse creation order
  // (pre(left) = pre(node) + 1, pre(right) = pre(node) + 1 + size(left)).
  // L, R, C and t go straight into the serialized tree (zeros where the
  // reference leaves them 0: leaves' L/R, merged nodes' C/t).
  std::vector<uint32_t>& size = sc.size;
  std::vector<NodeInfo>& info = sc.info;
  size.resize(nn);
  info.resize(nn);
  const size_t nm = nn - distinct;
  for (size_t d = 0; d < distinct; d++) size[d] = 1;
  for (size_t m = 0; m < nm; m++) size[distinct + m] = size[kids[2 * m]] + size[kids[2 * m + 1]] + 1;
  const size_t tsz = tree_size_for(node_count);
  out->tree_bytes.assign(8 + 4 + tsz, 0);
  uint8_t* tb = out->tree_bytes.data();
  {
    const unsigned long long nc = node_count;
    const uint32_t ts = (uint32_t)tsz;
    memcpy(tb, &nc, 8);
    memcpy(tb + 8, &ts, 4);  // then sysEndianType 0
  }
  const int wdt = node_count <= 256 ? 1 : (node_count <= 65536 ? 2 : 4);
  uint8_t* Lb = tb + 13;
  uint8_t* Rb = Lb + (size_t)wdt * node_count;
  uint8_t* Cb = Rb + (size_t)wdt * node_count;
  uint8_t* Tb = Cb + 4 * node_count;
  info[root] = NodeInfo{0ull, 0u, 0u};
  int deepest = 0;
  auto walk = [&](auto tag) {
    using Wd = decltype(tag);
    Wd* Lw = reinterpret_cast<Wd*>(Lb);
    Wd* Rw = reinterpret_cast<Wd*>(Rb);
    for (size_t m = nm; m-- > 0;) {
      const NodeInfo nd = info[distinct + m];
      const int l = kids[2 * m], r = kids[2 * m + 1];
      const uint32_t dc = nd.depth + 1, pl = nd.pre + 1, pr = nd.pre + 1 + size[l];
      info[l] = NodeInfo{nd.code << 1, pl, dc};
      info[r] = NodeInfo{(nd.code << 1) | 1ull, pr, dc};
      Wd vl = (Wd)pl, vr = (Wd)pr;
      memcpy(Lw + nd.pre, &vl, sizeof(Wd));
      memcpy(Rw + nd.pre, &vr, sizeof(Wd));
      deepest = (int)dc > deepest ? (int)dc : deepest;
    }
  };
  if (wdt == 1) walk(uint8_t{});
  else if (wdt == 2) walk(uint16_t{});
  else walk(uint32_t{});
  if (deepest > 64) {
    set_error(CPSZ_ERR_UNSUPPORTED, "Huffman code longer than 64 bits");
    return false;
  }
  out->max_len = deepest;
  out->entries.resize(distinct);
  for (size_t d = 0; d < distinct; d++) {
    const NodeInfo nd = info[d];
    memcpy(Cb + 4 * (size_t)nd.pre, &leaf_sym[d], 4);
    Tb[nd.pre] = 1;
    out->entries[d] = HuffEntry{nd.code, leaf_sym[d], nd.depth};
    out->total_bits += leaf_freq[d] * (unsigned long long)nd.depth;
  }
  return true;
}

int huff_upload(cpsz_b200_ctx* ctx, const HuffCodebook& cb, HuffEntry* h_stage, HuffEntry* d_ent,
                unsigned long long* code, uint8_t* len) {
  const size_t n = cb.entries.size();
  const HuffEntry* src = cb.entries.data();
  if (h_stage) {
    memcpy(h_stage, src, n * sizeof(HuffEntry));
    src = h_stage;
  }
  CPSZ_CUDA_TRY(cudaMemcpyAsync(d_ent, src, n * sizeof(HuffEntry), cudaMemcpyHostToDevice, ctx->stream));
  return launch_codebook_scatter(ctx, d_ent, n, code, len);
}

void huff_tables(const HuffCodebook& cb, size_t bins, unsigned long long* code, uint8_t* len) {
  if (code) memset(code, 0, bins * sizeof(unsigned long long));
  if (len) memset(len, 0, bins);
  for (const HuffEntry& e : cb.entries) {
    if (e.sym >= bins) continue;
    if (code) code[e.sym] = e.code;
    if (len) len[e.sym] = (uint8_t)e.len;
  }
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
