// huffman_host.h -- host side of the SZ-1.x Huffman codec: tree construction
// from a device histogram with the reference's exact tie-breaking, the tree's
// byte serialization, and decoder tables rebuilt from serialized trees.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "kernels.h"

namespace cpsz {

struct HuffCodebook {
  std::vector<HuffEntry> entries;        // the symbols that occur, ascending, with their codes
  std::vector<uint8_t> tree_bytes;       // node_count(8) tree_size(4) tree(tree_size)
  unsigned long long total_bits = 0;     // sum over symbols of freq * len
  int max_len = 0;
  size_t distinct = 0;
};

// Builds the codebook for a histogram over `bins` symbols (state_num =
// bins/2 in the reference's terms; node_count counts the symbols < state_num).
// Returns false (with an error set) if the histogram is empty or a code would
// exceed 64 bits.
bool huff_build(const unsigned long long* hist, size_t bins, size_t state_num, HuffCodebook* out);

// Device tables of the codebook: its entries go up to d_ent (room for
// cb.entries.size()) on ctx->stream and are scattered into code / len.  With
// h_stage (page-locked, room for the entries) the entries are copied there
// first, so the upload is asynchronous; without, they go up from the
// codebook's own (pageable) memory.
int huff_upload(cpsz_b200_ctx* ctx, const HuffCodebook& cb, HuffEntry* h_stage, HuffEntry* d_ent,
                unsigned long long* code, uint8_t* len);

// Full per-symbol tables over `bins` symbols (code right-aligned; len 0 = absent).
void huff_tables(const HuffCodebook& cb, size_t bins, unsigned long long* code, uint8_t* len);

// Section size: 8 + 4 + tree_size + 8 + ceil(total_bits/8).
inline size_t huff_section_bytes(const HuffCodebook& cb) { return cb.tree_bytes.size() + 8 + (cb.total_bits + 7) / 8; }

struct HuffDecoderHost {
  std::vector<uint32_t> lut;    // 1 << 12 entries
  std::vector<uint32_t> child;  // 2 per node
  std::vector<uint32_t> sym;
  std::vector<uint8_t> leaf;
  int node_count = 0;
  bool root_is_leaf = false;
  uint32_t root_sym = 0;
  size_t tree_size = 0;
  size_t nbytes = 0;           // bit-stream bytes
  size_t bits_offset = 0;      // offset of the bit stream from the section start
  size_t section_bytes = 0;    // whole section
};

// Parses a Huffman section (src/sz_decompression_utils.cpp:92-108 layout) of
// at most `avail` bytes.  Validates node indices (pre-order: children have
// larger indices than their parent) so decoding always terminates.
bool huff_parse(const unsigned char* p, size_t avail, size_t max_symbol, HuffDecoderHost* out);

}  // namespace cpsz
