// zstd_format_check.cpp -- CPU check of cpsz_b200/csrc/zstd_format.h (test
// infrastructure, built and run by tests/test_zstd_format.py): frames written
// with the header's sequence coder and a plain greedy hash matcher must decode
// with the system libzstd to the original bytes.  The matcher here is only a
// driver for the format code; the GPU kernels find their own matches.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "zstd_format.h"

extern "C" {
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
unsigned ZSTD_isError(size_t code);
const char* ZSTD_getErrorName(size_t code);
unsigned long long ZSTD_getFrameContentSize(const void* src, size_t srcSize);
}

using namespace cpsz::zstd;

static uint32_t rd32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}

// greedy matches inside [begin, end), candidates anywhere in [0, pos) within the window
static void find_sequences(const uint8_t* src, size_t begin, size_t end, std::vector<Seq>& seqs, size_t& tail) {
  static std::vector<uint32_t> table(1 << 14);
  std::fill(table.begin(), table.end(), 0);
  size_t anchor = begin, p = begin;
  while (p + kMinMatch <= end) {
    const uint32_t h = (rd32(src + p) * 2654435761u) >> 18;
    const size_t c = table[h];
    table[h] = (uint32_t)p + 1;
    if (c && rd32(src + c - 1) == rd32(src + p) && p - (c - 1) <= ((size_t)1 << kWindowLog)) {
      size_t q = c - 1, L = kMinMatch;
      while (p + L < end && src[q + L] == src[p + L]) L++;
      seqs.push_back(Seq{(uint32_t)(p - anchor), (uint32_t)L, (uint32_t)(p - q)});
      p += L;
      anchor = p;
    } else {
      p++;
    }
  }
  tail = end - anchor;
}

static size_t encode_frame(const uint8_t* src, size_t n, std::vector<uint8_t>& out, const Tables& T, size_t block,
                           int* kinds) {
  out.resize(kFrameHeader + n + (n / block + 2) * 64 + 64);
  size_t at = write_frame_header(out.data(), n);
  const size_t nb = n ? (n + block - 1) / block : 1;
  std::vector<Seq> seqs;
  std::vector<uint8_t> body(block + 256);
  for (size_t b = 0; b < nb; b++) {
    const size_t s0 = b * block, len = (n == 0) ? 0 : (s0 + block < n ? block : n - s0);
    const bool last = b + 1 == nb;
    bool rle = len > 0;
    for (size_t i = 1; i < len && rle; i++) rle = src[s0 + i] == src[s0];
    if (rle && len > 1) {
      write_block_header(&out[at], last, 1, (uint32_t)len);
      out[at + 3] = src[s0];
      at += 4;
      kinds[1]++;
      continue;
    }
    seqs.clear();
    size_t tail = 0;
    find_sequences(src, s0, s0 + len, seqs, tail);
    // literals: the bytes no match covers, in order
    size_t nlit = tail, pos = s0;
    for (const Seq& q : seqs) nlit += q.lit;
    size_t k = write_raw_literals_header((uint32_t)nlit, body.data());
    for (const Seq& q : seqs) {
      memcpy(&body[k], src + pos, q.lit);
      k += q.lit;
      pos += q.lit + q.ml;
    }
    memcpy(&body[k], src + pos, tail);
    k += tail;
    size_t sq = (k < body.size()) ? write_sequences(T, seqs.data(), (int)seqs.size(), &body[k], body.size() - k) : 0;
    if (sq && k + sq < len) {
      write_block_header(&out[at], last, 2, (uint32_t)(k + sq));
      memcpy(&out[at + 3], body.data(), k + sq);
      at += 3 + k + sq;
      kinds[2]++;
    } else {
      write_block_header(&out[at], last, 0, (uint32_t)len);
      memcpy(&out[at + 3], src + s0, len);
      at += 3 + len;
      kinds[0]++;
    }
  }
  out.resize(at);
  return at;
}

static int check(const char* name, const std::vector<uint8_t>& data, const Tables& T, size_t block) {
  std::vector<uint8_t> frame;
  int kinds[3] = {0, 0, 0};
  encode_frame(data.data(), data.size(), frame, T, block, kinds);
  if (ZSTD_getFrameContentSize(frame.data(), frame.size()) != data.size()) {
    printf("FAIL %s: content size\n", name);
    return 1;
  }
  std::vector<uint8_t> back(data.size() + 1);
  const size_t r = ZSTD_decompress(back.data(), back.size(), frame.data(), frame.size());
  if (ZSTD_isError(r)) {
    printf("FAIL %s: %s\n", name, ZSTD_getErrorName(r));
    return 1;
  }
  if (r != data.size() || memcmp(back.data(), data.data(), r) != 0) {
    printf("FAIL %s: decoded bytes differ\n", name);
    return 1;
  }
  printf("ok %s: %zu -> %zu bytes (raw %d, rle %d, compressed %d blocks)\n", name, data.size(), frame.size(), kinds[0],
         kinds[1], kinds[2]);
  return 0;
}

int main(int argc, char** argv) {
  Tables T;
  build_tables(&T);
  int fails = 0;
  uint64_t s = 12345;
  auto rnd = [&]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (uint32_t)(s >> 33);
  };
  std::vector<uint8_t> d;
  fails += check("empty", d, T, kBlockMax);
  d.assign(1, 7);
  fails += check("one byte", d, T, kBlockMax);
  d.assign(300000, 0);
  fails += check("zeros", d, T, kBlockMax);
  d.resize(500000);
  for (auto& x : d) x = (uint8_t)rnd();
  fails += check("random", d, T, kBlockMax);
  // repeated phrases of varied lengths and distances: long literal runs,
  // short and long matches, every length and offset code range
  d.clear();
  std::vector<uint8_t> phrase(70000);
  for (auto& x : phrase) x = (uint8_t)rnd();
  while (d.size() < 3000000) {
    const uint32_t r = rnd();
    if (r % 5 == 0) {
      for (int i = 0; i < (int)(r % 300); i++) d.push_back((uint8_t)rnd());
    } else {
      const size_t len = 4 + (rnd() % ((r % 7 == 0) ? 66000 : 40)), off = rnd() % 60000;
      for (size_t i = 0; i < len; i++) d.push_back(phrase[(off + i) % phrase.size()]);
    }
  }
  fails += check("phrases", d, T, kBlockMax);
  fails += check("phrases, 16 KB blocks", d, T, 16384);
  // skewed bytes with runs (like a Huffman stream of a peaked distribution)
  d.clear();
  while (d.size() < 1000000) {
    const uint32_t r = rnd();
    const int run = (r & 3) ? (int)(r >> 28) : 0;
    for (int i = 0; i < run; i++) d.push_back(0);
    d.push_back((uint8_t)(rnd() & 0x3f));
  }
  fails += check("skewed", d, T, kBlockMax);
  if (argc > 1) {
    FILE* f = fopen(argv[1], "rb");
    if (f) {
      fseek(f, 0, SEEK_END);
      d.resize(ftell(f));
      fseek(f, 0, SEEK_SET);
      if (fread(d.data(), 1, d.size(), f) != d.size()) d.clear();
      fclose(f);
      fails += check(argv[1], d, T, kBlockMax);
    }
  }
  printf(fails ? "FAILED\n" : "ALL OK\n");
  return fails ? 1 : 0;
}
