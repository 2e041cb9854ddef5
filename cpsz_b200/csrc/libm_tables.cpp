// libm_tables.cpp -- scan, cache and upload of the host log2f / exp2f tables
// (the scheme is described in libm.h).
#include "libm.h"

#include <dlfcn.h>
#include <gnu/libc-version.h>
#include <unistd.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "runtime.h"

namespace cpsz {

namespace {

constexpr int kKeys = 512;
constexpr long double kHardUlps = 1.0L / 262144.0L;  // 2^-18
// GPU double log2 / exp2 errors are below 2^-28 float ulp; the bands carry a
// margin of 2^-26 on top of the largest distance the scan saw.
constexpr double kMargin = 1.0 / 67108864.0;
constexpr double kBitmapBand = 0.01;  // binades misrounding this far get a bitmap
constexpr char kMagic[8] = {'C', 'P', 'S', 'Z', 'L', 'M', '0', '2'};

struct HostFn {
  std::vector<uint32_t> hard_in, hard_out, mis;
  double band[kKeys];
};
struct HostTables {
  HostFn fn[2];  // log2f, exp2f
};

float f_of(uint32_t b) {
  float f;
  memcpy(&f, &b, 4);
  return f;
}
uint32_t b_of(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
}

struct Part {
  std::vector<uint32_t> hard_in, hard_out, mis;
  double band[kKeys];
  bool bad = false;
};

// Classifies input bits `xb` with host result h and long-double result ex.
void classify(Part& p, uint32_t xb, float h, long double ex) {
  const float f = (float)ex;  // correctly rounded (long double -> float)
  if ((long double)f == ex || std::isnan(ex)) {
    if (b_of(h) != b_of(f) && !(std::isnan(h) && std::isnan(f))) {
      p.hard_in.push_back(xb);
      p.hard_out.push_back(b_of(h));
    }
    return;
  }
  const float g = std::nextafter(f, ex > (long double)f ? INFINITY : -INFINITY);
  const long double mid = ((long double)f + (long double)g) / 2;
  const long double ulp = fabsl((long double)g - (long double)f);
  const long double d = (std::isinf(f) || std::isinf(g)) ? 0.0L : fabsl(ex - mid) / ulp;
  if (d < kHardUlps) {
    if (b_of(h) != b_of(f) || std::isinf(f) || std::isinf(g)) {
      p.hard_in.push_back(xb);
      p.hard_out.push_back(b_of(h));
    }
    return;
  }
  if (b_of(h) != b_of(f)) {
    if (b_of(h) != b_of(g)) p.bad = true;
    p.mis.push_back(xb);
    const int key = (int)(xb >> 23);
    if ((double)d > p.band[key]) p.band[key] = (double)d;
  }
}

void scan_range(int which, uint64_t lo, uint64_t hi, Part* p) {
  for (int k = 0; k < kKeys; k++) p->band[k] = -1;
  for (uint64_t b = lo; b < hi; b++) {
    const float x = f_of((uint32_t)b);
    if (which == 0) {
      if (!(x > 0) || std::isinf(x)) continue;
      classify(*p, (uint32_t)b, log2f(x), log2l((long double)x));
    } else {
      if (!(x >= -99.0f && x <= 128.0f)) continue;
      classify(*p, (uint32_t)b, exp2f(x), exp2l((long double)x));
    }
  }
}

int scan(int which, HostFn* out) {
  unsigned nt = std::thread::hardware_concurrency();
  if (const char* e = getenv("CPSZ_B200_TABLE_THREADS")) nt = (unsigned)atoi(e);
  if (nt < 1) nt = 1;
  if (nt > 256) nt = 256;
  // 4096 chunks of 2^20 bit patterns handed out dynamically (the domains
  // cover only parts of the bit range, so static halves would idle)
  constexpr int kChunks = 4096;
  constexpr uint64_t kChunk = (1ull << 32) / kChunks;
  std::vector<Part> parts(kChunks);
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++)
    th.emplace_back([&] {
      for (int c = next++; c < kChunks; c = next++) scan_range(which, c * kChunk, (c + 1) * kChunk, &parts[c]);
    });
  for (auto& t : th) t.join();
  for (int k = 0; k < kKeys; k++) out->band[k] = -1;
  // chunk ranges ascend, so the concatenation stays sorted
  for (auto& p : parts) {
    if (p.bad) return set_error(CPSZ_ERR_UNSUPPORTED, "host %s misrounds beyond the adjacent float",
                                which ? "exp2f" : "log2f");
    out->hard_in.insert(out->hard_in.end(), p.hard_in.begin(), p.hard_in.end());
    out->hard_out.insert(out->hard_out.end(), p.hard_out.begin(), p.hard_out.end());
    out->mis.insert(out->mis.end(), p.mis.begin(), p.mis.end());
    for (int k = 0; k < kKeys; k++)
      if (p.band[k] > out->band[k]) out->band[k] = p.band[k];
  }
  return CPSZ_OK;
}

std::string default_path() {
  if (const char* e = getenv("CPSZ_B200_LIBM_TABLES")) return e;
  Dl_info info;
  if (dladdr((void*)&default_path, &info) && info.dli_fname) {
    std::string s = info.dli_fname;
    size_t slash = s.rfind('/');
    if (slash != std::string::npos) return s.substr(0, slash) + "/libm_f32_tables.bin";
  }
  return "libm_f32_tables.bin";
}

bool load_file(const std::string& path, HostTables* T) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  bool ok = false;
  char magic[8];
  uint32_t vlen = 0;
  std::string ver;
  do {
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kMagic, 8) != 0) break;
    if (fread(&vlen, 4, 1, f) != 1 || vlen > 256) break;
    ver.resize(vlen);
    if (vlen && fread(&ver[0], 1, vlen, f) != vlen) break;
    if (ver != gnu_get_libc_version()) break;
    bool good = true;
    for (int k = 0; k < 2 && good; k++) {
      HostFn& F = T->fn[k];
      uint32_t nh = 0, nm = 0;
      good = fread(&nh, 4, 1, f) == 1 && fread(&nm, 4, 1, f) == 1 && nh < (1u << 26) && nm < (1u << 26);
      if (!good) break;
      F.hard_in.resize(nh);
      F.hard_out.resize(nh);
      F.mis.resize(nm);
      good = fread(F.band, 8, kKeys, f) == (size_t)kKeys && fread(F.hard_in.data(), 4, nh, f) == nh &&
             fread(F.hard_out.data(), 4, nh, f) == nh && fread(F.mis.data(), 4, nm, f) == nm;
    }
    ok = good;
  } while (0);
  fclose(f);
  return ok;
}

void save_file(const std::string& path, const HostTables& T) {
  std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) return;  // read-only location: keep the tables in memory only
  const char* ver = gnu_get_libc_version();
  uint32_t vlen = (uint32_t)strlen(ver);
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(&vlen, 4, 1, f) == 1 && fwrite(ver, 1, vlen, f) == vlen;
  for (int k = 0; k < 2 && ok; k++) {
    const HostFn& F = T.fn[k];
    uint32_t nh = (uint32_t)F.hard_in.size(), nm = (uint32_t)F.mis.size();
    ok = fwrite(&nh, 4, 1, f) == 1 && fwrite(&nm, 4, 1, f) == 1 && fwrite(F.band, 8, kKeys, f) == (size_t)kKeys &&
         fwrite(F.hard_in.data(), 4, nh, f) == nh && fwrite(F.hard_out.data(), 4, nh, f) == nh &&
         fwrite(F.mis.data(), 4, nm, f) == nm;
  }
  ok = (fclose(f) == 0) && ok;
  if (ok) ok = rename(tmp.c_str(), path.c_str()) == 0;
  if (!ok) remove(tmp.c_str());
}

std::mutex g_mu;
HostTables* g_host = nullptr;

int host_tables(const char* path, const HostTables** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_host) {
    std::string p = path ? std::string(path) : default_path();
    HostTables* T = new HostTables();
    if (!load_file(p, T)) {
      *T = HostTables();
      int rc = scan(0, &T->fn[0]);
      if (rc == CPSZ_OK) rc = scan(1, &T->fn[1]);
      if (rc != CPSZ_OK) {
        delete T;
        return rc;
      }
      save_file(p, *T);
    }
    g_host = T;
  }
  *out = g_host;
  return CPSZ_OK;
}

}  // namespace

int libm_tables_prepare(const char* path) {
  const HostTables* T;
  return host_tables(path, &T);
}

int libm_tables_device(cpsz_b200_ctx* ctx, LibmTables* out) {
  if (ctx->libm_mem) {
    *out = *(const LibmTables*)ctx->libm_view;
    return CPSZ_OK;
  }
  const HostTables* T;
  CPSZ_TRY(host_tables(nullptr, &T));
  // layout: per function hard_in | hard_out | hard_off | mis | mis_off | band | bmp_slot | bitmaps
  struct Lay {
    size_t hard_in, hard_out, hard_off, mis, mis_off, band, slot, bmp;
    int nslots;
  } lay[2];
  size_t bytes = 0;
  auto take = [&](size_t b) {
    size_t at = bytes;
    bytes += align_up(b, 256);
    return at;
  };
  std::vector<int> slots[2];
  for (int k = 0; k < 2; k++) {
    const HostFn& F = T->fn[k];
    slots[k].assign(kKeys, -1);
    int ns = 0;
    for (int key = 0; key < kKeys; key++)
      if (F.band[key] > kBitmapBand) slots[k][key] = ns++;
    lay[k].nslots = ns;
    lay[k].hard_in = take(F.hard_in.size() * 4 + 4);
    lay[k].hard_out = take(F.hard_out.size() * 4 + 4);
    lay[k].hard_off = take((kKeys + 1) * 4);
    lay[k].mis = take(F.mis.size() * 4 + 4);
    lay[k].mis_off = take((kKeys + 1) * 4);
    lay[k].band = take(kKeys * 8);
    lay[k].slot = take(kKeys * 4);
    lay[k].bmp = take((size_t)ns * (1u << 18) * 4 + 4);
  }
  std::vector<uint8_t> host(bytes, 0);
  for (int k = 0; k < 2; k++) {
    const HostFn& F = T->fn[k];
    uint8_t* h = host.data();
    memcpy(h + lay[k].hard_in, F.hard_in.data(), F.hard_in.size() * 4);
    memcpy(h + lay[k].hard_out, F.hard_out.data(), F.hard_out.size() * 4);
    memcpy(h + lay[k].mis, F.mis.data(), F.mis.size() * 4);
    uint32_t* hoff = (uint32_t*)(h + lay[k].hard_off);
    uint32_t* moff = (uint32_t*)(h + lay[k].mis_off);
    size_t a = 0, b = 0;
    for (int key = 0; key <= kKeys; key++) {
      while (a < F.hard_in.size() && (int)(F.hard_in[a] >> 23) < key) a++;
      while (b < F.mis.size() && (int)(F.mis[b] >> 23) < key) b++;
      hoff[key] = (uint32_t)a;
      moff[key] = (uint32_t)b;
    }
    double* band = (double*)(h + lay[k].band);
    int* slot = (int*)(h + lay[k].slot);
    uint32_t* bmp = (uint32_t*)(h + lay[k].bmp);
    for (int key = 0; key < kKeys; key++) {
      band[key] = F.band[key] >= 0 ? F.band[key] + kMargin : -1.0;
      slot[key] = slots[k][key];
    }
    for (uint32_t x : F.mis) {
      int s = slots[k][x >> 23];
      if (s < 0) continue;
      uint32_t m = x & 0x7fffffu;
      bmp[(size_t)s * (1u << 18) + (m >> 5)] |= 1u << (m & 31);
    }
  }
  void* d = nullptr;
  CPSZ_CUDA_TRY(cudaMalloc(&d, bytes));
  CPSZ_CUDA_TRY(cudaMemcpy(d, host.data(), bytes, cudaMemcpyHostToDevice));
  LibmTables* v = new LibmTables();
  char* base = (char*)d;
  LibmFn* fns[2] = {&v->log2f, &v->exp2f};
  for (int k = 0; k < 2; k++) {
    LibmFn& F = *fns[k];
    F.hard_in = (const uint32_t*)(base + lay[k].hard_in);
    F.hard_out = (const uint32_t*)(base + lay[k].hard_out);
    F.hard_off = (const uint32_t*)(base + lay[k].hard_off);
    F.mis = (const uint32_t*)(base + lay[k].mis);
    F.mis_off = (const uint32_t*)(base + lay[k].mis_off);
    F.band = (const double*)(base + lay[k].band);
    F.bmp_slot = (const int*)(base + lay[k].slot);
    F.bmp = (const uint32_t*)(base + lay[k].bmp);
  }
  ctx->libm_mem = d;
  ctx->libm_view = v;
  *out = *v;
  return CPSZ_OK;
}

}  // namespace cpsz

extern "C" int cpsz_b200_libm_tables_prepare(const char* path) {
  cpsz::clear_error();
  return cpsz::libm_tables_prepare(path);
}
