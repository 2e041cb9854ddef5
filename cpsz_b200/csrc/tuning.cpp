// tuning.cpp -- the launch-shape table (tuning.h): storage, lookup, the JSON
// reader for the sweep's output and the C ABI around them.
#include "tuning.h"

#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "runtime.h"

namespace cpsz {

namespace {

// name, default, valid range
const TuneInfo kInfo[TUNE_COUNT] = {
    {"eb2d.tile", 0, 0, 5},
    {"wave2d.ctas_per_sm", 0, 0, 16},
    {"eb3d.fill", 4, 1, 32},
    {"eb3d.min_chunk", 8, 1, 256},
    {"h2d.chunks", 8, 1, 32},
    {"wave2d.overlap", 1, 0, 1},
    {"eb2d.skew", 1, 0, 64},
};

struct Entry {
  size_t min_points;
  int value;
};

std::shared_mutex g_mu;
std::vector<Entry> g_tab[TUNE_COUNT];  // sorted by min_points, unique thresholds
std::atomic<uint64_t> g_gen{0};        // bumped by every change of the table
std::once_flag g_once;
int g_auto_rc = CPSZ_OK;
std::string g_auto_err, g_loaded_from;

int find_param(const char* name) {
  if (!name) return -1;
  for (int p = 0; p < TUNE_COUNT; p++)
    if (!strcmp(kInfo[p].name, name)) return p;
  return -1;
}

void put(std::vector<Entry>& v, size_t min_points, int value) {
  for (Entry& e : v)
    if (e.min_points == min_points) {
      e.value = value;
      return;
    }
  v.push_back({min_points, value});
  std::sort(v.begin(), v.end(), [](const Entry& a, const Entry& b) { return a.min_points < b.min_points; });
}

// ---- a small JSON reader: objects, arrays, strings, numbers, literals ------
struct Json {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  double num = 0;
  std::string str;
  std::vector<Json> items;                              // ARR
  std::vector<std::pair<std::string, Json>> members;  // OBJ
  const Json* get(const char* k) const {
    for (auto& m : members)
      if (m.first == k) return &m.second;
    return nullptr;
  }
};

struct Reader {
  const char* p;
  const char* end;
  std::string err;
  void ws() {
    while (p < end && isspace((unsigned char)*p)) p++;
  }
  bool fail(const char* what) {
    if (err.empty()) err = what;
    return false;
  }
  bool string(std::string& out) {
    if (p >= end || *p != '"') return fail("expected a string");
    p++;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        if (++p >= end) break;
        char c = *p;
        out.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c);  // \uXXXX is not needed by the table
      } else {
        out.push_back(*p);
      }
      p++;
    }
    if (p >= end) return fail("unterminated string");
    p++;
    return true;
  }
  bool value(Json& v, int depth) {
    if (depth > 32) return fail("nesting too deep");
    ws();
    if (p >= end) return fail("unexpected end");
    if (*p == '{') {
      v.kind = Json::OBJ;
      p++;
      ws();
      if (p < end && *p == '}') return p++, true;
      for (;;) {
        ws();
        std::string k;
        if (!string(k)) return false;
        ws();
        if (p >= end || *p != ':') return fail("expected ':'");
        p++;
        v.members.emplace_back(k, Json());
        if (!value(v.members.back().second, depth + 1)) return false;
        ws();
        if (p < end && *p == ',') {
          p++;
          continue;
        }
        if (p < end && *p == '}') return p++, true;
        return fail("expected ',' or '}'");
      }
    }
    if (*p == '[') {
      v.kind = Json::ARR;
      p++;
      ws();
      if (p < end && *p == ']') return p++, true;
      for (;;) {
        v.items.emplace_back();
        if (!value(v.items.back(), depth + 1)) return false;
        ws();
        if (p < end && *p == ',') {
          p++;
          continue;
        }
        if (p < end && *p == ']') return p++, true;
        return fail("expected ',' or ']'");
      }
    }
    if (*p == '"') {
      v.kind = Json::STR;
      return string(v.str);
    }
    auto lit = [&](const char* w) {
      size_t n = strlen(w);
      if ((size_t)(end - p) >= n && !strncmp(p, w, n)) {
        p += n;
        return true;
      }
      return false;
    };
    if (lit("true")) return v.kind = Json::BOOL, v.num = 1, true;
    if (lit("false")) return v.kind = Json::BOOL, v.num = 0, true;
    if (lit("null")) return v.kind = Json::NUL, true;
    std::string num;
    while (p < end && (isdigit((unsigned char)*p) || strchr("+-.eE", *p))) num.push_back(*p++);
    if (num.empty()) return fail("unexpected character");
    char* e = nullptr;
    v.kind = Json::NUM;
    v.num = strtod(num.c_str(), &e);
    if (!e || *e) return fail("malformed number");
    return true;
  }
};

// Parses the table text into per-parameter entry lists (nothing is installed
// unless the whole file is valid).
int parse_table(const std::string& text, std::vector<Entry> (&out)[TUNE_COUNT]) {
  Reader r{text.data(), text.data() + text.size(), {}};
  Json root;
  if (!r.value(root, 0)) return set_error(CPSZ_ERR_INVALID, "tuning table: %s", r.err.c_str());
  r.ws();
  if (r.p != r.end) return set_error(CPSZ_ERR_INVALID, "tuning table: trailing characters");
  if (root.kind != Json::OBJ) return set_error(CPSZ_ERR_INVALID, "tuning table: top level is not an object");
  const Json* fmt = root.get("format");
  if (!fmt || fmt->kind != Json::STR || fmt->str != "cpsz_b200-tuning-1")
    return set_error(CPSZ_ERR_INVALID, "tuning table: format is not \"cpsz_b200-tuning-1\"");
  const Json* ent = root.get("entries");
  if (!ent || ent->kind != Json::ARR) return set_error(CPSZ_ERR_INVALID, "tuning table: no \"entries\" array");
  for (size_t k = 0; k < ent->items.size(); k++) {
    const Json& e = ent->items[k];
    const Json* pn = e.get("param");
    const Json* mp = e.get("min_points");
    const Json* va = e.get("value");
    if (e.kind != Json::OBJ || !pn || pn->kind != Json::STR || !mp || mp->kind != Json::NUM || !va ||
        va->kind != Json::NUM)
      return set_error(CPSZ_ERR_INVALID, "tuning table: entry %zu needs \"param\", \"min_points\", \"value\"", k);
    const int p = find_param(pn->str.c_str());
    if (p < 0) return set_error(CPSZ_ERR_INVALID, "tuning table: unknown parameter \"%s\"", pn->str.c_str());
    if (mp->num < 0 || mp->num > 9.0e18 || va->num != (double)(int)va->num || va->num < kInfo[p].lo ||
        va->num > kInfo[p].hi)
      return set_error(CPSZ_ERR_INVALID, "tuning table: entry %zu (%s) out of range", k, pn->str.c_str());
    put(out[p], (size_t)mp->num, (int)va->num);
  }
  return CPSZ_OK;
}

int load_file(const std::string& path, bool missing_ok) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    if (missing_ok) return CPSZ_OK;
    return set_error(CPSZ_ERR_INVALID, "tuning table %s: cannot open", path.c_str());
  }
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  fclose(f);
  std::vector<Entry> t[TUNE_COUNT];
  int rc = parse_table(text, t);
  if (rc != CPSZ_OK) return set_error(rc, "%s (%s)", cpsz_b200_last_error(), path.c_str());
  std::unique_lock<std::shared_mutex> lk(g_mu);
  for (int p = 0; p < TUNE_COUNT; p++) g_tab[p] = std::move(t[p]);
  g_loaded_from = path;
  g_gen++;
  return CPSZ_OK;
}

std::string default_path() {
  Dl_info info;
  if (dladdr((void*)&default_path, &info) && info.dli_fname) {
    std::string s(info.dli_fname);
    size_t a = s.rfind('/');
    if (a != std::string::npos) {
      size_t b = s.rfind('/', a ? a - 1 : 0);
      if (b != std::string::npos) return s.substr(0, b) + "/tuning_b200.json";
    }
  }
  return "tuning_b200.json";
}

// An explicit set / clear / load means the caller manages the table: the
// default file is then never loaded over it.
void suppress_autoload() { std::call_once(g_once, [] {}); }

}  // namespace

const TuneInfo& tune_info(int p) { return kInfo[p]; }

uint64_t tune_generation() { return g_gen.load(); }

int tune_get(TuneParam p, size_t points) {
  if (p == TUNE_WAVE2D_OVERLAP) {
    static const bool env_off = [] {
      const char* e = getenv("CPSZ_B200_OVERLAP");
      return e && !strcmp(e, "0");
    }();
    if (env_off) return 0;
  }
  std::shared_lock<std::shared_mutex> lk(g_mu);
  int v = kInfo[p].def;
  for (const Entry& e : g_tab[p]) {
    if (e.min_points > points) break;
    v = e.value;
  }
  return v;
}

int tune_autoload() {
  std::call_once(g_once, [] {
    const char* env = getenv("CPSZ_B200_TUNING");
    if (env && (!*env || !strcmp(env, "none"))) return;
    g_auto_rc = env ? load_file(env, false) : load_file(default_path(), true);
    if (g_auto_rc != CPSZ_OK) g_auto_err = cpsz_b200_last_error();
  });
  if (g_auto_rc != CPSZ_OK) return set_error(g_auto_rc, "%s", g_auto_err.c_str());
  return CPSZ_OK;
}

}  // namespace cpsz

using namespace cpsz;

extern "C" {

int cpsz_b200_tuning_param_count(void) { return TUNE_COUNT; }

int cpsz_b200_tuning_param_info(int index, const char** name, int* def, int* lo, int* hi) {
  if (index < 0 || index >= TUNE_COUNT) return set_error(CPSZ_ERR_INVALID, "tuning parameter %d out of range", index);
  if (name) *name = kInfo[index].name;
  if (def) *def = kInfo[index].def;
  if (lo) *lo = kInfo[index].lo;
  if (hi) *hi = kInfo[index].hi;
  return CPSZ_OK;
}

int cpsz_b200_tuning_set(const char* param, size_t min_points, int value) {
  const int p = find_param(param);
  if (p < 0) return set_error(CPSZ_ERR_INVALID, "unknown tuning parameter \"%s\"", param ? param : "(null)");
  if (value < kInfo[p].lo || value > kInfo[p].hi)
    return set_error(CPSZ_ERR_INVALID, "tuning %s = %d outside [%d, %d]", kInfo[p].name, value, kInfo[p].lo,
                     kInfo[p].hi);
  suppress_autoload();
  std::unique_lock<std::shared_mutex> lk(g_mu);
  put(g_tab[p], min_points, value);
  g_gen++;
  return CPSZ_OK;
}

int cpsz_b200_tuning_get(const char* param, size_t points, int* value) {
  const int p = find_param(param);
  if (p < 0) return set_error(CPSZ_ERR_INVALID, "unknown tuning parameter \"%s\"", param ? param : "(null)");
  if (!value) return set_error(CPSZ_ERR_INVALID, "tuning_get: null output");
  *value = tune_get((TuneParam)p, points);
  return CPSZ_OK;
}

int cpsz_b200_tuning_clear(void) {
  suppress_autoload();
  std::unique_lock<std::shared_mutex> lk(g_mu);
  for (auto& v : g_tab) v.clear();
  g_loaded_from.clear();
  g_gen++;
  return CPSZ_OK;
}

int cpsz_b200_tuning_load(const char* path) {
  clear_error();
  suppress_autoload();
  return path ? load_file(path, false) : load_file(default_path(), false);
}

}  // extern "C"

extern "C" const char* cpsz_b200_tuning_source(void) {
  std::shared_lock<std::shared_mutex> lk(g_mu);
  static thread_local std::string copy;
  copy = g_loaded_from;
  return copy.c_str();
}
