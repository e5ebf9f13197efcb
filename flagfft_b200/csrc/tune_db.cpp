#include "tune_db.hpp"

#include <dlfcn.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdlib>
#include <filesystem>
#include <mutex>

namespace ffb {

const char *tune_planner_fingerprint() { return "ffb-planner-1-reference-semantics"; }
const char *tune_codegen_fingerprint() { return "ffb-kernels-1-sm100a-onchip"; }
const char *tune_runtime_fingerprint() { return "ffb-runtime-1"; }

std::string batch_bucket(int64_t batch) {  // src/exec/tuned_plan.cpp:21-35
  if (batch <= 1) return "1";
  if (batch <= 8) return "2-8";
  if (batch <= 64) return "9-64";
  if (batch <= 512) return "65-512";
  return "513+";
}

static bool env_true(const char *v) {
  if (!v) return false;
  std::string s(v);
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return !(s.empty() || s == "0" || s == "false" || s == "off" || s == "no");
}

std::optional<std::string> tune_db_path() {  // src/exec/tuned_plan.cpp:49-58
  if (env_true(std::getenv("FLAGFFT_TUNE_DISABLE"))) return std::nullopt;
  const char *p = std::getenv("FLAGFFT_TUNE_DB");
  if (p && *p) return std::string(p);
  char buf[4096];
  ssize_t len = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  std::filesystem::path dir = len > 0 ? std::filesystem::path(std::string(buf, (size_t)len)).parent_path()
                                      : std::filesystem::current_path();
  return (dir / ".flagfft" / "tuned_plans.sqlite").string();
}

namespace {

// The handful of SQLite C API entry points used, bound at run time.
struct Sqlite {
  void *h = nullptr;
  int (*open_v2)(const char *, void **, int, const char *) = nullptr;
  int (*close)(void *) = nullptr;
  int (*prepare_v2)(void *, const char *, int, void **, const char **) = nullptr;
  int (*bind_int64)(void *, int, long long) = nullptr;
  int (*bind_double)(void *, int, double) = nullptr;
  int (*bind_text)(void *, int, const char *, int, void (*)(void *)) = nullptr;
  int (*step)(void *) = nullptr;
  const unsigned char *(*column_text)(void *, int) = nullptr;
  int (*finalize)(void *) = nullptr;
  int (*exec)(void *, const char *, void *, void *, char **) = nullptr;
  bool ok = false;
};

Sqlite &sqlite() {
  static Sqlite s;
  static std::once_flag once;
  std::call_once(once, [] {
    s.h = dlopen("libsqlite3.so.0", RTLD_NOW | RTLD_LOCAL);
    if (!s.h) s.h = dlopen("libsqlite3.so", RTLD_NOW | RTLD_LOCAL);
    if (!s.h) return;
#define FFB_SYM(field, name) s.field = reinterpret_cast<decltype(s.field)>(dlsym(s.h, name))
    FFB_SYM(open_v2, "sqlite3_open_v2");
    FFB_SYM(close, "sqlite3_close");
    FFB_SYM(prepare_v2, "sqlite3_prepare_v2");
    FFB_SYM(bind_int64, "sqlite3_bind_int64");
    FFB_SYM(bind_double, "sqlite3_bind_double");
    FFB_SYM(bind_text, "sqlite3_bind_text");
    FFB_SYM(step, "sqlite3_step");
    FFB_SYM(column_text, "sqlite3_column_text");
    FFB_SYM(finalize, "sqlite3_finalize");
    FFB_SYM(exec, "sqlite3_exec");
#undef FFB_SYM
    s.ok = s.open_v2 && s.close && s.prepare_v2 && s.bind_int64 && s.bind_double && s.bind_text && s.step &&
           s.column_text && s.finalize && s.exec;
  });
  return s;
}

constexpr int kOpenReadOnly = 0x1, kOpenReadWrite = 0x2, kOpenCreate = 0x4;
constexpr int kRow = 100, kDone = 101;
void (*const kTransient)(void *) = reinterpret_cast<void (*)(void *)>(-1);

const char *kCreate =
    "CREATE TABLE IF NOT EXISTS tuned_measurements ("
    " id INTEGER PRIMARY KEY AUTOINCREMENT, schema_version INTEGER, status TEXT, rank INTEGER,"
    " device_arch TEXT, fft_length INTEGER, batch_bucket TEXT, dtype TEXT, direction TEXT, norm TEXT,"
    " input_layout TEXT, planner_fingerprint TEXT, codegen_fingerprint TEXT, runtime_fingerprint TEXT,"
    " benchmark_fingerprint TEXT, median_ms REAL, source TEXT, measured_at TEXT, plan_json TEXT)";

}  // namespace

std::optional<std::string> tune_lookup(const TuneKey &key) {  // src/utils/plan_json.cpp:163-207
  auto path = tune_db_path();
  if (!path) return std::nullopt;
  std::error_code ec;
  if (!std::filesystem::is_regular_file(*path, ec)) return std::nullopt;
  Sqlite &s = sqlite();
  if (!s.ok) return std::nullopt;
  void *db = nullptr;
  if (s.open_v2(path->c_str(), &db, kOpenReadOnly, nullptr) != 0) {
    if (db) s.close(db);
    return std::nullopt;
  }
  std::optional<std::string> out;
  void *st = nullptr;
  const char *sql =
      "SELECT plan_json FROM tuned_measurements WHERE schema_version=? AND status='valid' AND rank=0 "
      "AND device_arch=? AND fft_length=? AND batch_bucket=? AND dtype=? AND direction=? AND norm=? "
      "AND input_layout=? AND planner_fingerprint=? AND codegen_fingerprint=? AND runtime_fingerprint=? "
      "ORDER BY measured_at DESC LIMIT 1";
  if (s.prepare_v2(db, sql, -1, &st, nullptr) == 0 && st) {
    std::string bucket = batch_bucket(key.batch);
    s.bind_int64(st, 1, kTuneSchemaVersion);
    s.bind_text(st, 2, key.device_arch.c_str(), -1, kTransient);
    s.bind_int64(st, 3, key.fft_length);
    s.bind_text(st, 4, bucket.c_str(), -1, kTransient);
    s.bind_text(st, 5, key.dtype.c_str(), -1, kTransient);
    s.bind_text(st, 6, key.direction.c_str(), -1, kTransient);
    s.bind_text(st, 7, "backward", -1, kTransient);
    s.bind_text(st, 8, "contiguous", -1, kTransient);
    s.bind_text(st, 9, tune_planner_fingerprint(), -1, kTransient);
    s.bind_text(st, 10, tune_codegen_fingerprint(), -1, kTransient);
    s.bind_text(st, 11, tune_runtime_fingerprint(), -1, kTransient);
    if (s.step(st) == kRow) {
      const unsigned char *t = s.column_text(st, 0);
      if (t) out = std::string(reinterpret_cast<const char *>(t));
    }
    s.finalize(st);
  }
  s.close(db);
  return out;
}

bool tune_store(const TuneKey &key, const std::string &plan_json, double median_ms, const std::string &source,
                const std::string &db_path) {
  Sqlite &s = sqlite();
  if (!s.ok) return false;
  std::error_code ec;
  auto parent = std::filesystem::path(db_path).parent_path();
  if (!parent.empty()) std::filesystem::create_directories(parent, ec);
  void *db = nullptr;
  if (s.open_v2(db_path.c_str(), &db, kOpenReadWrite | kOpenCreate, nullptr) != 0) {
    if (db) s.close(db);
    return false;
  }
  bool ok = s.exec(db, kCreate, nullptr, nullptr, nullptr) == 0;
  void *st = nullptr;
  const char *sql =
      "INSERT INTO tuned_measurements (schema_version, status, rank, device_arch, fft_length, batch_bucket, dtype,"
      " direction, norm, input_layout, planner_fingerprint, codegen_fingerprint, runtime_fingerprint,"
      " benchmark_fingerprint, median_ms, source, measured_at, plan_json)"
      " VALUES (?, 'valid', 0, ?, ?, ?, ?, ?, 'backward', 'contiguous', ?, ?, ?, 'ffb-bench-1', ?, ?,"
      " strftime('%Y-%m-%dT%H:%M:%f', 'now'), ?)";
  if (ok && s.prepare_v2(db, sql, -1, &st, nullptr) == 0 && st) {
    std::string bucket = batch_bucket(key.batch);
    s.bind_int64(st, 1, kTuneSchemaVersion);
    s.bind_text(st, 2, key.device_arch.c_str(), -1, kTransient);
    s.bind_int64(st, 3, key.fft_length);
    s.bind_text(st, 4, bucket.c_str(), -1, kTransient);
    s.bind_text(st, 5, key.dtype.c_str(), -1, kTransient);
    s.bind_text(st, 6, key.direction.c_str(), -1, kTransient);
    s.bind_text(st, 7, tune_planner_fingerprint(), -1, kTransient);
    s.bind_text(st, 8, tune_codegen_fingerprint(), -1, kTransient);
    s.bind_text(st, 9, tune_runtime_fingerprint(), -1, kTransient);
    s.bind_double(st, 10, median_ms);
    s.bind_text(st, 11, source.c_str(), -1, kTransient);
    s.bind_text(st, 12, plan_json.c_str(), -1, kTransient);
    ok = s.step(st) == kDone;
    s.finalize(st);
  } else {
    ok = false;
  }
  s.close(db);
  return ok;
}

}  // namespace ffb
