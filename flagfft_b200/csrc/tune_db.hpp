// Tune database: per-request forced plan trees in SQLite, read at plan time.
//
// Keeps the reference's table, key columns and lookup rule
// (src/utils/plan_json.cpp:163-207, src/exec/tuned_plan.cpp:21-58): the most
// recent valid rank-0 row for (schema, arch, length, batch bucket, dtype,
// direction, norm, layout, fingerprints) supplies the plan JSON.  SQLite is
// loaded at run time (libsqlite3.so.0); without it the lookup finds nothing.
#pragma once

#include <cstdint>
#include <optional>
#include <string>

namespace ffb {

struct TuneKey {
  std::string device_arch;  // "sm_100"
  int64_t fft_length = 0;
  int64_t batch = 1;
  std::string dtype;      // "complex64" / "complex128"
  std::string direction;  // "forward" / "inverse"
};

constexpr int64_t kTuneSchemaVersion = 3;
const char *tune_planner_fingerprint();
const char *tune_codegen_fingerprint();
const char *tune_runtime_fingerprint();

std::string batch_bucket(int64_t batch);

// Path of the DB: $FLAGFFT_TUNE_DB, else <executable dir>/.flagfft/tuned_plans.sqlite;
// none when $FLAGFFT_TUNE_DISABLE is set to a true value.
std::optional<std::string> tune_db_path();

std::optional<std::string> tune_lookup(const TuneKey &key);

// Insert one measured row (used by the autotuner).  Creates the table when
// missing.  Returns false when SQLite is unavailable or the write failed.
bool tune_store(const TuneKey &key, const std::string &plan_json, double median_ms, const std::string &source,
                const std::string &db_path);

}  // namespace ffb
