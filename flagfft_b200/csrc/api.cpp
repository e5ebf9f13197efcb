// The flagfft.h C ABI: descriptor validation, plan lifecycle and Exec entry
// points, keeping the reference's argument checks and status codes
// (src/exec/c_api_plan.cpp, src/exec/c_api_exec.cpp, src/exec/c_api_internal.cpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <optional>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/flagfft.h"
#include "../../include/flagfft_b200.h"
#include "exec.hpp"
#include "plan.hpp"
#include "tune_db.hpp"

struct flagfftPlan_t {
  void *impl = nullptr;
};

namespace ffb {
namespace {

enum class Precision { F32, F64 };

struct PlanDesc {  // src/exec/c_api_internal.hpp:14-32
  int rank = 0;
  std::vector<int64_t> n, inembed, onembed;
  int64_t istride = 1, idist = 0, ostride = 1, odist = 0, batch = 1;
  flagfftType type = FLAGFFT_C2C;
  bool is_double = false;
  bool real_forward = false, real_inverse = false;
  int device = 0;
  std::string arch;
  int64_t smem_optin = 232448;
};

struct Plan {
  PlanDesc desc;
  bool initialized = false;
  bool destroyed = false;
  cudaStream_t stream = nullptr;
  NodePtr root;
  std::unique_ptr<Program> fwd, inv;
  // 1-D real plans executed in place read / write padded rows of 2(n/2+1)
  // reals (src/exec/raw_nodes.cpp:425-429, 466-470)
  std::unique_ptr<Program> fwd_ip, inv_ip;
  // batch plans (flagfftB200PlanBatch): groups of uneven lengths
  bool is_batch = false;
  std::vector<BatchGroup> groups;
  std::unique_ptr<BatchProgram> bfwd, binv;
  std::string description;
  std::string json;
  std::mutex mutex;
};

Plan *checked(flagfftHandle h) {  // c_api_internal.cpp:170-175
  if (h == nullptr || h->impl == nullptr) return nullptr;
  return static_cast<Plan *>(h->impl);
}

flagfftResult type_info(flagfftType t, PlanDesc &d) {  // c_api_internal.cpp:5-52
  switch (t) {
    case FLAGFFT_C2C: d.is_double = false; return FLAGFFT_SUCCESS;
    case FLAGFFT_Z2Z: d.is_double = true; return FLAGFFT_SUCCESS;
    case FLAGFFT_R2C: d.is_double = false; d.real_forward = true; return FLAGFFT_SUCCESS;
    case FLAGFFT_D2Z: d.is_double = true; d.real_forward = true; return FLAGFFT_SUCCESS;
    case FLAGFFT_C2R: d.is_double = false; d.real_inverse = true; return FLAGFFT_SUCCESS;
    case FLAGFFT_Z2D: d.is_double = true; d.real_inverse = true; return FLAGFFT_SUCCESS;
  }
  return FLAGFFT_INVALID_TYPE;
}

// src/exec/c_api_internal.cpp:60-89: 1-D, unit strides, tight or padded-real distances.
bool supported_1d(const PlanDesc &d) {
  if (d.rank != 1 || d.batch <= 0 || d.n.size() != 1 || d.n[0] <= 0) return false;
  const int64_t n = d.n[0], half = n / 2 + 1, padded = 2 * half;
  const int64_t in_len = d.real_inverse ? half : n;
  const int64_t out_len = d.real_forward ? half : n;
  const bool idist_ok = d.idist == in_len || (d.real_forward && d.idist == padded);
  const bool odist_ok = d.odist == out_len || (d.real_inverse && d.odist == padded);
  const bool iemb_ok = d.inembed.size() == 1 && (d.inembed[0] == in_len || (d.real_forward && d.inembed[0] == padded));
  const bool oemb_ok =
      d.onembed.size() == 1 && (d.onembed[0] == out_len || (d.real_inverse && d.onembed[0] == padded));
  return d.istride == 1 && d.ostride == 1 && idist_ok && odist_ok && iemb_ok && oemb_ok;
}

// src/exec/c_api_internal.cpp:91-120: 2-D, unit strides, tightly packed batches.
bool supported_2d(const PlanDesc &d) {
  if (d.rank != 2 || d.batch <= 0 || d.n.size() != 2 || d.n[0] <= 0 || d.n[1] <= 0) return false;
  if (d.istride != 1 || d.ostride != 1) return false;
  const int64_t n0 = d.n[0], n1 = d.n[1], h1 = n1 / 2 + 1;
  const int64_t in_logical = d.real_inverse ? n0 * h1 : n0 * n1;
  const int64_t out_logical = d.real_forward ? n0 * h1 : n0 * n1;
  return d.idist == in_logical && d.odist == out_logical;
}

flagfftResult ensure_device(PlanDesc &d) {  // src/adaptor/backend/cuda/adaptor.cpp:215-244
#ifdef FFB_HOST_EMULATION
  d.device = 0;
  d.arch = "sm_100";
  d.smem_optin = 232448;
  return FLAGFFT_SUCCESS;
#endif
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return FLAGFFT_INVALID_DEVICE;
  }
  if (cudaFree(nullptr) != cudaSuccess) {
    cudaGetLastError();
    return FLAGFFT_INVALID_DEVICE;
  }
  int major = 0, minor = 0, optin = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (major != 10) return FLAGFFT_INVALID_DEVICE;  // kernels are built for sm_100a only
  d.device = dev;
  d.arch = "sm_" + std::to_string(major) + std::to_string(minor);
  d.smem_optin = optin > 0 ? optin : 48 * 1024;
  return FLAGFFT_SUCCESS;
}

// Tuned tree for one request, or null (src/exec/c_api_plan.cpp:27-39).  The
// stored object wraps the tree under "root" (src/utils/plan_json.cpp:147-156).
NodePtr tuned_tree(Planner &pl, const PlanDesc &d, int64_t length, int64_t batch, const char *direction) {
  TuneKey k;
  k.device_arch = d.arch;
  k.fft_length = length;
  k.batch = batch;
  k.dtype = d.is_double ? "complex128" : "complex64";
  k.direction = direction;
  auto row = tune_lookup(k);
  if (!row) return nullptr;
  try {
    Json j = Json::parse(*row);
    NodePtr n = node_from_json(pl, j.has("root") ? j.at("root") : j);
    return raw_supported(n) && n->length == length ? n : nullptr;
  } catch (const std::exception &) {
    return nullptr;
  }
}

NodePtr root_for(Planner &pl, const PlanDesc &d, int64_t n, int64_t batch) {
  NodePtr tf = tuned_tree(pl, d, n, batch, "forward");
  NodePtr ti = tuned_tree(pl, d, n, batch, "inverse");
  return build_raw_root(pl, n, tf, ti);
}

flagfftResult build_plan(flagfftHandle *out, PlanDesc desc) {  // src/exec/c_api_plan.cpp:43-245
  if (out == nullptr) return FLAGFFT_INVALID_VALUE;
  *out = nullptr;
  const bool is_2d = supported_2d(desc);
  if (!supported_1d(desc) && !is_2d) return FLAGFFT_NOT_SUPPORTED;
  flagfftResult dr = ensure_device(desc);
  if (dr != FLAGFFT_SUCCESS) return dr;
  try {
    auto plan = std::make_unique<Plan>();
    plan->desc = desc;
    Planner planner(desc.is_double, desc.smem_optin);
    const Transform tr = desc.real_forward ? Transform::R2C : desc.real_inverse ? Transform::C2R : Transform::C2C;
    if (is_2d) {
      const int64_t n0 = desc.n[0], n1 = desc.n[1];
      const int64_t h1 = n1 / 2 + 1;
      NodePtr row = root_for(planner, desc, n1, desc.batch * n0);
      NodePtr col = root_for(planner, desc, n0, desc.batch * (tr == Transform::C2C ? n1 : h1));
      if (!raw_supported(row) || !raw_supported(col)) return FLAGFFT_NOT_SUPPORTED;
      plan->root = make_two_dim_node(n0, n1, row, col);
      if (tr != Transform::C2R)
        plan->fwd = lower_2d(plan->root, planner, desc.is_double, tr, false, n0, n1, desc.batch);
      if (tr != Transform::R2C)
        plan->inv = lower_2d(plan->root, planner, desc.is_double, tr, true, n0, n1, desc.batch);
    } else {
      const int64_t n = desc.n[0];
      plan->root = root_for(planner, desc, n, desc.batch);
      if (!raw_supported(plan->root)) return FLAGFFT_NOT_SUPPORTED;
      Layout lay;
      lay.batch = desc.batch;
      lay.idist = desc.idist;
      lay.odist = desc.odist;
      if (tr != Transform::C2R) plan->fwd = lower(plan->root, planner, desc.is_double, tr, false, n, lay, false);
      if (tr != Transform::R2C) plan->inv = lower(plan->root, planner, desc.is_double, tr, true, n, lay, false);
      if (tr == Transform::R2C) plan->fwd_ip = lower(plan->root, planner, desc.is_double, tr, false, n, lay, true);
      if (tr == Transform::C2R) plan->inv_ip = lower(plan->root, planner, desc.is_double, tr, true, n, lay, true);
    }
    plan->json = plan->root->to_json();
    plan->initialized = true;
    auto h = std::make_unique<flagfftPlan_t>();
    h->impl = plan.release();
    *out = h.release();
    return FLAGFFT_SUCCESS;
  } catch (const std::bad_alloc &) {
    return FLAGFFT_ALLOC_FAILED;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "[flagfft] plan setup failed: %s\n", e.what());
    return FLAGFFT_SETUP_FAILED;
  }
}

flagfftResult run(Plan *plan, const Program *prog, const void *in, void *out) {
  cudaError_t e = prog->run(in, out, plan->stream);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "[flagfft] Exec failed: %s\n", cudaGetErrorString(e));
    std::fflush(stderr);
    return FLAGFFT_EXEC_FAILED;
  }
  return FLAGFFT_SUCCESS;
}

// Shared checks of every Exec entry point (src/exec/c_api_exec.cpp:9-21).
template <typename F>
flagfftResult exec_common(flagfftHandle h, const void *in, void *out, flagfftType want, bool has_dir, int dir,
                          F pick) {
  Plan *plan = checked(h);
  if (plan == nullptr || plan->destroyed || !plan->initialized) return FLAGFFT_INVALID_PLAN;
  if (in == nullptr || out == nullptr) return FLAGFFT_INVALID_VALUE;
  if (plan->desc.type != want) return FLAGFFT_INVALID_TYPE;
  if (has_dir && dir != FLAGFFT_FORWARD && dir != FLAGFFT_INVERSE) return FLAGFFT_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(plan->mutex);
  if (plan->is_batch) {
    BatchProgram *bp = dir == FLAGFFT_INVERSE ? plan->binv.get() : plan->bfwd.get();
    cudaError_t e = cudaErrorInvalidValue;
    try {
      if (bp) e = bp->run(in, out, plan->stream);
    } catch (const std::bad_alloc &) {
      return FLAGFFT_ALLOC_FAILED;
    } catch (const std::exception &ex) {
      std::fprintf(stderr, "[flagfft] batch Exec failed: %s\n", ex.what());
      return FLAGFFT_EXEC_FAILED;
    }
    if (e != cudaSuccess) {
      std::fprintf(stderr, "[flagfft] batch Exec failed: %s\n", cudaGetErrorString(e));
      std::fflush(stderr);
      return FLAGFFT_EXEC_FAILED;
    }
    return FLAGFFT_SUCCESS;
  }
  const Program *prog = pick(plan, in == out);
  if (prog == nullptr) return FLAGFFT_EXEC_FAILED;
  return run(plan, prog, in, out);
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" flagfftResult flagfftPlanMany(flagfftHandle *plan, int rank, int *n, int *inembed, int istride, int idist,
                                         int *onembed, int ostride, int odist, flagfftType type, int batch) {
  if (plan == nullptr) return FLAGFFT_INVALID_VALUE;
  *plan = nullptr;
  if (rank <= 0 || n == nullptr || batch <= 0) return FLAGFFT_INVALID_VALUE;
  for (int i = 0; i < rank; ++i)
    if (n[i] <= 0) return FLAGFFT_INVALID_SIZE;
  PlanDesc d;
  d.rank = rank;
  for (int i = 0; i < rank; ++i) d.n.push_back(n[i]);
  d.istride = istride;
  d.idist = idist;
  d.ostride = ostride;
  d.odist = odist;
  d.batch = batch;
  d.type = type;
  flagfftResult tr = type_info(type, d);
  if (tr != FLAGFFT_SUCCESS) return tr;
  // default embeds (src/exec/c_api_plan.cpp:307-333)
  if (inembed != nullptr) {
    for (int i = 0; i < rank; ++i) d.inembed.push_back(inembed[i]);
  } else if (d.real_inverse && rank == 1) {
    d.inembed = {d.n[0] / 2 + 1};
  } else if (d.real_inverse && rank == 2) {
    d.inembed = {d.n[0], d.n[1] / 2 + 1};
  } else {
    d.inembed = d.n;
  }
  if (onembed != nullptr) {
    for (int i = 0; i < rank; ++i) d.onembed.push_back(onembed[i]);
  } else if (d.real_forward && rank == 1) {
    d.onembed = {d.n[0] / 2 + 1};
  } else if (d.real_forward && rank == 2) {
    d.onembed = {d.n[0], d.n[1] / 2 + 1};
  } else {
    d.onembed = d.n;
  }
  return build_plan(plan, std::move(d));
}

extern "C" flagfftResult flagfftPlan1d(flagfftHandle *plan, int nx, flagfftType type, int batch) {
  int n[1] = {nx};
  const bool rf = type == FLAGFFT_R2C || type == FLAGFFT_D2Z;
  const bool ri = type == FLAGFFT_C2R || type == FLAGFFT_Z2D;
  const int half = nx / 2 + 1;
  return flagfftPlanMany(plan, 1, n, nullptr, 1, ri ? half : nx, nullptr, 1, rf ? half : nx, type, batch);
}

extern "C" flagfftResult flagfftPlan2d(flagfftHandle *plan, int nx, int ny, flagfftType type) {
  int n[2] = {nx, ny};
  const bool rf = type == FLAGFFT_R2C || type == FLAGFFT_D2Z;
  const bool ri = type == FLAGFFT_C2R || type == FLAGFFT_Z2D;
  const int hy = ny / 2 + 1;
  return flagfftPlanMany(plan, 2, n, nullptr, 1, ri ? nx * hy : nx * ny, nullptr, 1, rf ? nx * hy : nx * ny, type,
                         1);
}

extern "C" flagfftResult flagfftPlan3d(flagfftHandle *plan, int nx, int ny, int nz, flagfftType type) {
  int n[3] = {nx, ny, nz};
  return flagfftPlanMany(plan, 3, n, nullptr, 1, nx * ny * nz, nullptr, 1, nx * ny * nz, type, 1);
}

extern "C" flagfftResult flagfftExecC2C(flagfftHandle h, flagfftComplex *in, flagfftComplex *out, int dir) {
  return exec_common(h, in, out, FLAGFFT_C2C, true, dir,
                     [&](Plan *p, bool) { return dir == FLAGFFT_INVERSE ? p->inv.get() : p->fwd.get(); });
}

extern "C" flagfftResult flagfftExecZ2Z(flagfftHandle h, flagfftDoubleComplex *in, flagfftDoubleComplex *out,
                                        int dir) {
  return exec_common(h, in, out, FLAGFFT_Z2Z, true, dir,
                     [&](Plan *p, bool) { return dir == FLAGFFT_INVERSE ? p->inv.get() : p->fwd.get(); });
}

extern "C" flagfftResult flagfftExecR2C(flagfftHandle h, flagfftReal *in, flagfftComplex *out) {
  return exec_common(h, in, out, FLAGFFT_R2C, false, 0, [](Plan *p, bool ip) { return ip && p->fwd_ip ? p->fwd_ip.get() : p->fwd.get(); });
}

extern "C" flagfftResult flagfftExecD2Z(flagfftHandle h, flagfftDoubleReal *in, flagfftDoubleComplex *out) {
  return exec_common(h, in, out, FLAGFFT_D2Z, false, 0, [](Plan *p, bool ip) { return ip && p->fwd_ip ? p->fwd_ip.get() : p->fwd.get(); });
}

extern "C" flagfftResult flagfftExecC2R(flagfftHandle h, flagfftComplex *in, flagfftReal *out) {
  return exec_common(h, in, out, FLAGFFT_C2R, false, 0, [](Plan *p, bool ip) { return ip && p->inv_ip ? p->inv_ip.get() : p->inv.get(); });
}

extern "C" flagfftResult flagfftExecZ2D(flagfftHandle h, flagfftDoubleComplex *in, flagfftDoubleReal *out) {
  return exec_common(h, in, out, FLAGFFT_Z2D, false, 0, [](Plan *p, bool ip) { return ip && p->inv_ip ? p->inv_ip.get() : p->inv.get(); });
}

extern "C" flagfftResult flagfftSetStream(flagfftHandle h, flagfftStream_t stream) {  // c_api_exec.cpp:169-177
  Plan *plan = checked(h);
  if (plan == nullptr || plan->destroyed) return FLAGFFT_INVALID_PLAN;
  std::lock_guard<std::mutex> lock(plan->mutex);
  plan->stream = static_cast<cudaStream_t>(stream);
  return FLAGFFT_SUCCESS;
}

extern "C" flagfftResult flagfftDestroy(flagfftHandle h) {  // c_api_exec.cpp:179-194
  if (h == nullptr) return FLAGFFT_INVALID_PLAN;
  Plan *plan = checked(h);
  if (plan != nullptr) {
    {
      std::lock_guard<std::mutex> lock(plan->mutex);
      plan->destroyed = true;
    }
    delete plan;
    h->impl = nullptr;
  }
  delete h;
  return FLAGFFT_SUCCESS;
}

extern "C" const char *flagfftGetPlanDescription(flagfftHandle h) {  // c_api_exec.cpp:196-236
  Plan *plan = checked(h);
  if (plan == nullptr || plan->destroyed || !plan->initialized) return nullptr;
  std::lock_guard<std::mutex> lock(plan->mutex);
  if (!plan->description.empty()) return plan->description.c_str();
  std::ostringstream o;
  const auto &d = plan->desc;
  o << "=== FlagFFT Plan ===\n";
  o << "rank=" << d.rank << " n=[" << d.n[0];
  for (size_t i = 1; i < d.n.size(); ++i) o << "," << d.n[i];
  o << "] batch=" << d.batch << " type=" << (int)d.type << "\n";
  if (plan->is_batch) {
    o << "\n-- Batch --\n" << plan->groups.size() << " groups\n";
    o << "\n-- Forward execution --\nB200BatchProgram(launches=" << plan->bfwd->launches() << ")\n"
      << plan->bfwd->describe() << "\n";
    o << "\n-- Inverse execution --\nB200BatchProgram(launches=" << plan->binv->launches() << ")\n"
      << plan->binv->describe() << "\n";
    plan->description = o.str();
    return plan->description.c_str();
  }
  o << "\n-- Plan tree --\n" << plan->root->describe() << "\n";
  o << "\n-- Forward execution --\n";
  if (plan->fwd)
    o << "B200Program(launches=" << plan->fwd->launches() << ")\n" << plan->fwd->describe() << "\n";
  else
    o << "(not compiled)\n";
  if (plan->inv) o << "\n-- Inverse execution --\nB200Program(launches=" << plan->inv->launches() << ")\n"
                   << plan->inv->describe() << "\n";
  plan->description = o.str();
  return plan->description.c_str();
}

extern "C" const char *flagfftB200Version(void) { return "flagfft-b200 0.1.0 sm_100a"; }

extern "C" int flagfftB200PlannerTree(int n, int is_double, long long smem_bytes, char *buf, int buflen) {
  if (n <= 0) return -1;
  try {
    Planner pl(is_double != 0, smem_bytes > 0 ? smem_bytes : 232448);
    NodePtr root = build_raw_root(pl, n, nullptr, nullptr);
    std::string s = root->to_json();
    if (buf && buflen > 0) {
      size_t c = std::min<size_t>(s.size(), (size_t)buflen - 1);
      std::memcpy(buf, s.data(), c);
      buf[c] = 0;
    }
    return (int)s.size();
  } catch (const std::exception &) {
    return -1;
  }
}

extern "C" int flagfftB200TuneCandidates(int n, int is_double, char *buf, int buflen) {
  if (n <= 0) return -1;
  try {
    Planner pl(is_double != 0, 232448);
    std::string s = "[";
    const auto c = pl.tune_candidates(n, 12);
    for (size_t i = 0; i < c.size(); ++i) s += (i ? ", " : "") + c[i]->to_json();
    s += "]";
    if (buf && buflen > 0) {
      size_t k = std::min<size_t>(s.size(), (size_t)buflen - 1);
      std::memcpy(buf, s.data(), k);
      buf[k] = 0;
    }
    return (int)s.size();
  } catch (const std::exception &) {
    return -1;
  }
}

extern "C" flagfftResult flagfftB200Tune(int n, flagfftType type, int batch, int direction, const char *db_path,
                                        char *report, int buflen, double *best_ms) {
  if (n <= 0) return FLAGFFT_INVALID_SIZE;
  if (batch <= 0) return FLAGFFT_INVALID_VALUE;
  if (type != FLAGFFT_C2C && type != FLAGFFT_Z2Z) return FLAGFFT_INVALID_TYPE;
  if (direction != FLAGFFT_FORWARD && direction != FLAGFFT_INVERSE) return FLAGFFT_INVALID_VALUE;
  PlanDesc d;
  d.rank = 1;
  d.n = {n};
  d.batch = batch;
  d.type = type;
  type_info(type, d);
  flagfftResult dr = ensure_device(d);
  if (dr != FLAGFFT_SUCCESS) return dr;
#ifdef FFB_HOST_EMULATION
  (void)db_path;
  (void)report;
  (void)buflen;
  (void)best_ms;
  return FLAGFFT_NOT_SUPPORTED;
#else
  try {
    Planner pl(d.is_double, d.smem_optin);
    const auto cands = pl.tune_candidates(n, 12);
    const size_t bytes = (size_t)batch * (size_t)n * (d.is_double ? 16 : 8);
    DevMem in(bytes), out(bytes);
    cudaMemset(in.ptr, 0x3c, bytes);  // timing does not depend on the values
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    Layout lay;
    lay.batch = batch;
    lay.idist = n;
    lay.odist = n;
    const bool inverse = direction == FLAGFFT_INVERSE;
    std::string rows;
    double best = 1e30, def_ms = -1;
    NodePtr best_node;
    for (size_t i = 0; i < cands.size(); ++i) {
      double ms = -1;
      try {
        auto prog = lower(cands[i], pl, d.is_double, Transform::C2C, inverse, n, lay, false);
        for (int w = 0; w < 2; ++w) prog->run(in.ptr, out.ptr, st);
        std::vector<double> t;
        for (int r = 0; r < 3; ++r) {
          cudaEventRecord(e0, st);
          for (int k = 0; k < 10; ++k) prog->run(in.ptr, out.ptr, st);
          cudaEventRecord(e1, st);
          cudaEventSynchronize(e1);
          float el = 0;
          cudaEventElapsedTime(&el, e0, e1);
          t.push_back(el / 10.0);
        }
        std::sort(t.begin(), t.end());
        ms = t[1];
        if (cudaGetLastError() != cudaSuccess) ms = -1;
      } catch (const std::exception &) {
        ms = -1;
      }
      if (i == 0) def_ms = ms;
      if (ms > 0 && ms < best) {
        best = ms;
        best_node = cands[i];
      }
      rows += std::string(rows.empty() ? "" : ", ") + "{\"key\": \"" + cands[i]->key_repr() +
              "\", \"ms\": " + std::to_string(ms) + "}";
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (!best_node) return FLAGFFT_EXEC_FAILED;
    bool stored = false;
    const auto path = db_path ? std::optional<std::string>(db_path) : tune_db_path();
    if (path) {
      TuneKey k;
      k.device_arch = d.arch;
      k.fft_length = n;
      k.batch = batch;
      k.dtype = d.is_double ? "complex128" : "complex64";
      k.direction = inverse ? "inverse" : "forward";
      stored = tune_store(k, "{\"root\": " + best_node->to_json() + "}", best, "flagfft-b200-autotune", *path);
    }
    if (best_ms) *best_ms = best;
    const std::string rep = "{\"n\": " + std::to_string(n) + ", \"batch\": " + std::to_string(batch) +
                            ", \"best_ms\": " + std::to_string(best) + ", \"default_ms\": " +
                            std::to_string(def_ms) + ", \"stored\": " + (stored ? "true" : "false") +
                            ", \"best\": " + best_node->to_json() + ", \"candidates\": [" + rows + "]}";
    if (report && buflen > 0) {
      size_t c = std::min<size_t>(rep.size(), (size_t)buflen - 1);
      std::memcpy(report, rep.data(), c);
      report[c] = 0;
    }
    return FLAGFFT_SUCCESS;
  } catch (const std::bad_alloc &) {
    return FLAGFFT_ALLOC_FAILED;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "[flagfft] tune failed: %s\n", e.what());
    return FLAGFFT_SETUP_FAILED;
  }
#endif
}

extern "C" const char *flagfftB200PlanJson(flagfftHandle h) {
  Plan *plan = checked(h);
  if (plan == nullptr || plan->destroyed || !plan->initialized) return nullptr;
  return plan->json.c_str();
}

extern "C" int flagfftB200LaunchCount(flagfftHandle h, int direction) {
  Plan *plan = checked(h);
  if (plan == nullptr || plan->destroyed || !plan->initialized) return -1;
  if (plan->is_batch) {
    const BatchProgram *bp = direction == FLAGFFT_INVERSE ? plan->binv.get() : plan->bfwd.get();
    return bp ? bp->launches() : -1;
  }
  const Program *p = direction == FLAGFFT_INVERSE ? plan->inv.get() : plan->fwd.get();
  return p ? p->launches() : -1;
}

extern "C" flagfftResult flagfftB200PlanBatch(flagfftHandle *out, int ngroups, const int *lengths, const int *counts,
                                             flagfftType type) {
  if (out == nullptr) return FLAGFFT_INVALID_VALUE;
  *out = nullptr;
  if (ngroups <= 0 || lengths == nullptr || counts == nullptr) return FLAGFFT_INVALID_VALUE;
  if (type != FLAGFFT_C2C && type != FLAGFFT_Z2Z) return FLAGFFT_INVALID_TYPE;
  PlanDesc d;
  d.rank = 1;
  d.type = type;
  d.is_double = type == FLAGFFT_Z2Z;
  int64_t total = 0;
  std::vector<BatchGroup> groups;
  for (int g = 0; g < ngroups; ++g) {
    if (lengths[g] <= 0) return FLAGFFT_INVALID_SIZE;
    if (counts[g] <= 0) return FLAGFFT_INVALID_VALUE;
    groups.push_back({lengths[g], counts[g]});
    total += (int64_t)lengths[g] * counts[g];
  }
  d.n = {total};
  d.batch = 1;
  flagfftResult dr = ensure_device(d);
  if (dr != FLAGFFT_SUCCESS) return dr;
  try {
    auto plan = std::make_unique<Plan>();
    plan->desc = d;
    plan->is_batch = true;
    plan->groups = groups;
    Planner planner(d.is_double, d.smem_optin);
    const char *g = std::getenv("FLAGFFT_BATCH_GRAPH");
    const bool graphs = g == nullptr || std::string(g) != "0";
    plan->bfwd = lower_batch(groups, planner, d.is_double, false, graphs);
    plan->binv = lower_batch(groups, planner, d.is_double, true, graphs);
    plan->root = make_direct_node(total);  // placeholder: a batch plan has one tree per group
    plan->json = "{\"batch_groups\": " + std::to_string(ngroups) + "}";
    plan->initialized = true;
    auto h = std::make_unique<flagfftPlan_t>();
    h->impl = plan.release();
    *out = h.release();
    return FLAGFFT_SUCCESS;
  } catch (const std::bad_alloc &) {
    return FLAGFFT_ALLOC_FAILED;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "[flagfft] batch plan setup failed: %s\n", e.what());
    return FLAGFFT_SETUP_FAILED;
  }
}

extern "C" flagfftResult flagfftB200DeviceWaitFailures(long long *count) {
  if (count == nullptr) return FLAGFFT_INVALID_VALUE;
  const long long a = ffb::tcols_wait_failures<float>(), b = ffb::tcols_wait_failures<double>();
  if (a < 0 || b < 0) return FLAGFFT_INVALID_DEVICE;
  *count = a + b;
  return FLAGFFT_SUCCESS;
}
