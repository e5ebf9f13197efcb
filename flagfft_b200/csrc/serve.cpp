// Request server: continuous batching of transforms of mixed type, length and
// batch count on one GPU.
//
// Callers submit requests (type, n, batch, direction, device input / output)
// from any thread.  A scheduler thread admits pending requests in arrival
// order into a "tick" while the HBM budget allows (each request is charged
// its input, output and workspace bytes) and a tick slot is free, lowers each
// request from a per-(type, n, direction) template program that stays
// resident (tables shared process-wide), and runs the tick's passes the way a
// batch plan does: pass p of every request forms phase p, whose ping-pong and
// register-column tiles go through one persistent work-queue launch per
// shared-memory class; other passes launch on their own.  Up to `max_ticks`
// ticks are in flight on their own streams, so requests that arrive while
// others run are admitted as soon as a slot and memory free up, and their work
// overlaps on the device.  A request's tiles depend only on the request
// itself, so its result is the same alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/flagfft_b200.h"
#include "batch.cuh"
#include "exec_internal.hpp"

namespace ffb {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool is_double_type(flagfftType t) { return t == FLAGFFT_Z2Z || t == FLAGFFT_D2Z || t == FLAGFFT_Z2D; }

// Element sizes (bytes) of a type's input and output.
void io_elems(flagfftType t, int64_t n, int64_t *in_b, int64_t *out_b) {
  const int64_t h = n / 2 + 1;
  switch (t) {
    case FLAGFFT_C2C: *in_b = 8 * n; *out_b = 8 * n; return;
    case FLAGFFT_Z2Z: *in_b = 16 * n; *out_b = 16 * n; return;
    case FLAGFFT_R2C: *in_b = 4 * n; *out_b = 8 * h; return;
    case FLAGFFT_D2Z: *in_b = 8 * n; *out_b = 16 * h; return;
    case FLAGFFT_C2R: *in_b = 8 * h; *out_b = 4 * n; return;
    case FLAGFFT_Z2D: *in_b = 16 * h; *out_b = 8 * n; return;
  }
  *in_b = *out_b = 0;
}

// A lowered program for batch 2 whose passes are re-targeted per request:
// a pass's batch dimension is nbatch when the template has nbatch == 2, else
// G (single-pass lowerings put the batch in G); workspaces scale per
// transform.
struct Template {
  std::unique_ptr<Program> prog;
  size_t ws0_per = 0, ws1_per = 0;  // workspace bytes per transform
};

struct Request {
  int64_t id = 0;
  flagfftType type = FLAGFFT_C2C;
  int64_t n = 0, batch = 0;
  int dir = FLAGFFT_FORWARD;
  const void *in = nullptr;
  void *out = nullptr;
  const Template *tpl = nullptr;
  size_t bytes = 0;  // budget charge
  double t_submit = 0, t_done = -1;
  int state = 0;  // 0 pending, 1 in flight, 2 done, 3 failed
  void *ws0 = nullptr, *ws1 = nullptr;
};

// Device arrays of one tick's persistent launches (one precision).
template <typename T>
struct TickWork {
  std::vector<TileArgs<T>> args;
  std::vector<int> kinds;
  std::vector<int> arg_phase, arg_cls;  // (phase, class) of each args entry
  std::vector<BatchItem> items;
  struct Launch {
    int first = 0, count = 0, threads = 0;
    size_t smem = 0;
  };
  std::vector<std::vector<Launch>> phases;  // [phase][class]
  // One device buffer holds the tick's arguments, kinds, items and zeroed
  // work-queue counters (16-byte aligned sections), filled from one pinned
  // host buffer by one copy.  A slot's next tick reuses both only after the
  // slot's previous tick finished on the device.  They grow without any
  // device-wide synchronisation: the device buffer is stream-ordered
  // (cudaMallocAsync / cudaFreeAsync on the slot's stream) and outgrown
  // pinned buffers are kept until the server ends (cudaFree and
  // cudaFreeHost wait for the whole device: a growth under load once held
  // the scheduler for half a second).
  void *d_all = nullptr;
  size_t cap = 0;
  void *h_all = nullptr;
  std::vector<void *> old_h;
  size_t off_kinds = 0, off_items = 0, off_counters = 0;
  const TileArgs<T> *dev_args() const { return reinterpret_cast<const TileArgs<T> *>(d_all); }
  const int *dev_kinds() const { return reinterpret_cast<const int *>(static_cast<char *>(d_all) + off_kinds); }
  const BatchItem *dev_items() const {
    return reinterpret_cast<const BatchItem *>(static_cast<char *>(d_all) + off_items);
  }
  int *dev_counters() const { return reinterpret_cast<int *>(static_cast<char *>(d_all) + off_counters); }
  // Room for `bytes` of arguments, kinds, items and counters; outgrown
  // buffers are released as the class comment says.
  bool reserve(size_t bytes, cudaStream_t st) {
    if (d_all && cap >= bytes) return true;
    void *nd = nullptr, *nh = nullptr;
#ifndef FFB_HOST_EMULATION
    if (cudaMallocAsync(&nd, bytes, st) != cudaSuccess) return false;
    if (d_all) cudaFreeAsync(d_all, st);
    if (cudaMallocHost(&nh, bytes) != cudaSuccess) nh = nullptr;
#else
    (void)st;
    nd = std::malloc(bytes);
    std::free(d_all);
    nh = std::malloc(bytes);
#endif
    d_all = nd;
    old_h.push_back(h_all);
    h_all = nh;
    cap = bytes;
    return nh != nullptr;
  }
  ~TickWork() {  // (the server synchronised the slot's stream before)
    old_h.push_back(h_all);
#ifndef FFB_HOST_EMULATION
    if (d_all) cudaFree(d_all);
    for (void *h : old_h)
      if (h) cudaFreeHost(h);
#else
    std::free(d_all);
    for (void *h : old_h) std::free(h);
#endif
  }
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<std::shared_ptr<Request>> reqs;
  TickWork<float> wf;
  TickWork<double> wd;
  void *ws = nullptr;  // the tick's workspaces, one allocation carved per request
  cudaEvent_t start = nullptr;  // ($FLAGFFT_SERVE_TRACE) the tick's first launch
};

template <typename T>
void upload_grow(DevPtr &d, size_t &cap, const void *host, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return;
  if (!d || cap < bytes) {
    cap = std::max(bytes, cap * 2);
    d = std::make_shared<DevMem>(cap);
  }
#ifndef FFB_HOST_EMULATION
  cudaMemcpyAsync(d->ptr, host, bytes, cudaMemcpyHostToDevice, st);
#else
  (void)st;
  std::memcpy(d->ptr, host, bytes);
#endif
}

}  // namespace

class Server {
 public:
  Server(int64_t budget, int max_ticks) : budget_(budget), slots_(std::max(1, max_ticks)) {
    const char *tr = std::getenv("FLAGFFT_SERVE_TRACE");
    trace_ = tr && tr[0] == '1';
#ifndef FFB_HOST_EMULATION
    cudaGetDevice(&device_);
    for (Slot &s : slots_) {
      cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
      // tick buffers for large ticks up front: growing pinned memory under
      // load (page-locking megabytes) held the scheduler for a fifth of a second
      s.wf.reserve(kTickBufferBytes, s.stream);
      s.wd.reserve(kTickBufferBytes, s.stream);
      cudaEventCreateWithFlags(&s.done, trace_ ? cudaEventDefault : cudaEventDisableTiming);
      if (trace_) cudaEventCreate(&s.start);
    }
    // keep freed workspace in the stream-ordered pool between ticks, and
    // grow the pool once now (an eighth of the budget, at most 4 GB) rather
    // than under load, where mapping new memory stalled a tick
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      const size_t reserve = (size_t)std::min<int64_t>(budget_ / 8, (int64_t)4 << 30);
      void *p = nullptr;
      if (reserve && cudaMallocAsync(&p, reserve, slots_[0].stream) == cudaSuccess) {
        cudaFreeAsync(p, slots_[0].stream);
        cudaStreamSynchronize(slots_[0].stream);
      }
    }
    cudaGetLastError();
#endif
    worker_ = std::thread([this] { loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    worker_.join();
    if (trace_)
      std::fprintf(stderr,
                   "[flagfft] server trace: ticks %lld, requests %lld, largest tick %lld requests, host time in tick "
                   "assembly and launch %.1f ms (longest %.2f ms, %lld requests), device time of ticks %.1f ms "
                   "(longest %.2f ms), longest scheduler pass with ticks in flight %.2f ms\n",
                   (long long)ticks_, (long long)completed_, (long long)max_tick_reqs_, host_launch_s_ * 1e3,
                   max_host_tick_s_ * 1e3, (long long)max_host_tick_reqs_, device_tick_ms_, max_device_tick_ms_,
                   max_loop_gap_s_ * 1e3);
#ifndef FFB_HOST_EMULATION
    for (Slot &s : slots_) {
      if (s.stream) cudaStreamSynchronize(s.stream);
      if (s.stream) cudaStreamDestroy(s.stream);
      if (s.done) cudaEventDestroy(s.done);
      if (s.start) cudaEventDestroy(s.start);
    }
#endif
  }

  flagfftResult prepare(flagfftType type, int64_t n, int dir) {
    try {
      std::lock_guard<std::mutex> lock(tpl_mu_);
      if (!template_for(type, n, dir)) return FLAGFFT_SETUP_FAILED;
    } catch (const std::bad_alloc &) {
      return FLAGFFT_ALLOC_FAILED;
    } catch (const std::exception &e) {
      std::fprintf(stderr, "[flagfft] server prepare failed: %s\n", e.what());
      return FLAGFFT_SETUP_FAILED;
    }
#ifndef FFB_HOST_EMULATION
    // One transform of the template through the tick path: the first launch
    // of each kernel it takes loads that kernel (lazy module loading), a
    // stall of the scheduler thread of up to milliseconds that, under load,
    // would land on the requests queued behind it.
    int64_t ib = 0, ob = 0;
    io_elems(type, n, &ib, &ob);
    void *in = nullptr, *out = nullptr;
    if (cudaMalloc(&in, (size_t)ib) != cudaSuccess || cudaMalloc(&out, (size_t)ob) != cudaSuccess) {
      cudaGetLastError();
      if (in) cudaFree(in);
      return FLAGFFT_ALLOC_FAILED;
    }
    cudaMemsetAsync(in, 0, (size_t)ib, cudaStreamPerThread);
    cudaStreamSynchronize(cudaStreamPerThread);
    int64_t id = 0;
    flagfftResult st = submit(type, n, 1, dir, in, out, &id);
    if (st == FLAGFFT_SUCCESS) st = wait(id, nullptr);
    cudaFree(in);
    cudaFree(out);
    return st;
#else
    return FLAGFFT_SUCCESS;
#endif
  }

  flagfftResult submit(flagfftType type, int64_t n, int64_t batch, int dir, const void *in, void *out, int64_t *id) {
    const Template *tpl = nullptr;
    try {
      std::lock_guard<std::mutex> lock(tpl_mu_);
      tpl = template_for(type, n, dir);
    } catch (const std::bad_alloc &) {
      return FLAGFFT_ALLOC_FAILED;
    } catch (const std::exception &e) {
      std::fprintf(stderr, "[flagfft] server: no program for n=%lld: %s\n", (long long)n, e.what());
      return FLAGFFT_SETUP_FAILED;
    }
    if (!tpl) return FLAGFFT_SETUP_FAILED;
    auto r = std::make_shared<Request>();
    r->type = type;
    r->n = n;
    r->batch = batch;
    r->dir = dir;
    r->in = in;
    r->out = out;
    r->tpl = tpl;
    int64_t ib = 0, ob = 0;
    io_elems(type, n, &ib, &ob);
    r->bytes = (size_t)batch * (size_t)(ib + ob) + (size_t)batch * (tpl->ws0_per + tpl->ws1_per);
    if ((int64_t)r->bytes > budget_) return FLAGFFT_INVALID_SIZE;
    r->t_submit = now_s();
    {
      std::lock_guard<std::mutex> lock(mu_);
      r->id = ++next_id_;
      *id = r->id;
      all_[r->id] = r;
      pending_.push_back(r);
    }
    cv_.notify_all();
    return FLAGFFT_SUCCESS;
  }

  flagfftResult wait(int64_t id, double *latency_ms) {
    std::unique_lock<std::mutex> lock(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) return FLAGFFT_INVALID_VALUE;
    std::shared_ptr<Request> r = it->second;
    done_cv_.wait(lock, [&] { return r->state >= 2; });
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
    all_.erase(id);
    return r->state == 2 ? FLAGFFT_SUCCESS : FLAGFFT_EXEC_FAILED;
  }

  // wait() bounded by timeout_ms: *done = 0 (ticket kept) when the request
  // has not finished by then.
  flagfftResult wait_for(int64_t id, double timeout_ms, double *latency_ms, int *done) {
    std::unique_lock<std::mutex> lock(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) return FLAGFFT_INVALID_VALUE;
    std::shared_ptr<Request> r = it->second;
    const bool fin = done_cv_.wait_for(lock, std::chrono::duration<double, std::milli>(std::max(0.0, timeout_ms)),
                                       [&] { return r->state >= 2; });
    *done = fin ? 1 : 0;
    if (!fin) return FLAGFFT_SUCCESS;
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
    all_.erase(id);
    return r->state == 2 ? FLAGFFT_SUCCESS : FLAGFFT_EXEC_FAILED;
  }

  void stats(int64_t *completed, int64_t *ticks, int64_t *in_use) {
    std::lock_guard<std::mutex> lock(mu_);
    if (completed) *completed = completed_;
    if (ticks) *ticks = ticks_;
    if (in_use) *in_use = in_use_;
  }

  // Continuous-batching evidence: the most ticks seen in flight at once, and
  // how many requests were admitted while another tick was on the GPU.
  void overlap(int64_t *max_in_flight, int64_t *admitted_while_busy) {
    std::lock_guard<std::mutex> lock(mu_);
    if (max_in_flight) *max_in_flight = max_in_flight_;
    if (admitted_while_busy) *admitted_while_busy = admitted_while_busy_;
  }

 private:
  // ---- templates
  const Template *template_for(flagfftType type, int64_t n, int dir) {
    const bool inv = type == FLAGFFT_C2R || type == FLAGFFT_Z2D || ((type == FLAGFFT_C2C || type == FLAGFFT_Z2Z) &&
                                                                    dir == FLAGFFT_INVERSE);
    const auto key = std::make_tuple((int)type, n, inv);
    auto it = tpls_.find(key);
    if (it != tpls_.end()) return it->second.get();
    const bool dbl = is_double_type(type);
    auto pl = planners_.find(dbl);
    if (pl == planners_.end()) pl = planners_.emplace(dbl, std::make_unique<Planner>(dbl, 232448)).first;
    const Transform tr = (type == FLAGFFT_R2C || type == FLAGFFT_D2Z)   ? Transform::R2C
                         : (type == FLAGFFT_C2R || type == FLAGFFT_Z2D) ? Transform::C2R
                                                                        : Transform::C2C;
    NodePtr root = build_raw_root(*pl->second, n, nullptr, nullptr);
    if (!raw_supported(root)) return nullptr;
    Layout lay;
    lay.batch = kTemplateBatch;
    int64_t ib = 0, ob = 0;
    io_elems(type, n, &ib, &ob);
    const int64_t esz_in = type == FLAGFFT_R2C ? 4 : type == FLAGFFT_D2Z ? 8 : dbl ? 16 : 8;
    const int64_t esz_out = type == FLAGFFT_C2R ? 4 : type == FLAGFFT_Z2D ? 8 : dbl ? 16 : 8;
    lay.idist = ib / esz_in;
    lay.odist = ob / esz_out;
    auto t = std::make_unique<Template>();
    t->prog = lower_batchable(root, *pl->second, dbl, tr, inv, n, lay);
    if (!servable(*t->prog)) return nullptr;
    t->ws0_per = t->prog->scratch0 ? t->prog->scratch0->bytes / kTemplateBatch : 0;
    t->ws1_per = t->prog->scratch1 ? t->prog->scratch1->bytes / kTemplateBatch : 0;
    const Template *raw = t.get();
    tpls_.emplace(key, std::move(t));
    return raw;
  }

  // Every pass of a template is a tile pass or re-sizes to a request's batch.
  static bool servable(const Program &prog) {
    for (const auto &pb : prog.passes)
      if (!dynamic_cast<const TilePass<float> *>(pb.get()) && !dynamic_cast<const TilePass<double> *>(pb.get()) &&
          !pb->rebatched(kTemplateBatch, kTemplateBatch))
        return false;
    return true;
  }

  // ---- tick assembly for one precision
  // (a template's tile passes carry its batch as the outer batch, or, for
  // single-pass lowerings, as the transform count per outer batch)
  template <typename T>
  static void retarget(TileArgs<T> &a, int64_t b) {
    if (a.nbatch == kTemplateBatch)
      a.nbatch = b;
    else
      a.G = (int)b;
  }

  // Adds request r's passes: persistent-capable ones to w, the others to own.
  template <typename T>
  static void add_request(TickWork<T> &w, const Request &r,
                          std::vector<std::vector<std::function<cudaError_t(cudaStream_t)>>> &own) {
    const Program &prog = *r.tpl->prog;
    for (size_t p = 0; p < prog.passes.size(); ++p) {
      if (w.phases.size() <= p) w.phases.resize(p + 1, std::vector<typename TickWork<T>::Launch>(kBatchClasses));
      if (own.size() <= p) own.resize(p + 1);
      const PassBase *pb = prog.passes[p].get();
      if (auto *tp = dynamic_cast<const TilePass<T> *>(pb)) {
        TileArgs<T> a = tp->a;
        retarget(a, r.batch);
        a.in = TilePass<T>::pick(tp->src, r.in, r.out, r.ws0, r.ws1);
        a.out = TilePass<T>::pick(tp->dst, r.in, r.out, r.ws0, r.ws1);
        size_t smem = tp->smem;
        int kind = -1;
        if (a.regcol) {
          kind = kBatchRegcol;
        } else if (!a.pp && !a.blue_cols && !a.tiles && tp->kind == CoreKind::Dit &&
                   (tp->io == IoKind::R2C || tp->io == IoKind::C2R)) {
          // a real request's on-chip core: the in-place tile body with the
          // pack / unpack, at the template's tile width
          kind = tp->io == IoKind::R2C ? kBatchR2C : kBatchC2R;
          if (smem + kBatchSmemHeader > 232448) kind = -1;
        } else if (a.pp && !a.blue_cols && !a.tiles && !a.rows_only && tp->io == IoKind::C2C) {
          kind = tp->kind == CoreKind::Dit         ? kBatchPpDit
                 : tp->kind == CoreKind::Bluestein ? kBatchPpBluestein
                 : tp->kind == CoreKind::Rader     ? kBatchPpRader
                                                   : kBatchPpConv;
          // the request's own tile width (independent of the other requests)
          const size_t per = pp_tile_smem(tp->a) / (size_t)tp->a.W;
          if (a.tpt <= kBatchWidth) {
            int64_t W = std::min<int64_t>({(int64_t)(kBatchWidth / a.tpt), (int64_t)a.G,
                                           (int64_t)std::max<size_t>(1, 110 * 1024 / per)});
            W = std::max<int64_t>(W, 1);
            if (W * std::llabs(a.ig) + a.core.L * std::llabs(a.ii) < (1ll << 31) &&
                W * std::llabs(a.og) + a.core.L * std::llabs(a.ok) < (1ll << 31)) {
              a.W = (int)W;
              a.wdiv = make_fastdiv((uint32_t)W);
            }
          }
          smem = per * (size_t)a.W;
          if (smem + kBatchSmemHeader > 232448) kind = -1;
        }
        if (kind < 0) {
          const CoreKind ck = tp->kind;
          const IoKind io = tp->io;
          own[p].push_back([a, ck, io, smem](cudaStream_t st) { return launch_tile<T>(a, ck, io, smem, st); });
          continue;
        }
        const int cls = batch_class(smem, a.W * a.tpt, kind == kBatchRegcol);
        auto &L = w.phases[p][(size_t)cls];
        L.threads = std::max(L.threads, kind == kBatchRegcol ? 128 : a.W * a.tpt);
        L.smem = std::max(L.smem, kind == kBatchRegcol ? (size_t)0 : smem);
        w.args.push_back(a);
        w.kinds.push_back(kind);
        w.arg_phase.push_back((int)p);
        w.arg_cls.push_back(cls);
        // items are numbered after all requests are in (tile counts need the class width)
      } else {
        // every other pass (Hermitian post / pre, widen / take, transposes)
        // at the request's batch; templates hold no other kind (servable())
        std::shared_ptr<PassBase> q = pb->rebatched(kTemplateBatch, r.batch);
        const void *in = r.in;
        void *out = r.out, *s0 = r.ws0, *s1 = r.ws1;
        own[p].push_back([q, in, out, s0, s1](cudaStream_t st) { return q->run(in, out, s0, s1, st); });
      }
    }
  }

  // Items of every (phase, class) of w, in the order args were added
  // (requests in arrival order), and the device uploads.
  template <typename T>
  static void finish_work(TickWork<T> &w) {
    const std::vector<int> &arg_phase = w.arg_phase, &arg_cls = w.arg_cls;
    w.items.clear();
    for (size_t p = 0; p < w.phases.size(); ++p)
      for (int c = 0; c < kBatchClasses; ++c) {
        auto &L = w.phases[p][(size_t)c];
        L.first = (int)w.items.size();
        for (size_t i = 0; i < w.args.size(); ++i) {
          if (arg_phase[i] != (int)p || arg_cls[i] != c) continue;
          const TileArgs<T> &a = w.args[i];
          const int width = w.kinds[i] == kBatchRegcol ? std::max(L.threads, 32) : a.W;
          const int tiles = (int)(((int64_t)a.G + width - 1) / width * a.nbatch);
          for (int t = 0; t < tiles; ++t) w.items.push_back({(int)i, t});
        }
        L.count = (int)w.items.size() - L.first;
      }
  }

  template <typename T>
  cudaError_t launch_work(TickWork<T> &w, size_t p, cudaStream_t st) {
    if (p >= w.phases.size()) return cudaSuccess;
    for (int c = 0; c < kBatchClasses; ++c) {
      const auto &L = w.phases[p][(size_t)c];
      if (L.count == 0) continue;
      // (every counter of the tick was zeroed once when the tick was assembled)
      int *counter = w.dev_counters() + p * kBatchClasses + (size_t)c;
      const int ctas = std::max(1, batch_resident_ctas<T>(std::max(L.threads, 32), L.smem));
      cudaError_t e = launch_batch<T>(w.dev_args(), w.dev_kinds(), w.dev_items() + L.first, L.count, counter,
                                      std::max(L.threads, 32), L.smem, ctas, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  // Builds and launches the tick of slot s (its requests already chosen).
  cudaError_t launch_tick(Slot &s) {
    TickWork<float> &wf = s.wf;
    TickWork<double> &wd = s.wd;
    wf.args.clear();
    wf.kinds.clear(); wf.phases.clear(); wf.arg_phase.clear(); wf.arg_cls.clear();
    wd.args.clear(); wd.kinds.clear(); wd.phases.clear(); wd.arg_phase.clear(); wd.arg_cls.clear();
    std::vector<std::vector<std::function<cudaError_t(cudaStream_t)>>> own;
    // every request's workspaces from one stream-ordered allocation per tick
    // (two allocations and two frees per request cost more host time than
    // the rest of a small request's assembly)
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    size_t ws_total = 0;
    for (auto &rp : s.reqs)
      ws_total += al(rp->tpl->ws0_per * (size_t)rp->batch) + al(rp->tpl->ws1_per * (size_t)rp->batch);
    if (ws_total) {
#ifndef FFB_HOST_EMULATION
      cudaError_t e = cudaMallocAsync(&s.ws, ws_total, s.stream);
      if (e != cudaSuccess) return e;
#else
      s.ws = std::malloc(ws_total);
#endif
    }
    size_t ws_at = 0;
    for (auto &rp : s.reqs) {
      Request &r = *rp;
      const size_t b0 = r.tpl->ws0_per * (size_t)r.batch, b1 = r.tpl->ws1_per * (size_t)r.batch;
      r.ws0 = b0 ? static_cast<char *>(s.ws) + ws_at : nullptr;
      ws_at += al(b0);
      r.ws1 = b1 ? static_cast<char *>(s.ws) + ws_at : nullptr;
      ws_at += al(b1);
      if (is_double_type(r.type))
        add_request<double>(wd, r, own);
      else
        add_request<float>(wf, r, own);
    }
    finish_work(wf);
    finish_work(wd);
    // uploads
    auto up = [&](auto &w) -> bool {
      if (w.args.empty()) return true;
      const size_t nc = w.phases.size() * kBatchClasses + 1;
      auto al = [](size_t v) { return (v + 15) / 16 * 16; };
      const size_t b_args = w.args.size() * sizeof(w.args[0]);
      w.off_kinds = al(b_args);
      w.off_items = w.off_kinds + al(w.kinds.size() * sizeof(int));
      w.off_counters = w.off_items + al(w.items.size() * sizeof(BatchItem));
      const size_t total = w.off_counters + nc * sizeof(int);
      if ((!w.d_all || w.cap < total) && !w.reserve(std::max({total, 2 * w.cap, (size_t)1 << 20}), s.stream))
        return false;
      char *h = static_cast<char *>(w.h_all);
      if (h == nullptr) return false;
      std::memcpy(h, w.args.data(), b_args);
      std::memcpy(h + w.off_kinds, w.kinds.data(), w.kinds.size() * sizeof(int));
      std::memcpy(h + w.off_items, w.items.data(), w.items.size() * sizeof(BatchItem));
      std::memset(h + w.off_counters, 0, nc * sizeof(int));  // every work-queue counter starts at zero
#ifndef FFB_HOST_EMULATION
      return cudaMemcpyAsync(w.d_all, h, total, cudaMemcpyHostToDevice, s.stream) == cudaSuccess;
#else
      std::memcpy(w.d_all, h, total);
      return true;
#endif
    };
    if (!up(wf) || !up(wd)) return cudaErrorMemoryAllocation;
    const size_t nph = std::max({wf.phases.size(), wd.phases.size(), own.size()});
    for (size_t p = 0; p < nph; ++p) {
      if (p < own.size())
        for (auto &f : own[p]) {
          cudaError_t e = f(s.stream);
          if (e != cudaSuccess) return e;
        }
      cudaError_t e = launch_work(wf, p, s.stream);
      if (e == cudaSuccess) e = launch_work(wd, p, s.stream);
      if (e != cudaSuccess) return e;
    }
    for (auto &rp : s.reqs) rp->ws0 = rp->ws1 = nullptr;
#ifndef FFB_HOST_EMULATION
    if (s.ws) cudaFreeAsync(s.ws, s.stream);
    s.ws = nullptr;
    return cudaEventRecord(s.done, s.stream);
#else
    std::free(s.ws);
    s.ws = nullptr;
    return cudaSuccess;
#endif
  }

  void retire(Slot &s, bool ok) {
#ifndef FFB_HOST_EMULATION
    if (trace_ && ok && s.start) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, s.start, s.done) == cudaSuccess) {
        device_tick_ms_ += ms;
        max_device_tick_ms_ = std::max(max_device_tick_ms_, (double)ms);
      }
      cudaGetLastError();
    }
#endif
    const double t = now_s();
    for (auto &rp : s.reqs) {
      rp->t_done = t;
      rp->state = ok ? 2 : 3;
      in_use_ -= (int64_t)rp->bytes;
      ++completed_;
    }
    s.reqs.clear();
    s.busy = false;
  }

  void loop() {
#ifndef FFB_HOST_EMULATION
    PdlOff no_pdl;  // this thread feeds several streams at once
#endif
    std::unique_lock<std::mutex> lock(mu_);
    double t_iter = now_s();
    while (true) {
      if (trace_) {  // the longest stretch between two passes of the loop while ticks were in flight
        const double t = now_s();
        bool any = false;
        for (Slot &s : slots_) any = any || s.busy;
        if (any) max_loop_gap_s_ = std::max(max_loop_gap_s_, t - t_iter);
        t_iter = t;
      }
      bool progressed = false;
      // retire finished ticks
      for (Slot &s : slots_) {
        if (!s.busy) continue;
#ifndef FFB_HOST_EMULATION
        cudaError_t q = cudaEventQuery(s.done);
        if (q == cudaErrorNotReady) continue;
        retire(s, q == cudaSuccess);
#else
        retire(s, true);
#endif
        progressed = true;
      }
      if (progressed) done_cv_.notify_all();
      // admit pending requests into a free slot
      Slot *free_slot = nullptr;
      for (Slot &s : slots_)
        if (!s.busy) {
          free_slot = &s;
          break;
        }
      // Under load (a tick already on the GPU) requests gather into fewer,
      // larger ticks: a tick starts once kCoalesceMin requests are pending
      // or the oldest has waited kCoalesceWait; with the GPU idle it starts
      // at once.  (Assembling a tick costs host time per tick, so at high
      // arrival rates small ticks cap the throughput: at 50k requests/s
      // with 16 / 50 us the scheduler thread saturated near 48k/s.)
      bool gpu_busy = false;
      for (Slot &s : slots_) gpu_busy = gpu_busy || s.busy;
      const bool start = !pending_.empty() && (!gpu_busy || stop_ || pending_.size() >= kCoalesceMin ||
                                               now_s() - pending_.front()->t_submit >= kCoalesceWait);
      if (free_slot && start) {
        while (!pending_.empty() && in_use_ + (int64_t)pending_.front()->bytes <= budget_ &&
               free_slot->reqs.size() < kMaxPerTick) {
          auto r = pending_.front();
          pending_.pop_front();
          in_use_ += (int64_t)r->bytes;
          r->state = 1;
          free_slot->reqs.push_back(r);
        }
        if (!free_slot->reqs.empty()) {
          if (gpu_busy) admitted_while_busy_ += (int64_t)free_slot->reqs.size();
          free_slot->busy = true;
          ++ticks_;
          int64_t in_flight = 0;
          for (Slot &s : slots_) in_flight += s.busy ? 1 : 0;
          max_in_flight_ = std::max(max_in_flight_, in_flight);
          lock.unlock();
#ifndef FFB_HOST_EMULATION
          cudaSetDevice(device_);
#endif
          max_tick_reqs_ = std::max<int64_t>(max_tick_reqs_, (int64_t)free_slot->reqs.size());
          const double th0 = trace_ ? now_s() : 0.0;
#ifndef FFB_HOST_EMULATION
          if (trace_ && free_slot->start) cudaEventRecord(free_slot->start, free_slot->stream);
#endif
          cudaError_t e = launch_tick(*free_slot);
          if (trace_) {
            const double dt = now_s() - th0;
            host_launch_s_ += dt;
            if (dt > max_host_tick_s_) {
              max_host_tick_s_ = dt;
              max_host_tick_reqs_ = (int64_t)free_slot->reqs.size();
            }
          }
          lock.lock();
          if (e != cudaSuccess) {
            std::fprintf(stderr, "[flagfft] server tick failed: %s\n", cudaGetErrorString(e));
            cudaGetLastError();
#ifndef FFB_HOST_EMULATION
            if (free_slot->ws) cudaFreeAsync(free_slot->ws, free_slot->stream);
            cudaStreamSynchronize(free_slot->stream);
#else
            std::free(free_slot->ws);
#endif
            free_slot->ws = nullptr;
            retire(*free_slot, false);
            done_cv_.notify_all();
          }
          continue;
        }
      }
      if (stop_ && pending_.empty()) {
        bool any = false;
        for (Slot &s : slots_) any = any || s.busy;
        if (!any) return;
      }
      bool busy = false;
      for (Slot &s : slots_) busy = busy || s.busy;
      if (busy)
        cv_.wait_for(lock, std::chrono::microseconds(20));
      else
        cv_.wait_for(lock, std::chrono::milliseconds(5), [&] { return stop_ || !pending_.empty(); });
    }
  }

  static constexpr size_t kMaxPerTick = 4096;
  static constexpr size_t kTickBufferBytes = 16u << 20;  // per slot and precision, reserved at creation
  static constexpr int64_t kTemplateBatch = 2;  // transforms a template program is lowered for
  static constexpr size_t kCoalesceMin = 32;
  static constexpr double kCoalesceWait = 100e-6;  // seconds

  int64_t budget_;
  int device_ = 0;
  std::vector<Slot> slots_;
  std::thread worker_;
  std::mutex mu_, tpl_mu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  std::deque<std::shared_ptr<Request>> pending_;
  std::unordered_map<int64_t, std::shared_ptr<Request>> all_;
  int64_t next_id_ = 0, completed_ = 0, ticks_ = 0, in_use_ = 0;
  int64_t max_in_flight_ = 0, admitted_while_busy_ = 0;
  bool trace_ = false;  // $FLAGFFT_SERVE_TRACE=1: tick timing, printed at destruction
  int64_t max_tick_reqs_ = 0;
  double host_launch_s_ = 0.0, device_tick_ms_ = 0.0, max_host_tick_s_ = 0.0, max_device_tick_ms_ = 0.0;
  int64_t max_host_tick_reqs_ = 0;
  double max_loop_gap_s_ = 0.0;
  std::map<std::tuple<int, int64_t, bool>, std::unique_ptr<Template>> tpls_;
  std::map<bool, std::unique_ptr<Planner>> planners_;
};

}  // namespace ffb

struct flagfftB200Server_st {
  ffb::Server *impl = nullptr;
};

using ffb::Server;

extern "C" flagfftResult flagfftB200ServerCreate(flagfftB200Server *srv, long long hbm_budget_bytes, int max_ticks) {
  if (srv == nullptr) return FLAGFFT_INVALID_VALUE;
  *srv = nullptr;
  if (hbm_budget_bytes <= 0 || max_ticks <= 0) return FLAGFFT_INVALID_VALUE;
#ifndef FFB_HOST_EMULATION
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
    cudaGetLastError();
    return FLAGFFT_INVALID_DEVICE;
  }
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) return FLAGFFT_INVALID_DEVICE;
#endif
  try {
    auto h = std::make_unique<flagfftB200Server_st>();
    h->impl = new Server(hbm_budget_bytes, max_ticks);
    *srv = h.release();
    return FLAGFFT_SUCCESS;
  } catch (const std::bad_alloc &) {
    return FLAGFFT_ALLOC_FAILED;
  } catch (const std::exception &) {
    return FLAGFFT_SETUP_FAILED;
  }
}

static bool server_type_ok(flagfftType t) {
  return t == FLAGFFT_C2C || t == FLAGFFT_Z2Z || t == FLAGFFT_R2C || t == FLAGFFT_D2Z || t == FLAGFFT_C2R ||
         t == FLAGFFT_Z2D;
}

extern "C" flagfftResult flagfftB200ServerPrepare(flagfftB200Server srv, flagfftType type, int n, int direction) {
  if (srv == nullptr || srv->impl == nullptr) return FLAGFFT_INVALID_PLAN;
  if (!server_type_ok(type)) return FLAGFFT_INVALID_TYPE;
  if (n <= 0) return FLAGFFT_INVALID_SIZE;
  return srv->impl->prepare(type, n, direction);
}

extern "C" flagfftResult flagfftB200ServerSubmit(flagfftB200Server srv, flagfftType type, int n, int batch,
                                                 int direction, const void *idata, void *odata, long long *ticket) {
  if (srv == nullptr || srv->impl == nullptr) return FLAGFFT_INVALID_PLAN;
  if (!server_type_ok(type)) return FLAGFFT_INVALID_TYPE;
  if (n <= 0) return FLAGFFT_INVALID_SIZE;
  if (batch <= 0 || batch > 65535 || idata == nullptr || odata == nullptr || ticket == nullptr)
    return FLAGFFT_INVALID_VALUE;
  if ((type == FLAGFFT_C2C || type == FLAGFFT_Z2Z) && direction != FLAGFFT_FORWARD && direction != FLAGFFT_INVERSE)
    return FLAGFFT_INVALID_VALUE;
  int64_t id = 0;
  flagfftResult r = srv->impl->submit(type, n, batch, direction, idata, odata, &id);
  *ticket = id;
  return r;
}

extern "C" flagfftResult flagfftB200ServerWait(flagfftB200Server srv, long long ticket, double *latency_ms) {
  if (srv == nullptr || srv->impl == nullptr) return FLAGFFT_INVALID_PLAN;
  return srv->impl->wait(ticket, latency_ms);
}

extern "C" flagfftResult flagfftB200ServerWaitFor(flagfftB200Server srv, long long ticket, double timeout_ms,
                                                  double *latency_ms, int *done) {
  if (srv == nullptr || srv->impl == nullptr || done == nullptr) return FLAGFFT_INVALID_VALUE;
  return srv->impl->wait_for(ticket, timeout_ms, latency_ms, done);
}

extern "C" flagfftResult flagfftB200ServerOverlap(flagfftB200Server srv, long long *max_ticks_in_flight,
                                                 long long *admitted_while_busy) {
  if (srv == nullptr || srv->impl == nullptr) return FLAGFFT_INVALID_VALUE;
  int64_t a = 0, b = 0;
  srv->impl->overlap(&a, &b);
  if (max_ticks_in_flight) *max_ticks_in_flight = a;
  if (admitted_while_busy) *admitted_while_busy = b;
  return FLAGFFT_SUCCESS;
}

extern "C" flagfftResult flagfftB200ServerStats(flagfftB200Server srv, long long *completed, long long *ticks,
                                                long long *bytes_in_use) {
  if (srv == nullptr || srv->impl == nullptr) return FLAGFFT_INVALID_PLAN;
  int64_t c = 0, t = 0, u = 0;
  srv->impl->stats(&c, &t, &u);
  if (completed) *completed = c;
  if (ticks) *ticks = t;
  if (bytes_in_use) *bytes_in_use = u;
  return FLAGFFT_SUCCESS;
}

extern "C" flagfftResult flagfftB200ServerDestroy(flagfftB200Server srv) {
  if (srv == nullptr) return FLAGFFT_INVALID_PLAN;
  delete srv->impl;
  delete srv;
  return FLAGFFT_SUCCESS;
}
