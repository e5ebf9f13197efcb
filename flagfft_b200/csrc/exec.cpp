// Lowering of plan trees onto on-chip FFT passes.
//
// Node -> pass mapping (reference node shapes from src/exec/raw_nodes.cpp):
//   leaf, or a four-step whose children flatten into radix lists, when the
//   whole length fits one CTA              -> one pass (DIT core)
//   Bluestein / Rader whose convolution fits one CTA
//                                          -> one fused pass (chirp or
//                                             permutation, forward FFT,
//                                             kernel product, inverse FFT,
//                                             unchirp / unpermute)
//   four-step whose children each fit      -> two passes through a workspace:
//                                             column FFTs with the W_N^{j2 k1}
//                                             twiddle fused into their store,
//                                             then row FFTs
//   R2C / C2R of even n                    -> the n/2-point complex core with
//                                             the pack / unpack fused into its
//                                             load and store
//   2-D RTRT                               -> a row pass and an in-place
//                                             column-tile pass (no transposes)
#include "exec.hpp"

#include <algorithm>
#include <functional>
#include <map>
#include <mutex>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>

#include "batch.cuh"
#include "exec_internal.hpp"
#include "tables.hpp"

namespace ffb {

#ifndef FFB_HOST_EMULATION
static thread_local bool t_pdl_off = false;

bool pdl_enabled() {
  static const bool on = [] {
    const char *v = std::getenv("FLAGFFT_PDL");
    return !(v && v[0] == '0');
  }();
  return on && !t_pdl_off;
}

PdlOff::PdlOff() : prev(t_pdl_off) { t_pdl_off = true; }
PdlOff::~PdlOff() { t_pdl_off = prev; }
#endif

// Host-side fault injection for tests: with FLAGFFT_FAULT_ALLOC=1 every
// device allocation a plan makes fails as if the device were out of memory
// (plan creation then returns FLAGFFT_ALLOC_FAILED).  Off unless set.
static bool alloc_fault_injected() {
  const char *v = std::getenv("FLAGFFT_FAULT_ALLOC");
  return v && v[0] == '1';
}

#ifndef FFB_HOST_EMULATION
DevMem::DevMem(size_t n) : bytes(n) {
  if (n == 0) return;
  if (alloc_fault_injected()) throw std::bad_alloc();
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    throw std::bad_alloc();
  }
}

DevMem::~DevMem() {
  if (ptr) cudaFree(ptr);
}

DevPtr upload(const void *host, size_t bytes) {
  auto m = std::make_shared<DevMem>(bytes);
  if (bytes && cudaMemcpy(m->ptr, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error("table upload failed");
  }
  return m;
}
#else
// Host-emulation build: "device" memory is host memory.
DevMem::DevMem(size_t n) : bytes(n) {
  if (n == 0) return;
  if (alloc_fault_injected()) throw std::bad_alloc();
  ptr = std::malloc(n);
  if (!ptr) throw std::bad_alloc();
}

DevMem::~DevMem() { std::free(ptr); }

DevPtr upload(const void *host, size_t bytes) {
  auto m = std::make_shared<DevMem>(bytes);
  if (bytes) std::memcpy(m->ptr, host, bytes);
  return m;
}
#endif

// Process-wide cache of plan tables (twiddles, chirps, kernel spectra,
// permutations) keyed by device and content: plans of the same lengths share
// one device copy, and a table lives while any plan holds it.
namespace {
std::mutex g_table_mu;
std::map<std::string, std::weak_ptr<DevMem>> g_tables;

int current_device() {
#ifdef FFB_HOST_EMULATION
  return 0;
#else
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return d;
#endif
}
}  // namespace

DevPtr shared_table(const std::string &key, const std::function<DevPtr()> &make) {
  const std::string k = std::to_string(current_device()) + "|" + key;
  std::lock_guard<std::mutex> lock(g_table_mu);
  auto it = g_tables.find(k);
  if (it != g_tables.end()) {
    if (DevPtr d = it->second.lock()) return d;
  }
  DevPtr d = make();
  g_tables[k] = d;
  return d;
}

cudaError_t Program::run(const void *in, void *out, cudaStream_t st) const {
  void *s0 = scratch0 ? scratch0->ptr : nullptr;
  void *s1 = scratch1 ? scratch1->ptr : nullptr;
  for (const auto &p : passes) {
    cudaError_t e = p->run(in, out, s0, s1, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

std::string Program::describe() const {
  std::ostringstream o;
  for (size_t i = 0; i < passes.size(); ++i) o << (i ? "\n" : "") << "  pass " << i << ": " << passes[i]->describe();
  return o.str();
}

int Program::launches() const {
  int n = 0;
  for (const auto &p : passes) n += p->launches();
  return n;
}

int64_t max_onchip_length(bool is_double) {
  // (padded(L) + one spare group) complex elements within the 227 KB opt-in limit
  const int64_t limit = 232448;
  const int64_t elem = is_double ? 16 : 8;
  const int64_t g = is_double ? 8 : 16;
  return (limit / elem - g) / g * g;
}

namespace {

// What one CTA-resident transform needs.
struct CoreSpec {
  CoreKind kind = CoreKind::Dit;
  int64_t n = 0;  // logical transform length
  int64_t L = 0;  // buffer (core) length
  std::vector<int> radices;
  NodePtr node;
};

// Radix list of a node that runs as one chain of stages, or empty.
static std::vector<int> flatten(const NodePtr &node) {
  if (!node) return {};
  if (node->kind == NodeKind::CtLeaf) {
    std::vector<int> r;
    for (int64_t f : node->factors) r.push_back((int)f);
    return r;
  }
  if (node->kind == NodeKind::FourStep) {
    const auto a = flatten(node->row);
    const auto b = flatten(node->col);
    if (a.empty() || b.empty()) return {};
    std::vector<int> r(a);
    for (int v : b) r.push_back(v);
    return r;
  }
  return {};
}

// ---------------------------------------------------------------------------
// Convolution length of a Bluestein node.  Any M >= 2n - 1 gives the same
// DFT; the plan's M is the reference planner's choice for its own kernels.
// The executor runs the convolution at the length its own stages do fastest:
// the one minimising M x (per-element cost of its cheapest radix chain).
// Per element-stage cost in instructions: a fixed part for addressing, the
// two shared-memory accesses, loop control and twiddle (kStageFixed), plus the
// codelet's and the twiddle multiply's arithmetic (~0.6 instructions per flop
// with fused multiply-adds).
// ---------------------------------------------------------------------------
namespace {
constexpr double kStageFixed = 28.0;

// flops of the forward codelet of radix R (engine.cuh's Dft / DftPrime /
// DftSplit structure)
double codelet_flops(int R) {
  switch (R) {
    case 2: return 4;
    case 3: return 12;
    case 4: return 16;
    case 6: return 48;
    case 8: return 56;
    case 9: return 96;
    case 10: return 148;
    case 12: return 132;
    case 15: return 264;
    case 16: return 173;
    default: {  // odd prime: pairs, then (R-1)/2 outputs of (R-1)/2 fused terms each
      const double H = (R - 1) / 2.0;
      return 8 * H * H + 10 * H;
    }
  }
}

double stage_cost(int R) { return kStageFixed + 0.6 * (codelet_flops(R) / R + 6.0 * (R - 1) / R); }

// Cheapest chain of supported radices with product m (per element), radices
// largest first; infinite when m has a prime factor above 19.
double chain_cost(int64_t m, std::vector<int> *radices, std::unordered_map<int64_t, std::pair<double, int>> &memo) {
  if (m == 1) {
    if (radices) radices->clear();
    return 0.0;
  }
  auto it = memo.find(m);
  if (it == memo.end()) {
    double best = 1e30;
    int best_r = 0;
    for (int64_t R : kSupportedRadices) {
      if (m % R) continue;
      const double c = stage_cost((int)R) + chain_cost(m / R, nullptr, memo);
      if (c < best) {
        best = c;
        best_r = (int)R;
      }
    }
    it = memo.emplace(m, std::make_pair(best, best_r)).first;
  }
  const double cost = it->second.first;
  if (radices) {
    // every value on the best chain was memoised by the recursion above
    radices->clear();
    for (int64_t v = m; v > 1 && memo.at(v).second != 0; v /= memo.at(v).second) radices->push_back(memo.at(v).second);
    std::sort(radices->rbegin(), radices->rend());
  }
  return cost;
}

// TMA column passes: on unless FLAGFFT_TMA_COLUMNS=0 (read at plan time).
static bool tma_columns_enabled() {
  const char *v = std::getenv("FLAGFFT_TMA_COLUMNS");
  return !(v && std::string(v) == "0");
}

// Set while lowering batch groups: the one-pass four-step Bluestein and the
// strided tile kernels (their own launches) give way to lowerings whose
// passes join the persistent launches.
thread_local bool t_no_one_pass = false;

// One-pass Bluestein in the pair form ($FLAGFFT_BLUESTEIN_PAIR=1, read at
// plan time): the N1 convolution rows split over a two-CTA cluster, in both
// precisions, instead of one CTA (single precision) or the three-pass chain
// (double precision).  Off by default: on B200 it measured slower at the
// benchmark lengths (C2C 10007 x 1024: 208.8 us against 176.7 us for one CTA,
// both before the product-form column twiddles they share; Z2Z 10007 x 256:
// 123.2 us against 102 us for three passes) -- a pair CTA runs 12 warps, and
// its row phase is no more efficient than the chain's.
bool bluestein_pair() {
  const char *v = std::getenv("FLAGFFT_BLUESTEIN_PAIR");
  return v && v[0] == '1';
}

// The compile-time radix sequence of length L (FFB_FIXED_SEQUENCES), if it
// has one: such a length runs on a row kernel with every index constant.
bool fixed_sequence(int64_t L, std::vector<int> *r) {
#define FFB_SEQ(len, ...)        \
  if (L == (len)) {              \
    if (r) *r = {__VA_ARGS__};   \
    return true;                 \
  }
  FFB_FIXED_SEQUENCES(FFB_SEQ)
#undef FFB_SEQ
  return false;
}

// Cost weight of a length with a compile-time sequence against the chain
// cost model (its row kernel ran 1.4-2x faster than the runtime-sequence
// kernel at 1701, 2048 and 4096 on B200).
constexpr double kFixedWeight = 0.6;

// On-chip convolution length for a length-n Bluestein: the M in
// [2n - 1, maxL] with the least M x chain cost (weighted for compile-time
// sequences); 0 if none fits.
int64_t choose_conv_length(int64_t n, int64_t maxL, std::vector<int> *radices) {
  std::unordered_map<int64_t, std::pair<double, int>> memo;
  int64_t best_m = 0;
  double best = 1e30;
  const int64_t lo = 2 * n - 1, hi = std::min<int64_t>(maxL, 2 * lo + 64);
  for (int64_t m = lo; m <= hi; ++m) {
    const double c = (double)m * chain_cost(m, nullptr, memo) * (fixed_sequence(m, nullptr) ? kFixedWeight : 1.0);
    if (c < best) {
      best = c;
      best_m = m;
    }
  }
  if (best_m && !fixed_sequence(best_m, radices)) chain_cost(best_m, radices, memo);
  return best_m;
}

// Four-step convolution M = n1 * n2: n1 one codelet (the column passes), n2
// on chip (the convolution rows).  Minimises M x chain cost of n2 (the column
// passes cost about the same for every n1), weighted for compile-time row
// sequences and for the shapes `one_pass` (the one-pass kernel's shape test,
// or null) accepts.
constexpr double kOnePassWeight = 0.35;
int64_t choose_split_conv(int64_t n, int64_t maxL, bool (*one_pass)(int, int), int64_t *n1_out,
                          std::vector<int> *row_radices) {
  std::unordered_map<int64_t, std::pair<double, int>> memo;
  static const int kCols[] = {16, 15, 13, 12, 11, 10, 9, 8};
  int64_t best_m = 0, best_n1 = 0;
  double best = 1e30;
  const int64_t lo = 2 * n - 1, hi = lo + lo / 4 + 64;
  for (int64_t m = lo; m <= hi; ++m)
    for (int n1 : kCols) {
      if (m % n1 || m / n1 > maxL) continue;
      const bool fixed = fixed_sequence(m / n1, nullptr);
      const double c = (double)m * chain_cost(m / n1, nullptr, memo) *
                       (one_pass && fixed && one_pass(n1, (int)(m / n1)) ? kOnePassWeight
                                                                             : fixed ? kFixedWeight : 1.0);
      if (c < best) {
        best = c;
        best_m = m;
        best_n1 = n1;
      }
    }
  if (!best_m) {
    // a convolution too long for a one-codelet column: columns of a
    // compile-time power-of-two sequence (strided tile passes, which carry
    // the chirp on load and store like the codelet columns), rows of at most
    // maxL points: M = n1 * n2 the smallest power of two >= 2n - 1
    int64_t m = 1;
    while (m < lo) m <<= 1;
    for (int64_t n1 = 32; n1 <= 16384 && !best_m; n1 <<= 1) {
      const int64_t n2 = m / n1;
      std::vector<int> r1;
      if (n2 >= 2 && n2 <= maxL && n2 <= 16384 && fixed_sequence(n1, &r1) && chain_cost(n2, nullptr, memo) < 1e29) {
        best_m = m;
        best_n1 = n1;
      }
    }
  }
  if (best_m) {
    *n1_out = best_n1;
    if (!fixed_sequence(best_m / best_n1, row_radices)) chain_cost(best_m / best_n1, row_radices, memo);
  }
  return best_m;
}

// The executor's own radix chain for length n (false when n has a prime
// factor above 19).
bool radix_chain(int64_t n, std::vector<int> *radices) {
  std::unordered_map<int64_t, std::pair<double, int>> memo;
  return chain_cost(n, radices, memo) < 1e29;
}

// The executor's own four-step split n = n1 x n2 (both chains, both on chip)
// with the least n x (chain cost of n1 + chain cost of n2); false if none.
bool own_four_step(int64_t n, int64_t maxL, int64_t *n1_out, std::vector<int> *r1, std::vector<int> *r2) {
  std::unordered_map<int64_t, std::pair<double, int>> memo;
  double best = 1e29;
  int64_t best_n1 = 0;
  for (int64_t a = 2; a * a <= n; ++a) {
    if (n % a) continue;
    for (int64_t n1 : {a, n / a}) {
      const int64_t n2 = n / n1;
      if (n1 > maxL || n2 > maxL) continue;
      const double c = chain_cost(n1, nullptr, memo) + chain_cost(n2, nullptr, memo);
      if (c < best) {
        best = c;
        best_n1 = n1;
      }
    }
  }
  if (!best_n1) return false;
  *n1_out = best_n1;
  chain_cost(best_n1, r1, memo);
  chain_cost(n / best_n1, r2, memo);
  return true;
}
}  // namespace

static Core make_dit_core(int64_t L, const std::vector<int> &r) {
  if ((int)r.size() > kMaxStages) throw std::runtime_error("too many radix stages");
  Core c{};
  c.L = (int)L;
  c.nst = (int)r.size();
  int64_t span = 1;
  for (size_t s = 0; s < r.size(); ++s) {
    c.radix[s] = r[s];
    c.span[s] = (int)span;
    c.sdiv[s] = make_fastdiv((uint32_t)span);
    c.rdiv[s] = make_fastdiv((uint32_t)r[s]);
    span *= r[s];
  }
  if (span != L) throw std::runtime_error("radices do not multiply to the core length");
  return c;
}

static Core make_dif_core(int64_t L, const std::vector<int> &r) {
  if ((int)r.size() > kMaxStages) throw std::runtime_error("too many radix stages");
  Core c{};
  c.L = (int)L;
  c.nst = (int)r.size();
  int64_t span = L;
  for (size_t s = 0; s < r.size(); ++s) {
    c.radix[s] = r[s];
    c.span[s] = (int)span;
    c.sdiv[s] = make_fastdiv((uint32_t)(span / r[s]));
    c.rdiv[s] = make_fastdiv((uint32_t)r[s]);
    span /= r[s];
  }
  if (span != 1) throw std::runtime_error("radices do not multiply to the core length");
  return c;
}

template <typename T>
class Builder {
 public:
  Builder(Program &prog, Planner &planner) : prog_(prog), planner_(planner) {}

  // A device table from the process-wide cache (built by `make` on a miss);
  // the program keeps a reference for its lifetime.
  template <typename V, class Make>
  const V *cached(const std::string &key, Make make) {
    DevPtr d = shared_table(std::string(sizeof(T) == 4 ? "f32|" : "f64|") + key, [&]() {
      std::vector<V> h = make();
      return upload(h.data(), h.size() * sizeof(V));
    });
    prog_.owned.push_back(d);
    return reinterpret_cast<const V *>(d->ptr);
  }

  static std::string radix_key(const std::vector<int> &r) {
    std::string k;
    for (int v : r) k += std::to_string(v) + ",";
    return k;
  }

  static constexpr int kMaxThreads = sizeof(T) == 4 ? 512 : 256;
  static constexpr int64_t kSMs = 148;

  // Two ping-pong buffers of a length-L transform fit one CTA.
  static bool pp_fits(int64_t L) {
    return (2 * (size_t)pp_size((int)L) + 3) * sizeof(cpx<T>) <= 232448;
  }

  // On-chip core for a complex transform node, if one exists.
  bool core_for(const NodePtr &node, CoreSpec &spec) const {
    const int64_t maxL = max_onchip_length(sizeof(T) == 8);
    if (node->length == 1) {  // the half-length core of a 2-point real transform
      spec = {CoreKind::Dit, 1, 1, {}, node};
      return true;
    }
    auto r = flatten(node);
    if (!r.empty() && node->length <= maxL) {
      fixed_sequence(node->length, &r);  // the same DFT on the compile-time sequence
      spec = {CoreKind::Dit, node->length, node->length, r, node};
      return true;
    }
    // a tree whose nodes do not flatten into one radix chain (a four-step
    // over Bluestein / Rader children): the executor's own chain when the
    // length has one and fits
    if (node->kind == NodeKind::FourStep && node->length <= maxL &&
        (fixed_sequence(node->length, &r) || radix_chain(node->length, &r))) {
      spec = {CoreKind::Dit, node->length, node->length, r, node};
      return true;
    }
    if (node->kind == NodeKind::Bluestein) {
      std::vector<int> rc;
      const int64_t m = choose_conv_length(node->length, maxL, &rc);
      if (m) {
        spec = {CoreKind::Bluestein, node->length, m, rc, node};
        return true;
      }
    }
    if (node->kind == NodeKind::Rader) {
      auto rc = flatten(node->child);
      if (rc.empty()) radix_chain(node->length - 1, &rc);  // the child tree is not one chain
      if (!rc.empty() && node->length - 1 <= maxL) {
        spec = {CoreKind::Rader, node->length, node->length - 1, rc, node};
        return true;
      }
      // p - 1 without a radix chain (a prime factor above 19): the same DFT
      // through a Bluestein convolution
      std::vector<int> bc;
      const int64_t m = rc.empty() ? choose_conv_length(node->length, maxL, &bc) : 0;
      if (m) {
        spec = {CoreKind::Bluestein, node->length, m, bc, node};
        return true;
      }
    }
    return false;
  }

  // Thread count per transform: one butterfly of the largest radix per thread.
  static int choose_tpt(int64_t L, const std::vector<int> &r) {
    if (r.empty()) return 1;
    int rmax = *std::max_element(r.begin(), r.end());
    int64_t t = (L + rmax - 1) / rmax;
    if (t <= 32) {
      int p = 1;
      while (p < t) p <<= 1;
      return p;
    }
    t = (t + 31) / 32 * 32;
    return (int)std::min<int64_t>(t, kMaxThreads);
  }

  // Threads per transform of the wide form (rows::rows_tpt_wide): for L's
  // compile-time sequence when it has a radix that is not a power of two,
  // one butterfly of its smallest radix >= 5 per thread; otherwise tpt.
  // Measured on B200 against the default: C2C 1701 x 1024 12.62 -> 12.31 us,
  // Z2Z 1701 x 256 9.58 -> 7.44, C2C 1701 x 256 7.18 -> 6.93; but slower at
  // large batch (C2C x 16384 126.9 -> 129.2, Z2Z x 4096 66.8 -> 71.0), so
  // passes of more than kWideMaxTransforms transforms keep the default.
  static constexpr int64_t kWideMaxTransforms = 2048;
  static int wide_tpt(int64_t L, const std::vector<int> &r, int tpt) {
    std::vector<int> seq;
    if (!fixed_sequence(L, &seq) || seq != r) return tpt;
    bool pow2 = true;
    int rmin = *std::max_element(r.begin(), r.end());
    for (int x : r) {
      pow2 = pow2 && (x & (x - 1)) == 0;
      if (x >= 5 && x < rmin) rmin = x;
    }
    return pow2 ? tpt : choose_tpt(L, {rmin});
  }

  // Fill a tile pass for G transforms per outer batch.
  TilePass<T> *add_pass(const CoreSpec &spec, IoKind io, bool inverse, int64_t nbatch, int64_t G, long long ib,
                        long long ig, long long ii, long long ob, long long og, long long ok, Buf src, Buf dst,
                        int64_t logical_n) {
    auto p = std::make_unique<TilePass<T>>();
    TileArgs<T> &a = p->a;
    a = TileArgs<T>{};
    a.nbatch = nbatch;
    a.ib = ib;
    a.ig = ig;
    a.ii = ii;
    a.ob = ob;
    a.og = og;
    a.ok = ok;
    a.G = (int)G;
    a.inv = inverse ? 1 : 0;
    a.n = (int)logical_n;
    const int64_t L = spec.L;
    const size_t limit = 232448;
    // Stockham ping-pong when two buffers of the transform fit (C2C passes);
    // the in-place DIT / DIF path otherwise.
    const size_t pp_per = (2 * (size_t)pp_size((int)L) + 3) * sizeof(cpx<T>);
    // a contiguous-row pass of a compile-time sequence runs on a row kernel,
    // which keeps one buffer per row (rows.cuh): it needs half of pp_per
    std::vector<int> seq, sorted_r = spec.radices;
    std::sort(sorted_r.rbegin(), sorted_r.rend());
    const size_t rows_per = ((size_t)pp_size((int)L) + 1) * sizeof(cpx<T>);
    const bool rows_only = io == IoKind::C2C && L > 1 && pp_per > limit && rows_per <= limit && ii == 1 &&
                           ok == 1 && ii <= ig && fixed_sequence(L, &seq) && seq == sorted_r;
    a.pp = (io == IoKind::C2C && L > 1 && (pp_per <= limit || rows_only)) ? 1 : 0;
    a.rows_only = (a.pp && pp_per > limit) ? 1 : 0;
    // ping-pong cores run their radices largest first (any order is the same
    // DFT; this one matches the compile-time sequences), and a convolution's
    // inverse core the same order; the in-place pair needs DIF then DIT with
    // the radices reversed
    std::vector<int> radices = spec.radices;
    if (a.pp) std::sort(radices.rbegin(), radices.rend());
    if (spec.kind == CoreKind::Dit) {
      a.core = make_dit_core(L, radices);
    } else {
      a.core = a.pp ? make_dit_core(L, radices) : make_dif_core(L, radices);
      std::vector<int> rev(radices.rbegin(), radices.rend());
      a.core2 = make_dit_core(L, a.pp ? radices : rev);
      if (spec.kind != CoreKind::Conv) fill_convolution(a, spec, inverse);  // Conv: caller supplies the kernel
    }
    // one-codelet transforms lying side by side in memory on both sides run
    // one per thread in registers
    if (spec.kind == CoreKind::Dit && io == IoKind::C2C && spec.radices.size() == 1 && spec.radices[0] == L &&
        regcol_supports((int)L) && ig == 1 && og == 1) {
      a.pp = 0;
      a.regcol = 1;
      a.W = 1;
      a.tpt = 1;
      p->kind = spec.kind;
      p->io = io;
      p->smem = 0;
      p->src = src;
      p->dst = dst;
      TilePass<T> *raw = p.get();
      prog_.passes.push_back(std::move(p));
      return raw;
    }
    if (spec.kind == CoreKind::Dit) {
      a.tw = table_stage_twiddles(a.core, false, inverse);
    } else {
      // convolution: forward core (DIF in place, DIT for Stockham), inverse core2
      a.tw = table_stage_twiddles(a.core, a.pp == 0, false);
      a.tw2 = table_stage_twiddles(a.core2, false, true);
    }
    // thread and tile shape: column tiles (transform index fastest in memory)
    // take consecutive transforms on consecutive threads
    const bool strided = ii > ig;
    a.wfast = strided ? 1 : 0;
    int tpt = choose_tpt(L, spec.radices);
    if (nbatch * G <= kWideMaxTransforms) tpt = wide_tpt(L, spec.radices, tpt);
    const size_t per = rows_only ? rows_per
                       : a.pp    ? pp_per
                                 : tile_smem_per_transform<T>((int)L) + Swz<T>::G * sizeof(cpx<T>);
    // Transforms per CTA: about 128 threads' worth, within a shared-memory
    // budget that leaves room for a second CTA per SM, and no more than keeps
    // ~2 CTAs per SM busy; column tiles take at least 8 transforms so each
    // row segment they read is 64-128 bytes.  (Against 256 threads' worth,
    // measured in one process on B200: C2C 256 x 262144 189 -> 168 us,
    // 1024 x 65536 175 -> 163, 1009 x 16384 179 -> 166, 256 x 16384 15.5 ->
    // 13.5, Z2Z 1024 x 32768 178 -> 164; no call slower; 512 threads' worth
    // was slower everywhere.)
    const size_t budget = std::max<size_t>(per, 110 * 1024);
    const int64_t w_thr = std::max<int64_t>(1, 128 / tpt);
    const int64_t w_smem = std::max<int64_t>(1, (int64_t)(std::min(budget, limit) / per));
    const int64_t w_par = std::max<int64_t>(1, (nbatch * G) / (2 * kSMs));
    int64_t W = std::min<int64_t>({w_thr, w_smem, w_par, G});
    if (strided) W = std::max<int64_t>(W, std::min<int64_t>({8, G, (int64_t)(limit / per)}));
    W = std::max<int64_t>(W, 1);
    if (W * tpt > kMaxThreads) tpt = std::max<int>(1, (int)(kMaxThreads / W));
    size_t smem_tiles = 0;
    {
      // a strided pass of a compile-time sequence: the tile kernel (one
      // buffer per transform, compile-time indexing), at least as wide as
      // the general tile
      int tw = 0, tthreads = 0;
      size_t tsm = 0;
      if (spec.kind == CoreKind::Dit && io == IoKind::C2C && a.pp && (ii > ig || ok > og) && !t_no_one_pass &&
          fixed_sequence(L, &seq) && seq == sorted_r && tiles_shape<T>((int)L, &tw, &tthreads, &tsm) &&
          std::min<int64_t>(tw, G) >= W) {
        a.tiles = 1;
        W = tw;
        tpt = tthreads;  // all threads of the CTA (the kernel splits them over the tile's transforms)
        smem_tiles = tsm;
      }
    }
    a.W = (int)W;
    a.tpt = tpt;
    // a strided pass of a TMA column sequence: the persistent TMA kernel
    // (the configuration above stays as its fallback)
    {
      int tc_threads = 0;
      size_t tc_smem = 0;
      if (spec.kind == CoreKind::Dit && io == IoKind::C2C && a.pp && !t_no_one_pass && tma_columns_enabled() &&
          fixed_sequence(L, &seq) && seq == sorted_r &&
          tcols_eligible<T>((int)L, nbatch, G, ib, ig, ii, ob, og, ok, &tc_threads, &tc_smem)) {
        a.tcols = 1;
        a.tc_threads = tc_threads;
        a.tc_smem = (int)tc_smem;
      }
    }
    // offsets inside one CTA's tile are 32-bit in the kernels
    if (W * std::llabs(ig) + L * std::llabs(ii) >= (1ll << 31) || W * std::llabs(og) + L * std::llabs(ok) >= (1ll << 31))
      throw std::runtime_error("tile extent above 2^31 elements");
    const size_t smem = a.tiles ? smem_tiles : per * (size_t)W;
    a.ldiv = make_fastdiv((uint32_t)L);
    a.wdiv = make_fastdiv((uint32_t)W);
    a.ndiv = make_fastdiv((uint32_t)std::max<int64_t>(1, logical_n));
    a.hdiv = make_fastdiv((uint32_t)std::max<int64_t>(1, logical_n / 2));
    p->kind = spec.kind;
    p->io = io;
    p->smem = smem;
    p->src = src;
    p->dst = dst;
    TilePass<T> *raw = p.get();
    prog_.passes.push_back(std::move(p));
    return raw;
  }

  // Per-stage twiddle blocks of a core for one direction; sets c.twoff.
  // Stage s's block holds R - 1 rows of `inner` entries (inner = span for
  // DIT / Stockham stages, span / R for DIF): entry j of row r - 1 is
  // W_{inner R}^{r j} (forward sign, the conjugate for the inverse).  A
  // length-L core's blocks hold L - 1 entries in all.  Cached per radix
  // sequence, stage kind and direction.
  const cpx<T> *table_stage_twiddles(Core &c, bool dif, bool inverse) {
    int64_t total = 0;
    std::string key = "tw|" + std::to_string(c.L) + (dif ? "|dif|" : "|dit|") + (inverse ? "inv|" : "fwd|");
    for (int s = 0; s < c.nst; ++s) {
      c.twoff[s] = (int)total;
      total += (int64_t)(c.radix[s] - 1) * (dif ? c.span[s] / c.radix[s] : c.span[s]);
      key += std::to_string(c.radix[s]) + ",";
    }
    const Core cc = c;
    return cached<cpx<T>>(key, [&]() {
      std::vector<cpx<T>> h((size_t)std::max<int64_t>(total, 1), mk((T)1, (T)0));
      for (int s = 0; s < cc.nst; ++s) {
        const int64_t R = cc.radix[s];
        const int64_t inner = dif ? cc.span[s] / R : cc.span[s];
        for (int64_t r = 1; r < R; ++r)
          for (int64_t j = 0; j < inner; ++j) {
            cld w = unit_root(r * j, inner * R, inverse ? 1 : -1);
            h[(size_t)(cc.twoff[s] + (r - 1) * inner + j)] = mk((T)w.real(), (T)w.imag());
          }
      }
      return h;
    });
  }

  // Real-transform twiddles W_n^k, k <= n/2.
  const cpx<T> *table_rtw(int64_t n) {
    return cached<cpx<T>>("rtw|" + std::to_string(n), [&]() {
      std::vector<cpx<T>> h((size_t)(n / 2 + 1));
      for (int64_t k = 0; k <= n / 2; ++k) {
        cld w = unit_root(k, n, -1);
        h[(size_t)k] = mk((T)w.real(), (T)w.imag());
      }
      return h;
    });
  }

  // The same twiddles as two short tables (RealTw): lo[m] = W_n^m, m < split,
  // hi[m] = W_n^(m split), m <= n/2 / split.
  RealTw<T> table_rtw_split(int64_t n) {
    const int64_t half = n / 2;
    const int64_t split = std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)(half + 1))));
    const int64_t nhi = half / split + 1;
    RealTw<T> t{};
    t.lo = cached<cpx<T>>("rtwlo|" + std::to_string(n) + "|" + std::to_string(split), [&]() {
      std::vector<cpx<T>> lo((size_t)split);
      for (int64_t m = 0; m < split; ++m) {
        cld w = unit_root(m, n, -1);
        lo[(size_t)m] = mk((T)w.real(), (T)w.imag());
      }
      return lo;
    });
    t.hi = cached<cpx<T>>("rtwhi|" + std::to_string(n) + "|" + std::to_string(split), [&]() {
      std::vector<cpx<T>> hi((size_t)nhi);
      for (int64_t m = 0; m < nhi; ++m) {
        cld w = unit_root(m * split, n, -1);
        hi[(size_t)m] = mk((T)w.real(), (T)w.imag());
      }
      return hi;
    });
    t.split = make_fastdiv((uint32_t)split);
    return t;
  }

  // Bluestein chirp exp(-+ i pi (j^2 mod 2n) / n), j < n (+ for the inverse).
  const cpx<T> *table_chirp(int64_t n, bool inverse) {
    return cached<cpx<T>>("chirp|" + std::to_string(n) + (inverse ? "|inv" : "|fwd"), [&]() {
      std::vector<cpx<T>> h((size_t)n);
      for (int64_t j = 0; j < n; ++j) {
        cld c = chirp_value(j, n, inverse ? 1 : -1);
        h[(size_t)j] = mk((T)c.real(), (T)c.imag());
      }
      return h;
    });
  }

  // Bluestein kernel spectrum B[k] / M laid out per row k1 of an n1 x n2
  // four-step: entry k1 * n2 + p holds B[k1 + n1 k2] for p = k2 (Stockham
  // passes) or the n2-point DIF position of k2 (in-place passes).
  const cpx<T> *table_bluestein_rows(int64_t n, const std::vector<int> &col_radices, int64_t n1, int64_t n2,
                                     bool inverse, bool natural) {
    const int64_t M = n1 * n2;
    const int sign = inverse ? 1 : -1;
    const std::string key = "bsrows|" + std::to_string(n) + "|" + std::to_string(n1) + "x" + std::to_string(n2) +
                            (inverse ? "|inv|" : "|fwd|") + (natural ? "nat|" : "dif|") + radix_key(col_radices);
    return cached<cpx<T>>(key, [&]() {
      std::vector<cld> b((size_t)M, cld(0));
      for (int64_t k = 0; k < n; ++k) {
        cld bc = chirp_value(k, n, -sign);
        b[(size_t)k] = bc;
        if (k) b[(size_t)(M - k)] = bc;
      }
      host_fft(b, -1);
      std::vector<cpx<T>> h((size_t)M);
      for (int64_t k1 = 0; k1 < n1; ++k1)
        for (int64_t k2 = 0; k2 < n2; ++k2) {
          cld v = b[(size_t)(k1 + n1 * k2)] / (long double)M;
          const int64_t p = natural ? k2 : dif_position(k2, col_radices);
          h[(size_t)(k1 * n2 + p)] = mk((T)v.real(), (T)v.imag());
        }
      return h;
    });
  }

  // Four-step post-twiddle W_N^m = hi[m / split] * lo[m % split].
  void set_post_twiddle(TileArgs<T> &a, int64_t N) {
    const int64_t split = (int64_t)std::ceil(std::sqrt((double)N));
    const int64_t nhi = (N + split - 1) / split;
    a.post_twiddle = 1;
    a.ptw_lo = cached<cpx<T>>("ptwlo|" + std::to_string(N), [&]() {
      std::vector<cpx<T>> lo((size_t)split);
      for (int64_t m = 0; m < split; ++m) {
        cld w = unit_root(m, N, -1);
        lo[(size_t)m] = mk((T)w.real(), (T)w.imag());
      }
      return lo;
    });
    a.ptw_hi = cached<cpx<T>>("ptwhi|" + std::to_string(N), [&]() {
      std::vector<cpx<T>> hi((size_t)nhi);
      for (int64_t m = 0; m < nhi; ++m) {
        cld w = unit_root(m * split, N, -1);
        hi[(size_t)m] = mk((T)w.real(), (T)w.imag());
      }
      return hi;
    });
    a.ptw_div = make_fastdiv((uint32_t)split);
  }

  // The same split tables as a transpose's twiddle W_N^{r c}.
  SplitTw<T> split_tw(int64_t N, bool inverse) {
    TileArgs<T> a{};
    set_post_twiddle(a, N);
    SplitTw<T> t;
    t.lo = a.ptw_lo;
    t.hi = a.ptw_hi;
    t.split = a.ptw_div;
    t.inv = inverse;
    return t;
  }

  // Tables of a multi-pass Rader chain for prime p (generator g): the
  // gather q -> g^-q, the scatter q -> g^q and FFT_m(b) / m in natural order,
  // b_q = W_p^{sign g^q} (src/plan/rader_utils.cpp:55-90,
  // src/codegen/tables.cpp:218-258).
  struct RaderChain {
    const int *perm_in, *perm_out;
    const cpx<T> *kern;
  };
  RaderChain rader_chain(int64_t p, int64_t g, bool inverse) {
    const int64_t m = p - 1;
    const std::string pk = std::to_string(p) + "|g" + std::to_string(g);
    const auto idx = rader_index_table(p, g);
    RaderChain r;
    r.perm_in = cached<int>("rcin|" + pk, [&]() {
      std::vector<int> v((size_t)m);
      for (int64_t q = 0; q < m; ++q) v[(size_t)q] = (int)idx[(size_t)(q == 0 ? 0 : m - q)];
      return v;
    });
    r.perm_out = cached<int>("rpout|" + pk, [&]() {
      std::vector<int> v((size_t)m);
      for (int64_t q = 0; q < m; ++q) v[(size_t)q] = (int)idx[(size_t)q];
      return v;
    });
    r.kern = cached<cpx<T>>("rchain|" + pk + (inverse ? "|inv" : "|fwd"), [&]() {
      std::vector<cld> b((size_t)m);
      for (int64_t q = 0; q < m; ++q) b[(size_t)q] = unit_root(idx[(size_t)q], p, inverse ? 1 : -1);
      return kernel_spectrum(b, true, {});
    });
    return r;
  }

 private:
  // Chirp, kernel spectrum and permutation tables of a Bluestein / Rader core.
  void fill_convolution(TileArgs<T> &a, const CoreSpec &spec, bool inverse) {
    const int sign = inverse ? 1 : -1;
    const int64_t L = spec.L;
    const std::string layout = std::string(a.pp ? "|nat|" : "|dif|") + radix_key(spec.radices);
    if (spec.kind == CoreKind::Bluestein) {
      const int64_t n = spec.n;
      a.chirp = table_chirp(n, inverse);
      a.kern = cached<cpx<T>>("bkern|" + std::to_string(n) + "|" + std::to_string(L) + (inverse ? "|inv" : "|fwd") +
                                  layout,
                              [&]() {
                                std::vector<cld> b((size_t)L, cld(0));
                                for (int64_t k = 0; k < n; ++k) {
                                  cld bc = chirp_value(k, n, -sign);
                                  b[(size_t)k] = bc;
                                  if (k) b[(size_t)(L - k)] = bc;
                                }
                                return kernel_spectrum(b, a.pp != 0, spec.radices);
                              });
    } else {
      const int64_t p = spec.n, m = p - 1;
      const int64_t g = spec.node->root;
      const std::string pk = std::to_string(p) + "|g" + std::to_string(g);
      auto idx = rader_index_table(p, g);
      // perm_in: q -> g^-q (m entries), then the log table k -> q (p entries)
      a.perm_in = cached<int>("rpin|" + pk, [&]() {
        std::vector<int> pin((size_t)(m + p), 0);
        for (int64_t q = 0; q < m; ++q) {
          pin[(size_t)q] = (int)idx[(size_t)(q == 0 ? 0 : m - q)];
          pin[(size_t)(m + idx[(size_t)q])] = (int)q;
        }
        return pin;
      });
      a.perm_out = cached<int>("rpout|" + pk, [&]() {
        std::vector<int> pout((size_t)m);
        for (int64_t q = 0; q < m; ++q) pout[(size_t)q] = (int)idx[(size_t)q];
        return pout;
      });
      a.kern = cached<cpx<T>>("rkern|" + pk + "|" + std::to_string(L) + (inverse ? "|inv" : "|fwd") + layout, [&]() {
        std::vector<cld> b((size_t)L, cld(0));
        for (int64_t q = 0; q < m; ++q) b[(size_t)q] = unit_root(idx[(size_t)q], p, sign);
        return kernel_spectrum(b, a.pp != 0, spec.radices);
      });
    }
  }

  // FFT(b) / L in natural order (Stockham cores) or DIF position order.
  static std::vector<cpx<T>> kernel_spectrum(std::vector<cld> &b, bool natural, const std::vector<int> &radices) {
    const int64_t L = (int64_t)b.size();
    host_fft(b, -1);
    std::vector<cpx<T>> kern((size_t)L);
    for (int64_t k = 0; k < L; ++k) {
      cld v = b[(size_t)k] / (long double)L;
      kern[(size_t)(natural ? k : dif_position(k, radices))] = mk((T)v.real(), (T)v.imag());
    }
    return kern;
  }

  Program &prog_;
  Planner &planner_;
};

// A length-n complex transform over `batch` rows (row distances idist / odist)
// from `src` to `dst`; `ws` is a workspace of batch * (n or the Bluestein
// convolution length) elements when the plan needs more than one pass.
// On-chip policy ($FLAGFFT_ONCHIP_POLICY): by default a transform that fits
// one CTA (two Stockham buffers, or in place) runs as one pass, except a
// Bluestein convolution that fits only in place, which takes the three-pass
// chain; "multipass" splits every tree that has a multi-pass lowering (one
// HBM round trip more, but smaller, more numerous CTAs); "inplace" keeps
// every transform that fits one CTA in one pass.
thread_local int t_policy_override = -1;  // set while lowering batch groups

// A program workspace of at least `bytes` (several lowerings of one program
// share it: they run one after the other).
static void ensure_scratch(DevPtr &d, size_t bytes) {
  if (!d || d->bytes < bytes) d = std::make_shared<DevMem>(bytes);
}

static int onchip_policy() {
  if (t_policy_override >= 0) return t_policy_override;
  const char *v = std::getenv("FLAGFFT_ONCHIP_POLICY");
  if (!v) return 0;
  std::string s(v);
  return s == "inplace" ? 1 : s == "multipass" ? 2 : 0;
}

// Plan-tree lowering ($FLAGFFT_TREE_LOWERING=1): a four-step whose child
// needs more than one pass, and a Rader prime whose p - 1 transform needs
// more than one pass, run as the tree says -- the reference's generic
// four-step (src/exec/raw_nodes.cpp:340-394: reshape, row child, twiddle
// reshape, column child, pack) and Rader chain (raw_nodes.cpp:252-305:
// gather, child FFT, kernel product, child FFT, scatter) around the
// children's own lowerings -- instead of the executor's own split or a
// Bluestein chain of the whole length (fewer HBM round trips, the default).
// A tree lowering keeps its working rows in workspace 1; a child that would
// need workspace 1 itself runs the executor's way.
static bool tree_lowering() {
  const char *v = std::getenv("FLAGFFT_TREE_LOWERING");
  return v && v[0] == '1';
}

template <typename T>
void lower_c2c(Builder<T> &bld, Program &prog, const NodePtr &root, bool inverse, int64_t n, int64_t batch,
               long long idist, long long odist, Buf src, Buf dst);

// True when node's lowering under the current policy is a tree lowering
// (it would use workspace 1).
template <typename T>
bool needs_tree_lowering(Builder<T> &bld, const NodePtr &node) {
  if (!tree_lowering() || !node) return false;
  CoreSpec a, b;
  if (node->kind == NodeKind::FourStep)
    return !(bld.core_for(node->row, a) && bld.core_for(node->col, b)) && !bld.core_for(node, a);
  if (node->kind == NodeKind::Rader) return !bld.core_for(node, a) || a.kind != CoreKind::Rader;
  return false;
}

// The plan tree's four-step over children of any lowering: x viewed as
// n1 x n2 (x[j1 n2 + j2]) is transposed to n2 rows of n1, the n1-point
// child runs on them, a twiddled transpose (W_N^{j2 k1}) gives n1 rows of
// n2, the n2-point child runs on those into workspace 1, and a last
// transpose gives X[k1 + n1 k2].  Workspace 1 holds the working rows; the
// children use workspace 0.
template <typename T>
bool lower_tree_four_step(Builder<T> &bld, Program &prog, const NodePtr &root, bool inverse, int64_t n,
                          int64_t batch, long long idist, long long odist, Buf src, Buf dst) {
  if (needs_tree_lowering(bld, root->row) || needs_tree_lowering(bld, root->col)) return false;
  if (src == Buf::Scratch1 || dst == Buf::Scratch1) return false;
  const int64_t n1 = root->n1, n2 = root->n2;
  // (the n2-point rows are formed in the output, so its rows are contiguous;
  // a child's multi-pass lowering takes at most 65535 rows)
  CoreSpec c1, c2;
  if (n1 * n2 != n || odist != n) return false;
  if ((!bld.core_for(root->row, c1) && batch * n2 > 65535) || (!bld.core_for(root->col, c2) && batch * n1 > 65535))
    return false;
  ensure_scratch(prog.scratch1, (size_t)(batch * n) * sizeof(cpx<T>));
  auto t1 = std::make_unique<TransposePass<T>>(src, Buf::Scratch1, batch, n1, n2);
  t1->sdist = idist;
  t1->ddist = n;
  prog.passes.push_back(std::move(t1));
  lower_c2c<T>(bld, prog, root->row, inverse, n1, batch * n2, n1, n1, Buf::Scratch1, Buf::Scratch1);
  auto t2 = std::make_unique<TransposePass<T>>(Buf::Scratch1, dst, batch, n2, n1);
  t2->sdist = n;
  t2->ddist = odist;
  t2->tw = bld.split_tw(n, inverse);
  prog.passes.push_back(std::move(t2));
  lower_c2c<T>(bld, prog, root->col, inverse, n2, batch * n1, n2, n2, dst, Buf::Scratch1);
  auto t3 = std::make_unique<TransposePass<T>>(Buf::Scratch1, dst, batch, n1, n2);
  t3->sdist = n;
  t3->ddist = odist;
  prog.passes.push_back(std::move(t3));
  return true;
}

// The plan tree's Rader chain over a multi-pass p - 1 transform: gather into
// workspace 1, the child forward, the kernel product (conjugated), the child
// forward again, scatter with x_0 added (the reference's conj(FFT(conj(.)))
// form of the inverse).  Workspace 1: batch rows of p - 1 plus 2 * batch.
template <typename T>
bool lower_tree_rader(Builder<T> &bld, Program &prog, const NodePtr &root, bool inverse, int64_t batch,
                      long long idist, long long odist, Buf src, Buf dst) {
  const NodePtr child = root->child;
  if (!child || needs_tree_lowering(bld, child)) return false;
  if (src == Buf::Scratch1 || dst == Buf::Scratch1) return false;
  const int64_t p = root->length, m = p - 1;
  if (batch > 65535) return false;
  ensure_scratch(prog.scratch1, (size_t)(batch * m + 2 * batch) * sizeof(cpx<T>));
  const auto r = bld.rader_chain(p, root->root, inverse);
  prog.passes.push_back(std::make_unique<RaderStepPass<T>>(0, src, Buf::Scratch1, dst, batch, p, idist, odist,
                                                           r.perm_in, r.kern));
  lower_c2c<T>(bld, prog, child, false, m, batch, m, m, Buf::Scratch1, Buf::Scratch1);
  prog.passes.push_back(std::make_unique<RaderStepPass<T>>(1, src, Buf::Scratch1, dst, batch, p, idist, odist,
                                                           r.perm_in, r.kern));
  lower_c2c<T>(bld, prog, child, false, m, batch, m, m, Buf::Scratch1, Buf::Scratch1);
  prog.passes.push_back(std::make_unique<RaderStepPass<T>>(2, src, Buf::Scratch1, dst, batch, p, idist, odist,
                                                           r.perm_out, r.kern));
  return true;
}

template <typename T>
void lower_c2c(Builder<T> &bld, Program &prog, const NodePtr &root, bool inverse, int64_t n, int64_t batch,
               long long idist, long long odist, Buf src, Buf dst) {
  if (needs_tree_lowering(bld, root)) {
    if (root->kind == NodeKind::FourStep &&
        lower_tree_four_step<T>(bld, prog, root, inverse, n, batch, idist, odist, src, dst))
      return;
    if (root->kind == NodeKind::Rader && lower_tree_rader<T>(bld, prog, root, inverse, batch, idist, odist, src, dst))
      return;
  }
  CoreSpec spec;
  const bool onchip = bld.core_for(root, spec);
  CoreSpec ca, cb;
  const bool mp_four = root->kind == NodeKind::FourStep && bld.core_for(root->row, ca) && bld.core_for(root->col, cb);
  // three-pass Bluestein chain at an executor-chosen split (also the
  // multi-pass lowering of a Rader prime)
  const bool mp_blue = root->kind == NodeKind::Bluestein || root->kind == NodeKind::Rader;
  const int policy = onchip_policy();
  // A Bluestein convolution that fits one CTA only in place (not as two
  // ping-pong buffers) runs faster as the three-pass chain: its 1-CTA-per-SM
  // in-place pass is latency-bound (C2C N=10007 on B200: 440 us fused vs
  // 414 us in three passes).
  const bool blue_in_place = onchip && (spec.kind == CoreKind::Bluestein || spec.kind == CoreKind::Rader) &&
                             !Builder<T>::pp_fits(spec.L);
  const bool use_onchip =
      onchip && (policy == 1 || ((policy != 2 || !(mp_four || mp_blue)) && !blue_in_place));
  if (use_onchip) {
    bld.add_pass(spec, IoKind::C2C, inverse, 1, batch, 0, idist, 1, 0, odist, 1, src, dst, n);
    return;
  }
  if (batch > 65535) throw std::runtime_error("multi-pass batch above 65535");
  CoreSpec sa, sb;
  int64_t f1 = 0;
  if (root->kind == NodeKind::FourStep && bld.core_for(root->row, sa) && bld.core_for(root->col, sb)) {
    f1 = root->n1;
  } else if (root->kind != NodeKind::Bluestein && root->kind != NodeKind::Rader) {
    // the executor's own split when the tree's children cannot run as cores
    std::vector<int> r1, r2;
    if (own_four_step(n, max_onchip_length(sizeof(T) == 8), &f1, &r1, &r2)) {
      sa = {CoreKind::Dit, f1, f1, r1, nullptr};
      sb = {CoreKind::Dit, n / f1, n / f1, r2, nullptr};
    }
  }
  if (f1) {
    {
      const int64_t n1 = f1, n2 = n / f1;
      ensure_scratch(prog.scratch0, (size_t)(batch * n) * sizeof(cpx<T>));
      // pass A: columns j2 (stride n2) of length n1, x W_n^{j2 k1}, rows Y[j2][k1]
      auto *pa = bld.add_pass(sa, IoKind::C2C, inverse, batch, n2, idist, 1, n2, n, n1, 1, src, Buf::Scratch0, n1);
      bld.set_post_twiddle(pa->a, n);
      // pass B: for each k1, length n2 over Y[j2][k1] -> X[k1 + n1 k2]
      bld.add_pass(sb, IoKind::C2C, inverse, batch, n1, n, 1, n1, odist, 1, n1, Buf::Scratch0, dst, n2);
      return;
    }
  }
  {
    // A Bluestein node whose convolution is too long for one CTA, or any
    // length the lowerings above cannot run (a Rader prime too long for one
    // CTA, a length whose factors are neither chains nor a split): three
    // passes through an M-point
    // workspace, M = n1 x n2 chosen by the executor (n1 one codelet, n2 on
    // chip), with the chirps, the kernel product and both four-step twiddles
    // fused (src/exec/raw_nodes.cpp:153-204 runs the same chain as 7 launches).
    int64_t n1 = 0;
    std::vector<int> row_radices;
    // the one-pass forms: single precision holds the N1 rows in one CTA;
    // the pair form (both precisions) splits them over a two-CTA cluster
    const bool pair = bluestein_pair();
    bool (*const one_pass)(int, int) = t_no_one_pass ? nullptr
                                       : pair        ? blue4_pair_shape
                                       : sizeof(T) == 4 ? blue4_shape
                                                        : nullptr;
    const int64_t M = choose_split_conv(n, max_onchip_length(sizeof(T) == 8), one_pass, &n1, &row_radices);
    std::vector<int> seq;
    if (M && one_pass && one_pass((int)n1, (int)(M / n1)) && fixed_sequence(M / n1, &seq) && seq == row_radices) {
      // the whole chain in one CTA (or CTA pair) per transform: n1 rows of
      // n2 points in shared memory (blue4.cuh)
      const int64_t n2 = M / n1;
      CoreSpec sc{CoreKind::Conv, n2, n2, row_radices, nullptr};
      auto *p = bld.add_pass(sc, IoKind::C2C, true, batch, 1, idist, 0, 1, odist, 0, 1, src, dst, n);
      TileArgs<T> &a = p->a;
      a.blue_cols = (int)n1;
      a.blue_pair = pair ? 1 : 0;
      a.G = 1;
      a.W = 1;
      a.n = (int)n;
      a.chirp = bld.table_chirp(n, inverse);
      a.kern = bld.table_bluestein_rows(n, row_radices, n1, n2, inverse, true);
      a.kern_stride = n2;
      bld.set_post_twiddle(a, M);
      p->smem = blue4_smem((int)n1, (int)n2, sizeof(cpx<T>), pair);
      p->note = "bluestein one pass: " + std::to_string(n1) + " x " + std::to_string(n2) +
                (pair ? " four-step in a two-CTA cluster" : " four-step in one CTA");
      return;
    }
    if (M) {
      const int64_t n2 = M / n1;
      // the column core: one codelet, or (long convolutions) a compile-time sequence
      std::vector<int> col_radices{(int)n1};
      if (n1 > 19) fixed_sequence(n1, &col_radices);
      const CoreSpec sa{CoreKind::Dit, n1, n1, col_radices, nullptr};
      const CoreSpec sb{CoreKind::Dit, n2, n2, row_radices, nullptr};
      ensure_scratch(prog.scratch0, (size_t)(batch * M) * sizeof(cpx<T>));
      const cpx<T> *chirp = bld.table_chirp(n, inverse);
      // A: a_j = x_j c_j (j = j1 n2 + j2 < n), FFT over j1, x W_M^{j2 k1} -> Y[k1][j2]
      auto *pa = bld.add_pass(sa, IoKind::C2C, false, batch, n2, idist, 1, n2, M, 1, n2, src, Buf::Scratch0, n);
      pa->a.chirp_mode = 1;
      pa->a.chirp = chirp;
      pa->a.cj_e = n2;
      pa->a.cj_g = 1;
      bld.set_post_twiddle(pa->a, M);
      pa->note = "bluestein 1/3: chirp + column FFT";
      // B: per k1: FFT over j2, x B[k1 + n1 k2] / M, inverse FFT over k2, x W_M^{-j2 k1}
      CoreSpec sc = sb;
      sc.kind = CoreKind::Conv;
      auto *pb = bld.add_pass(sc, IoKind::C2C, true, batch, n1, M, n2, 1, M, n2, 1, Buf::Scratch0, Buf::Scratch0, n2);
      pb->a.kern = bld.table_bluestein_rows(n, sb.radices, n1, n2, inverse, pb->a.pp != 0);
      pb->a.kern_stride = n2;
      bld.set_post_twiddle(pb->a, M);
      pb->note = "bluestein 2/3: row convolution";
      // C: inverse FFT over k1 -> j1, y_j = conv_j c_j for j = j1 n2 + j2 < n
      auto *pc = bld.add_pass(sa, IoKind::C2C, true, batch, n2, M, 1, n2, odist, 1, n2, Buf::Scratch0, dst, n);
      pc->a.chirp_mode = 2;
      pc->a.chirp = chirp;
      pc->a.cj_e = n2;
      pc->a.cj_g = 1;
      pc->note = "bluestein 3/3: column inverse FFT + chirp";
      return;
    }
  }
  throw std::runtime_error("plan tree has no lowering on this engine: " + root->key_repr());
}

template <typename T>
std::unique_ptr<Program> lower_t(const NodePtr &root, Planner &planner, Transform t, bool inverse, int64_t n,
                                 const Layout &lay, bool in_place_real) {
  auto prog = std::make_unique<Program>();
  Builder<T> bld(*prog, planner);
  const int64_t batch = lay.batch;

  if (t == Transform::C2C) {
    lower_c2c<T>(bld, *prog, root, inverse, n, batch, lay.idist, lay.odist, Buf::In, Buf::Out);
    return prog;
  }

  // Real transforms.  Even n: n/2-point complex core with the pack / unpack
  // fused into its load and store; odd n: the n-point core on real data.
  const bool even = (n % 2) == 0;
  const int64_t L = n / 2;
  NodePtr core_node = even ? build_raw_root(planner, L, nullptr, nullptr) : root;
  const int64_t idist = (t == Transform::R2C && in_place_real) ? std::max<int64_t>(lay.idist, 2 * (L + 1)) : lay.idist;
  const int64_t odist = (t == Transform::C2R && in_place_real) ? std::max<int64_t>(lay.odist, 2 * (L + 1)) : lay.odist;
  CoreSpec spec;
  if (bld.core_for(core_node, spec)) {
    if (t == Transform::R2C) {
      auto *p = bld.add_pass(spec, even ? IoKind::R2C : IoKind::R2CFull, false, 1, batch, 0, idist, even ? 2 : 1, 0,
                             odist, 1, Buf::In, Buf::Out, n);
      if (even) p->a.rtw = bld.table_rtw(n);
      p->note = even ? "n/2-point complex core" : "n-point complex core";
    } else {
      auto *p = bld.add_pass(spec, even ? IoKind::C2R : IoKind::C2RFull, true, 1, batch, 0, idist, 1, 0, odist,
                             even ? 2 : 1, Buf::In, Buf::Out, n);
      if (even) p->a.rtw = bld.table_rtw(n);
      p->note = even ? "n/2-point complex core" : "n-point complex core";
    }
    return prog;
  }
  CoreSpec sa, sb;
  // (the pack / unpack rides on a Dit core: pass A of R2C, pass B of C2R)
  if (even && core_node->kind == NodeKind::FourStep && bld.core_for(core_node->row, sa) &&
      bld.core_for(core_node->col, sb) && (t == Transform::R2C ? sa.kind : sb.kind) == CoreKind::Dit) {
    if (batch > 65535) throw std::runtime_error("multi-pass batch above 65535");
    const int64_t n1 = core_node->n1, n2 = core_node->n2;
    const RealTw<T> rtw = bld.table_rtw_split(n);
    prog->scratch0 = std::make_shared<DevMem>((size_t)(batch * L) * sizeof(cpx<T>));
    if (t == Transform::R2C) {
      // A: z_j = x_2j + i x_2j+1 (j = j1 n2 + j2), FFT over j1, x W_L^{j2 k1} -> Y[j2][k1];
      // with an even row distance the pairs are the rows read as complex
      // elements, and the pass is a plain complex one (tile kernels apply)
      auto *pa = idist % 2 == 0
                     ? bld.add_pass(sa, IoKind::C2C, false, batch, n2, idist / 2, 1, n2, L, n1, 1, Buf::In,
                                    Buf::Scratch0, n1)
                     : bld.add_pass(sa, IoKind::PackC2C, false, batch, n2, idist, 2, 2 * n2, L, n1, 1, Buf::In,
                                    Buf::Scratch0, n1);
      bld.set_post_twiddle(pa->a, L);
      // B: FFT over j2 -> Z[k1 + n1 k2] in the output rows; when those rows
      // start off 16-byte boundaries (odd complex64 distances: n/2 + 1), in
      // place in the workspace, whose rows the TMA column kernel can copy,
      // and the Hermitian post pass moves the result to the output
      if (batch > 1 && (odist * (long long)sizeof(cpx<T>)) % 16 != 0) {
        bld.add_pass(sb, IoKind::C2C, false, batch, n1, L, 1, n1, L, 1, n1, Buf::Scratch0, Buf::Scratch0, n2);
        prog->passes.push_back(
            std::make_unique<RealPass<T>>(true, Buf::Scratch0, Buf::Out, batch, L, odist, L, rtw));
      } else {
        bld.add_pass(sb, IoKind::C2C, false, batch, n1, L, 1, n1, odist, 1, n1, Buf::Scratch0, Buf::Out, n2);
        prog->passes.push_back(std::make_unique<RealPass<T>>(true, Buf::Out, Buf::Out, batch, odist, odist, L, rtw));
      }
    } else {
      prog->scratch1 = std::make_shared<DevMem>((size_t)(batch * L) * sizeof(cpx<T>));
      prog->passes.push_back(
          std::make_unique<RealPass<T>>(false, Buf::In, Buf::Scratch1, batch, idist, L, L, rtw));
      auto *pa = bld.add_pass(sa, IoKind::C2C, true, batch, n2, L, 1, n2, L, n1, 1, Buf::Scratch1, Buf::Scratch0, n1);
      bld.set_post_twiddle(pa->a, L);
      // B: inverse FFT over j2, z_j -> x_2j, x_2j+1 (j = k1 + n1 k2): with an
      // even row distance, complex elements of the output rows
      if (odist % 2 == 0)
        bld.add_pass(sb, IoKind::C2C, true, batch, n1, L, 1, n1, odist / 2, 1, n1, Buf::Scratch0, Buf::Out, n2);
      else
        bld.add_pass(sb, IoKind::C2CUnpack, true, batch, n1, L, 1, n1, odist, 2, 2 * n1, Buf::Scratch0, Buf::Out,
                     n2);
    }
    return prog;
  }
  if (even && (t == Transform::R2C ? idist % 2 == 0 : odist % 2 == 0)) {
    // Any other even n: the complex transform of length n/2 over the rows
    // reinterpreted as complex (whatever lowering that length takes), then
    // the Hermitian post-processing in place on the output (R2C); or the
    // pre-processing into a workspace, then the complex transform into the
    // output rows reinterpreted as complex (C2R).
    if (batch > 65535) throw std::runtime_error("multi-pass batch above 65535");
    const RealTw<T> rtw = bld.table_rtw_split(n);
    if (t == Transform::R2C) {
      lower_c2c<T>(bld, *prog, core_node, false, L, batch, idist / 2, odist, Buf::In, Buf::Out);
      prog->passes.push_back(std::make_unique<RealPass<T>>(true, Buf::Out, Buf::Out, batch, odist, odist, L, rtw));
    } else {
      prog->scratch1 = std::make_shared<DevMem>((size_t)(batch * L) * sizeof(cpx<T>));
      prog->passes.push_back(std::make_unique<RealPass<T>>(false, Buf::In, Buf::Scratch1, batch, idist, L, L, rtw));
      lower_c2c<T>(bld, *prog, core_node, true, L, batch, L, odist / 2, Buf::Scratch1, Buf::Out);
    }
    return prog;
  }
  {
    // Any length: widen to complex, the n-point complex transform of any
    // lowering, then the half spectrum (R2C); or the Hermitian expansion,
    // the inverse complex transform and the real part (C2R).
    if (batch > 65535) throw std::runtime_error("multi-pass batch above 65535");
    auto ws = std::make_shared<DevMem>((size_t)(batch * n) * sizeof(cpx<T>));
    prog->scratch1 = ws;
    // (the complex transform runs in place on scratch1: every lowering reads
    // a tile whole before writing it, and a multi-pass one goes through its
    // own workspace, scratch0)
    if (t == Transform::R2C) {
      prog->passes.push_back(std::make_unique<ConvertPass<T>>(0, Buf::In, Buf::Scratch1, batch, idist, n, n));
      lower_c2c<T>(bld, *prog, root, false, n, batch, n, n, Buf::Scratch1, Buf::Scratch1);
      prog->passes.push_back(std::make_unique<ConvertPass<T>>(1, Buf::Scratch1, Buf::Out, batch, n, odist, n));
    } else {
      prog->passes.push_back(std::make_unique<ConvertPass<T>>(2, Buf::In, Buf::Scratch1, batch, idist, n, n));
      lower_c2c<T>(bld, *prog, root, true, n, batch, n, n, Buf::Scratch1, Buf::Scratch1);
      prog->passes.push_back(std::make_unique<ConvertPass<T>>(3, Buf::Scratch1, Buf::Out, batch, n, odist, n));
    }
    return prog;
  }
}

template <typename T>
std::unique_ptr<Program> lower_2d_t(const NodePtr &root, Planner &planner, Transform t, bool inverse, int64_t n0,
                                    int64_t n1, int64_t batch) {
  auto prog = std::make_unique<Program>();
  Builder<T> bld(*prog, planner);
  CoreSpec rs, cs;
  const int64_t h1 = n1 / 2 + 1;
  if (batch > 65535) throw std::runtime_error("2-D batch above 65535");
  if (t == Transform::C2C) {
    if (bld.core_for(root->row, rs) && bld.core_for(root->col, cs)) {
      bld.add_pass(rs, IoKind::C2C, inverse, 1, batch * n0, 0, n1, 1, 0, n1, 1, Buf::In, Buf::Out, n1);
      bld.add_pass(cs, IoKind::C2C, inverse, batch, n1, n0 * n1, 1, n1, n0 * n1, 1, n1, Buf::Out, Buf::Out, n0);
      return prog;
    }
    // An axis too long for one CTA (src/exec/raw_nodes.cpp:549-610 runs any
    // child per axis): the rows with whatever lowering their tree takes,
    // the matrix transposed, the other axis as rows, transposed back.
    lower_c2c<T>(bld, *prog, root->row, inverse, n1, batch * n0, n1, n1, Buf::In, Buf::Out);
    ensure_scratch(prog->scratch1, (size_t)(batch * n0 * n1) * sizeof(cpx<T>));
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::Out, Buf::Scratch1, batch, n0, n1));
    lower_c2c<T>(bld, *prog, root->col, inverse, n0, batch * n1, n0, n0, Buf::Scratch1, Buf::Scratch1);
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::Scratch1, Buf::Out, batch, n1, n0));
    return prog;
  }
  const bool even = (n1 % 2) == 0;
  NodePtr row_core = even ? build_raw_root(planner, n1 / 2, nullptr, nullptr) : root->row;
  if (!bld.core_for(row_core, rs)) throw std::runtime_error("2-D real row axis too long for one CTA");
  const bool col_onchip = bld.core_for(root->col, cs);
  if (t == Transform::R2C) {
    if (col_onchip) {
      // rows into the workspace, then column tiles into the output (safe in place)
      ensure_scratch(prog->scratch0, (size_t)(batch * n0 * h1) * sizeof(cpx<T>));
      auto *p = bld.add_pass(rs, even ? IoKind::R2C : IoKind::R2CFull, false, 1, batch * n0, 0, n1, even ? 2 : 1, 0,
                             h1, 1, Buf::In, Buf::Scratch0, n1);
      if (even) p->a.rtw = bld.table_rtw(n1);
      bld.add_pass(cs, IoKind::C2C, false, batch, h1, n0 * h1, 1, h1, n0 * h1, 1, h1, Buf::Scratch0, Buf::Out, n0);
      return prog;
    }
    // a column axis too long for one CTA: rows into the output, transpose,
    // the columns as rows (any lowering), transpose back
    auto *p = bld.add_pass(rs, even ? IoKind::R2C : IoKind::R2CFull, false, 1, batch * n0, 0, n1, even ? 2 : 1, 0,
                           h1, 1, Buf::In, Buf::Out, n1);
    if (even) p->a.rtw = bld.table_rtw(n1);
    ensure_scratch(prog->scratch1, (size_t)(batch * n0 * h1) * sizeof(cpx<T>));
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::Out, Buf::Scratch1, batch, n0, h1));
    lower_c2c<T>(bld, *prog, root->col, false, n0, batch * h1, n0, n0, Buf::Scratch1, Buf::Scratch1);
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::Scratch1, Buf::Out, batch, h1, n0));
    return prog;
  }
  if (col_onchip) {
    ensure_scratch(prog->scratch0, (size_t)(batch * n0 * h1) * sizeof(cpx<T>));
    bld.add_pass(cs, IoKind::C2C, true, batch, h1, n0 * h1, 1, h1, n0 * h1, 1, h1, Buf::In, Buf::Scratch0, n0);
  } else {
    // columns first (transposed to rows, any lowering, transposed back into
    // the workspace the row pass reads)
    ensure_scratch(prog->scratch1, (size_t)(batch * n0 * h1) * sizeof(cpx<T>));
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::In, Buf::Scratch1, batch, n0, h1));
    lower_c2c<T>(bld, *prog, root->col, true, n0, batch * h1, n0, n0, Buf::Scratch1, Buf::Scratch1);
    ensure_scratch(prog->scratch0, (size_t)(batch * n0 * h1) * sizeof(cpx<T>));
    prog->passes.push_back(std::make_unique<TransposePass<T>>(Buf::Scratch1, Buf::Scratch0, batch, h1, n0));
  }
  auto *p = bld.add_pass(rs, even ? IoKind::C2R : IoKind::C2RFull, true, 1, batch * n0, 0, h1, 1, 0, n1, even ? 2 : 1,
                         Buf::Scratch0, Buf::Out, n1);
  if (even) p->a.rtw = bld.table_rtw(n1);
  return prog;
}

}  // namespace

std::unique_ptr<Program> lower(const NodePtr &root, Planner &planner, bool is_double, Transform t, bool inverse,
                               int64_t n, const Layout &layout, bool in_place_real) {
  return is_double ? lower_t<double>(root, planner, t, inverse, n, layout, in_place_real)
                   : lower_t<float>(root, planner, t, inverse, n, layout, in_place_real);
}

std::unique_ptr<Program> lower_2d(const NodePtr &root, Planner &planner, bool is_double, Transform t, bool inverse,
                                  int64_t n0, int64_t n1, int64_t batch) {
  return is_double ? lower_2d_t<double>(root, planner, t, inverse, n0, n1, batch)
                   : lower_2d_t<float>(root, planner, t, inverse, n0, n1, batch);
}

std::unique_ptr<Program> lower_batchable(const NodePtr &root, Planner &planner, bool is_double, Transform t,
                                         bool inverse, int64_t n, const Layout &layout) {
  struct Scope {  // the thread's lowering switches, restored on every exit
    bool one = t_no_one_pass;
    int pol = t_policy_override;
    ~Scope() {
      t_no_one_pass = one;
      t_policy_override = pol;
    }
  } scope;
  t_no_one_pass = true;
  auto prog = lower(root, planner, is_double, t, inverse, n, layout, false);
  bool in_place = false;
  for (const auto &ps : prog->passes) {
    if (is_double) {
      auto *tp = dynamic_cast<const TilePass<double> *>(ps.get());
      if (tp && !tp->a.pp && !tp->a.regcol) in_place = true;
    } else {
      auto *tp = dynamic_cast<const TilePass<float> *>(ps.get());
      if (tp && !tp->a.pp && !tp->a.regcol) in_place = true;
    }
  }
  if (in_place) {
    t_policy_override = 2;
    prog = lower(root, planner, is_double, t, inverse, n, layout, false);
  }
  return prog;
}

// ---------------------------------------------------------------------------
// Batch programs
// ---------------------------------------------------------------------------
namespace {

template <typename T>
struct BatchProgramT final : BatchProgram {
  struct Group {
    int64_t n = 0, count = 0, offset = 0;
    std::unique_ptr<Program> prog;
  };
  struct PassRef {
    int group, pass, kind;  // kind: a BatchKind, or -1 for a pass launched on its own
    int cls;                // shared-memory class of a persistent pass
  };
  struct Launch {  // one persistent launch: the passes of one class of one phase
    int threads = 0;
    size_t smem = 0;
  };
  struct Phase {
    std::vector<PassRef> passes;
    Launch cls[kBatchClasses];
  };
  // Device state for one (input, output) pair: resolved pass arguments, the
  // work items of every launch, the queue counters and the captured graph.
  struct Bound {
    const void *in = nullptr;
    void *out = nullptr;
    DevPtr args, kinds, items, counters;
    std::vector<int> first_item, nitems, ctas;  // per (phase, class)
    std::vector<TileArgs<T>> host_args;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Bound() {
#ifndef FFB_HOST_EMULATION
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
#endif
    }
  };

  bool inverse = false, graphs = true;
  std::vector<Group> groups;
  std::vector<Phase> phases;
  std::vector<std::unique_ptr<Bound>> bound;  // most recent last
  std::mutex mu;
#ifndef FFB_HOST_EMULATION
  cudaStream_t side[kBatchClasses] = {};
  cudaEvent_t fork = nullptr, join[kBatchClasses] = {};
#endif

  static constexpr size_t kMaxBound = 4;

  ~BatchProgramT() override {
    bound.clear();
#ifndef FFB_HOST_EMULATION
    for (int c = 0; c < kBatchClasses; ++c) {
      if (side[c]) cudaStreamDestroy(side[c]);
      if (join[c]) cudaEventDestroy(join[c]);
    }
    if (fork) cudaEventDestroy(fork);
#endif
  }

  const TilePass<T> *tile_pass(const PassRef &r) const {
    return dynamic_cast<const TilePass<T> *>(groups[(size_t)r.group].prog->passes[(size_t)r.pass].get());
  }

  std::unique_ptr<Bound> bind(const void *in, void *out) {
    auto b = std::make_unique<Bound>();
    b->in = in;
    b->out = out;
    std::vector<int> kinds;
    std::vector<BatchItem> items;
    for (const Phase &ph : phases) {
      struct Cost {
        double c;
        int args, tiles;
      };
      std::vector<Cost> order[kBatchClasses];
      for (const PassRef &r : ph.passes) {
        if (r.kind < 0) continue;
        const Group &g = groups[(size_t)r.group];
        const TilePass<T> *tp = tile_pass(r);
        TileArgs<T> a = tp->a;
        const cpx<T> *gin = reinterpret_cast<const cpx<T> *>(in) + g.offset;
        cpx<T> *gout = reinterpret_cast<cpx<T> *>(out) + g.offset;
        void *s0 = g.prog->scratch0 ? g.prog->scratch0->ptr : nullptr;
        void *s1 = g.prog->scratch1 ? g.prog->scratch1->ptr : nullptr;
        a.in = TilePass<T>::pick(tp->src, gin, gout, s0, s1);
        a.out = TilePass<T>::pick(tp->dst, gin, gout, s0, s1);
        const int idx = (int)b->host_args.size();
        b->host_args.push_back(a);
        kinds.push_back(r.kind);
        const int width = r.kind == kBatchRegcol ? std::max(ph.cls[r.cls].threads, 32) : a.W;
        const int tiles = (int)(((int64_t)a.G + width - 1) / width * a.nbatch);
        // longest items first: per-tile work ~ transforms x length x stages
        const double c = r.kind == kBatchRegcol ? 0.0 : (double)a.W * a.core.L * (a.core.nst + a.core2.nst);
        order[r.cls].push_back({c, idx, tiles});
      }
      for (int c = 0; c < kBatchClasses; ++c) {
        std::stable_sort(order[c].begin(), order[c].end(), [](const Cost &x, const Cost &y) { return x.c > y.c; });
        b->first_item.push_back((int)items.size());
        for (const Cost &o : order[c])
          for (int t = 0; t < o.tiles; ++t) items.push_back({o.args, t});
        b->nitems.push_back((int)items.size() - b->first_item.back());
        b->ctas.push_back(std::max(1, b->nitems.back() ? batch_resident_ctas<T>(std::max(ph.cls[c].threads, 32),
                                                                                ph.cls[c].smem)
                                                       : 1));
      }
    }
    // (a phase of passes that all launch on their own has no items; keep the
    // uploads non-empty)
    std::vector<TileArgs<T>> args_up = b->host_args;
    if (args_up.empty()) args_up.push_back(TileArgs<T>{});
    if (kinds.empty()) kinds.push_back(-1);
    if (items.empty()) items.push_back({0, 0});
    b->args = upload(args_up.data(), args_up.size() * sizeof(TileArgs<T>));
    b->kinds = upload(kinds.data(), kinds.size() * sizeof(int));
    b->items = upload(items.data(), items.size() * sizeof(BatchItem));
    std::vector<int> zeros(phases.size() * kBatchClasses + 1, 0);
    b->counters = upload(zeros.data(), zeros.size() * sizeof(int));
    return b;
  }

  cudaError_t launch_class(const Bound &b, size_t p, int c, cudaStream_t st) {
    const size_t k = p * kBatchClasses + (size_t)c;
    if (b.nitems[k] == 0) return cudaSuccess;
    const Launch &L = phases[p].cls[c];
    int *counter = reinterpret_cast<int *>(b.counters->ptr) + k;
#ifndef FFB_HOST_EMULATION
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
#else
    cudaError_t e = cudaSuccess;
    *counter = 0;
#endif
    e = launch_batch<T>(reinterpret_cast<const TileArgs<T> *>(b.args->ptr), reinterpret_cast<const int *>(b.kinds->ptr),
                        reinterpret_cast<const BatchItem *>(b.items->ptr) + b.first_item[k], b.nitems[k], counter,
                        std::max(L.threads, 32), L.smem, b.ctas[k], st);
    if (e != cudaSuccess)
      std::fprintf(stderr, "[flagfft] batch phase %zu class %d launch (%d CTAs x %d threads, %zu B shared): %s\n", p, c,
                   b.ctas[k], std::max(L.threads, 32), L.smem, cudaGetErrorString(e));
    return e;
  }

  // The launches of every phase on stream st: the persistent launches of a
  // phase's classes run concurrently on side streams (forked from and joined
  // back into st), the passes launched on their own run on st meanwhile.
  cudaError_t enqueue(const Bound &b, cudaStream_t st) {
    for (size_t p = 0; p < phases.size(); ++p) {
      const Phase &ph = phases[p];
#ifndef FFB_HOST_EMULATION
      cudaError_t e = cudaEventRecord(fork, st);
      if (e != cudaSuccess) return e;
      for (int c = 0; c < kBatchClasses; ++c) {
        if (b.nitems[p * kBatchClasses + (size_t)c] == 0) continue;
        if ((e = cudaStreamWaitEvent(side[c], fork, 0)) != cudaSuccess) return e;
        if ((e = launch_class(b, p, c, side[c])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(join[c], side[c])) != cudaSuccess) return e;
      }
#else
      for (int c = 0; c < kBatchClasses; ++c) {
        cudaError_t e = launch_class(b, p, c, st);
        if (e != cudaSuccess) return e;
      }
#endif
      for (const PassRef &r : ph.passes) {
        if (r.kind >= 0) continue;
        const Group &g = groups[(size_t)r.group];
        const cpx<T> *gin = reinterpret_cast<const cpx<T> *>(b.in) + g.offset;
        cpx<T> *gout = reinterpret_cast<cpx<T> *>(b.out) + g.offset;
        void *s0 = g.prog->scratch0 ? g.prog->scratch0->ptr : nullptr;
        void *s1 = g.prog->scratch1 ? g.prog->scratch1->ptr : nullptr;
        cudaError_t e2 = g.prog->passes[(size_t)r.pass]->run(gin, gout, s0, s1, st);
        if (e2 != cudaSuccess) {
          std::fprintf(stderr, "[flagfft] batch phase %zu: own launch of group %d pass %d: %s\n", p, r.group, r.pass,
                       cudaGetErrorString(e2));
          return e2;
        }
      }
#ifndef FFB_HOST_EMULATION
      for (int c = 0; c < kBatchClasses; ++c) {
        if (b.nitems[p * kBatchClasses + (size_t)c] == 0) continue;
        if ((e = cudaStreamWaitEvent(st, join[c], 0)) != cudaSuccess) return e;
      }
#endif
    }
    return cudaSuccess;
  }

  cudaError_t ensure_streams() {
#ifndef FFB_HOST_EMULATION
    if (fork) return cudaSuccess;
    cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (int c = 0; c < kBatchClasses && e == cudaSuccess; ++c) {
      e = cudaStreamCreateWithFlags(&side[c], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[c], cudaEventDisableTiming);
    }
    return e;
#else
    return cudaSuccess;
#endif
  }

  cudaError_t run(const void *in, void *out, cudaStream_t st) override {
    std::lock_guard<std::mutex> lock(mu);
    cudaError_t se = ensure_streams();
    if (se != cudaSuccess) return se;
    Bound *b = nullptr;
    for (size_t i = 0; i < bound.size(); ++i)
      if (bound[i]->in == in && bound[i]->out == out) {
        std::unique_ptr<Bound> hit = std::move(bound[i]);
        bound.erase(bound.begin() + (long)i);
        bound.push_back(std::move(hit));
        b = bound.back().get();
        break;
      }
    if (b == nullptr) {
      if (bound.size() >= kMaxBound) {
#ifndef FFB_HOST_EMULATION
        cudaStreamSynchronize(st);  // the oldest binding's buffers may still be in use
#endif
        bound.erase(bound.begin());
      }
      bound.push_back(bind(in, out));
      b = bound.back().get();
    }
#ifndef FFB_HOST_EMULATION
    if (graphs) {
      if (b->exec == nullptr) {
        cudaStream_t cap = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        const char *step = "begin capture";
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          cudaError_t le = enqueue(*b, cap);
          step = "end capture";
          e = cudaStreamEndCapture(cap, &b->graph);
          if (le != cudaSuccess) {
            e = le;
            step = "captured launches";
          }
        }
        if (e == cudaSuccess) {
          step = "instantiate";
          e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        }
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) {
          std::fprintf(stderr, "[flagfft] batch graph %s: %s\n", step, cudaGetErrorString(e));
          cudaGetLastError();
          return e;
        }
      }
      return cudaGraphLaunch(b->exec, st);
    }
#endif
    return enqueue(*b, st);
  }

  std::string describe() const override {
    std::ostringstream o;
    o << "  " << groups.size() << " length groups, " << phases.size() << " phases (" << (graphs ? "CUDA graph" : "direct")
      << ")";
    for (size_t p = 0; p < phases.size(); ++p) {
      int persistent[kBatchClasses] = {}, own = 0;
      for (const PassRef &r : phases[p].passes) {
        if (r.kind >= 0)
          persistent[r.cls]++;
        else
          ++own;
      }
      o << "\n  phase " << p << ":";
      for (int c = 0; c < kBatchClasses; ++c)
        if (persistent[c])
          o << " [" << persistent[c] << " passes, one persistent launch of " << std::max(phases[p].cls[c].threads, 32)
            << " threads, " << phases[p].cls[c].smem << " B shared]";
      o << " " << own << " launched on their own";
    }
    const size_t show = std::min<size_t>(groups.size(), 16);
    for (size_t g = 0; g < show; ++g)
      o << "\n  group " << g << ": n=" << groups[g].n << " x" << groups[g].count << " at element " << groups[g].offset
        << "\n" << groups[g].prog->describe();
    if (show < groups.size()) o << "\n  ... " << groups.size() - show << " more groups";
    return o.str();
  }

  int launches() const override {
    int n = 0;
    for (const Phase &ph : phases) {
      bool any[kBatchClasses] = {};
      for (const PassRef &r : ph.passes) {
        if (r.kind >= 0)
          any[r.cls] = true;
        else
          ++n;
      }
      for (bool a : any) n += a ? 1 : 0;
    }
    return n;
  }
};

template <typename T>
std::unique_ptr<BatchProgram> lower_batch_t(const std::vector<BatchGroup> &groups, Planner &planner, bool inverse,
                                            bool use_graphs) {
  auto bp = std::make_unique<BatchProgramT<T>>();
  bp->inverse = inverse;
  bp->graphs = use_graphs;
  int64_t offset = 0;
  for (const BatchGroup &g : groups) {
    if (g.n <= 0 || g.count <= 0) throw std::runtime_error("batch group with a non-positive length or count");
    typename BatchProgramT<T>::Group grp;
    grp.n = g.n;
    grp.count = g.count;
    grp.offset = offset;
    offset += g.n * g.count;
    NodePtr root = build_raw_root(planner, g.n, nullptr, nullptr);
    Layout lay;
    lay.batch = g.count;
    lay.idist = g.n;
    lay.odist = g.n;
    t_no_one_pass = true;
    try {
      grp.prog = lower_t<T>(root, planner, Transform::C2C, inverse, g.n, lay, false);
    } catch (...) {
      t_no_one_pass = false;
      throw;
    }
    t_no_one_pass = false;
    // in-place passes cannot join a persistent launch: prefer a multi-pass lowering
    bool in_place = false;
    for (const auto &ps : grp.prog->passes) {
      auto *tp = dynamic_cast<const TilePass<T> *>(ps.get());
      if (tp && !tp->a.pp && !tp->a.regcol) in_place = true;
    }
    if (in_place) {
      t_policy_override = 2;
      t_no_one_pass = true;
      try {
        grp.prog = lower_t<T>(root, planner, Transform::C2C, inverse, g.n, lay, false);
      } catch (...) {
        t_policy_override = -1;
        t_no_one_pass = false;
        throw;
      }
      t_policy_override = -1;
      t_no_one_pass = false;
    }
    bp->groups.push_back(std::move(grp));
  }
  // Retile ping-pong passes for the shared launches: as many transforms per
  // tile as fill kBatchWidth threads within ~110 KB of shared memory (a
  // standalone plan of a small batch keeps its tiles narrow to spread them
  // over the SMs; in a batch the other groups do that).
  for (auto &g : bp->groups)
    for (auto &ps : g.prog->passes) {
      auto *tp = dynamic_cast<TilePass<T> *>(ps.get());
      if (!tp || !tp->a.pp || tp->a.regcol || tp->a.blue_cols || tp->a.tiles || tp->a.rows_only ||
          tp->a.tpt > kBatchWidth)
        continue;
      TileArgs<T> &a = tp->a;
      const size_t per = pp_tile_smem(a) / (size_t)a.W;
      int64_t W = std::min<int64_t>({(int64_t)(kBatchWidth / a.tpt), (int64_t)a.G,
                                     (int64_t)std::max<size_t>(1, 110 * 1024 / per)});
      W = std::max<int64_t>(W, a.W);
      if (W * std::llabs(a.ig) + a.core.L * std::llabs(a.ii) >= (1ll << 31) ||
          W * std::llabs(a.og) + a.core.L * std::llabs(a.ok) >= (1ll << 31))
        continue;
      a.W = (int)W;
      a.wdiv = make_fastdiv((uint32_t)W);
      tp->smem = per * (size_t)W;
    }
  size_t nph = 0;
  for (const auto &g : bp->groups) nph = std::max(nph, g.prog->passes.size());
  bp->phases.resize(nph);
  for (size_t gi = 0; gi < bp->groups.size(); ++gi) {
    const auto &g = bp->groups[gi];
    for (size_t pi = 0; pi < g.prog->passes.size(); ++pi) {
      auto &ph = bp->phases[pi];
      int kind = -1, cls = 0;
      if (auto *tp = dynamic_cast<const TilePass<T> *>(g.prog->passes[pi].get())) {
        if (tp->a.regcol) {
          kind = kBatchRegcol;
        } else if (tp->a.pp && !tp->a.blue_cols && !tp->a.tiles && !tp->a.rows_only && tp->io == IoKind::C2C) {
          kind = tp->kind == CoreKind::Dit         ? kBatchPpDit
                 : tp->kind == CoreKind::Bluestein ? kBatchPpBluestein
                 : tp->kind == CoreKind::Rader     ? kBatchPpRader
                                                   : kBatchPpConv;
        }
        // a persistent item runs the general ping-pong body: size its shared
        // memory from the tile itself
        const size_t item_smem = kind >= 0 && kind != kBatchRegcol ? pp_tile_smem(tp->a) : 0;
        if (kind >= 0 && kind != kBatchRegcol && item_smem + kBatchSmemHeader > 232448) kind = -1;
        if (kind >= 0) {
          cls = batch_class(item_smem, tp->a.W * tp->a.tpt, kind == kBatchRegcol);
          auto &L = ph.cls[cls];
          L.threads = std::max(L.threads, kind == kBatchRegcol ? 128 : tp->a.W * tp->a.tpt);
          L.smem = std::max(L.smem, item_smem);
        }
      }
      ph.passes.push_back({(int)gi, (int)pi, kind, cls});
    }
  }
  return bp;
}

}  // namespace

std::unique_ptr<BatchProgram> lower_batch(const std::vector<BatchGroup> &groups, Planner &planner, bool is_double,
                                          bool inverse, bool use_graphs) {
  return is_double ? lower_batch_t<double>(groups, planner, inverse, use_graphs)
                   : lower_batch_t<float>(groups, planner, inverse, use_graphs);
}

}  // namespace ffb
