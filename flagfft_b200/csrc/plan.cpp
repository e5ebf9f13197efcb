// Planner restatement.  Each function cites the reference function whose
// behaviour it keeps; the cost model's formulas and the candidate order are
// kept exactly (including floating-point expression order) because ties are
// broken by them and the plan tree must match the reference's.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <sstream>
#include <stdexcept>

#include "json.hpp"

namespace ffb {

const std::vector<int64_t> kSupportedRadices = {19, 17, 16, 15, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
// Every supported radix has a specialised codelet (base.hpp:48-50), so no
// factor of a supported factorisation is a "generic" radix.
static bool is_generic_radix(int64_t r) {
  return std::find(kSupportedRadices.begin(), kSupportedRadices.end(), r) == kSupportedRadices.end();
}

std::string node_kind_name(NodeKind k) {  // src/utils/base.cpp plan_node_kind_name
  switch (k) {
    case NodeKind::CtLeaf: return "ct_leaf";
    case NodeKind::FourStep: return "four_step";
    case NodeKind::DirectDft: return "direct_dft";
    case NodeKind::StockhamAutosort: return "stockham_autosort";
    case NodeKind::Bluestein: return "bluestein";
    case NodeKind::Rader: return "rader";
    case NodeKind::TwoDim: return "two_dim";
  }
  return "unknown";
}

int64_t ceil_pow2(int64_t v) {
  int64_t r = 1;
  while (r < v) r <<= 1;
  return r;
}

int64_t lane_block_for(int64_t lanes) { return lanes <= 1 ? 1 : ceil_pow2(lanes); }

// ---------------------------------------------------------------------------
// nodes
// ---------------------------------------------------------------------------

NodePtr make_leaf_node(int64_t n, std::vector<int64_t> factors, int64_t remainder, int64_t lanes, int64_t warps,
                       std::vector<int64_t> generic, int64_t smem) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::CtLeaf;
  p->length = n;
  p->factors = std::move(factors);
  p->remainder = remainder;
  p->lanes = lanes;
  p->num_warps = warps;
  p->generic_radices = std::move(generic);
  p->smem_size = smem;
  return p;
}

NodePtr make_four_step_node(int64_t n, int64_t n1, int64_t n2, NodePtr row, NodePtr col) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::FourStep;
  p->length = n;
  p->n1 = n1;
  p->n2 = n2;
  p->row = std::move(row);
  p->col = std::move(col);
  return p;
}

NodePtr make_bluestein_node(int64_t n, int64_t m, NodePtr child) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::Bluestein;
  p->length = n;
  p->conv_length = m;
  p->child = std::move(child);
  return p;
}

NodePtr make_rader_node(int64_t prime, int64_t g, std::vector<int64_t> idx, NodePtr child) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::Rader;
  p->length = prime;
  p->root = g;
  p->idx = std::move(idx);
  p->conv_length = prime - 1;
  p->child = std::move(child);
  return p;
}

NodePtr make_two_dim_node(int64_t n0, int64_t n1, NodePtr row, NodePtr col) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::TwoDim;
  p->length = n0 * n1;
  p->n1 = n0;
  p->n2 = n1;
  p->row = std::move(row);
  p->col = std::move(col);
  return p;
}

NodePtr make_direct_node(int64_t n) {
  auto p = std::make_shared<PlanNode>();
  p->kind = NodeKind::DirectDft;
  p->length = n;
  return p;
}

static std::string ints_br(const std::vector<int64_t> &v) {
  std::string s = "[";
  for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + std::to_string(v[i]);
  return s + "]";
}

// Text shape of src/plan/nodes.cpp:25-71 (describe()).
std::string PlanNode::describe(int indent) const {
  std::ostringstream o;
  std::string pad((size_t)indent, ' ');
  switch (kind) {
    case NodeKind::CtLeaf:
      o << pad << "LeafPlan(n=" << length << ", factors=" << ints_br(factors) << ", lanes=" << lanes
        << ", num_warps=" << num_warps;
      if (!generic_radices.empty()) o << ", generic_radices=" << ints_br(generic_radices);
      o << ", smem_size=" << smem_size << ")";
      break;
    case NodeKind::DirectDft:
      o << pad << "DirectDFT(n=" << length << ")";
      break;
    case NodeKind::StockhamAutosort:
      o << pad << "Stockham(n=" << length << ", factors=" << ints_br(factors) << ")";
      break;
    case NodeKind::FourStep:
      o << pad << "FourStep(n=" << length << ", n1=" << n1 << ", n2=" << n2 << ")\n"
        << row->describe(indent + 2) << "\n"
        << col->describe(indent + 2);
      break;
    case NodeKind::Bluestein:
      o << pad << "Bluestein(n=" << length << ", conv_length=" << conv_length << ")\n" << child->describe(indent + 2);
      break;
    case NodeKind::Rader:
      o << pad << "Rader(p=" << length << ", root=" << root << ", conv_length=" << (length - 1) << ")\n"
        << child->describe(indent + 2);
      break;
    case NodeKind::TwoDim:
      o << pad << "TwoDim(strategy=RTRT, n0=" << n1 << ", n1=" << n2 << ")\n"
        << row->describe(indent + 2) << "\n"
        << col->describe(indent + 2);
      break;
  }
  return o.str();
}

// JSON shape of src/utils/plan_json.cpp:18-57 (plan_node_to_json).
std::string PlanNode::to_json() const {
  std::ostringstream o;
  o << "{\"kind\":\"" << node_kind_name(kind) << "\",\"length\":" << length;
  switch (kind) {
    case NodeKind::CtLeaf:
      o << ",\"factors\":" << json_ints(factors) << ",\"remainder\":" << remainder << ",\"lanes\":" << lanes
        << ",\"num_warps\":" << num_warps << ",\"generic_radices\":" << json_ints(generic_radices)
        << ",\"smem_size\":" << smem_size;
      break;
    case NodeKind::FourStep:
      o << ",\"n1\":" << n1 << ",\"n2\":" << n2 << ",\"row\":" << row->to_json() << ",\"col\":" << col->to_json();
      break;
    case NodeKind::Bluestein:
      o << ",\"conv_length\":" << conv_length << ",\"fft_plan\":" << child->to_json();
      break;
    case NodeKind::Rader:
      o << ",\"prime\":" << length << ",\"root\":" << root << ",\"idx\":" << json_ints(idx)
        << ",\"conv_length\":" << (length - 1) << ",\"conv_plan\":" << child->to_json();
      break;
    case NodeKind::TwoDim:
      o << ",\"n0\":" << n1 << ",\"n1\":" << n2 << ",\"strategy\":\"RTRT\",\"row\":" << row->to_json()
        << ",\"col\":" << col->to_json();
      break;
    case NodeKind::DirectDft:
      o << ",\"impl\":\"direct\"";
      break;
    case NodeKind::StockhamAutosort:
      o << ",\"factors\":" << json_ints(factors);
      break;
  }
  o << "}";
  return o.str();
}

// src/utils/plan_key.cpp:14-48 (PlanKey::repr), schema 3.
std::string PlanNode::key_repr() const {
  std::ostringstream o;
  o << "schema=3;kind=" << node_kind_name(kind) << ";length=" << length;
  const std::vector<int64_t> &f = kind == NodeKind::Rader ? idx : factors;
  if (!f.empty()) o << ";factors=[" << json_ints(f).substr(1, json_ints(f).size() - 2) << "]";
  if (kind == NodeKind::CtLeaf) {
    std::string g = json_ints(generic_radices);
    o << ";remainder=" << remainder << ";lanes=" << lanes << ";num_warps=" << num_warps << ";generic_radices=["
      << g.substr(1, g.size() - 2) << "];smem_size=" << smem_size;
  }
  if (kind == NodeKind::FourStep) o << ";n1=" << n1 << ";n2=" << n2;
  if (kind == NodeKind::TwoDim) o << ";n0=" << n1 << ";n1=" << n2;
  if (kind == NodeKind::Bluestein) o << ";conv_length=" << conv_length;
  if (kind == NodeKind::Rader) {
    std::string s = json_ints(idx);
    o << ";conv_length=" << (length - 1) << ";root=" << root << ";idx=[" << s.substr(1, s.size() - 2) << "]";
  }
  std::vector<NodePtr> kids;
  if (kind == NodeKind::FourStep || kind == NodeKind::TwoDim) kids = {row, col};
  if (kind == NodeKind::Bluestein || kind == NodeKind::Rader) kids = {child};
  if (!kids.empty()) {
    o << ";children=[";
    for (size_t i = 0; i < kids.size(); ++i) o << (i ? "|" : "") << "{" << kids[i]->key_repr() << "}";
    o << "]";
  }
  return o.str();
}

// ---------------------------------------------------------------------------
// number theory (src/plan/rader_utils.cpp:40-90)
// ---------------------------------------------------------------------------

bool is_prime_length(int64_t n) {
  if (n < 2) return false;
  if (n % 2 == 0) return n == 2;
  for (int64_t d = 3; d * d <= n; d += 2)
    if (n % d == 0) return false;
  return true;
}

static int64_t powmod(int64_t b, int64_t e, int64_t m) {
  int64_t r = 1;
  b %= m;
  while (e > 0) {
    if (e & 1) r = (int64_t)((__int128)r * b % m);
    b = (int64_t)((__int128)b * b % m);
    e >>= 1;
  }
  return r;
}

int64_t find_primitive_root(int64_t p) {
  if (!is_prime_length(p)) throw std::runtime_error("Rader primitive root requires a prime length");
  if (p == 2) return 1;
  const int64_t phi = p - 1;
  std::vector<int64_t> fac;
  int64_t t = phi;
  for (int64_t d = 2; d * d <= t; ++d) {
    if (t % d) continue;
    fac.push_back(d);
    while (t % d == 0) t /= d;
  }
  if (t > 1) fac.push_back(t);
  for (int64_t g = 2; g < p; ++g) {
    bool ok = true;
    for (int64_t q : fac)
      if (powmod(g, phi / q, p) == 1) {
        ok = false;
        break;
      }
    if (ok) return g;
  }
  throw std::runtime_error("failed to find primitive root for prime length");
}

std::vector<int64_t> rader_index_table(int64_t p, int64_t g) {
  std::vector<int64_t> idx((size_t)(p - 1));
  int64_t v = 1;
  for (int64_t q = 0; q < p - 1; ++q) {
    idx[(size_t)q] = v;
    v = (v * g) % p;
  }
  return idx;
}

bool raw_supported(const NodePtr &n) {
  if (!n) return false;
  switch (n->kind) {
    case NodeKind::CtLeaf: return true;
    case NodeKind::FourStep:
    case NodeKind::TwoDim: return raw_supported(n->row) && raw_supported(n->col);
    case NodeKind::Bluestein:
    case NodeKind::Rader: return raw_supported(n->child);
    default: return false;
  }
}

// ---------------------------------------------------------------------------
// planner
// ---------------------------------------------------------------------------

Planner::Planner(bool is_double, int64_t smem) : is_double_(is_double), smem_limit_(smem) {}

// src/plan/factorization.cpp:5-28 (greedy over the radix list)
std::vector<int64_t> Planner::greedy(int64_t n, int64_t *rem_out) const {
  if (n <= 0) throw std::runtime_error("FFT length must be positive");
  std::vector<int64_t> f;
  int64_t rem = n;
  while (rem > 1) {
    bool found = false;
    for (int64_t r : kSupportedRadices) {
      if (rem % r == 0) {
        f.push_back(r);
        rem /= r;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  *rem_out = rem;
  return f;
}

// src/plan/factorization.cpp:30-55 (all ordered factorisations, sorted, unique)
const std::vector<std::vector<int64_t>> &Planner::factorizations(int64_t n) {
  auto it = fact_cache_.find(n);
  if (it != fact_cache_.end()) return it->second;
  std::vector<std::vector<int64_t>> out;
  for (int64_t r : kSupportedRadices) {
    if (n % r) continue;
    if (n == r) {
      out.push_back({r});
      continue;
    }
    for (const auto &tail : factorizations(n / r)) {
      std::vector<int64_t> f{r};
      f.insert(f.end(), tail.begin(), tail.end());
      out.push_back(std::move(f));
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return fact_cache_[n] = std::move(out);
}

// src/plan/factorization.cpp:71-84 (largest divisor of gcd(n/f_i) up to 128)
int64_t Planner::choose_lanes(int64_t n, const std::vector<int64_t> &f) const {
  int64_t g = n / f.front();
  for (size_t i = 1; i < f.size(); ++i) g = std::gcd(g, n / f[i]);
  for (int64_t c = std::min(g, kMaxLanes); c > 0; --c)
    if (g % c == 0) return c;
  return 1;
}

// src/plan/factorization.cpp:129-136
int64_t Planner::choose_num_warps(int64_t lanes) const {
  int64_t warps = std::max<int64_t>(1, (lane_block_for(lanes) + 31) / 32);
  int64_t c = 1;
  while (c < warps) c *= 2;
  return std::min<int64_t>(c, 8);
}

// src/plan/cost_model.cpp:10-24
double Planner::leaf_cost(int64_t n, const std::vector<int64_t> &f) const {
  int64_t lanes = choose_lanes(n, f);
  int64_t warps = choose_num_warps(lanes);
  int64_t generic = 0;
  for (int64_t r : f)
    if (is_generic_radix(r)) ++generic;
  double base = static_cast<double>(n * static_cast<int64_t>(f.size()) * warps) / static_cast<double>(lanes);
  return base + static_cast<double>(generic * n);
}

// src/plan/factorization.cpp:86-105 (lexicographic score; first best kept)
std::vector<int64_t> Planner::leaf_score(int64_t n, const std::vector<int64_t> &f) {
  int64_t lanes = choose_lanes(n, f);
  int64_t generic = 0;
  for (int64_t r : f)
    if (is_generic_radix(r)) ++generic;
  int64_t warm = static_cast<int64_t>(std::llround(leaf_cost(n, f) * 1024.0));
  std::vector<int64_t> s = {-warm, -static_cast<int64_t>(f.size()), lanes, -lane_block_for(lanes), -generic};
  s.insert(s.end(), f.begin(), f.end());
  return s;
}

// src/plan/factorization.cpp:107-127
const std::vector<int64_t> &Planner::leaf_factors(int64_t n) {
  auto it = leaf_cache_.find(n);
  if (it != leaf_cache_.end()) return it->second;
  const auto &cands = factorizations(n);
  std::vector<int64_t> best;
  if (cands.empty()) {
    int64_t rem = 1;
    best = greedy(n, &rem);
    if (rem != 1 || best.empty()) throw std::runtime_error("length is not fully factorable by supported radices");
  } else {
    best = cands.front();
    auto best_score = leaf_score(n, best);
    for (const auto &c : cands) {
      auto s = leaf_score(n, c);
      if (s > best_score) {
        best = c;
        best_score = std::move(s);
      }
    }
  }
  return leaf_cache_[n] = best;
}

// src/plan/factorization.cpp:138-162
int64_t Planner::leaf_smem_elements(int64_t n, const std::vector<int64_t> &f) const {
  return f.size() <= 1 ? 0 : ceil_pow2(n);
}

bool Planner::use_leaf(int64_t n, const std::vector<int64_t> &f) const {
  int64_t bytes = 4 * leaf_smem_elements(n, f) * (is_double_ ? 8 : 4);
  return n <= kLeafMaxN && bytes <= smem_limit_;
}

// src/plan/factorization.cpp:170-193
NodePtr Planner::leaf_plan(int64_t n, const std::vector<int64_t> &f) {
  int64_t lanes = choose_lanes(n, f);
  std::vector<int64_t> generic;
  for (int64_t r : f)
    if (is_generic_radix(r) && std::find(generic.begin(), generic.end(), r) == generic.end()) generic.push_back(r);
  std::sort(generic.begin(), generic.end());
  return make_leaf_node(n, f, 1, lanes, choose_num_warps(lanes), generic, leaf_smem_elements(n, f));
}

// src/plan/cost_model.cpp:30-33
double Planner::four_step_cost(int64_t n1, int64_t n2) {
  return static_cast<double>(n2) * cost_for(n1) + static_cast<double>(n1) * cost_for(n2) +
         static_cast<double>(n1 * n2);
}

// src/plan/cost_model.cpp:45-66
int Planner::priority(const NodePtr &n) const {
  switch (n->kind) {
    case NodeKind::CtLeaf: return 0;
    case NodeKind::FourStep: return 1;
    case NodeKind::StockhamAutosort: return 2;
    case NodeKind::Bluestein:
    case NodeKind::Rader: return 3;
    case NodeKind::DirectDft: return 4;
    case NodeKind::TwoDim: return 5;
  }
  return 99;
}

// src/plan/auto_candidates.cpp:7-26
const std::vector<int64_t> &Planner::divisors(int64_t n) {
  auto it = divisor_cache_.find(n);
  if (it != divisor_cache_.end()) return it->second;
  std::vector<int64_t> d;
  int64_t root = static_cast<int64_t>(std::sqrt(static_cast<double>(n)));
  for (int64_t x = 1; x <= root; ++x) {
    if (n % x) continue;
    d.push_back(x);
    if (n / x != x) d.push_back(n / x);
  }
  std::sort(d.begin(), d.end());
  return divisor_cache_[n] = std::move(d);
}

// src/plan/auto_candidates.cpp:28-40
int64_t Planner::next_conv_length(int64_t minimum) const {
  if (minimum <= 1) return 1;
  int64_t power = ceil_pow2(minimum);
  for (int64_t c = minimum; c <= power; ++c) {
    int64_t rem = 1;
    auto f = greedy(c, &rem);
    if (rem == 1 && !f.empty()) return c;
  }
  return power;
}

// src/plan/auto_candidates.cpp:56-106 (candidate order matters for ties)
std::vector<Planner::Candidate> Planner::candidates(int64_t n) {
  if (n <= 0) throw std::runtime_error("FFT length must be positive");
  std::vector<Candidate> c;
  int64_t rem = 1;
  auto g = greedy(n, &rem);
  if (rem == 1 && !g.empty() && use_leaf(n, g)) {
    const auto &f = leaf_factors(n);
    NodePtr node = leaf_plan(n, f);
    c.push_back({node, leaf_cost(n, f), priority(node)});
  }
  if (n <= kDirectDftMaxN) {
    NodePtr node = make_direct_node(n);
    c.push_back({node, static_cast<double>(n * n), priority(node)});
  }
  if (n == 16384 && use_leaf(64, {4, 4, 4}) && use_leaf(256, {4, 8, 8})) {
    NodePtr row = leaf_plan(64, {4, 4, 4});
    NodePtr col = leaf_plan(256, {4, 8, 8});
    NodePtr node = make_four_step_node(n, 64, 256, row, col);
    c.push_back({node, four_step_cost(64, 256) * 0.5, priority(node)});
  }
  for (int64_t n1 : std::vector<int64_t>(divisors(n))) {
    if (n1 <= 1 || n1 >= n) continue;
    int64_t n2 = n / n1;
    try {
      NodePtr row = auto_node(n1);
      NodePtr col = auto_node(n2);
      NodePtr node = make_four_step_node(n, n1, n2, row, col);
      double balance = std::abs(std::log(static_cast<double>(n1)) - std::log(static_cast<double>(n2)));
      c.push_back({node, four_step_cost(n1, n2) + balance, priority(node)});
    } catch (const std::exception &) {
    }
  }
  if (c.empty() && n > kDirectDftMaxN) {
    int64_t m = next_conv_length(2 * n - 1);
    NodePtr node = make_bluestein_node(n, m, auto_node(m));
    c.push_back({node, 3.0 * cost_for(m) + static_cast<double>(n + m), priority(node)});
    if (is_prime_length(n)) {
      int64_t root = find_primitive_root(n);
      NodePtr rader = make_rader_node(n, root, rader_index_table(n, root), auto_node(n - 1));
      int64_t conv = n - 1;
      c.push_back({rader, 3.0 * cost_for(conv) + static_cast<double>(n + 3 * conv), priority(rader)});
    }
  }
  return c;
}

// src/plan/tune_candidates.cpp:141-152 (min cost, then priority; first minimum)
const Planner::Candidate &Planner::select(const std::vector<Candidate> &c) {
  if (c.empty()) throw std::runtime_error("no FFT plan candidates were generated");
  return *std::min_element(c.begin(), c.end(), [](const Candidate &a, const Candidate &b) {
    if (a.cost != b.cost) return a.cost < b.cost;
    return a.priority < b.priority;
  });
}

// src/plan/tune_candidates.cpp:154-163
NodePtr Planner::auto_node(int64_t n) {
  auto it = node_cache_.find(n);
  if (it != node_cache_.end()) return it->second;
  auto c = candidates(n);
  const Candidate &best = select(c);
  node_cache_[n] = best.node;
  cost_cache_[n] = best.cost;
  return best.node;
}

// src/plan/builder_context.cpp:42-48
NodePtr Planner::build(int64_t n) {
  if (n <= 0) throw std::runtime_error("FFT length must be positive");
  return auto_node(n);
}

// src/plan/builder_context.cpp:55-67
double Planner::cost_for(int64_t n) {
  auto it = cost_cache_.find(n);
  if (it != cost_cache_.end()) return it->second;
  auto c = candidates(n);
  if (c.empty()) throw std::runtime_error("length " + std::to_string(n) + " has no supported FFT implementation route");
  double v = select(c).cost;
  cost_cache_[n] = v;
  return v;
}

std::vector<NodePtr> Planner::tune_candidates(int64_t n, int limit) {
  std::vector<NodePtr> out;
  std::vector<std::string> seen;
  auto add = [&](const NodePtr &node) {
    if (!node || (int)out.size() >= limit || !raw_supported(node)) return;
    const std::string k = node->key_repr();
    if (std::find(seen.begin(), seen.end(), k) != seen.end()) return;
    seen.push_back(k);
    out.push_back(node);
  };
  NodePtr def = build_raw_root(*this, n, nullptr, nullptr);
  add(def);
  // leaf radix orders (descending, ascending) of the default factor multiset
  int64_t rem = 1;
  auto g = greedy(n, &rem);
  if (rem == 1 && !g.empty() && n <= kLeafMaxN) {
    std::vector<int64_t> f = leaf_factors(n);
    std::vector<int64_t> asc = f, desc = f;
    std::sort(asc.begin(), asc.end());
    std::sort(desc.rbegin(), desc.rend());
    for (const auto &o : {desc, asc, g})
      if (use_leaf(n, o)) add(leaf_plan(n, o));
  }
  // four-step splits, most balanced first, children from the default planner
  std::vector<std::pair<double, int64_t>> pairs;
  for (int64_t n1 : divisors(n)) {
    if (n1 <= 1 || n1 >= n) continue;
    pairs.push_back({std::abs(std::log((double)n1) - std::log((double)(n / n1))), n1});
  }
  std::sort(pairs.begin(), pairs.end());
  int splits = 0;
  for (const auto &pr : pairs) {
    if (splits >= 4) break;
    try {
      add(make_four_step_node(n, pr.second, n / pr.second, auto_node(pr.second), auto_node(n / pr.second)));
      ++splits;
    } catch (const std::exception &) {
    }
  }
  // convolution routes for primes and lengths without a leaf
  if (n > kDirectDftMaxN && (is_prime_length(n) || rem != 1)) {
    const int64_t m = next_conv_length(2 * n - 1);
    add(make_bluestein_node(n, m, auto_node(m)));
    if (is_prime_length(n)) {
      const int64_t root = find_primitive_root(n);
      add(make_rader_node(n, root, rader_index_table(n, root), auto_node(n - 1)));
    }
  }
  return out;
}

NodePtr build_raw_root(Planner &planner, int64_t n, const NodePtr &tuned_fwd, const NodePtr &tuned_inv) {
  NodePtr root = (tuned_fwd && raw_supported(tuned_fwd)) ? tuned_fwd : planner.build(n);
  if (!raw_supported(root)) root = (tuned_inv && raw_supported(tuned_inv)) ? tuned_inv : planner.build(n);
  if (!raw_supported(root) && is_prime_length(n) && n > kDirectDftMaxN) {
    int64_t g = find_primitive_root(n);
    NodePtr cand = make_rader_node(n, g, rader_index_table(n, g), planner.build(n - 1));
    if (raw_supported(cand)) root = cand;
  }
  if (!raw_supported(root)) {
    int64_t m = ceil_pow2(2 * n - 1);
    NodePtr cand = make_bluestein_node(n, m, planner.build(m));
    if (raw_supported(cand)) root = cand;
  }
  return root;
}

// src/plan/plan_deserialize.cpp:6-77
static NodePtr node_from(Planner &pl, const Json &j) {
  std::string kind = j.at("kind").str;
  int64_t length = j.at("length").i64();
  if (kind == "ct_leaf") {
    auto f = j.at("factors").ivec();
    int64_t prod = 1;
    for (int64_t r : f) {
      if (std::find(kSupportedRadices.begin(), kSupportedRadices.end(), r) == kSupportedRadices.end())
        throw std::runtime_error("forced plan uses an unsupported radix");
      prod *= r;
    }
    if (f.empty() || prod != length) throw std::runtime_error("forced leaf factors do not multiply to its length");
    int64_t rem = j.has("remainder") ? j.at("remainder").i64() : 1;
    int64_t lanes = j.has("lanes") ? j.at("lanes").i64() : pl.choose_lanes(length, f);
    int64_t warps = j.has("num_warps") ? j.at("num_warps").i64() : pl.choose_num_warps(lanes);
    std::vector<int64_t> generic;
    if (j.has("generic_radices")) generic = j.at("generic_radices").ivec();
    int64_t smem = j.has("smem_size") ? j.at("smem_size").i64() : (f.size() <= 1 ? 0 : ceil_pow2(length));
    return make_leaf_node(length, f, rem, lanes, warps, generic, smem);
  }
  if (kind == "four_step") {
    int64_t n1 = j.at("n1").i64(), n2 = j.at("n2").i64();
    if (n1 * n2 != length) throw std::runtime_error("forced four-step sizes do not multiply to its length");
    return make_four_step_node(length, n1, n2, node_from(pl, j.at("row")), node_from(pl, j.at("col")));
  }
  if (kind == "bluestein") {
    int64_t m = j.at("conv_length").i64();
    if (m < 2 * length - 1) throw std::runtime_error("forced Bluestein convolution is too short");
    NodePtr ch = node_from(pl, j.at("fft_plan"));
    if (ch->length != m) throw std::runtime_error("forced Bluestein child length mismatch");
    return make_bluestein_node(length, m, ch);
  }
  if (kind == "rader") {
    if (!is_prime_length(length)) throw std::runtime_error("forced Rader length is not prime");
    int64_t g = j.at("root").i64();
    std::vector<int64_t> idx = j.has("idx") ? j.at("idx").ivec() : rader_index_table(length, g);
    if (idx != rader_index_table(length, g)) throw std::runtime_error("forced Rader index table is inconsistent");
    NodePtr ch = node_from(pl, j.at("conv_plan"));
    if (ch->length != length - 1) throw std::runtime_error("forced Rader child length mismatch");
    return make_rader_node(length, g, idx, ch);
  }
  if (kind == "direct_dft") return make_direct_node(length);
  if (kind == "two_dim") {
    return make_two_dim_node(j.at("n0").i64(), j.at("n1").i64(), node_from(pl, j.at("row")), node_from(pl, j.at("col")));
  }
  throw std::runtime_error("unsupported plan node kind in forced plan: " + kind);
}

NodePtr node_from_json(Planner &planner, const std::string &json) { return node_from(planner, Json::parse(json)); }
NodePtr node_from_json(Planner &planner, const Json &json) { return node_from(planner, json); }

}  // namespace ffb
