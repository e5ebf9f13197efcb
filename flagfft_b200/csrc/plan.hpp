// Planner: restates the reference planner's semantics (src/plan/*.cpp) so the
// plan tree -- factorisation, algorithm choice (leaf / four-step / Bluestein /
// Rader / 2-D RTRT) and cost model -- is the one the reference builds for the
// same request.  The executor (exec.cpp) then lowers that tree onto the sm_100a
// kernels, fusing nodes into as few HBM passes as on-chip capacity allows.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "json.hpp"

namespace ffb {

// src/utils/include/flagfft/base.hpp:30-51 (constants the cost model depends on)
constexpr int64_t kDirectDftMaxN = 64;
constexpr int64_t kLeafMaxN = 4096;
constexpr int64_t kMaxLanes = 128;
constexpr int64_t kDynamicSmemFallbackBytes = 48 * 1024;
extern const std::vector<int64_t> kSupportedRadices;  // {19,17,16,15,13,12,11,10,9,8,7,6,5,4,3,2}

enum class NodeKind { CtLeaf, FourStep, DirectDft, StockhamAutosort, Bluestein, Rader, TwoDim };

std::string node_kind_name(NodeKind k);

struct PlanNode;
using NodePtr = std::shared_ptr<PlanNode>;

// Plan tree node (src/utils/include/flagfft/plan.hpp:14-98).
struct PlanNode {
  NodeKind kind = NodeKind::CtLeaf;
  int64_t length = 0;
  // leaf
  std::vector<int64_t> factors;
  int64_t remainder = 1;
  int64_t lanes = 0;
  int64_t num_warps = 0;
  std::vector<int64_t> generic_radices;
  int64_t smem_size = 0;
  // four-step (n1 = row length, n2 = col length) / two-dim (n1 = n0, n2 = n1)
  int64_t n1 = 0, n2 = 0;
  NodePtr row, col;
  // Bluestein / Rader
  int64_t conv_length = 0;
  int64_t root = 0;
  std::vector<int64_t> idx;
  NodePtr child;

  std::string describe(int indent = 0) const;
  std::string to_json() const;   // reference plan_node_to_json shape
  std::string key_repr() const;  // reference PlanKey::repr shape
};

NodePtr make_leaf_node(int64_t n, std::vector<int64_t> factors, int64_t remainder, int64_t lanes,
                       int64_t warps, std::vector<int64_t> generic, int64_t smem);
NodePtr make_four_step_node(int64_t n, int64_t n1, int64_t n2, NodePtr row, NodePtr col);
NodePtr make_bluestein_node(int64_t n, int64_t m, NodePtr child);
NodePtr make_rader_node(int64_t p, int64_t g, std::vector<int64_t> idx, NodePtr child);
NodePtr make_two_dim_node(int64_t n0, int64_t n1, NodePtr row, NodePtr col);
NodePtr make_direct_node(int64_t n);

bool is_prime_length(int64_t n);
int64_t find_primitive_root(int64_t p);
std::vector<int64_t> rader_index_table(int64_t p, int64_t g);
int64_t ceil_pow2(int64_t v);
int64_t lane_block_for(int64_t lanes);

// A node the executor can run (src/exec/c_api_internal.cpp:122-140): direct
// DFT and Stockham nodes are not.
bool raw_supported(const NodePtr &n);

class Planner {
 public:
  // dtype: false = complex64/float32, true = complex128/float64
  Planner(bool is_double, int64_t max_dynamic_smem_bytes);

  NodePtr build(int64_t n);
  double cost_for(int64_t n);
  // Alternative raw-supported trees for the autotuner, the default tree
  // first: other orders of the leaf radices, balanced four-step splits with
  // the default child trees, and Bluestein / Rader for primes; at most
  // `limit`, distinct by key.
  std::vector<NodePtr> tune_candidates(int64_t n, int limit);
  int64_t choose_lanes(int64_t n, const std::vector<int64_t> &factors) const;
  int64_t choose_num_warps(int64_t lanes) const;

 private:
  struct Candidate {
    NodePtr node;
    double cost;
    int priority;
  };
  std::vector<int64_t> greedy(int64_t n, int64_t *rem) const;
  const std::vector<std::vector<int64_t>> &factorizations(int64_t n);
  std::vector<int64_t> leaf_score(int64_t n, const std::vector<int64_t> &f);
  const std::vector<int64_t> &leaf_factors(int64_t n);
  int64_t leaf_smem_elements(int64_t n, const std::vector<int64_t> &f) const;
  bool use_leaf(int64_t n, const std::vector<int64_t> &f) const;
  NodePtr leaf_plan(int64_t n, const std::vector<int64_t> &f);
  double leaf_cost(int64_t n, const std::vector<int64_t> &f) const;
  double four_step_cost(int64_t n1, int64_t n2);
  int priority(const NodePtr &n) const;
  const std::vector<int64_t> &divisors(int64_t n);
  int64_t next_conv_length(int64_t minimum) const;
  std::vector<Candidate> candidates(int64_t n);
  static const Candidate &select(const std::vector<Candidate> &c);
  NodePtr auto_node(int64_t n);

  bool is_double_;
  int64_t smem_limit_;
  std::unordered_map<int64_t, NodePtr> node_cache_;
  std::unordered_map<int64_t, double> cost_cache_;
  std::unordered_map<int64_t, std::vector<int64_t>> divisor_cache_;
  std::unordered_map<int64_t, std::vector<std::vector<int64_t>>> fact_cache_;
  std::unordered_map<int64_t, std::vector<int64_t>> leaf_cache_;
};

// Root plan for a 1-D length with the raw-support fallbacks of
// src/exec/c_api_plan.cpp:9-25,169-194 (tuned tree first if one is given).
NodePtr build_raw_root(Planner &planner, int64_t n, const NodePtr &tuned_fwd, const NodePtr &tuned_inv);

// Plan tree from the reference plan-JSON node shape (src/plan/plan_deserialize.cpp:6-77).
NodePtr node_from_json(Planner &planner, const std::string &json);
NodePtr node_from_json(Planner &planner, const Json &json);

}  // namespace ffb
