// Test infrastructure only: drives the reference's own planner sources
// (src/plan/*.cpp, compiled unmodified by oracle/Makefile) and prints the plan
// tree it builds for each requested length as one JSON object per line, in the
// node shape of the reference's plan serialiser (src/utils/plan_json.cpp:18-57).
//
// The raw-support fallbacks applied after PlanBuilder::build restate
// src/exec/c_api_plan.cpp:9-25 (Rader for primes > 64, else Bluestein with a
// power-of-two convolution) and the root/fallback order of c_api_plan.cpp:169-194.
//
// Usage: plan_dump N:c N:z N0xN1:c ...   (c = complex64, z = complex128)
#include <iostream>
#include <sstream>
#include <string>

#include "flagfft/core.hpp"
#include "plan/rader_utils.hpp"

using namespace flagfft;

namespace {

bool raw_ok(const PlanNodePtr &n) {
  if (std::dynamic_pointer_cast<LeafPlanNode>(n)) return true;
  if (auto f = std::dynamic_pointer_cast<FourStepPlanNode>(n)) return raw_ok(f->row_plan) && raw_ok(f->col_plan);
  if (auto b = std::dynamic_pointer_cast<BluesteinPlanNode>(n)) return raw_ok(b->fft_plan);
  if (auto r = std::dynamic_pointer_cast<RaderPlanNode>(n)) return raw_ok(r->conv_plan);
  return false;
}

std::string ints(const std::vector<int64_t> &v) {
  std::ostringstream o;
  o << "[";
  for (size_t i = 0; i < v.size(); ++i) o << (i ? "," : "") << v[i];
  o << "]";
  return o.str();
}

std::string to_json(const PlanNodePtr &n) {
  std::ostringstream o;
  o << "{\"kind\":\"" << plan_node_kind_name(n->kind) << "\",\"length\":" << n->length;
  if (auto l = std::dynamic_pointer_cast<LeafPlanNode>(n)) {
    o << ",\"factors\":" << ints(l->factors) << ",\"remainder\":" << l->remainder << ",\"lanes\":" << l->lanes
      << ",\"num_warps\":" << l->num_warps << ",\"generic_radices\":" << ints(l->generic_radices)
      << ",\"smem_size\":" << l->smem_size;
  } else if (auto f = std::dynamic_pointer_cast<FourStepPlanNode>(n)) {
    o << ",\"n1\":" << f->n1 << ",\"n2\":" << f->n2 << ",\"row\":" << to_json(f->row_plan)
      << ",\"col\":" << to_json(f->col_plan);
  } else if (auto b = std::dynamic_pointer_cast<BluesteinPlanNode>(n)) {
    o << ",\"conv_length\":" << b->conv_length << ",\"fft_plan\":" << to_json(b->fft_plan);
  } else if (auto r = std::dynamic_pointer_cast<RaderPlanNode>(n)) {
    o << ",\"prime\":" << r->prime << ",\"root\":" << r->root << ",\"conv_length\":" << (r->prime - 1)
      << ",\"conv_plan\":" << to_json(r->conv_plan);
  }
  o << "}";
  return o.str();
}

PlanNodePtr raw_root(PlanBuilder &b, int64_t n, const FFTRequest &r) {
  PlanNodePtr root = b.build(n, r);
  if (!raw_ok(root) && is_prime_length(n) && n > kDirectDftMaxN) {
    int64_t g = find_primitive_root(n);
    PlanNodePtr cand = std::make_shared<RaderPlanNode>(n, g, build_rader_index_table(n, g), b.build(n - 1, r));
    if (raw_ok(cand)) root = cand;
  }
  if (!raw_ok(root)) {
    int64_t m = ceil_power_of_two(2 * n - 1);
    PlanNodePtr cand = std::make_shared<BluesteinPlanNode>(n, m, b.build(m, r));
    if (raw_ok(cand)) root = cand;
  }
  return root;
}

}  // namespace

int main(int argc, char **argv) {
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto p = s.find(':');
    bool z = s.substr(p + 1) == "z";
    std::string dims = s.substr(0, p);
    FFTRequest r;
    r.input_dtype = z ? "complex128" : "complex64";
    r.output_dtype = r.input_dtype;
    r.device_type = "cuda";
    r.device_index = 0;
    r.direction = "forward";
    PlanBuilder b;
    try {
      int64_t n = std::stoll(dims);
      r.requested_n = n;
      PlanNodePtr root = raw_root(b, n, r);
      std::cout << "{\"n\":" << n << ",\"dtype\":\"" << r.input_dtype << "\",\"raw\":" << (raw_ok(root) ? 1 : 0)
                << ",\"root\":" << to_json(root) << "}\n";
    } catch (const std::exception &e) {
      std::cout << "{\"n\":" << dims << ",\"dtype\":\"" << r.input_dtype << "\",\"error\":\"" << e.what()
                << "\"}\n";
    }
  }
  return 0;
}
