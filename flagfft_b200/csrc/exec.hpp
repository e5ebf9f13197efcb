// Executor: lowers a plan tree (plan.hpp) onto on-chip FFT passes (kernels.cu)
// and owns the plan's device tables and workspaces.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "plan.hpp"

namespace ffb {

// Device allocation owned by a plan.
struct DevMem {
  void *ptr = nullptr;
  size_t bytes = 0;
  explicit DevMem(size_t n);
  ~DevMem();
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
};
using DevPtr = std::shared_ptr<DevMem>;

DevPtr upload(const void *host, size_t bytes);

enum class Transform { C2C, R2C, C2R };

// Buffer a pass reads or writes.
enum class Buf : int { In = 0, Out = 1, Scratch0 = 2, Scratch1 = 3 };

struct PassBase {
  virtual ~PassBase() = default;
  virtual cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const = 0;
  virtual std::string describe() const = 0;
  virtual int launches() const { return 1; }
  // A copy of this pass for `to` transforms where it was lowered for `from`
  // (batch-proportional passes; nullptr for a pass that cannot be re-sized).
  virtual std::shared_ptr<PassBase> rebatched(long long from, long long to) const {
    (void)from;
    (void)to;
    return nullptr;
  }
};

// One direction of one plan: a fixed sequence of passes.
struct Program {
  std::vector<std::unique_ptr<PassBase>> passes;
  std::vector<DevPtr> owned;  // tables and workspaces
  DevPtr scratch0, scratch1;
  cudaError_t run(const void *in, void *out, cudaStream_t st) const;
  std::string describe() const;
  int launches() const;
};

// Layout of one batched 1-D or 2-D request in elements of its own types.
struct Layout {
  int64_t batch = 1;
  int64_t idist = 0;  // input transform distance (input element type)
  int64_t odist = 0;  // output transform distance (output element type)
};

// 1-D: `root` is the plan tree of the length-n complex transform (for R2C /
// C2R the executor derives its own half-length tree with `planner` when n is
// even).  2-D: `root` is a TwoDim node.
std::unique_ptr<Program> lower(const NodePtr &root, Planner &planner, bool is_double, Transform t, bool inverse,
                               int64_t n, const Layout &layout, bool in_place_real);
std::unique_ptr<Program> lower_2d(const NodePtr &root, Planner &planner, bool is_double, Transform t, bool inverse,
                                  int64_t n0, int64_t n1, int64_t batch);

// The same 1-D lowering with every tile pass in a form the persistent
// work-queue kernel takes (no strided tile / TMA column kernels, no one-pass
// four-step Bluestein, a multi-pass chain instead of an in-place pass), as
// batch plans and server templates use it: their requests' passes then join
// one launch per phase instead of launching one by one.
std::unique_ptr<Program> lower_batchable(const NodePtr &root, Planner &planner, bool is_double, Transform t,
                                         bool inverse, int64_t n, const Layout &layout);

// Largest core length one CTA can hold.
int64_t max_onchip_length(bool is_double);

// Batched complex transforms of uneven lengths: `count` transforms of length
// `n` per group, groups packed back to back (group g starts at element
// sum_{h<g} count_h n_h of the input and of the output).
struct BatchGroup {
  int64_t n = 0;
  int64_t count = 0;
};

// One direction of a batch plan: every group's passes gathered into phases
// (phase p holds the p-th pass of every group) that each run as one
// persistent launch over a work queue, replayed through a CUDA graph.
struct BatchProgram {
  virtual ~BatchProgram() = default;
  virtual cudaError_t run(const void *in, void *out, cudaStream_t st) = 0;
  virtual std::string describe() const = 0;
  virtual int launches() const = 0;
};

std::unique_ptr<BatchProgram> lower_batch(const std::vector<BatchGroup> &groups, Planner &planner, bool is_double,
                                          bool inverse, bool use_graphs);

}  // namespace ffb
