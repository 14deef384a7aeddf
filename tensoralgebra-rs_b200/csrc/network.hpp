// N-ary contraction networks: a list of labelled input tensors, the labels
// and layout of the output, and a pairwise contraction path, executed as a
// sequence of binary contractions whose intermediates stay in device memory.
//
// The reference keeps the N-ary layer (einsum) above its stack, in its
// callers (docs/architecture.md:54): a caller such as tenferro-rs contracts a
// network by calling Problem::from_labels / Plan::execute_into once per pair.
// This is that caller on the GPU. Each step is an ordinary product (plan
// built once, at network creation); intermediates are dense column-major with
// their labels ordered [free labels of the first operand, free labels of the
// second, shared (batch) labels], in one device arena; a list of networks runs
// step by step, each step of every network in one grouped submission
// (contract_batched), so independent networks share launches and CUDA graphs.
#pragma once

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "runtime.hpp"

namespace tprims {

struct NetworkOperand {
  Operand op;  // layout (element offset 0) and conjugation
  std::vector<int64_t> labels;
};

struct NetworkStep {
  int a = 0, b = 0;             // operand ids: inputs 0..n-1, the result of step s is n + s
  std::vector<int64_t> la, lb;  // labels of the two operands
  std::vector<int64_t> labels;  // labels of the result
  std::vector<int64_t> dims;    // extents of the result
  size_t offset = 0;            // byte offset of an intermediate result in the arena
  size_t bytes = 0;
  bool last = false;            // writes the network's output
  std::unique_ptr<Product> plan;
};

struct Network {
  DType dtype = DType::F64;
  std::vector<NetworkOperand> inputs;
  NetworkOperand output;
  std::vector<std::pair<int, int>> path;  // positions in the operand list (opt_einsum convention)
  bool greedy = false;                    // the path was chosen here
  std::vector<NetworkStep> steps;
  size_t arena_bytes = 0;
  std::mutex mu;
  std::map<int, void*> arena;  // per device, when the caller passes no workspace

  // Validates labels and extents, completes the path (greedy when `path` is
  // empty) and builds one plan per step.
  static Network* create(DType dtype, std::vector<NetworkOperand> inputs, NetworkOperand output,
                         std::vector<std::pair<int, int>> path);
  ~Network();
  double macs() const;
  std::string report() const;
};

// Greedy pairwise path: repeatedly the pair of operands that share a label
// (any pair when none do) with the fewest multiply-accumulates, ties to the
// smaller result. Positions follow the opt_einsum convention: both operands
// are removed and the result is appended.
std::vector<std::pair<int, int>> greedy_path(const std::vector<std::vector<int64_t>>& labels,
                                             const std::vector<int64_t>& out_labels,
                                             const std::map<int64_t, int64_t>& extents);

// Runs networks on the executor: step s of every network that has one forms
// one grouped submission, in order of s. alpha and beta apply to each
// network's last step (D = alpha * network + beta * D); inputs[i][j] is the
// origin of input j of network i, outs[i] the output origin, workspaces[i] a
// device buffer of the network's arena_bytes or null (the network's own arena).
void execute_networks(Executor& ex, int n, Network* const* nets, const Scalar* alpha, const Scalar* beta,
                      const void* const* const* inputs, void* const* outs, void* const* workspaces);

}  // namespace tprims
