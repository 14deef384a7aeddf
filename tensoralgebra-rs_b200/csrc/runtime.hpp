// Executors and prepared products: the state behind TAPP_executor and
// TAPP_tensor_product handles.
//
// A product snapshots its validated Problem and PackedPlan at creation (the
// reference's product.rs:83-195 does the same on the CPU); it holds no data
// pointer and no executor. Device copies of the oriented scatter vectors are
// made lazily, once per device, on first execution.
//
// An executor owns one CUDA stream on one device, a workspace arena that grows
// and is then reused (no allocation in the steady state), and a device status
// word that bounded-wait kernels report into. TAPP execution is synchronous
// (crates/tprims-capi/src/execute.rs:153): every call drains the stream before
// it returns, unless the executor was switched to asynchronous mode.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "plan.hpp"

namespace tprims {

// Per-kernel-family timing of an executor (opt-in): CUDA events recorded on
// the executor's stream around every launch, resolved when the stream drains.
struct KernelTimes {
  struct Pending {
    std::string name;
    cudaEvent_t beg, end;
  };
  struct Total {
    double ms = 0;
    long launches = 0;
  };
  std::vector<Pending> pending;
  std::map<std::string, Total> totals;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take();
  void resolve();  // after the stream is drained
  ~KernelTimes();
};

struct Executor {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t capture_stream = nullptr;  // grouped-graph captures only
  bool sync = true;
  bool profile = false;
  bool grouping = true;
  size_t ws_limit = SIZE_MAX;  // cap of the workspace arena (allocation-failure injection)
  int drain_limit_s = 300;     // bound of one wait for the stream to drain
  KernelTimes times;
  size_t pool_size = 0, budget = 1;  // recorded for the pooled-executor extension
  void* ws = nullptr;
  size_t ws_bytes = 0;
  unsigned* status = nullptr;  // device word
  int num_sms = 148;
  std::mutex mu;
  std::atomic<int> inflight{0};
  // CUDA graphs of grouped submissions, keyed by the item list.
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    void* buf = nullptr;  // descriptors, tile starts, claim counters
    uint64_t last_use = 0;
    std::vector<int> single;  // items of the list that run individually
  };
  std::map<uint64_t, Graph> graphs;
  uint64_t graph_clock = 0;

  static Executor* create(int device, uintptr_t stream);
  ~Executor();
  // A device buffer of at least `bytes` from the arena (contents undefined).
  void* workspace(size_t bytes);
};

struct DeviceScatters {
  int64_t* buf = nullptr;
  dev::Scatters s{};
};

struct Product {
  Problem problem;
  PackedPlan packed;
  OrientedView view;
  Scheme scheme = Scheme::Plain;
  int ozaki_slices = 0;
  int kernel_pin = 0;
  // Batch strides of the oriented view for the tiny batched kernel.
  dev::TinyStrides tiny_h{};
  // Unique over the process lifetime (never reused, unlike the address), so a
  // cached grouped graph can never be replayed for a newer plan.
  const uint64_t uid;
  std::mutex mu;
  std::map<int, DeviceScatters> dev;  // per device
  // Adjoint contractions of Plan::vjp, built on first use.
  std::unique_ptr<Product> adj_a, adj_b;

  explicit Product(const Problem& p);
  ~Product();
  // Device copy of the 12 scatter vectors, uploaded on first use on `stream`
  // (which this call then drains once).
  const dev::Scatters& scatters(int device, cudaStream_t stream);
  std::string report() const;
};

// One execution's operands as the caller passed them.
struct Item {
  const void* a;
  const void* b;
  const void* c;
  void* d;
};

// Element type of a product as the scalar pointers alpha/beta carry it.
struct Scalar {
  double re = 0, im = 0;
  bool is_zero() const { return re == 0 && im == 0; }
  bool is_one() const { return re == 1 && im == 0; }
};
Scalar read_scalar(DType t, const void* p);

// The semantic preflight (Plan::check_raw, plan/mod.rs:384-428) plus the C-ABI
// null rules (execute.rs:34-39).
void validate_item(const Product& p, const Item& it, bool beta_zero);

// Run one validated item on the executor (stage host operands, launch,
// copy back, drain when synchronous).
void execute_item(Product& p, Executor& ex, Scalar alpha, Scalar beta, const Item& it);

// A grouped submission of validated items (contract_batched).
void execute_items(Executor& ex, int n, Product* const* plans, const Scalar* alpha, const Scalar* beta,
                   const Item* items);

// Plan::vjp: cotangents of A and B.
void execute_vjp(Product& p, Executor& ex, Scalar alpha, const void* A, const void* B, const void* dD, void* dA,
                 void* dB);

// The split-precision path on the caller's stream with no device allocation:
// scratch in a fixed device array (k_noalloc.cu). Synchronous on `stream`.
void execute_split_noalloc(Product& p, cudaStream_t stream, Scalar alpha, Scalar beta, const Item& it);

// Drain the stream (bounded) and turn a non-zero device status word into an error.
void finish(Executor& ex);
void drain(Executor& ex);

// JSON of the executor's per-kernel totals ({"name": {"ms": .., "launches": ..}}).
std::string kernel_times_json(Executor& ex, bool reset);

void check_cuda(cudaError_t e, const char* what);

}  // namespace tprims
