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

// One launch configuration of the plain path: a tile family, a split-K
// factor (1: none; K is cut into `splits` chunks of `chunk`) or the tiny
// batched kernel.
struct PlainChoice {
  int kernel = 0;
  int splits = 1;
  int64_t chunk = 0;
  bool tiny = false;
  bool operator==(const PlainChoice& o) const {
    return kernel == o.kernel && splits == o.splits && chunk == o.chunk && tiny == o.tiny;
  }
};

// How a product's launch configuration was decided.
enum class ChoiceSource { Model = 0, Pinned = 1, Autotuned = 2, Cached = 3 };

// Autotuner result for one Problem signature (single contractions) or one
// list signature (grouped lists: `policy` is the tile policy of the list).
struct TuneEntry {
  PlainChoice choice;
  int policy = 0;
  double ms = 0;     // best measured time of one execution (0: not measured)
  int tried = 0;     // candidates timed
  bool tuned = true; // false: the model's choice, kept without timing
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
  // Launch-failure injection: the launch this many launches from now is
  // refused on the host with an error, before it reaches the stream (-1: off).
  int fail_launch_after = -1;
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
  // Autotuner cache, keyed by Problem signature (single contractions) and by
  // list signature (grouped lists); persisted with save_tuning / load_tuning.
  std::map<std::string, TuneEntry> tune;
  std::map<std::string, TuneEntry> list_tune;
  std::string device_name;
  // Streamed host execution (host operands split into chunks along the
  // output's outermost column axis; copies in, kernels and copies out of
  // successive chunks overlap): switch, copy streams and events, the latter
  // created on first use.
  bool streaming = true;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> stream_events;
  // Side streams and fork/join events: the persistent launches of a grouped
  // submission's tile families run concurrently (a later family fills the
  // tail of an earlier one), and so do the two split-precision packs.
  std::vector<cudaStream_t> family_streams;
  std::vector<cudaEvent_t> family_events;

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
  PackedPlan packed;  // statistics and run structure; its scatter vectors moved into `view`
  OrientedView view;
  Scheme scheme = Scheme::Plain;
  int ozaki_slices = 0;
  int kernel_pin = 0;
  int split_pin = 0;       // 0: chosen; 1: never split K; s > 1: exactly s chunks
  bool autotune = false;   // time the candidates on first execution per executor
  std::string signature;   // dtype, folded axes and conjugations (scheme added per call)
  // The launch configuration of the last plain execution and how it was chosen.
  PlainChoice last{};
  ChoiceSource last_source = ChoiceSource::Model;
  bool executed = false;
  // Batch strides of the oriented view for the tiny batched kernel.
  dev::TinyStrides tiny_h{};
  // Unique over the process lifetime (never reused, unlike the address), so a
  // cached grouped graph can never be replayed for a newer plan.
  const uint64_t uid;
  mutable std::mutex mu;
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

// Plan::check_raw (plan/mod.rs:384-428): the aliasing preflight from the
// origins alone, nothing dereferenced, a null origin treated as absent: D
// overlapping A or B, a separate C overlapping D without being the same mapping
// at the same origin. Throws ERR_ALIASED.
void check_raw(const Product& p, const Item& it);
// check_raw plus the C-ABI null rules (execute.rs:34-39).
void validate_item(const Product& p, const Item& it, bool beta_zero);

// Run one validated item on the executor (stage host operands, launch,
// copy back, drain when synchronous).
void execute_item(Product& p, Executor& ex, Scalar alpha, Scalar beta, const Item& it);

// A grouped submission of validated items (contract_batched).
void execute_items(Executor& ex, int n, Product* const* plans, const Scalar* alpha, const Scalar* beta,
                   const Item* items);

// Longest-first balance of items over parts: items in decreasing cost (ties
// by index) each go to the least-loaded part whose device is the item's home
// (home < 0: any part). Returns the part of each item; ERR_DEVICE when an
// item's home has no part.
std::vector<int> balance_parts(const std::vector<double>& costs, const std::vector<int>& homes,
                               const std::vector<int>& part_devices);

// contract_batched over several executors (one per GPU, or several per GPU):
// the validated items are balanced by their multiply-accumulates over the
// executors of the device that holds each item's output (host outputs go
// anywhere), each executor's share is one grouped submission on its own stream,
// and every stream is drained before returning. No data moves between devices.
void execute_items_sharded(Executor* const* exs, int n_exec, int n, Product* const* plans, const Scalar* alpha,
                           const Scalar* beta, const Item* items);

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

// Every device allocation of the library goes through device_alloc, which
// counts it; device_allocations() is the process-wide count (diagnostics: a
// steady-state execution must leave it unchanged).
cudaError_t device_alloc(void** p, size_t bytes);
uint64_t device_allocations();

// ---- autotuner (autotune.cpp) ----

// A product's Problem signature: dtype, folded axes (extent and the strides
// of A, B, C, D), orientation and conjugations. Spaces never occur in it.
std::string problem_signature(const Product& p);
// The signature under the product's current scheme, plus whether the call
// reads C: the key of the autotuner cache.
std::string tune_key(const Product& p, bool c_read);
// Plain-path candidates for a shape: every tile family of the dtype, each with
// the split-K factors that keep at most four CTAs per SM in flight, and the
// tiny batched kernel where it applies. The model's choice comes first.
std::vector<PlainChoice> plain_candidates(int dtype, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms);
// The model's choice (heuristics), honouring the tile and split pins.
PlainChoice model_choice(const Product& p, int num_sms);
// Scratch bytes a plain choice needs (split-K partials).
size_t plain_scratch(const PlainChoice& c, const Product& p);
// Whether a choice (from a tuning-cache file, say) is valid for a product: a
// family of the product's dtype, the tiny kernel only where it applies, and
// split-K chunks in whole 64-deep blocks whose count is exactly `splits`
// (so that every k is covered once).
bool choice_fits(const PlainChoice& c, const Product& p);
// Tile family of a grouped item under a list tile policy (0: model, 1: large
// tiles, 2: small tiles, 3: tall 128 x 32 tiles for narrow f64/c64 outputs).
int grouped_family(const Product& p, int policy);
constexpr int GROUP_POLICIES = 4;
// The versioned text form of an executor's cache, and its inverse (entries of
// another device kind are skipped; a malformed file is an error).
std::string tuning_text(const Executor& ex);
void load_tuning_text(Executor& ex, const std::string& text);
// A parsed cache file: the header's SM count and device tag, and its entries.
struct TuningFile {
  int sms = 0;
  std::string device;
  std::map<std::string, TuneEntry> singles, lists;
};
TuningFile parse_tuning_text(const std::string& text);
std::string tuning_json(const Executor& ex);
std::string choice_name(const PlainChoice& c, int dtype);

}  // namespace tprims
