// The exported C ABI: TAPP symbols, tprims extensions and the B200 additions.
//
// Argument checks and their order follow the reference's C layer
// (crates/tprims-capi/src/product.rs:83-195, execute.rs:14-279,
// tensor_info.rs:58-221, handle.rs, status.rs); status codes and the one
// error-to-status table are those of status.rs:13-43 and abi.rs:97-113.
// Every entry point catches all C++ exceptions: nothing unwinds across the C
// boundary, and the message of the last failure is kept per thread.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/tprims_b200.h"
#include "network.hpp"
#include "runtime.hpp"

using namespace tprims;

namespace {

thread_local std::string g_last_error;

template <class F>
int ffi(F&& body) {
  try {
    body();
    if (!g_last_error.empty()) g_last_error.clear();
    return TPRIMS_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    g_last_error = "out of memory";
    return TPRIMS_ERR_INTERNAL;
  } catch (const std::exception& e) {
    g_last_error = std::string("panic: ") + e.what();
    return TPRIMS_ERR_PANIC;
  } catch (...) {
    g_last_error = "panic";
    return TPRIMS_ERR_PANIC;
  }
}

[[noreturn]] void null_arg(const std::string& what) { throw Error(ERR_INVALID_ARGUMENT, what + " is null or zero"); }

struct TensorInfo {
  int dtype;
  std::vector<int64_t> extents, strides;
};

struct HandleState {
  uint64_t reserved = 0;  // non-empty, so every handle is a distinct address
};

// An executor handle: the CUDA resources are created on first use, so that a
// host without a GPU can still create handles and plan.
struct ExecHandle {
  int device = -1;
  uintptr_t stream = 0;
  size_t pool_size = 0, budget = 1;
  bool sync = true;
  std::unique_ptr<Executor> ex;
  std::mutex mu;

  Executor& get() {
    std::lock_guard<std::mutex> lk(mu);
    if (!ex) {
      ex.reset(Executor::create(device, stream));
      ex->sync = sync;
      ex->pool_size = pool_size;
      ex->budget = budget;
    }
    return *ex;
  }
};

// Executor 0: one lazily created executor per device, kept for the process.
ExecHandle* default_exec() {
  static std::mutex mu;
  static std::vector<ExecHandle*> per_dev;
  int d = 0;
  check_cuda(cudaGetDevice(&d), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(mu);
  if ((int)per_dev.size() <= d) per_dev.resize(d + 1, nullptr);
  if (!per_dev[d]) {
    per_dev[d] = new ExecHandle();
    per_dev[d]->device = d;
  }
  return per_dev[d];
}

ExecHandle* resolve_exec(TAPP_executor exec) {
  return exec == 0 ? default_exec() : reinterpret_cast<ExecHandle*>(exec);
}

int elem_size(int dtype) {
  switch (dtype) {
    case TAPP_F32: return 4;
    case TAPP_F64: return 8;
    case TAPP_C32: return 8;
    case TAPP_C64: return 16;
  }
  return 0;
}

bool op_conj(int op, const char* name) {
  if (op == TAPP_IDENTITY) return false;
  if (op == TAPP_CONJUGATE) return true;
  throw Error(ERR_UNSUPPORTED, "element operation " + std::to_string(op) + " on " + name + " is not supported");
}

Product& product_of(TAPP_tensor_product plan) {
  if (plan == 0) null_arg("plan");
  return *reinterpret_cast<Product*>(plan);
}

// Execute a list of items of one product (validated first, as a whole).
void run_items(Product& p, TAPP_executor exec, const void* alpha, const void* beta, const std::vector<Item>& items) {
  if (!alpha) null_arg("alpha");
  if (!beta) null_arg("beta");
  const Scalar al = read_scalar(p.problem.dtype, alpha), be = read_scalar(p.problem.dtype, beta);
  for (const Item& it : items) validate_item(p, it, be.is_zero());
  if (items.empty()) return;
  ExecHandle* h = resolve_exec(exec);
  Executor& ex = h->get();
  ex.inflight++;
  struct Done {
    Executor& e;
    ~Done() { e.inflight--; }
  } done{ex};
  if (items.size() == 1) {
    execute_item(p, ex, al, be, items[0]);
  } else {
    std::vector<Product*> ps(items.size(), &p);
    std::vector<Scalar> als(items.size(), al), bes(items.size(), be);
    execute_items(ex, (int)items.size(), ps.data(), als.data(), bes.data(), items.data());
  }
}

Operand operand_from(const int64_t* ext, const int64_t* str, int rank, int op, const char* name) {
  if (rank < 0) throw Error(ERR_SHAPE, "negative mode count");
  if (rank > 0 && (!ext || !str)) null_arg(std::string("extents or strides of ") + name);
  Operand o;
  o.layout = layout_from_signed(ext, str, rank, 0);
  o.conj = op_conj(op, name);
  return o;
}

DType dtype_from(int t) {
  switch (t) {
    case TAPP_F32: return DType::F32;
    case TAPP_F64: return DType::F64;
    case TAPP_C32: return DType::C32;
    case TAPP_C64: return DType::C64;
  }
  throw Error(ERR_DTYPE, "unsupported datatype");
}

}  // namespace

// ------------------------------------------------------------------ status

extern "C" bool TAPP_check_success(TAPP_error error) { return error == TPRIMS_OK; }

static const char* describe(int s) {
  switch (s) {
    case TPRIMS_OK: return "success";
    case TPRIMS_ERR_INVALID_ARGUMENT: return "null pointer, invalid handle or invalid argument";
    case TPRIMS_ERR_SHAPE: return "inconsistent or overflowing extents or strides";
    case TPRIMS_ERR_DTYPE: return "unsupported or mismatched data type";
    case TPRIMS_ERR_DEVICE: return "unsupported device";
    case TPRIMS_ERR_READ_ONLY: return "output is read-only";
    case TPRIMS_ERR_ALIASED: return "output aliases an operand or overlaps itself";
    case TPRIMS_ERR_WOULD_MATERIALIZE: return "the operation would copy an operand";
    case TPRIMS_ERR_NUMERICAL: return "numerical failure";
    case TPRIMS_BUSY: return "executor has calls in flight";
    case TPRIMS_ERR_WOULD_DEADLOCK: return "executor destroyed from one of its own workers";
    case TPRIMS_ERR_PANIC: return "a panic was caught at the ABI boundary";
    case TPRIMS_ERR_INTERNAL: return "internal error";
    case TPRIMS_ERR_LABELS: return "invalid index labels";
    case TPRIMS_ERR_UNSUPPORTED: return "operation not supported by this implementation";
  }
  return "unknown error";
}

extern "C" size_t TAPP_explain_error(TAPP_error error, size_t maxlen, char* message) {
  const char* s = describe(error);
  const size_t len = std::strlen(s);
  if (message && maxlen > 0) {
    const size_t n = len < maxlen - 1 ? len : maxlen - 1;
    std::memcpy(message, s, n);
    message[n] = 0;
  }
  return len;
}

extern "C" const char* tprims_last_error(void) { return g_last_error.c_str(); }
extern "C" uint32_t tprims_abi_version(void) { return TPRIMS_ABI_VERSION; }
extern "C" int32_t tprims_has_part(const char* part) {
  if (!part) return 0;
  return (std::strcmp(part, "core") == 0 || std::strcmp(part, "tapp") == 0 || std::strcmp(part, "cuda") == 0) ? 1
                                                                                                             : 0;
}
extern "C" const char* TAPP_implementation_name(void) {
  return "tprims-b200: packed block-scatter contraction on sm_100a (SIMT/DMMA plain, tcgen05 split precision)";
}
extern "C" const char* TAPP_implementation_version(void) { return "0.1.0"; }

// -------------------------------------------------------------- attributes

extern "C" TAPP_error TAPP_attr_set(TAPP_attr, TAPP_key, void*) {
  return ffi([] { throw Error(ERR_UNSUPPORTED, "no attribute keys are defined"); });
}
extern "C" TAPP_error TAPP_attr_get(TAPP_attr, TAPP_key, void** value) {
  if (value) *value = nullptr;
  return ffi([] { throw Error(ERR_UNSUPPORTED, "no attribute keys are defined"); });
}
extern "C" TAPP_error TAPP_attr_clear(TAPP_attr, TAPP_key) {
  return ffi([] { throw Error(ERR_UNSUPPORTED, "no attribute keys are defined"); });
}

// ----------------------------------------------------------------- handles

extern "C" TAPP_error TAPP_create_handle(TAPP_handle* handle) {
  return ffi([&] {
    if (!handle) null_arg("handle out-parameter");
    *handle = reinterpret_cast<TAPP_handle>(new HandleState());
  });
}
extern "C" TAPP_error TAPP_destroy_handle(TAPP_handle handle) {
  return ffi([&] {
    if (handle == 0) null_arg("handle");
    delete reinterpret_cast<HandleState*>(handle);
  });
}
extern "C" TAPP_error TAPP_destroy_status(TAPP_status) {
  return ffi([] {});
}

// --------------------------------------------------------------- executors

extern "C" TAPP_error TAPP_create_executor(TAPP_executor* exec) {
  return ffi([&] {
    if (!exec) null_arg("executor out-parameter");
    *exec = reinterpret_cast<TAPP_executor>(new ExecHandle());
  });
}

extern "C" TAPP_error tprims_b200_executor_create(TAPP_executor* exec, int device, uintptr_t stream) {
  return ffi([&] {
    if (!exec) null_arg("executor out-parameter");
    auto* h = new ExecHandle();
    h->device = device;
    h->stream = stream;
    *exec = reinterpret_cast<TAPP_executor>(h);
  });
}

extern "C" TAPP_error tprims_tapp_executor_create_rayon(TAPP_executor* out, size_t nthreads,
                                                        const tprims_rayon_opts*) {
  return ffi([&] {
    if (!out) null_arg("executor out-parameter");
    if (nthreads == 0) throw Error(ERR_INVALID_ARGUMENT, "nthreads must be at least 1");
    auto* h = new ExecHandle();
    h->pool_size = nthreads == 1 ? 0 : nthreads;
    h->budget = nthreads;
    *out = reinterpret_cast<TAPP_executor>(h);
  });
}

extern "C" TAPP_error tprims_tapp_executor_set_budget(TAPP_executor exec, size_t budget) {
  return ffi([&] {
    if (exec == 0) return;
    if (budget == 0) throw Error(ERR_INVALID_ARGUMENT, "budget must be at least 1");
    auto* h = reinterpret_cast<ExecHandle*>(exec);
    if (h->pool_size == 0) return;
    h->budget = budget < h->pool_size ? budget : h->pool_size;
  });
}

extern "C" TAPP_error tprims_tapp_executor_get_threads(TAPP_executor exec, size_t* pool_size, size_t* budget) {
  return ffi([&] {
    size_t ps = 0, b = 1;
    if (exec != 0) {
      auto* h = reinterpret_cast<ExecHandle*>(exec);
      ps = h->pool_size;
      b = h->pool_size == 0 ? 1 : h->budget;
    }
    if (pool_size) *pool_size = ps;
    if (budget) *budget = b;
  });
}

extern "C" TAPP_error TAPP_destroy_executor(TAPP_executor exec) {
  return ffi([&] {
    if (exec == 0) return;
    auto* h = reinterpret_cast<ExecHandle*>(exec);
    if (h->ex && h->ex->inflight.load() > 0) throw Error(BUSY, "executor has calls in flight");
    delete h;
  });
}

extern "C" TAPP_error tprims_b200_executor_stream(TAPP_executor exec, uintptr_t* stream) {
  return ffi([&] {
    if (!stream) null_arg("stream out-parameter");
    *stream = reinterpret_cast<uintptr_t>(resolve_exec(exec)->get().stream);
  });
}

extern "C" TAPP_error tprims_b200_executor_set_sync(TAPP_executor exec, int sync) {
  return ffi([&] {
    ExecHandle* h = resolve_exec(exec);
    h->sync = sync != 0;
    if (h->ex) h->ex->sync = sync != 0;
  });
}

extern "C" TAPP_error tprims_b200_executor_synchronize(TAPP_executor exec) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ex.device);
    try {
      finish(ex);
    } catch (...) {
      if (prev >= 0) cudaSetDevice(prev);
      throw;
    }
    if (prev >= 0) cudaSetDevice(prev);
  });
}

// ------------------------------------------------------------ tensor infos

extern "C" TAPP_error TAPP_create_tensor_info(TAPP_tensor_info* info, TAPP_datatype type, int nmode,
                                              const int64_t* extents, const int64_t* strides) {
  return ffi([&] {
    if (!info) null_arg("info out-parameter");
    if (nmode < 0) throw Error(ERR_SHAPE, "negative mode count");
    if (elem_size(type) == 0) throw Error(ERR_DTYPE, "unsupported datatype");
    if (nmode > 0 && (!extents || !strides)) null_arg("extents or strides");
    auto* t = new TensorInfo();
    t->dtype = type;
    if (nmode > 0) {
      t->extents.assign(extents, extents + nmode);
      t->strides.assign(strides, strides + nmode);
    }
    *info = reinterpret_cast<TAPP_tensor_info>(t);
  });
}

extern "C" TAPP_error TAPP_destroy_tensor_info(TAPP_tensor_info info) {
  return ffi([&] {
    if (info == 0) null_arg("info");
    delete reinterpret_cast<TensorInfo*>(info);
  });
}

extern "C" int TAPP_get_nmodes(TAPP_tensor_info info) {
  if (info == 0) return -1;
  return (int)reinterpret_cast<TensorInfo*>(info)->extents.size();
}

extern "C" TAPP_error TAPP_set_nmodes(TAPP_tensor_info info, int nmodes) {
  return ffi([&] {
    if (info == 0) null_arg("info");
    if (nmodes < 0) throw Error(ERR_SHAPE, "negative mode count");
    auto* t = reinterpret_cast<TensorInfo*>(info);
    t->extents.resize(nmodes, 1);  // new modes: extent 1, stride 0
    t->strides.resize(nmodes, 0);
  });
}

extern "C" void TAPP_get_extents(TAPP_tensor_info info, int64_t* extents) {
  if (info == 0 || !extents) return;
  auto* t = reinterpret_cast<TensorInfo*>(info);
  std::memcpy(extents, t->extents.data(), t->extents.size() * sizeof(int64_t));
}

extern "C" TAPP_error TAPP_set_extents(TAPP_tensor_info info, const int64_t* extents) {
  return ffi([&] {
    if (info == 0) null_arg("info");
    if (!extents) null_arg("extents");
    auto* t = reinterpret_cast<TensorInfo*>(info);
    std::memcpy(t->extents.data(), extents, t->extents.size() * sizeof(int64_t));
  });
}

extern "C" void TAPP_get_strides(TAPP_tensor_info info, int64_t* strides) {
  if (info == 0 || !strides) return;
  auto* t = reinterpret_cast<TensorInfo*>(info);
  std::memcpy(strides, t->strides.data(), t->strides.size() * sizeof(int64_t));
}

extern "C" TAPP_error TAPP_set_strides(TAPP_tensor_info info, const int64_t* strides) {
  return ffi([&] {
    if (info == 0) null_arg("info");
    if (!strides) null_arg("strides");
    auto* t = reinterpret_cast<TensorInfo*>(info);
    std::memcpy(t->strides.data(), strides, t->strides.size() * sizeof(int64_t));
  });
}

// ---------------------------------------------------------------- products

extern "C" TAPP_error TAPP_create_tensor_product(TAPP_tensor_product* plan, TAPP_handle handle, TAPP_element_op op_A,
                                                 TAPP_tensor_info A, const int64_t* idx_A, TAPP_element_op op_B,
                                                 TAPP_tensor_info B, const int64_t* idx_B, TAPP_element_op op_C,
                                                 TAPP_tensor_info C, const int64_t* idx_C, TAPP_element_op op_D,
                                                 TAPP_tensor_info D, const int64_t* idx_D, TAPP_prectype prec) {
  return ffi([&] {
    if (!plan) null_arg("plan out-parameter");
    if (handle == 0) null_arg("library handle");
    if (!A || !B || !C || !D) null_arg("tensor info");
    auto* ta = reinterpret_cast<TensorInfo*>(A);
    auto* tb = reinterpret_cast<TensorInfo*>(B);
    auto* tc = reinterpret_cast<TensorInfo*>(C);
    auto* td = reinterpret_cast<TensorInfo*>(D);
    if (ta->dtype != tb->dtype || ta->dtype != tc->dtype || ta->dtype != td->dtype)
      throw Error(ERR_DTYPE, "operands have different storage types");
    const int storage_prec = (ta->dtype == TAPP_F32 || ta->dtype == TAPP_C32) ? TAPP_F32F32_ACCUM_F32
                                                                              : TAPP_F64F64_ACCUM_F64;
    if (prec != TAPP_DEFAULT_PREC && prec != storage_prec)
      throw Error(ERR_UNSUPPORTED,
                  "computational precision " + std::to_string(prec) + " differs from the storage precision");
    const bool ca = op_conj(op_A, "A"), cb = op_conj(op_B, "B"), cc = op_conj(op_C, "C"), cd = op_conj(op_D, "D");
    auto labels = [](const int64_t* p, const TensorInfo* t, const char* name) {
      const size_t n = t->extents.size();
      if (n == 0) return std::vector<int64_t>();
      if (!p) null_arg(std::string("labels of ") + name);
      return std::vector<int64_t>(p, p + n);
    };
    auto la = labels(idx_A, ta, "A"), lb = labels(idx_B, tb, "B"), lc = labels(idx_C, tc, "C"),
         ld = labels(idx_D, td, "D");
    const DType dt = dtype_from(ta->dtype);
    auto spec = [](const TensorInfo* t, bool conj) {
      Operand o;
      o.layout = layout_from_signed(t->extents.data(), t->strides.data(), (int)t->extents.size(), 0);
      o.conj = conj;
      return o;
    };
    Operand oa = spec(ta, ca), ob = spec(tb, cb), oc = spec(tc, cc), od = spec(td, cd);
    Problem p = Problem::from_labels(dt, oa, ob, CMode::Separate, oc, od, la, lb, true, lc, ld);
    *plan = reinterpret_cast<TAPP_tensor_product>(new Product(p));
  });
}

extern "C" TAPP_error TAPP_destroy_tensor_product(TAPP_tensor_product plan) {
  return ffi([&] {
    if (plan == 0) null_arg("plan");
    delete reinterpret_cast<Product*>(plan);
  });
}

extern "C" TAPP_error tprims_b200_product_from_dot_general(
    TAPP_tensor_product* plan, TAPP_datatype dtype, int rank_a, const int64_t* ext_a, const int64_t* str_a,
    TAPP_element_op op_a, int rank_b, const int64_t* ext_b, const int64_t* str_b, TAPP_element_op op_b, int rank_d,
    const int64_t* ext_d, const int64_t* str_d, TAPP_element_op op_d, int n_contract, const int64_t* lhs_contract,
    const int64_t* rhs_contract, int n_batch, const int64_t* lhs_batch, const int64_t* rhs_batch) {
  return ffi([&] {
    if (!plan) null_arg("plan out-parameter");
    const DType dt = dtype_from(dtype);
    Operand a = operand_from(ext_a, str_a, rank_a, op_a, "A");
    Operand b = operand_from(ext_b, str_b, rank_b, op_b, "B");
    Operand d = operand_from(ext_d, str_d, rank_d, op_d, "D");
    if (n_contract < 0 || n_batch < 0) throw Error(ERR_INVALID_ARGUMENT, "negative axis-list length");
    if ((n_contract > 0 && (!lhs_contract || !rhs_contract)) || (n_batch > 0 && (!lhs_batch || !rhs_batch)))
      null_arg("axis list");
    std::vector<int64_t> lc(lhs_contract, lhs_contract + n_contract), rc(rhs_contract, rhs_contract + n_contract);
    std::vector<int64_t> lbt(lhs_batch, lhs_batch + n_batch), rbt(rhs_batch, rhs_batch + n_batch);
    Problem p = Problem::from_dot_general(dt, a, b, d, lc, rc, lbt, rbt);
    *plan = reinterpret_cast<TAPP_tensor_product>(new Product(p));
  });
}

extern "C" TAPP_error tprims_b200_product_set_precision(TAPP_tensor_product plan, int scheme, int slices) {
  return ffi([&] {
    Product& p = product_of(plan);
    const DType t = p.problem.dtype;
    switch (scheme) {
      case TPRIMS_PREC_PLAIN: p.scheme = Scheme::Plain; break;
      case TPRIMS_PREC_BF16X3:
      case TPRIMS_PREC_BF16X6:
        if (t != DType::F32) throw Error(ERR_UNSUPPORTED, "the BF16 split schemes apply to f32 storage");
        p.scheme = scheme == TPRIMS_PREC_BF16X3 ? Scheme::Bf16x3 : Scheme::Bf16x6;
        break;
      case TPRIMS_PREC_OZAKI_INT8:
        if (t != DType::F64 && t != DType::C64)
          throw Error(ERR_UNSUPPORTED, "the Ozaki INT8 scheme applies to f64 and c64 storage");
        if (slices != 0 && (slices < 4 || slices > 8))
          throw Error(ERR_INVALID_ARGUMENT, "Ozaki slice count must be 0 (default) or 4..8");
        p.scheme = Scheme::OzakiInt8;
        // Six 8-bit slices (21 products) reach about 3e-14 relative error on
        // unit-range data; seven reach the FP64 rounding floor.
        p.ozaki_slices = slices == 0 ? 6 : slices;
        return;
      default:
        throw Error(ERR_INVALID_ARGUMENT, "unknown precision scheme " + std::to_string(scheme));
    }
  });
}

extern "C" TAPP_error tprims_b200_product_set_tile(TAPP_tensor_product plan, int kernel_id) {
  return ffi([&] {
    Product& p = product_of(plan);
    if (kernel_id < 0 || kernel_id > dev::PLAIN_LAST)
      throw Error(ERR_INVALID_ARGUMENT, "unknown kernel id " + std::to_string(kernel_id));
    p.kernel_pin = kernel_id;
  });
}

extern "C" TAPP_error tprims_b200_product_check_raw(TAPP_tensor_product plan, const void* A, const void* B,
                                                    const void* C, const void* D) {
  return ffi([&] { check_raw(product_of(plan), Item{A, B, C, const_cast<void*>(D)}); });
}

extern "C" TAPP_error tprims_b200_product_set_split_k(TAPP_tensor_product plan, int splits) {
  return ffi([&] {
    Product& p = product_of(plan);
    if (splits < 0 || splits > 64)
      throw Error(ERR_INVALID_ARGUMENT, "split-K factor must be 0 (chosen), 1 (never) or 2..64");
    p.split_pin = splits;
  });
}

extern "C" TAPP_error tprims_b200_product_set_autotune(TAPP_tensor_product plan, int on) {
  return ffi([&] { product_of(plan).autotune = on != 0; });
}

extern "C" size_t tprims_b200_product_report(TAPP_tensor_product plan, char* buf, size_t maxlen) {
  std::string s;
  if (ffi([&] { s = product_of(plan).report(); }) != TPRIMS_OK) return 0;
  if (buf && maxlen > 0) {
    const size_t n = s.size() < maxlen - 1 ? s.size() : maxlen - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

// ---------------------------------------------------------------- execution

extern "C" TAPP_error TAPP_execute_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                           const void* alpha, const void* A, const void* B, const void* beta,
                                           const void* C, void* D) {
  return ffi([&] {
    if (status) *status = 0;
    Product& p = product_of(plan);
    run_items(p, exec, alpha, beta, {Item{A, B, C, D}});
  });
}

extern "C" TAPP_error TAPP_execute_batched_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                                   int num_batches, const void* alpha, const void** A,
                                                   const void** B, const void* beta, const void** C, void** D) {
  return ffi([&] {
    if (status) *status = 0;
    if (num_batches < 0) throw Error(ERR_SHAPE, "negative batch count");
    Product& p = product_of(plan);
    if (!A || !B || !D) null_arg("A, B or D pointer array");
    std::vector<Item> items;
    for (int i = 0; i < num_batches; ++i) items.push_back(Item{A[i], B[i], C ? C[i] : nullptr, D[i]});
    run_items(p, exec, alpha, beta, items);
  });
}

extern "C" TAPP_error tprims_b200_contract_batched(TAPP_executor exec, int n, const tprims_b200_batch_item* items) {
  return ffi([&] {
    if (n < 0) throw Error(ERR_SHAPE, "negative item count");
    if (n > 0 && !items) null_arg("item array");
    std::vector<Product*> ps;
    std::vector<Scalar> als, bes;
    std::vector<Item> its;
    // All-or-nothing: every item is checked before anything runs (batch.rs:127-130).
    for (int i = 0; i < n; ++i) {
      Product& p = product_of(items[i].plan);
      if (!items[i].alpha) null_arg("alpha");
      if (!items[i].beta) null_arg("beta");
      const Scalar al = read_scalar(p.problem.dtype, items[i].alpha), be = read_scalar(p.problem.dtype, items[i].beta);
      Item it{items[i].A, items[i].B, items[i].C, items[i].D};
      validate_item(p, it, be.is_zero());
      ps.push_back(&p);
      als.push_back(al);
      bes.push_back(be);
      its.push_back(it);
    }
    if (n == 0) return;
    Executor& ex = resolve_exec(exec)->get();
    execute_items(ex, n, ps.data(), als.data(), bes.data(), its.data());
  });
}

// ---- N-ary networks

namespace {
Network& network_of(tprims_b200_network net) {
  if (net == 0) null_arg("network");
  return *reinterpret_cast<Network*>(net);
}
}  // namespace

extern "C" TAPP_error tprims_b200_network_create(tprims_b200_network* net, TAPP_datatype dtype, int n_inputs,
                                                 const int* nmodes, const int64_t* const* extents,
                                                 const int64_t* const* strides, const int64_t* const* labels,
                                                 const TAPP_element_op* ops, int out_nmode,
                                                 const int64_t* out_extents, const int64_t* out_strides,
                                                 const int64_t* out_labels, int n_steps, const int* path) {
  return ffi([&] {
    if (!net) null_arg("network out-parameter");
    if (n_inputs < 0 || out_nmode < 0 || n_steps < 0) throw Error(ERR_SHAPE, "negative count");
    if (n_inputs > 0 && (!nmodes || !extents || !strides || !labels)) null_arg("input descriptions");
    const DType dt = dtype_from(dtype);
    auto operand = [&](int rank, const int64_t* e, const int64_t* st, const int64_t* l, bool conj,
                       const std::string& what) {
      if (rank < 0) throw Error(ERR_SHAPE, what + ": negative rank");
      if (rank > 0 && (!e || !l)) null_arg(what + " extents or labels");
      NetworkOperand o;
      std::vector<int64_t> dense;
      if (rank > 0 && !st) {  // null strides: column-major
        int64_t acc = 1;
        for (int k = 0; k < rank; ++k) {
          dense.push_back(acc);
          acc *= std::max<int64_t>(e[k], 1);
        }
        st = dense.data();
      }
      o.op.layout = layout_from_signed(e, st, rank, 0);
      o.op.conj = conj;
      o.labels.assign(l, l + rank);
      return o;
    };
    std::vector<NetworkOperand> ins;
    for (int i = 0; i < n_inputs; ++i)
      ins.push_back(operand(nmodes[i], extents[i], strides[i], labels[i],
                            ops ? op_conj(ops[i], "a network input") : false, "input " + std::to_string(i)));
    NetworkOperand out = operand(out_nmode, out_extents, out_strides, out_labels, false, "output");
    std::vector<std::pair<int, int>> pth;
    if (n_steps > 0) {
      if (!path) null_arg("path");
      for (int s = 0; s < n_steps; ++s) pth.push_back({path[2 * s], path[2 * s + 1]});
    }
    *net = reinterpret_cast<tprims_b200_network>(Network::create(dt, std::move(ins), std::move(out), std::move(pth)));
  });
}

extern "C" TAPP_error tprims_b200_network_destroy(tprims_b200_network net) {
  return ffi([&] {
    if (net == 0) null_arg("network");
    delete reinterpret_cast<Network*>(net);
  });
}

extern "C" TAPP_error tprims_b200_network_set_precision(tprims_b200_network net, int scheme, int slices) {
  return ffi([&] {
    Network& n = network_of(net);
    for (auto& s : n.steps) {
      const TAPP_error e = tprims_b200_product_set_precision(reinterpret_cast<TAPP_tensor_product>(s.plan.get()),
                                                           scheme, slices);
      if (e != TPRIMS_OK) throw Error(e, g_last_error);
    }
  });
}

extern "C" TAPP_error tprims_b200_network_set_autotune(tprims_b200_network net, int on) {
  return ffi([&] {
    for (auto& s : network_of(net).steps) s.plan->autotune = on != 0;
  });
}

extern "C" TAPP_error tprims_b200_network_workspace_size(tprims_b200_network net, size_t* bytes) {
  return ffi([&] {
    if (!bytes) null_arg("bytes out-parameter");
    *bytes = network_of(net).arena_bytes;
  });
}

extern "C" size_t tprims_b200_network_report(tprims_b200_network net, char* buf, size_t maxlen) {
  std::string s;
  if (ffi([&] { s = network_of(net).report(); }) != TPRIMS_OK) return 0;
  if (buf && maxlen > 0) {
    const size_t n = s.size() < maxlen - 1 ? s.size() : maxlen - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

extern "C" TAPP_error tprims_b200_networks_execute(TAPP_executor exec, int n, const tprims_b200_network* nets,
                                                   const void* const* alphas, const void* const* const* inputs,
                                                   const void* const* betas, void* const* outs,
                                                   void* const* workspaces) {
  return ffi([&] {
    if (n < 0) throw Error(ERR_SHAPE, "negative network count");
    if (n == 0) return;
    if (!nets || !alphas || !inputs || !betas || !outs) null_arg("network arrays");
    std::vector<Network*> ns;
    std::vector<Scalar> al, be;
    for (int i = 0; i < n; ++i) {
      Network& net = network_of(nets[i]);
      if (!alphas[i]) null_arg("alpha");
      if (!betas[i]) null_arg("beta");
      if (!inputs[i]) null_arg("input pointers");
      if (!outs[i]) null_arg("output");
      for (size_t j = 0; j < net.inputs.size(); ++j)
        if (!inputs[i][j]) null_arg("input " + std::to_string(j));
      ns.push_back(&net);
      al.push_back(read_scalar(net.dtype, alphas[i]));
      be.push_back(read_scalar(net.dtype, betas[i]));
    }
    Executor& ex = resolve_exec(exec)->get();
    execute_networks(ex, n, ns.data(), al.data(), be.data(), inputs, outs, workspaces);
  });
}

extern "C" TAPP_error tprims_b200_network_execute(tprims_b200_network net, TAPP_executor exec, const void* alpha,
                                                  const void* const* inputs, const void* beta, void* out,
                                                  void* workspace) {
  void* ws[1] = {workspace};
  const void* const* ins[1] = {inputs};
  const void* al[1] = {alpha};
  const void* be[1] = {beta};
  void* outs[1] = {out};
  return tprims_b200_networks_execute(exec, 1, &net, al, ins, be, outs, ws);
}

extern "C" TAPP_error tprims_b200_balance(int n, const double* costs, const int* homes, int n_parts,
                                         const int* part_devices, int* assignment) {
  return ffi([&] {
    if (n < 0 || n_parts < 0) throw Error(ERR_SHAPE, "negative count");
    if (n > 0 && (!costs || !assignment)) null_arg("costs or assignment");
    if (n_parts > 0 && !part_devices) null_arg("part devices");
    std::vector<double> c(costs, costs + n);
    std::vector<int> h(n, -1);
    if (homes)
      for (int i = 0; i < n; ++i) h[i] = homes[i];
    const std::vector<int> d(part_devices, part_devices + n_parts);
    const std::vector<int> part = balance_parts(c, h, d);
    for (int i = 0; i < n; ++i) assignment[i] = part[i];
  });
}

extern "C" TAPP_error tprims_b200_contract_batched_sharded(const TAPP_executor* execs, int n_exec, int n,
                                                           const tprims_b200_batch_item* items) {
  return ffi([&] {
    if (n < 0 || n_exec < 0) throw Error(ERR_SHAPE, "negative count");
    if (n > 0 && !items) null_arg("item array");
    if (n_exec == 0 || !execs) throw Error(ERR_INVALID_ARGUMENT, "no executors");
    std::vector<Product*> ps;
    std::vector<Scalar> als, bes;
    std::vector<Item> its;
    // All-or-nothing: every item is checked before anything runs (batch.rs:127-130).
    for (int i = 0; i < n; ++i) {
      Product& p = product_of(items[i].plan);
      if (!items[i].alpha) null_arg("alpha");
      if (!items[i].beta) null_arg("beta");
      const Scalar al = read_scalar(p.problem.dtype, items[i].alpha), be = read_scalar(p.problem.dtype, items[i].beta);
      Item it{items[i].A, items[i].B, items[i].C, items[i].D};
      validate_item(p, it, be.is_zero());
      ps.push_back(&p);
      als.push_back(al);
      bes.push_back(be);
      its.push_back(it);
    }
    if (n == 0) return;
    std::vector<Executor*> exs;
    for (int e = 0; e < n_exec; ++e) {
      if (execs[e] == 0) null_arg("executor " + std::to_string(e));
      exs.push_back(&resolve_exec(execs[e])->get());
    }
    execute_items_sharded(exs.data(), n_exec, n, ps.data(), als.data(), bes.data(), its.data());
  });
}

extern "C" TAPP_error tprims_b200_product_vjp(TAPP_tensor_product plan, TAPP_executor exec, const void* alpha,
                                              const void* A, const void* B, const void* dD, void* dA, void* dB) {
  return ffi([&] {
    Product& p = product_of(plan);
    if (!alpha) null_arg("alpha");
    if (!A || !B || !dD) null_arg("A, B or dD pointer");
    Executor& ex = resolve_exec(exec)->get();
    execute_vjp(p, ex, read_scalar(p.problem.dtype, alpha), A, B, dD, dA, dB);
  });
}

// ------------------------------------------------------------------ DLPack

extern "C" tprims_tensor tprims_tensor_borrow_versioned(DLManagedTensorVersioned* m) {
  tprims_tensor t{nullptr, 0};
  if (!m || m->version.major != 1) return t;
  t.view = &m->dl_tensor;
  t.flags = m->flags;
  return t;
}

extern "C" tprims_tensor tprims_tensor_borrow_raw(DLTensor* t, uint64_t flags) { return tprims_tensor{t, flags}; }

namespace {

int dl_dtype(const DLTensor* v) {
  if (v->dtype.lanes != 1) throw Error(ERR_DTYPE, "lanes = " + std::to_string(v->dtype.lanes) + " (must be 1)");
  if (v->dtype.code == kDLFloat && v->dtype.bits == 32) return TAPP_F32;
  if (v->dtype.code == kDLFloat && v->dtype.bits == 64) return TAPP_F64;
  if (v->dtype.code == kDLComplex && v->dtype.bits == 64) return TAPP_C32;
  if (v->dtype.code == kDLComplex && v->dtype.bits == 128) return TAPP_C64;
  throw Error(ERR_DTYPE, "unsupported dtype code " + std::to_string(v->dtype.code) + " bits " +
                             std::to_string(v->dtype.bits));
}

// The origin of a DLTensor whose shape/strides must match the planned layout.
const void* dl_origin(const tprims_tensor& t, const Operand& planned, DType dt, const char* name) {
  const DLTensor* v = t.view;
  if (!v) null_arg(std::string("DLTensor ") + name);
  if (dl_dtype(v) != (int)dt) throw Error(ERR_DTYPE, std::string(name) + " has a different dtype from the plan");
  if (v->device.device_type != kDLCPU && v->device.device_type != kDLCUDA && v->device.device_type != kDLCUDAHost &&
      v->device.device_type != kDLCUDAManaged)
    throw Error(ERR_DEVICE, std::string(name) + ": unsupported device type");
  if ((size_t)v->ndim != planned.layout.rank())
    throw Error(ERR_SHAPE, std::string(name) + ": the view's layout differs from the planned layout");
  std::vector<int64_t> strides(v->ndim);
  int64_t acc = 1;
  for (int i = v->ndim - 1; i >= 0; --i) {
    strides[i] = v->strides ? v->strides[i] : acc;
    acc *= v->shape[i];
  }
  for (int i = 0; i < v->ndim; ++i)
    if (v->shape[i] != planned.layout.dims[i] || strides[i] != planned.layout.strides[i])
      throw Error(ERR_SHAPE, std::string(name) + ": the view's layout differs from the planned layout");
  const size_t real = dtype_double(dt) ? 8 : 4;
  const uintptr_t p = reinterpret_cast<uintptr_t>(v->data) + v->byte_offset;
  if (p % real != 0) throw Error(ERR_INVALID_ARGUMENT, std::string(name) + ": misaligned data pointer");
  return reinterpret_cast<const void*>(p);
}

}  // namespace

extern "C" TAPP_error tprims_b200_execute_product_dlpack(TAPP_tensor_product plan, TAPP_executor exec,
                                                         TAPP_status* status, const void* alpha, tprims_tensor A,
                                                         tprims_tensor B, const void* beta, tprims_tensor C,
                                                         tprims_tensor D) {
  return ffi([&] {
    if (status) *status = 0;
    Product& p = product_of(plan);
    const DType dt = p.problem.dtype;
    const void* a = dl_origin(A, p.problem.a, dt, "A");
    const void* b = dl_origin(B, p.problem.b, dt, "B");
    const void* c = C.view ? dl_origin(C, p.problem.c, dt, "C") : nullptr;
    void* d = const_cast<void*>(dl_origin(D, p.problem.d, dt, "D"));
    run_items(p, exec, alpha, beta, {Item{a, b, c, d}});
  });
}

extern "C" int64_t tprims_b200_product_scatter(TAPP_tensor_product plan, int which, int64_t* out, int64_t cap) {
  int64_t n = -1;
  ffi([&] {
    const std::vector<const std::vector<int64_t>*> vs = unorient(product_of(plan).view);
    if (which < 0 || which >= 12) throw Error(ERR_INVALID_ARGUMENT, "scatter index out of range");
    const auto& v = *vs[which];
    n = (int64_t)v.size();
    if (out)
      for (int64_t i = 0; i < n && i < cap; ++i) out[i] = v[i];
  });
  return n;
}

extern "C" TAPP_error tprims_b200_executor_set_profiling(TAPP_executor exec, int on) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.profile = on != 0;
  });
}

extern "C" size_t tprims_b200_executor_kernel_times(TAPP_executor exec, char* buf, size_t maxlen, int reset) {
  std::string s;
  if (ffi([&] {
        Executor& ex = resolve_exec(exec)->get();
        std::lock_guard<std::mutex> lk(ex.mu);
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(ex.device);
        drain(ex);
        ex.times.resolve();
        s = kernel_times_json(ex, reset != 0);
        if (prev >= 0) cudaSetDevice(prev);
      }) != TPRIMS_OK)
    return 0;
  if (buf && maxlen > 0) {
    const size_t n = s.size() < maxlen - 1 ? s.size() : maxlen - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

extern "C" TAPP_error tprims_b200_executor_save_tuning(TAPP_executor exec, const char* path) {
  return ffi([&] {
    if (!path || !*path) throw Error(ERR_INVALID_ARGUMENT, "tuning cache path is null or empty");
    Executor& ex = resolve_exec(exec)->get();
    std::string text;
    {
      std::lock_guard<std::mutex> lk(ex.mu);
      text = tuning_text(ex);
    }
    std::FILE* f = std::fopen(path, "wb");
    if (!f) throw Error(ERR_INVALID_ARGUMENT, std::string("cannot open tuning cache for writing: ") + path);
    const size_t n = std::fwrite(text.data(), 1, text.size(), f);
    const int closed = std::fclose(f);
    if (n != text.size() || closed != 0)
      throw Error(ERR_INTERNAL, std::string("short write of tuning cache: ") + path);
  });
}

extern "C" TAPP_error tprims_b200_executor_load_tuning(TAPP_executor exec, const char* path) {
  return ffi([&] {
    if (!path || !*path) throw Error(ERR_INVALID_ARGUMENT, "tuning cache path is null or empty");
    Executor& ex = resolve_exec(exec)->get();
    std::FILE* f = std::fopen(path, "rb");
    if (!f) throw Error(ERR_INVALID_ARGUMENT, std::string("cannot open tuning cache: ") + path);
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    std::fclose(f);
    std::lock_guard<std::mutex> lk(ex.mu);
    load_tuning_text(ex, text);  // all-or-nothing: nothing is added when a line is malformed
  });
}

extern "C" TAPP_error tprims_b200_tuning_file_info(const char* path, int* sms, char* device, size_t device_len,
                                                  int* singles, int* lists) {
  return ffi([&] {
    if (!path || !*path) throw Error(ERR_INVALID_ARGUMENT, "tuning cache path is null or empty");
    std::FILE* f = std::fopen(path, "rb");
    if (!f) throw Error(ERR_INVALID_ARGUMENT, std::string("cannot open tuning cache: ") + path);
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    std::fclose(f);
    const TuningFile tf = parse_tuning_text(text);
    if (sms) *sms = tf.sms;
    if (singles) *singles = (int)tf.singles.size();
    if (lists) *lists = (int)tf.lists.size();
    if (device && device_len > 0) {
      const size_t k = std::min(tf.device.size(), device_len - 1);
      std::memcpy(device, tf.device.data(), k);
      device[k] = 0;
    }
  });
}

extern "C" TAPP_error tprims_b200_executor_clear_tuning(TAPP_executor exec) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.tune.clear();
    ex.list_tune.clear();
  });
}

extern "C" size_t tprims_b200_executor_tuning(TAPP_executor exec, char* buf, size_t maxlen) {
  std::string s;
  if (ffi([&] {
        Executor& ex = resolve_exec(exec)->get();
        std::lock_guard<std::mutex> lk(ex.mu);
        s = tuning_json(ex);
      }) != TPRIMS_OK)
    return 0;
  if (buf && maxlen > 0) {
    const size_t n = s.size() < maxlen - 1 ? s.size() : maxlen - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

extern "C" uint64_t tprims_b200_device_allocations(void) { return device_allocations(); }

extern "C" TAPP_error tprims_b200_executor_inject_launch_failure(TAPP_executor exec, int after) {
  return ffi([&] {
    if (after < -1) throw Error(ERR_INVALID_ARGUMENT, "launch count must be -1 (off) or >= 0");
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.fail_launch_after = after;
  });
}

extern "C" TAPP_error tprims_b200_executor_set_grouping(TAPP_executor exec, int on) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.grouping = on != 0;
  });
}

extern "C" TAPP_error tprims_b200_executor_set_streaming(TAPP_executor exec, int on) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.streaming = on != 0;
  });
}

extern "C" TAPP_error tprims_b200_executor_set_workspace_limit(TAPP_executor exec, size_t bytes) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    ex.ws_limit = bytes == 0 ? SIZE_MAX : bytes;
  });
}

extern "C" TAPP_error tprims_b200_executor_selftest_wait(TAPP_executor exec, uint64_t limit_ns) {
  return ffi([&] {
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ex.device);
    struct Restore {
      int d;
      ~Restore() {
        if (d >= 0) cudaSetDevice(d);
      }
    } restore{prev};
    // The flag is a zeroed word of the status allocation that nothing writes.
    unsigned* flag = ex.status + 32;
    check_cuda(cudaMemsetAsync(flag, 0, sizeof(unsigned), ex.stream), "selftest flag");
    check_cuda(dev::launch_wait_selftest(flag, ex.status, limit_ns, ex.stream), "selftest launch");
    finish(ex);
  });
}

extern "C" TAPP_error tprims_b200_executor_probe_peak(TAPP_executor exec, int which, double* tflops) {
  return ffi([&] {
    if (!tflops) null_arg("tflops out-parameter");
    if (which < 0 || which > 3)
      throw Error(ERR_INVALID_ARGUMENT,
                  "probe must be 0 (FP64 DMMA), 1 (FP32 FFMA), 2 (INT8 tcgen05) or 3 (BF16 tcgen05)");
    Executor& ex = resolve_exec(exec)->get();
    std::lock_guard<std::mutex> lk(ex.mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ex.device);
    struct Restore {
      int d;
      ~Restore() {
        if (d >= 0) cudaSetDevice(d);
      }
    } restore{prev};
    void* sink = ex.workspace(4096);
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    const bool tc = which >= 2;
    const int blocks = tc ? ex.num_sms : ex.num_sms * 8;
    const int iters = which == 0 ? 4096 : (tc ? 20000 : 65536);
    double best = 0, flops = 0;
    for (int rep = 0; rep < 5; ++rep) {
      check_cuda(cudaEventRecord(e0, ex.stream), "cudaEventRecord");
      if (tc)
        check_cuda(dev::launch_tc_probe(which == 2 ? 1 : 0, blocks, iters, ex.status, ex.stream, &flops),
                   "tensor probe launch");
      else
        check_cuda(dev::launch_probe(which, sink, blocks, iters, ex.stream, &flops), "probe launch");
      check_cuda(cudaEventRecord(e1, ex.stream), "cudaEventRecord");
      check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0;
      check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    finish(ex);  // a tensor probe that gave up on its bounded wait reports here
    *tflops = best;
  });
}

extern "C" TAPP_error tprims_b200_execute_product_noalloc(TAPP_tensor_product plan, uintptr_t stream,
                                                         const void* alpha, const void* A, const void* B,
                                                         const void* beta, const void* C, void* D) {
  return ffi([&] {
    Product& p = product_of(plan);
    if (!alpha) null_arg("alpha");
    if (!beta) null_arg("beta");
    const Scalar al = read_scalar(p.problem.dtype, alpha), be = read_scalar(p.problem.dtype, beta);
    const Item it{A, B, C, D};
    validate_item(p, it, be.is_zero());
    execute_split_noalloc(p, reinterpret_cast<cudaStream_t>(stream), al, be, it);
  });
}
