/* libtprims_b200: a B200 (sm_100a) executor behind the TAPP C ABI of libtprims.
 *
 * Every entry point is plain C: integer handles (intptr_t), raw pointers and
 * sizes. Nothing here names a CUDA, PyTorch or C++ type, so a C, Rust, Julia or
 * Python host binds it exactly as it binds the CPU libtprims.
 *
 * Part 1 repeats the standard TAPP declarations (numeric values and prototypes
 * are ABI and are kept identical to the pinned upstream headers the reference
 * ships in the headers of crates/tprims-capi/include/tapp/). When the upstream <tapp.h> has
 * already been included, part 1 is skipped and its declarations are used.
 *
 * Part 2 repeats the tprims extensions of crates/tprims-capi/include/tprims/
 * core.h and tapp_ext.h (status codes, last error, ABI version, DLPack borrows,
 * the pooled-executor constructor).
 *
 * Part 3 is new to this library: a CUDA executor, the DLPack execute call that
 * accepts kDLCUDA operands, the precision-scheme setter (plain, 3xBF16, 6xBF16,
 * Ozaki INT8), the plan report, the dot_general front end, the batched list
 * call and the vector-Jacobian product. */
#ifndef TPRIMS_B200_H
#define TPRIMS_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
#define TPRIMS_B200_EXPORT extern "C" __attribute__((visibility("default")))
#else
#define TPRIMS_B200_EXPORT __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------ part 1 */
#ifndef TAPP_TAPP_H_
#define TAPP_TAPP_H_

typedef int TAPP_error;
typedef intptr_t TAPP_handle;
typedef intptr_t TAPP_executor;
typedef intptr_t TAPP_status;
typedef intptr_t TAPP_tensor_info;
typedef intptr_t TAPP_tensor_product;
typedef intptr_t TAPP_attr;
typedef int TAPP_key;
typedef int TAPP_datatype;
typedef int TAPP_prectype;
typedef int TAPP_element_op;

/* tapp/datatype.h */
enum {
  TAPP_F32 = 0,
  TAPP_F64 = 1,
  TAPP_C32 = 2,
  TAPP_C64 = 3,
  TAPP_F16 = 4,
  TAPP_BF16 = 5,
  TAPP_FLOAT = TAPP_F32,
  TAPP_DOUBLE = TAPP_F64,
  TAPP_SCOMPLEX = TAPP_C32,
  TAPP_DCOMPLEX = TAPP_C64
};
enum {
  TAPP_DEFAULT_PREC = -1,
  TAPP_F32F32_ACCUM_F32 = 0,
  TAPP_F64F64_ACCUM_F64 = 1,
  TAPP_F16F16_ACCUM_F16 = 4,
  TAPP_F16F16_ACCUM_F32 = 5,
  TAPP_BF16BF16_ACCUM_F32 = 6
};
/* tapp/product.h */
enum { TAPP_IDENTITY = 0, TAPP_CONJUGATE = 1 };
#define TAPP_IN_PLACE NULL

/* tapp/error.h — crates/tprims-capi/src/status.rs:69 and :81 */
TPRIMS_B200_EXPORT bool TAPP_check_success(TAPP_error error);
TPRIMS_B200_EXPORT size_t TAPP_explain_error(TAPP_error error, size_t maxlen, char* message);
/* tapp/attributes.h — crates/tprims-capi/src/handle.rs:83-127 (every key refused) */
TPRIMS_B200_EXPORT TAPP_error TAPP_attr_set(TAPP_attr attr, TAPP_key key, void* value);
TPRIMS_B200_EXPORT TAPP_error TAPP_attr_get(TAPP_attr attr, TAPP_key key, void** value);
TPRIMS_B200_EXPORT TAPP_error TAPP_attr_clear(TAPP_attr attr, TAPP_key key);
/* tapp/handle.h — crates/tprims-capi/src/handle.rs:35 and :52 */
TPRIMS_B200_EXPORT TAPP_error TAPP_create_handle(TAPP_handle* handle);
TPRIMS_B200_EXPORT TAPP_error TAPP_destroy_handle(TAPP_handle handle);
/* tapp/executor.h — crates/tprims-capi/src/executor.rs:278 and :299. Here an
   executor is one CUDA stream on the current device plus its workspace. */
TPRIMS_B200_EXPORT TAPP_error TAPP_create_executor(TAPP_executor* exec);
TPRIMS_B200_EXPORT TAPP_error TAPP_destroy_executor(TAPP_executor exec);
/* tapp/status.h — crates/tprims-capi/src/handle.rs:133 (a no-op: execution is synchronous) */
TPRIMS_B200_EXPORT TAPP_error TAPP_destroy_status(TAPP_status status);
/* tapp/tensor.h — crates/tprims-capi/src/tensor_info.rs:58-221 */
TPRIMS_B200_EXPORT TAPP_error TAPP_create_tensor_info(TAPP_tensor_info* info, TAPP_datatype type, int nmode,
                                                      const int64_t* extents, const int64_t* strides);
TPRIMS_B200_EXPORT TAPP_error TAPP_destroy_tensor_info(TAPP_tensor_info info);
TPRIMS_B200_EXPORT int TAPP_get_nmodes(TAPP_tensor_info info);
TPRIMS_B200_EXPORT TAPP_error TAPP_set_nmodes(TAPP_tensor_info info, int nmodes);
TPRIMS_B200_EXPORT void TAPP_get_extents(TAPP_tensor_info info, int64_t* extents);
TPRIMS_B200_EXPORT TAPP_error TAPP_set_extents(TAPP_tensor_info info, const int64_t* extents);
TPRIMS_B200_EXPORT void TAPP_get_strides(TAPP_tensor_info info, int64_t* strides);
TPRIMS_B200_EXPORT TAPP_error TAPP_set_strides(TAPP_tensor_info info, const int64_t* strides);
/* tapp/product.h — crates/tprims-capi/src/product.rs:83 and :198 */
TPRIMS_B200_EXPORT TAPP_error TAPP_create_tensor_product(
    TAPP_tensor_product* plan, TAPP_handle handle, TAPP_element_op op_A, TAPP_tensor_info A, const int64_t* idx_A,
    TAPP_element_op op_B, TAPP_tensor_info B, const int64_t* idx_B, TAPP_element_op op_C, TAPP_tensor_info C,
    const int64_t* idx_C, TAPP_element_op op_D, TAPP_tensor_info D, const int64_t* idx_D, TAPP_prectype prec);
TPRIMS_B200_EXPORT TAPP_error TAPP_destroy_tensor_product(TAPP_tensor_product plan);
/* crates/tprims-capi/src/execute.rs:192. Synchronous: returns when D is written. */
TPRIMS_B200_EXPORT TAPP_error TAPP_execute_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                                   const void* alpha, const void* A, const void* B, const void* beta,
                                                   const void* C, void* D);
/* crates/tprims-capi/src/execute.rs:235. Items are validated first, then run. */
TPRIMS_B200_EXPORT TAPP_error TAPP_execute_batched_product(TAPP_tensor_product plan, TAPP_executor exec,
                                                           TAPP_status* status, int num_batches, const void* alpha,
                                                           const void** A, const void** B, const void* beta,
                                                           const void** C, void** D);
#endif /* TAPP_TAPP_H_ */

/* ------------------------------------------------------------------ part 2 */
#ifndef TPRIMS_CORE_H
#define TPRIMS_CORE_H
#define TPRIMS_ABI_VERSION 100 /* 0.1.0, crates/tprims-capi/src/lib.rs:140 */

typedef int32_t tprims_status;
/* crates/tprims-capi/src/status.rs:13-43 */
#define TPRIMS_OK 0
#define TPRIMS_ERR_INVALID_ARGUMENT 1
#define TPRIMS_ERR_SHAPE 2
#define TPRIMS_ERR_DTYPE 3
#define TPRIMS_ERR_DEVICE 4
#define TPRIMS_ERR_READ_ONLY 5
#define TPRIMS_ERR_ALIASED 6
#define TPRIMS_ERR_WOULD_MATERIALIZE 7
#define TPRIMS_ERR_NUMERICAL 8
#define TPRIMS_BUSY 9
#define TPRIMS_ERR_WOULD_DEADLOCK 10
#define TPRIMS_ERR_PANIC 12
#define TPRIMS_ERR_INTERNAL 13
#define TPRIMS_ERR_LABELS 14
#define TPRIMS_ERR_UNSUPPORTED 15

/* DLPack 1.x ABI subset (the struct layouts are the DLPack standard's). */
#ifndef DLPACK_DLPACK_H_
#define DLPACK_DLPACK_H_
typedef enum { kDLCPU = 1, kDLCUDA = 2, kDLCUDAHost = 3, kDLCUDAManaged = 13 } DLDeviceType;
typedef struct { DLDeviceType device_type; int32_t device_id; } DLDevice;
typedef enum { kDLInt = 0, kDLUInt = 1, kDLFloat = 2, kDLBfloat = 4, kDLComplex = 5, kDLBool = 6 } DLDataTypeCode;
typedef struct { uint8_t code; uint8_t bits; uint16_t lanes; } DLDataType;
typedef struct {
  void* data;
  DLDevice device;
  int32_t ndim;
  DLDataType dtype;
  int64_t* shape;
  int64_t* strides;
  uint64_t byte_offset;
} DLTensor;
typedef struct { uint32_t major; uint32_t minor; } DLPackVersion;
typedef struct DLManagedTensorVersioned {
  DLPackVersion version;
  void* manager_ctx;
  void (*deleter)(struct DLManagedTensorVersioned* self);
  uint64_t flags;
  DLTensor dl_tensor;
} DLManagedTensorVersioned;
#endif

/* crates/tprims-capi/include/tprims/core.h: a borrowed operand, never freed here. */
typedef struct { DLTensor* view; uint64_t flags; } tprims_tensor;
TPRIMS_B200_EXPORT tprims_tensor tprims_tensor_borrow_versioned(struct DLManagedTensorVersioned* m); /* tensor.rs:26 */
TPRIMS_B200_EXPORT tprims_tensor tprims_tensor_borrow_raw(DLTensor* t, uint64_t flags);       /* tensor.rs:55 */
TPRIMS_B200_EXPORT const char* tprims_last_error(void);                                      /* status.rs:168 */
TPRIMS_B200_EXPORT uint32_t tprims_abi_version(void);                                        /* lib.rs:143 */
TPRIMS_B200_EXPORT int32_t tprims_has_part(const char* part);                                /* lib.rs:154 */
TPRIMS_B200_EXPORT const char* TAPP_implementation_name(void);                               /* handle.rs:141 */
TPRIMS_B200_EXPORT const char* TAPP_implementation_version(void);                            /* handle.rs:158 */
#endif /* TPRIMS_CORE_H */

#ifndef TPRIMS_TAPP_EXT_H
#define TPRIMS_TAPP_EXT_H
typedef struct { size_t stack_size; } tprims_rayon_opts;
/* crates/tprims-capi/src/executor.rs:320-392. Kept for source compatibility:
   nthreads == 0 is refused as in the reference; otherwise a CUDA executor on the
   current device is created and nthreads is recorded as its host budget. */
TPRIMS_B200_EXPORT TAPP_error tprims_tapp_executor_create_rayon(TAPP_executor* out, size_t nthreads,
                                                                const tprims_rayon_opts* opts);
TPRIMS_B200_EXPORT TAPP_error tprims_tapp_executor_set_budget(TAPP_executor exec, size_t budget);
TPRIMS_B200_EXPORT TAPP_error tprims_tapp_executor_get_threads(TAPP_executor exec, size_t* pool_size,
                                                               size_t* budget);
#endif /* TPRIMS_TAPP_EXT_H */

/* ------------------------------------------------------------------ part 3 */
#ifdef __cplusplus
extern "C" {
#endif

/* Executor on CUDA device `device` (-1 = the current device). `stream` is a
   cudaStream_t passed as an integer; 0 makes the executor create its own
   stream, a blocking one (ordered with work on the legacy default stream).
   No reference counterpart: the reference's executors are CPU thread pools
   (executor.rs:278-392). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_create(TAPP_executor* out, int device, uintptr_t stream);
/* The executor's stream, as an integer cudaStream_t. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_stream(TAPP_executor exec, uintptr_t* stream);
/* Execution mode of an executor: 1 = synchronous (the TAPP default: every
   execute returns after the stream is drained), 0 = asynchronous (device
   operands only; the call returns once the work is enqueued). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_set_sync(TAPP_executor exec, int sync);
/* Drain the executor's stream and report any kernel-side error status word. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_synchronize(TAPP_executor exec);

/* Grouped submission of lists (contract_batched, TAPP_execute_batched_product):
   with `on` != 0 (the default) the plain-precision items whose operands are in
   device memory run as one persistent grouped launch per kernel family,
   replayed from a cached CUDA graph; with 0 every item is its own launch. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_set_grouping(TAPP_executor exec, int on);
/* Streamed execution of host operands (no counterpart in the reference, whose
   operands are always host memory): with `on` != 0 (the default) a single
   contraction of at least 32 MiB whose A, B and D are all host memory, whose
   C is not read and which writes every element of D is split into chunks
   along the outermost column axis of its output; the copy in of one chunk,
   the kernels of the previous one and the copy out of the one before run at
   once on the executor's stream and two copy streams. The call stays
   synchronous and the result is the same as unstreamed (the kernels are the
   same). Layouts whose chunks cannot be moved as whole pitched copies (not
   nested, or negative strides) run unstreamed. 0 = always unstreamed. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_set_streaming(TAPP_executor exec, int on);
/* Failure detection without a GPU fault. tprims_b200_executor_set_workspace_limit
   caps the executor's workspace arena (0 = no cap): a call that needs more is
   refused with TPRIMS_ERR_INTERNAL before anything runs (allocation-failure
   injection). tprims_b200_executor_selftest_wait launches one kernel that waits
   on a flag nothing sets and gives up after `limit_ns`; the executor reports
   the recorded timeout as TPRIMS_ERR_INTERNAL and stays usable. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_set_workspace_limit(TAPP_executor exec, size_t bytes);
/* Launch-failure injection (simulated stream errors, on the host): the
   contraction launch `after` launches from now (0 = the next) is refused with
   TPRIMS_ERR_INTERNAL before anything of it reaches the GPU; its output is
   left as it was and later calls run normally. -1 switches the hook off. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_inject_launch_failure(TAPP_executor exec, int after);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_selftest_wait(TAPP_executor exec, uint64_t limit_ns);
/* Measured pipe peak for roofline denominators (diagnostics): which = 0 runs
   the FP64 DMMA pipe (mma.sync m8n8k4), 1 the FP32 FFMA pipe, with
   register-only operation chains on every SM; 2 the INT8 and 3 the BF16
   tensor pipe (dense 128 x 256 tcgen05.mma products from shared memory into
   TMEM, one CTA per SM); *tflops receives the best of a few timed launches
   (CUDA events on the executor's stream), in TFLOP/s or TOP/s. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_probe_peak(TAPP_executor exec, int which, double* tflops);
/* The executor's autotuner cache, persisted as a versioned text file (the
   reference has no tuning state to persist; this is the build's only
   checkpoint). save writes every entry; load adds the entries of a file
   written on the same kind of device (SM count and name; others are skipped)
   and refuses a malformed file with INVALID_ARGUMENT, adding nothing. clear
   empties the cache; tuning returns it as JSON (full length, like snprintf). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_save_tuning(TAPP_executor exec, const char* path);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_load_tuning(TAPP_executor exec, const char* path);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_clear_tuning(TAPP_executor exec);
/* Checks a cache file without an executor (no GPU needed): the header's SM
   count and device name, and the number of single-contraction and list
   entries; a malformed file is INVALID_ARGUMENT, another version UNSUPPORTED.
   Any out-parameter may be NULL. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_tuning_file_info(const char* path, int* sms, char* device,
                                                          size_t device_len, int* singles, int* lists);
TPRIMS_B200_EXPORT size_t tprims_b200_executor_tuning(TAPP_executor exec, char* buf, size_t maxlen);
/* Number of device allocations the library has made in this process (every
   cudaMalloc of executors, workspaces, scatter vectors, grouped-list
   descriptors and network arenas). Diagnostics: once a call has run, repeating
   it leaves the count unchanged (the counterpart of the reference's allocation
   counter tests, tprims-contract tests packed_workspace_alloc.rs). */
TPRIMS_B200_EXPORT uint64_t tprims_b200_device_allocations(void);
/* Per-kernel timing (diagnostics, off by default): with `on` != 0 the executor
   records CUDA events on its stream around every kernel launch. The totals
   are resolved whenever the stream is drained. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_executor_set_profiling(TAPP_executor exec, int on);
/* JSON {"kernel family": {"ms": total, "launches": n}, ...} of the resolved
   totals (the stream is drained first); `reset` != 0 clears them. Returns the
   full length, like snprintf. */
TPRIMS_B200_EXPORT size_t tprims_b200_executor_kernel_times(TAPP_executor exec, char* buf, size_t maxlen, int reset);

/* Precision schemes. PLAIN is the drop-in (FP32 SIMT / FP64 DMMA, complex by
   four real products); the others are split-precision tensor-core schemes whose
   error bound is stated in the plan report. */
enum {
  TPRIMS_PREC_PLAIN = 0,
  TPRIMS_PREC_BF16X3 = 1, /* f32: hi/lo BF16 split, 3 products, FP32 accumulation */
  TPRIMS_PREC_BF16X6 = 2, /* f32: 3-way BF16 split, 6 products, FP32 accumulation */
  TPRIMS_PREC_OZAKI_INT8 = 3 /* f64/c64: INT8 slices, exact INT32 accumulation */
};
/* Choose the precision scheme of a product. `slices` is the INT8 slice count
   for TPRIMS_PREC_OZAKI_INT8 (4..8; 0 = the default, 6) and is ignored
   otherwise. Refused (UNSUPPORTED) for a dtype the scheme does not apply to.
   The reference has no counterpart (its C ABI has no tuning call, product.rs:48). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_set_precision(TAPP_tensor_product plan, int scheme, int slices);
/* Pin the plain-path tile family (0 = chosen per shape). Rows x cols of the
   oriented M/N tile: 1 f32 128x128, 2 f32 64x64, 3 f64 64x64, 4 f64 32x32,
   5 c32 64x64, 6 c64 64x32, 7 c64 32x32, 8 f64 128x32, 9 c64 128x32 (direct
   tiles: the gather is part of the tile); packed families (a pack pass into
   dense panels, then TMA-fed tiles; single contractions only, a grouped list
   runs its items on direct tiles): 10 f32 128x128, 11 c32 64x128 as 1m (the
   2M x N x 2K real embedding), 12 f64 64x64, 13 c64 64x32 as 3m (three real
   products per complex MAC), 14 f32 128x64 and 15 c32 64x64 as 1m (half-width
   tiles, two CTAs per SM). A direct family of another dtype is refused at
   execution with TPRIMS_ERR_INTERNAL, a packed one with
   TPRIMS_ERR_INVALID_ARGUMENT. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_set_tile(TAPP_tensor_product plan, int kernel_id);
/* Plan::check_raw (crates/tprims-contract/src/plan/mod.rs:384): the aliasing
   preflight of a call from its origins alone (nothing is dereferenced; a NULL
   origin is absent): TPRIMS_ERR_ALIASED when D's reachable address range
   overlaps A's or B's, or a separate C's without being the same mapping at the
   same origin; TPRIMS_OK otherwise. Every execute entry runs it first. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_check_raw(TAPP_tensor_product plan, const void* A, const void* B,
                                                            const void* C, const void* D);
/* Pin the split-K factor of the plain path: 0 = chosen (model or autotuner),
   1 = never split K, 2..64 = cut K into that many chunks of whole 64-deep
   blocks (fewer when K is short). Split partials are summed in a fixed order.
   The counterpart of the reference's frozen partition (select/resolve.rs:164),
   which never splits K; INVALID_ARGUMENT outside 0..64. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_set_split_k(TAPP_tensor_product plan, int splits);
/* Autotuning (PlanConfig's `autotune` switch; the reference freezes its choice
   from an analytical model instead, contract resolve.rs:42, kernel
   blocking/model.rs:220). With `on` != 0 and no pins, the first plain
   execution of the plan's Problem signature (dtype, folded extents and
   strides, conjugations, scheme, whether C is read) on an executor times every
   candidate tile family and split-K factor on the executor's stream and keeps
   the fastest in the executor's cache; later executions of any plan with that
   signature use it. A grouped list whose plans all autotune has its tile policy
   measured the same way, keyed by the list's signatures. Results stay within
   the plain path's stated error; D is left as one execution leaves it (a D
   that is also C is restored between the timed runs). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_set_autotune(TAPP_tensor_product plan, int on);
/* A NUL-terminated JSON description of the plan (the counterpart of
   Plan::report, crates/tprims-contract/src/plan/mod.rs:237). Returns the full
   length, like snprintf. */
TPRIMS_B200_EXPORT size_t tprims_b200_product_report(TAPP_tensor_product plan, char* buf, size_t maxlen);

/* Problem::from_dot_general (crates/tprims-contract/src/api/problem.rs:396):
   D has extents [lhs_free, rhs_free, batch]; C is D itself (CSpec::Output).
   `*_contract` and `*_batch` are axis lists of A and B. Produces a product
   usable with TAPP_execute_product (C = NULL overwrites D; C = D accumulates in
   place). dtype is a TAPP_datatype. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_from_dot_general(
    TAPP_tensor_product* plan, TAPP_datatype dtype, int rank_a, const int64_t* ext_a, const int64_t* str_a,
    TAPP_element_op op_a, int rank_b, const int64_t* ext_b, const int64_t* str_b, TAPP_element_op op_b, int rank_d,
    const int64_t* ext_d, const int64_t* str_d, TAPP_element_op op_d, int n_contract, const int64_t* lhs_contract,
    const int64_t* rhs_contract, int n_batch, const int64_t* lhs_batch, const int64_t* rhs_batch);

/* Inspection for tests and diagnostics: copy scatter vector `which` of the
   packed plan before orientation (0 a_m, 1 a_k, 2 b_k, 3 b_n, 4 c_m, 5 c_n,
   6 d_m, 7 d_n, 8 h_a, 9 h_b, 10 h_c, 11 h_d; the fields of PackedPlan,
   crates/tprims-contract/src/plan/analysis.rs:139-150) into `out` (at most
   `cap` entries). Returns the vector's length, or -1 for a bad argument. */
TPRIMS_B200_EXPORT int64_t tprims_b200_product_scatter(TAPP_tensor_product plan, int which, int64_t* out,
                                                       int64_t cap);

/* DLPack execution (the extension the reference declines: dlpack.rs:87 rejects
   kDLCUDA). Operands are kDLCUDA on the executor's device, kDLCUDAHost or
   kDLCPU; lanes == 1; NULL strides mean row-major; C.view may be NULL only with
   a zero beta. The tensors' shapes and strides must equal the plan's. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_execute_product_dlpack(TAPP_tensor_product plan, TAPP_executor exec,
                                                                 TAPP_status* status, const void* alpha,
                                                                 tprims_tensor A, tprims_tensor B, const void* beta,
                                                                 tprims_tensor C, tprims_tensor D);

/* contract_batched (crates/tprims-contract/src/batch.rs:125): a heterogeneous
   list, validated all-or-nothing before any D is written, then executed as one
   grouped submission on the executor's stream. */
typedef struct {
  TAPP_tensor_product plan;
  const void* alpha;
  const void* A;
  const void* B;
  const void* beta;
  const void* C;
  void* D;
} tprims_b200_batch_item;
TPRIMS_B200_EXPORT TAPP_error tprims_b200_contract_batched(TAPP_executor exec, int n,
                                                           const tprims_b200_batch_item* items);

/* N-ary contraction networks. The reference keeps the N-ary layer (einsum)
   above its stack (docs/architecture.md:54): its callers contract a network
   pair by pair through Problem::from_labels / Plan::execute_into. These calls
   are that caller on the GPU. A network is created from its input tensors
   (extents, signed element strides or NULL for column-major, labels, and
   TAPP_IDENTITY / TAPP_CONJUGATE per input), the output's layout and labels,
   and a pairwise path of n_steps = n_inputs - 1 steps given as 2 * n_steps
   positions in the current operand list (opt_einsum convention: both operands
   are removed and the result appended); n_steps = 0 chooses a greedy path.
   Labels follow the TAPP rules per step: labels shared by the two operands
   and needed later are batch, others shared are contracted, a label of one
   operand needed nowhere else is summed, an output label found in no input is
   UNSUPPORTED, extents of one label must agree (SHAPE). Intermediates are
   dense column-major in a device arena of tprims_b200_network_workspace_size
   bytes (the caller's `workspace`, or the network's own when NULL).
   Execution computes out = alpha * network + beta * out (out is read only when
   beta != 0), synchronously like TAPP_execute_product; inputs and out may be
   host or device memory. tprims_b200_networks_execute runs a list of
   networks, step s of every network as one grouped submission. */
typedef intptr_t tprims_b200_network;
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_create(tprims_b200_network* net, TAPP_datatype dtype, int n_inputs,
                                                         const int* nmodes, const int64_t* const* extents,
                                                         const int64_t* const* strides,
                                                         const int64_t* const* labels, const TAPP_element_op* ops,
                                                         int out_nmode, const int64_t* out_extents,
                                                         const int64_t* out_strides, const int64_t* out_labels,
                                                         int n_steps, const int* path);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_destroy(tprims_b200_network net);
/* Precision scheme and autotuning of every step's plan (as for a product). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_set_precision(tprims_b200_network net, int scheme, int slices);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_set_autotune(tprims_b200_network net, int on);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_workspace_size(tprims_b200_network net, size_t* bytes);
/* JSON: the path, each step's operands, labels, extents, arena offset and plan
   report. Returns the full length, like snprintf. */
TPRIMS_B200_EXPORT size_t tprims_b200_network_report(tprims_b200_network net, char* buf, size_t maxlen);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_network_execute(tprims_b200_network net, TAPP_executor exec,
                                                          const void* alpha, const void* const* inputs,
                                                          const void* beta, void* out, void* workspace);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_networks_execute(TAPP_executor exec, int n, const tprims_b200_network* nets,
                                                           const void* const* alphas,
                                                           const void* const* const* inputs,
                                                           const void* const* betas, void* const* outs,
                                                           void* const* workspaces);

/* Scale-out without collectives: contract_batched over several executors
   (one per GPU, or several per GPU). The items are validated all-or-nothing,
   balanced longest-first by their multiply-accumulates over the executors of
   the device that holds each item's D (a host D may go anywhere; a device with
   no executor in `execs` is TPRIMS_ERR_DEVICE), and each executor's share runs
   as one grouped submission on its own stream, all streams side by side; no
   data moves between devices. tprims_b200_balance is the assignment alone:
   item i of cost costs[i] and home device homes[i] (NULL or < 0: any) goes to
   part assignment[i] of n_parts parts on part_devices. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_contract_batched_sharded(const TAPP_executor* execs, int n_exec, int n,
                                                                   const tprims_b200_batch_item* items);
TPRIMS_B200_EXPORT TAPP_error tprims_b200_balance(int n, const double* costs, const int* homes, int n_parts,
                                                  const int* part_devices, int* assignment);

/* Plan::vjp. For D = alpha*op_A(A)*op_B(B) (+ beta*C), given the cotangent dD,
   write dA (when non-NULL) and dB (when non-NULL) in the layouts of A and B:
   dA = conj-correct adjoint contraction of dD with B, scattered onto A's
   repeated-index diagonal (every element off the diagonal is set to zero), and
   likewise dB. No reference counterpart (the reference has no AD). */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_product_vjp(TAPP_tensor_product plan, TAPP_executor exec, const void* alpha,
                                                      const void* A, const void* B, const void* dD, void* dA, void* dB);

/* Split-precision execution that allocates no device memory. No counterpart
   in the reference. For callers that cannot call cudaMalloc: code running
   inside a memory pool that another component owns (a framework's caching
   allocator, a server that reserved the GPU's memory up front), or code that
   must not let cudaMalloc / cudaFree synchronise the device. Same operands and
   semantics as TAPP_execute_product, for an F32 plan set to
   TPRIMS_PREC_BF16X3 or TPRIMS_PREC_BF16X6 (others: TPRIMS_ERR_UNSUPPORTED);
   A, B, C and D must be in the current device's memory (else
   TPRIMS_ERR_DEVICE). Runs on `stream` (a cudaStream_t as an integer; 0 = the
   legacy default stream) of the current device and returns after that stream
   has drained; a stream that has not drained within 60 s (it waits on an event
   nobody records, say) gives TPRIMS_ERR_INTERNAL instead of blocking forever.
   Its scratch is one fixed 64 MiB device array inside this library, held on
   every GPU that loads the library until the process exits; a contraction
   that needs more (about M = N = K = 2048 at bf16x6 fits) is refused with
   TPRIMS_ERR_SHAPE before anything runs. The first call on a device looks
   the array's address up (this may load the library's device code), so make
   it before any stream capture on that device; the address is looked up
   again when the device's current context changes (after a cudaDeviceReset),
   but a reset while a call is in flight is not supported. All calls share
   the array: calls that overlap on one GPU, from two streams or two threads,
   race on it and give wrong results. */
TPRIMS_B200_EXPORT TAPP_error tprims_b200_execute_product_noalloc(TAPP_tensor_product plan, uintptr_t stream,
                                                                  const void* alpha, const void* A, const void* B,
                                                                  const void* beta, const void* C, void* D);

#ifdef __cplusplus
}
#endif
#endif /* TPRIMS_B200_H */
