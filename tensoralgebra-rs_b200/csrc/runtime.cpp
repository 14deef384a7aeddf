// Executors, device state of products, operand staging and kernel dispatch.
#include "runtime.hpp"

#include "network.hpp"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <climits>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <sstream>
#include <vector>

namespace tprims {

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();  // clear a sticky launch error of this thread
  const int st = (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
                     ? ERR_DEVICE
                     : ERR_INTERNAL;
  throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
std::atomic<uint64_t> g_device_allocations{0};
}  // namespace

cudaError_t device_alloc(void** p, size_t bytes) {
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) g_device_allocations.fetch_add(1, std::memory_order_relaxed);
  return e;
}

uint64_t device_allocations() { return g_device_allocations.load(std::memory_order_relaxed); }

namespace {

// An NVTX range for the scope (a no-op unless a profiler is attached), so the
// library's calls show up by name on an Nsight or ncu --nvtx timeline.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Makes `device` current for the scope and restores the caller's device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {
    check_cuda(cudaGetDevice(&prev), "cudaGetDevice");
    if (prev != device) check_cuda(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
  }
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

Executor* Executor::create(int device, uintptr_t stream) {
  int ndev = 0;
  check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0) check_cuda(cudaGetDevice(&device), "cudaGetDevice");
  if (device >= ndev) throw Error(ERR_DEVICE, "no CUDA device " + std::to_string(device));
  std::unique_ptr<Executor> ex(new Executor());
  ex->device = device;
  DeviceGuard g(device);
  if (stream == 0) {
    // A blocking stream: ordered after work on the legacy default stream (where
    // a caller such as torch writes the operands by default) and before work
    // issued there afterwards, so no explicit synchronisation is needed around a call.
    check_cuda(cudaStreamCreateWithFlags(&ex->stream, cudaStreamDefault), "cudaStreamCreate");
    ex->own_stream = true;
  } else {
    ex->stream = reinterpret_cast<cudaStream_t>(stream);
  }
  check_cuda(device_alloc(reinterpret_cast<void**>(&ex->status), 256), "cudaMalloc(status)");
  check_cuda(cudaMemsetAsync(ex->status, 0, 256, ex->stream), "cudaMemset(status)");
  check_cuda(cudaStreamSynchronize(ex->stream), "cudaStreamSynchronize");
  check_cuda(cudaDeviceGetAttribute(&ex->num_sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
  cudaDeviceProp prop;
  check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  ex->device_name = prop.name;
  return ex.release();
}

Executor::~Executor() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (cudaStream_t fs : family_streams) cudaStreamSynchronize(fs);
  for (auto& kv : graphs) {
    cudaGraphExecDestroy(kv.second.exec);
    cudaFree(kv.second.buf);
  }
  if (ws) cudaFree(ws);
  if (status) cudaFree(status);
  if (copy_in) cudaStreamSynchronize(copy_in);
  if (copy_out) cudaStreamSynchronize(copy_out);
  for (cudaEvent_t e : stream_events) cudaEventDestroy(e);
  if (copy_in) cudaStreamDestroy(copy_in);
  if (copy_out) cudaStreamDestroy(copy_out);
  if (own_stream && stream) cudaStreamDestroy(stream);
  if (capture_stream) cudaStreamDestroy(capture_stream);
  for (cudaEvent_t e : family_events) cudaEventDestroy(e);
  for (cudaStream_t fs : family_streams) cudaStreamDestroy(fs);
  if (prev >= 0) cudaSetDevice(prev);
}

void* Executor::workspace(size_t bytes) {
  if (bytes <= ws_bytes) return ws;
  if (bytes > ws_limit)
    throw Error(ERR_INTERNAL, "workspace of " + std::to_string(bytes) + " bytes exceeds the executor's limit of " +
                                  std::to_string(ws_limit) + " bytes");
  // Growing: earlier work on the stream may still use the old arena.
  check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  if (ws) cudaFree(ws);
  ws = nullptr;
  ws_bytes = 0;
  const size_t want = std::max(bytes, ws_bytes + ws_bytes / 2);
  check_cuda(device_alloc(&ws, want), "cudaMalloc(workspace)");
  ws_bytes = want;
  return ws;
}

namespace {
std::atomic<uint64_t> g_product_uid{1};
}

namespace {
// The stride of a scatter vector that is an arithmetic sequence from 0, else INT64_MIN.
int64_t sequence_stride(const std::vector<int64_t>& v) {
  if (v.empty() || v[0] != 0) return INT64_MIN;
  const int64_t s = v.size() > 1 ? v[1] : 0;
  for (size_t i = 1; i < v.size(); ++i)
    if (v[i] != (int64_t)i * s) return INT64_MIN;
  return s;
}
}  // namespace

Product::Product(const Problem& p) : problem(p), uid(g_product_uid.fetch_add(1)) {
  packed = PackedPlan::from_problem(p);
  const bool swap = packed.transposes_gemm(32);
  view = orient(packed, swap);
  tiny_h = dev::TinyStrides{sequence_stride(view.h_a), sequence_stride(view.h_b), sequence_stride(view.h_c),
                            sequence_stride(view.h_d)};
  signature = problem_signature(*this);
}

Product::~Product() {
  for (auto& kv : dev) {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(kv.first);
    cudaFree(kv.second.buf);
    if (prev >= 0) cudaSetDevice(prev);
  }
}

const dev::Scatters& Product::scatters(int device, cudaStream_t stream) {
  std::lock_guard<std::mutex> lk(mu);
  auto it = dev.find(device);
  if (it != dev.end()) return it->second.s;
  // The 12 scatter vectors, then the block scatters (blocks of
  // dev::SCATTER_BLOCK) of a_m, a_k, b_k and b_n for the pack passes.
  const std::vector<int64_t> blk[4] = {
      build_block_scatter(view.a_m, dev::SCATTER_BLOCK), build_block_scatter(view.a_k, dev::SCATTER_BLOCK),
      build_block_scatter(view.b_k, dev::SCATTER_BLOCK), build_block_scatter(view.b_n, dev::SCATTER_BLOCK)};
  static_assert(IRREGULAR == dev::SCATTER_IRREGULAR, "one sentinel for irregular blocks");
  const std::vector<int64_t>* vs[16] = {&view.a_m, &view.a_k, &view.b_k, &view.b_n, &view.c_m, &view.c_n,
                                        &view.d_m, &view.d_n, &view.h_a, &view.h_b, &view.h_c, &view.h_d,
                                        &blk[0],   &blk[1],   &blk[2],   &blk[3]};
  std::vector<int64_t> host;
  size_t offs[16];
  for (int i = 0; i < 16; ++i) {
    offs[i] = host.size();
    host.insert(host.end(), vs[i]->begin(), vs[i]->end());
    host.push_back(0);  // never empty
    while (host.size() % 4) host.push_back(0);
  }
  DeviceScatters ds;
  check_cuda(device_alloc(reinterpret_cast<void**>(&ds.buf), host.size() * sizeof(int64_t)), "cudaMalloc(scatters)");
  // A plain cudaMemcpy from pageable memory may return before its DMA lands,
  // and it is ordered on the legacy stream, which a non-blocking stream does
  // not wait for: copy on the caller's stream and wait for it, so that the
  // vectors are complete for every stream that uses them afterwards.
  cudaError_t e = cudaMemcpyAsync(ds.buf, host.data(), host.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    cudaFree(ds.buf);
    check_cuda(e, "scatter vector upload");
  }
  const int64_t* b = ds.buf;
  ds.s = dev::Scatters{b + offs[0], b + offs[1], b + offs[2],  b + offs[3],  b + offs[4],  b + offs[5],
                       b + offs[6], b + offs[7], b + offs[8], b + offs[9], b + offs[10], b + offs[11]};
  ds.s.blk_a_m = b + offs[12];
  ds.s.blk_a_k = b + offs[13];
  ds.s.blk_b_k = b + offs[14];
  ds.s.blk_b_n = b + offs[15];
  return dev.emplace(device, ds).first->second.s;
}

namespace {

const char* scheme_name(Scheme s) {
  switch (s) {
    case Scheme::Plain: return "plain";
    case Scheme::Bf16x3: return "bf16x3";
    case Scheme::Bf16x6: return "bf16x6";
    case Scheme::OzakiInt8: return "ozaki-int8";
  }
  return "?";
}

std::string axes_json(const std::vector<Axis>& ax) {
  std::ostringstream o;
  o << "[";
  for (size_t i = 0; i < ax.size(); ++i) {
    if (i) o << ",";
    o << "{\"extent\":" << ax[i].extent << ",\"sa\":" << ax[i].sa << ",\"sb\":" << ax[i].sb << ",\"sc\":" << ax[i].sc
      << ",\"sd\":" << ax[i].sd << "}";
  }
  o << "]";
  return o.str();
}

// Relative Frobenius error bound a scheme is designed for (stated, measured in
// the tests): unit roundoff of the storage type times a small factor for the
// plain path; the dropped split terms for the split paths.
double stated_bound(DType t, Scheme s) {
  switch (s) {
    case Scheme::Plain: return dtype_double(t) ? 1e-13 : 1e-6;
    case Scheme::Bf16x3: return 1e-5;
    case Scheme::Bf16x6: return 1e-6;
    case Scheme::OzakiInt8: return 1e-12;
  }
  return 0;
}

}  // namespace

namespace {
size_t scheme_scratch(const Product& pr, const PlainChoice& pc, int num_sms);
}  // namespace

std::string Product::report() const {
  std::ostringstream o;
  const auto& st = packed.stats;
  // The configuration of the last plain execution when there was one, else
  // the model's choice (148 SMs) under the pins.
  PlainChoice pc;
  ChoiceSource src;
  {
    std::lock_guard<std::mutex> lk(mu);
    pc = executed ? last : model_choice(*this, 148);
    src = executed ? last_source : ((kernel_pin || split_pin) ? ChoiceSource::Pinned : ChoiceSource::Model);
  }
  const bool tiny = scheme == Scheme::Plain && pc.tiny;
  const int kernel = pc.kernel, splits = pc.splits;
  static const char* src_names[4] = {"model", "pinned", "autotuned", "tuning-cache"};
  std::string family = tiny ? std::string("sm100.") + dtype_name(problem.dtype) + ".tiny-batched"
                       : scheme == Scheme::Plain ? dev::plain_kernel_name(kernel)
                       : scheme == Scheme::Bf16x3 ? "sm100.f32.tcgen05.bf16x3.128x256x32"
                       : scheme == Scheme::Bf16x6 ? "sm100.f32.tcgen05.bf16x6.128x256x32"
                                                  : std::string("sm100.") + dtype_name(problem.dtype) +
                                                        ".tcgen05.ozaki-int8.s" + std::to_string(ozaki_slices) +
                                                        ".128x64x64";
  o << "{\"algorithm\":\"packed\",\"dtype\":\"" << dtype_name(problem.dtype) << "\",\"m\":" << st.m
    << ",\"n\":" << st.n << ",\"k\":" << st.k << ",\"batch\":" << st.batch
    << ",\"is_pure_gemm\":" << (st.is_pure_gemm ? "true" : "false") << ",\"m_axes\":" << axes_json(st.m_axes)
    << ",\"n_axes\":" << axes_json(st.n_axes) << ",\"k_axes\":" << axes_json(st.k_axes)
    << ",\"h_axes\":" << axes_json(st.h_axes) << ",\"swapped\":" << (view.swapped ? "true" : "false")
    << ",\"a_kfast\":" << (view.a_kfast ? "true" : "false") << ",\"b_kfast\":" << (view.b_kfast ? "true" : "false")
    << ",\"d_mfast\":" << (view.d_mfast ? "true" : "false") << ",\"scheme\":\"" << scheme_name(scheme)
    << "\",\"family\":\"" << family << "\",\"split_k\":" << (scheme == Scheme::Plain && !tiny ? splits : 1)
    << ",\"tail_parts\":"
    << ((scheme == Scheme::Bf16x3 || scheme == Scheme::Bf16x6)
            ? dev::split_tail_parts(dev::split_layout((int)scheme, view.M, view.N, view.K, view.H), 148)
            : 1)
    << ",\"scratch_bytes\":" << scheme_scratch(*this, pc, 148);
  if (scheme == Scheme::Plain && !tiny) {
    // The CTA tile and the CTAs of the main launch (before the 1-D grid's
    // wrap-around) for 148 SMs.
    int bm = 0, bn = 0;
    dev::plain_tile_shape(kernel, &bm, &bn);
    const int64_t tiles = bm > 0 ? ((view.M + bm - 1) / bm) * ((view.N + bn - 1) / bn) * view.H : 0;
    o << ",\"tile\":[" << bm << "," << bn << "],\"ctas\":" << tiles * splits;
  }
  o << ",\"autotune_candidates\":[";
  if (scheme == Scheme::Plain) {
    const auto cands = plain_candidates((int)problem.dtype, view.M, view.N, view.K, view.H, 148);
    for (size_t i = 0; i < cands.size(); ++i)
      o << (i ? "," : "") << "\"" << choice_name(cands[i], (int)problem.dtype) << "\"";
  }
  o << "]"
    << ",\"choice\":\"" << (scheme == Scheme::Plain ? src_names[(int)src] : "fixed")
    << "\",\"autotune\":" << (autotune ? "true" : "false") << ",\"signature\":\"" << signature << "\""
    << ",\"stated_rel_error\":" << stated_bound(problem.dtype, scheme)
    << ",\"regular_rows\":" << regular_fraction(build_block_scatter(view.d_m, 32))
    << ",\"regular_cols\":" << regular_fraction(build_block_scatter(view.d_n, 32))
    << ",\"macs\":" << problem.macs() << "}";
  return o.str();
}

Scalar read_scalar(DType t, const void* p) {
  Scalar s;
  switch (t) {
    case DType::F32: { float v; std::memcpy(&v, p, 4); s.re = v; break; }
    case DType::F64: { double v; std::memcpy(&v, p, 8); s.re = v; break; }
    case DType::C32: { float v[2]; std::memcpy(v, p, 8); s.re = v[0]; s.im = v[1]; break; }
    case DType::C64: { double v[2]; std::memcpy(v, p, 16); s.re = v[0]; s.im = v[1]; break; }
  }
  return s;
}

namespace {

// Byte range [lo, hi) an operand can address from `origin` (null: none).
bool byte_range(const Problem& p, int slot, const void* origin, __int128* lo, __int128* hi) {
  if (!origin) return false;
  const Span& sp = p.spans[slot];
  if (sp.empty) return false;
  const Operand& op = slot == SA ? p.a : slot == SB ? p.b : slot == SC ? p.c : p.d;
  const __int128 off = op.layout.offset, sz = (__int128)dtype_size(p.dtype);
  const __int128 base = (__int128)(uintptr_t)origin;
  *lo = base + (sp.lo - off) * sz;
  *hi = base + (sp.hi - off + 1) * sz;
  return true;
}

bool overlaps(const Problem& p, int s1, const void* o1, int s2, const void* o2) {
  __int128 a0, a1, b0, b1;
  if (!byte_range(p, s1, o1, &a0, &a1) || !byte_range(p, s2, o2, &b0, &b1)) return false;
  return a0 < b1 && b0 < a1;
}

}  // namespace

void check_raw(const Product& pr, const Item& it) {
  const Problem& p = pr.problem;
  if (p.out_empty || !it.d) return;
  if (overlaps(p, SD, it.d, SA, it.a)) throw Error(ERR_ALIASED, "D overlaps A");
  if (overlaps(p, SD, it.d, SB, it.b)) throw Error(ERR_ALIASED, "D overlaps B");
  if (p.cmode == CMode::Separate && it.c) {
    const bool same = it.c == it.d && p.c_matches_d;
    if (!same && overlaps(p, SD, it.d, SC, it.c)) throw Error(ERR_ALIASED, "C and D overlap without being the same mapping");
  }
}

void validate_item(const Product& pr, const Item& it, bool beta_zero) {
  if (!it.a || !it.b || !it.d) throw Error(ERR_INVALID_ARGUMENT, "A, B or D data pointer is null or zero");
  if (!it.c && !beta_zero)
    throw Error(ERR_UNSUPPORTED,
                "a null C (TAPP_IN_PLACE) with a nonzero beta is ambiguous in TAPP and not supported; pass D as C to "
                "accumulate in place");
  check_raw(pr, it);
}

namespace {

enum class Where { Device, Host };

Where classify(const void* ptr, int device) {
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return Where::Host;
  }
  if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
    if (at.type == cudaMemoryTypeDevice && at.device != device)
      throw Error(ERR_DEVICE, "operand lives on CUDA device " + std::to_string(at.device) + ", the executor on " +
                                  std::to_string(device));
    return Where::Device;
  }
  return Where::Host;
}

struct Staged {
  const void* host = nullptr;  // origin as passed
  char* dev_origin = nullptr;  // origin on the device
  char* buf = nullptr;         // start of the copied span
  size_t bytes = 0;
  int64_t lo_bytes = 0;  // byte offset of the span start from the origin
  bool staged = false;
};

// Element offsets an operand addresses relative to its origin, in bytes.
void span_bytes(const Problem& p, int slot, int64_t* lo, size_t* bytes) {
  const Span& sp = p.spans[slot];
  const Operand& op = slot == SA ? p.a : slot == SB ? p.b : slot == SC ? p.c : p.d;
  const int64_t sz = (int64_t)dtype_size(p.dtype);
  *lo = (int64_t)(sp.lo - op.layout.offset) * sz;
  *bytes = (size_t)((sp.hi - sp.lo + 1) * sz);
}

// Whether the contraction writes every element of D's span (so a staged D
// need not be copied in): the distinct output elements (M * N * batch after
// repeated labels collapse) fill the span exactly.
bool fully_written(const Product& pr) {
  const Span& sp = pr.problem.spans[SD];
  const __int128 n = (__int128)pr.packed.stats.m * pr.packed.stats.n * pr.packed.stats.batch;
  return n == sp.hi - sp.lo + 1;
}

dev::Epilogue make_epilogue(const Product& pr, Scalar alpha, Scalar beta, bool c_read) {
  dev::Epilogue e{};
  e.alpha_re = alpha.re;
  e.alpha_im = alpha.im;
  e.beta_re = beta.re;
  e.beta_im = beta.im;
  e.beta_zero = c_read ? 0 : 1;
  const bool cplx = dtype_complex(pr.problem.dtype);
  e.conj_c = (cplx && pr.view.conj_c && c_read) ? 1 : 0;
  e.conj_d = (cplx && pr.view.conj_d) ? 1 : 0;
  e.plain = (!c_read && alpha.is_one() && !e.conj_d) ? 1 : 0;
  return e;
}

// Records the launch of one kernel family on the executor's stream when the
// executor profiles; a no-op otherwise.
struct Timed {
  Executor& ex;
  KernelTimes::Pending p{};
  Timed(Executor& e, const std::string& name) : ex(e) {
    if (!ex.profile) return;
    p.name = name;
    p.beg = ex.times.take();
    p.end = ex.times.take();
    cudaEventRecord(p.beg, ex.stream);
  }
  ~Timed() {
    if (!ex.profile) return;
    cudaEventRecord(p.end, ex.stream);
    ex.times.pending.push_back(p);
  }
};

// Side streams and fork/join events of the executor, created on first use
// (the executor's lock serialises the calls that use them).
void ensure_side(Executor& ex, size_t streams, size_t events) {
  while (ex.family_streams.size() < streams) {
    cudaStream_t s = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate(side)");
    ex.family_streams.push_back(s);
  }
  while (ex.family_events.size() < events) {
    cudaEvent_t e = nullptr;
    check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(side)");
    ex.family_events.push_back(e);
  }
}

// Fork a side stream off the executor's stream (its work starts after what is
// already queued there) and join it back (the executor's stream waits for
// everything queued on the side).
cudaStream_t fork_side(Executor& ex) {
  ensure_side(ex, 1, 2);
  check_cuda(cudaEventRecord(ex.family_events[0], ex.stream), "cudaEventRecord");
  check_cuda(cudaStreamWaitEvent(ex.family_streams[0], ex.family_events[0], 0), "cudaStreamWaitEvent");
  return ex.family_streams[0];
}
void join_side(Executor& ex) {
  check_cuda(cudaEventRecord(ex.family_events[1], ex.family_streams[0]), "cudaEventRecord");
  check_cuda(cudaStreamWaitEvent(ex.stream, ex.family_events[1], 0), "cudaStreamWaitEvent");
}

// One plain execution in the configuration `c` (scratch: the split-K partials).
void launch_plain(Product& pr, Executor& ex, const dev::GemmArgs& g, const PlainChoice& c, char* scratch,
                  size_t scratch_bytes) {
  const int dt = (int)pr.problem.dtype;
  if (c.tiny) {
    Timed t(ex, "tiny_batched");
    check_cuda(dev::launch_tiny_batched(dt, g, pr.tiny_h, ex.num_sms, ex.stream), "tiny batched launch");
    return;
  }
  if (dev::is_packed_kernel(c.kernel)) {
    // Pack pass into dense panels, then the TMA-fed tile (split-K partials
    // after the panels when split).
    if (dev::packed_dtype(c.kernel) != dt)
      throw Error(ERR_INVALID_ARGUMENT, std::string("kernel family ") + dev::plain_kernel_name(c.kernel) +
                                            " does not take " + dtype_name(pr.problem.dtype) + " operands");
    if (!dev::packed_fits(c.kernel, g.M, g.N, g.K, g.H))
      throw Error(ERR_UNSUPPORTED, std::string("kernel family ") + dev::plain_kernel_name(c.kernel) +
                                       " cannot take this shape (batch, rows or depth beyond its grid)");
    dev::PackedLayout L = dev::packed_layout(c.kernel, g.M, g.N, g.K, g.H);
    {
      const auto step = [](const std::vector<int64_t>& x) {
        return x.size() > 1 ? std::llabs(x[1] - x[0]) : (long long)INT64_MAX;
      };
      const OrientedView& v = pr.view;
      L.a_hfast = (v.H >= 8 && step(v.h_a) < std::min(step(v.a_m), step(v.a_k))) ? 1 : 0;
      L.b_hfast = (v.H >= 8 && step(v.h_b) < std::min(step(v.b_n), step(v.b_k))) ? 1 : 0;
    }
    const size_t panels = dev::packed_workspace_bytes(L);
    const size_t part = c.splits > 1 ? (size_t)c.splits * g.H * g.M * g.N * dtype_size(pr.problem.dtype) + 256 : 0;
    if (panels + part + 256 > scratch_bytes) throw Error(ERR_INTERNAL, "packed workspace too small");
    char* pp = reinterpret_cast<char*>(align_up((uintptr_t)scratch, 256));
    dev::GemmArgs gs = g;
    if (c.splits > 1) {
      gs.k_chunk = c.chunk;
      gs.partial = reinterpret_cast<void*>(align_up((uintptr_t)(pp + panels), 256));
    }
    {
      Timed t(ex, "plain_pack");
      // A' and B' packs overlap: B' on a side stream joined back before the GEMM.
      cudaStream_t side = fork_side(ex);
      check_cuda(dev::launch_packed_pack(gs, L, pp, ex.stream, side), "plain pack launch");
      join_side(ex);
    }
    {
      Timed t(ex, dev::plain_kernel_name(c.kernel));
      check_cuda(dev::launch_packed_gemm(gs, L, pp, ex.stream), "packed contraction launch");
    }
    if (c.splits > 1) {
      Timed t(ex, "splitk_reduce");
      check_cuda(dev::launch_splitk_reduce(dt, gs, c.splits, ex.stream), "split-K reduce launch");
    }
    return;
  }
  if (c.splits > 1) {
    // Split-K: partial tiles into the scratch, then the reduce + epilogue.
    const size_t need = (size_t)c.splits * g.H * g.M * g.N * dtype_size(pr.problem.dtype);
    if (need + 256 > scratch_bytes) throw Error(ERR_INTERNAL, "split-K workspace too small");
    dev::GemmArgs gs = g;
    gs.k_chunk = c.chunk;
    gs.partial = reinterpret_cast<void*>(align_up((uintptr_t)scratch, 256));
    {
      Timed t(ex, dev::plain_kernel_name(c.kernel));
      check_cuda(dev::launch_plain_gemm(dt, c.kernel, gs, ex.stream), "plain contraction launch");
    }
    Timed t(ex, "splitk_reduce");
    check_cuda(dev::launch_splitk_reduce(dt, gs, c.splits, ex.stream), "split-K reduce launch");
    return;
  }
  Timed t(ex, dev::plain_kernel_name(c.kernel));
  check_cuda(dev::launch_plain_gemm(dt, c.kernel, g, ex.stream), "plain contraction launch");
}

// The fault-injection hook: counts launches down and refuses the chosen one.
void injected_failure_check(Executor& ex) {
  if (ex.fail_launch_after < 0) return;
  if (ex.fail_launch_after-- == 0)
    throw Error(ERR_INTERNAL, "injected launch failure (tprims_b200_executor_inject_launch_failure)");
}

void launch_contraction(Product& pr, Executor& ex, const dev::GemmArgs& g, bool output_only, const PlainChoice& pc,
                        char* scratch, size_t scratch_bytes) {
  injected_failure_check(ex);
  const int dt = (int)pr.problem.dtype;
  if (output_only) {
    Timed t(ex, "output_pass");
    check_cuda(dev::launch_output_pass(dt, g, ex.stream), "output pass launch");
    return;
  }
  switch (pr.scheme) {
    case Scheme::Plain:
      launch_plain(pr, ex, g, pc, scratch, scratch_bytes);
      return;
    case Scheme::Bf16x3:
    case Scheme::Bf16x6: {
      const dev::SplitLayout L = dev::split_layout((int)pr.scheme, g.M, g.N, g.K, g.H);
      const size_t planes_bytes = dev::split_workspace_bytes(L);
      if (planes_bytes + dev::split_tail_bytes(L, ex.num_sms) > scratch_bytes)
        throw Error(ERR_INTERNAL, "split workspace too small");
      char* ap = reinterpret_cast<char*>(align_up((uintptr_t)scratch, 256));
      char* bp = ap + (size_t)L.planes * L.H * L.m_pad * L.k_pad * 2;
      char* tail = reinterpret_cast<char*>(align_up((uintptr_t)(ap + planes_bytes), 256));
      {
        // The two packs are independent: B's runs on a side stream forked
        // from the executor's stream and joined back before the GEMM, so the
        // two memory-bound passes overlap (and fill each other's tails).
        Timed t(ex, "split_pack");
        cudaStream_t side = fork_side(ex);
        check_cuda(dev::launch_split_pack_f32(g, 1, L, bp, side), "split pack B");
        check_cuda(dev::launch_split_pack_f32(g, 0, L, ap, ex.stream), "split pack A");
        join_side(ex);
      }
      Timed t(ex, pr.scheme == Scheme::Bf16x3 ? "tc_bf16x3_gemm" : "tc_bf16x6_gemm");
      check_cuda(dev::launch_tc_bf16_gemm(g, L, ap, bp, (int)pr.scheme, ex.stream, tail),
                 "tcgen05 contraction launch");
      return;
    }
    case Scheme::OzakiInt8: {
      dev::OzakiLayout L = dev::ozaki_layout(pr.ozaki_slices, dtype_complex(pr.problem.dtype), g.M, g.N, g.K, g.H);
      // Batch-innermost packing when the batch index has the smallest stride.
      const auto step = [](const std::vector<int64_t>& x) {
        return x.size() > 1 ? std::llabs(x[1] - x[0]) : (long long)INT64_MAX;
      };
      const OrientedView& v = pr.view;
      L.a_hfast = (v.H >= 32 && L.m_pad <= 65535 && step(v.h_a) < std::min(step(v.a_m), step(v.a_k))) ? 1 : 0;
      L.b_hfast = (v.H >= 32 && L.n_pad <= 65535 && step(v.h_b) < std::min(step(v.b_n), step(v.b_k))) ? 1 : 0;
      if (dev::ozaki_workspace_bytes(L) > scratch_bytes) throw Error(ERR_INTERNAL, "Ozaki workspace too small");
      char* ws = reinterpret_cast<char*>(align_up((uintptr_t)scratch, 256));
      {
        Timed t(ex, "ozaki_pack");
        cudaStream_t side = fork_side(ex);  // B' packs on a side stream, joined back below
        check_cuda(dev::launch_ozaki_pack(g, L, ws, ex.stream, side), "Ozaki slice pack");
        join_side(ex);
      }
      const int nkb = (int)(L.k_pad / 64);
      for (int kb0 = 0; kb0 < nkb; kb0 += L.kb_chunk) {
        const int kb1 = std::min(nkb, kb0 + L.kb_chunk);
        dev::GemmArgs gc = g;
        if (kb0 > 0) {
          // Later K chunks accumulate into D: beta = 1, C = D, op_C = op_D
          // (the KC-slab rule of the reference's driver/tile.rs:331-350).
          gc.C = g.D;
          gc.s.c_m = g.s.d_m;
          gc.s.c_n = g.s.d_n;
          gc.s.h_c = g.s.h_d;
          gc.e.beta_re = 1.0;
          gc.e.beta_im = 0.0;
          gc.e.beta_zero = 0;
          gc.e.plain = 0;
          gc.e.conj_c = g.e.conj_d;
        }
        Timed t(ex, "ozaki_gemm");
        check_cuda(dev::launch_ozaki_gemm(gc, L, ws, kb0, kb1, ex.stream), "Ozaki INT8 contraction launch");
      }
      return;
    }
  }
}

size_t scheme_scratch(const Product& pr, const PlainChoice& pc, int num_sms) {
  const auto& v = pr.view;
  if (pr.scheme == Scheme::Plain) return plain_scratch(pc, pr);
  if (pr.scheme == Scheme::Bf16x3 || pr.scheme == Scheme::Bf16x6) {
    const dev::SplitLayout L = dev::split_layout((int)pr.scheme, v.M, v.N, v.K, v.H);
    return dev::split_workspace_bytes(L) + dev::split_tail_bytes(L, num_sms) + 512;
  }
  if (pr.scheme == Scheme::OzakiInt8)
    return dev::ozaki_workspace_bytes(
        dev::ozaki_layout(pr.ozaki_slices, dtype_complex(pr.problem.dtype), v.M, v.N, v.K, v.H));
  return 0;
}

}  // namespace

cudaEvent_t KernelTimes::take() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  check_cuda(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

void KernelTimes::resolve() {
  for (auto& p : pending) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.beg, p.end) == cudaSuccess) {
      totals[p.name].ms += ms;
      totals[p.name].launches += 1;
    }
    pool.push_back(p.beg);
    pool.push_back(p.end);
  }
  pending.clear();
}

KernelTimes::~KernelTimes() {
  for (auto e : pool) cudaEventDestroy(e);
  for (auto& p : pending) {
    cudaEventDestroy(p.beg);
    cudaEventDestroy(p.end);
  }
}

std::string kernel_times_json(Executor& ex, bool reset) {
  std::ostringstream o;
  o << "{";
  bool first = true;
  for (auto& kv : ex.times.totals) {
    if (!first) o << ",";
    first = false;
    o << "\"" << kv.first << "\":{\"ms\":" << kv.second.ms << ",\"launches\":" << kv.second.launches << "}";
  }
  o << "}";
  if (reset) ex.times.totals.clear();
  return o.str();
}

// Drain the stream, giving up (with an error) after a deadline instead of
// blocking forever on work that does not finish.
void drain(Executor& ex) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaStreamQuery(ex.stream);
    if (q == cudaSuccess) return;
    if (q != cudaErrorNotReady) check_cuda(q, "kernel execution");
    const auto waited = std::chrono::steady_clock::now() - t0;
    if (waited > std::chrono::seconds(ex.drain_limit_s))
      throw Error(ERR_INTERNAL, "the executor's stream did not drain within " + std::to_string(ex.drain_limit_s) +
                                    " s");
    // Spin for the first 200 us (short synchronous calls), then poll gently.
    if (waited > std::chrono::microseconds(200)) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

void finish(Executor& ex) {
  drain(ex);
  if (!ex.times.pending.empty()) ex.times.resolve();
  unsigned word = 0;
  check_cuda(cudaMemcpy(&word, ex.status, sizeof(word), cudaMemcpyDeviceToHost), "status read");
  if (word != 0) {
    cudaMemsetAsync(ex.status, 0, sizeof(unsigned), ex.stream);
    cudaStreamSynchronize(ex.stream);
    if (word & dev::STATUS_WAIT_TIMEOUT)
      throw Error(ERR_INTERNAL, "a kernel gave up on a bounded wait (device status word " + std::to_string(word) + ")");
    throw Error(ERR_INTERNAL, "a kernel reported device status word " + std::to_string(word));
  }
}

namespace {

// Kernel arguments of one item with device-resident operands. Orientation:
// the kernels see A' and B', and the swap exchanges the operands.
dev::GemmArgs build_args(Product& pr, Executor& ex, Scalar alpha, Scalar beta, bool c_read, const char* a_dev,
                         const char* b_dev, const char* c_dev, char* d_dev) {
  dev::GemmArgs g{};
  g.s = pr.scatters(ex.device, ex.stream);
  g.A = pr.view.swapped ? b_dev : a_dev;
  g.B = pr.view.swapped ? a_dev : b_dev;
  g.C = c_dev;
  g.D = d_dev;
  g.M = pr.view.M;
  g.N = pr.view.N;
  g.K = pr.view.K;
  g.H = pr.view.H;
  const bool cplx = dtype_complex(pr.problem.dtype);
  g.conj_a = cplx && pr.view.conj_a;
  g.conj_b = cplx && pr.view.conj_b;
  g.a_kfast = pr.view.a_kfast;
  g.b_kfast = pr.view.b_kfast;
  g.d_mfast = pr.view.d_mfast;
  g.e = make_epilogue(pr, alpha, beta, c_read);
  g.status = ex.status;
  return g;
}

// Events for the autotuner's measurements.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    check_cuda(cudaEventCreate(&a), "cudaEventCreate");
    check_cuda(cudaEventCreate(&b), "cudaEventCreate");
  }
  ~EventPair() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// Profiling is suspended while the autotuner measures (its runs are not the
// caller's work).
struct ProfileOff {
  Executor& ex;
  bool prev;
  explicit ProfileOff(Executor& e) : ex(e), prev(e.profile) { ex.profile = false; }
  ~ProfileOff() { ex.profile = prev; }
};

// Milliseconds of `fn`'s work on the executor's stream (the stream drains).
template <class F>
double time_on_stream(Executor& ex, EventPair& ev, F&& fn) {
  check_cuda(cudaEventRecord(ev.a, ex.stream), "cudaEventRecord");
  fn();
  check_cuda(cudaEventRecord(ev.b, ex.stream), "cudaEventRecord");
  drain(ex);
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, ev.a, ev.b), "cudaEventElapsedTime");
  return ms;
}

// Repetitions of a measurement by the duration of its first run: short runs
// are repeated more, since their times scatter more.
int tune_reps(double first_ms) { return first_ms < 0.05 ? 10 : first_ms < 1.0 ? 5 : first_ms < 20.0 ? 3 : 1; }

// Times every plain candidate of the item (minimum over repetitions after one
// warm-up run) and returns the fastest; the model's choice is kept unless a
// candidate is at least 3 % faster. Each run writes D; when the call reads D
// (in-place accumulation) `d_span` is saved to `snapshot` first and restored
// before every run and at the end, so the caller's execution afterwards sees
// the original D.
TuneEntry autotune_plain(Product& pr, Executor& ex, const dev::GemmArgs& g, char* scratch, size_t scratch_bytes,
                         char* d_span, char* snapshot, size_t span_bytes) {
  NvtxRange range("tprims.autotune");
  ProfileOff off(ex);
  const auto restore = [&] {
    if (snapshot)
      check_cuda(cudaMemcpyAsync(d_span, snapshot, span_bytes, cudaMemcpyDeviceToDevice, ex.stream),
                 "autotune restore of D");
  };
  if (snapshot)
    check_cuda(cudaMemcpyAsync(snapshot, d_span, span_bytes, cudaMemcpyDeviceToDevice, ex.stream),
               "autotune snapshot of D");
  EventPair ev;
  const std::vector<PlainChoice> cands =
      plain_candidates((int)pr.problem.dtype, pr.view.M, pr.view.N, pr.view.K, pr.view.H, ex.num_sms);
  TuneEntry best;
  best.ms = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    const PlainChoice& c = cands[i];
    if (plain_scratch(c, pr) > scratch_bytes) continue;
    double t = 0;
    try {
      const auto run = [&] { launch_plain(pr, ex, g, c, scratch, scratch_bytes); };
      restore();
      const double first = time_on_stream(ex, ev, run);
      t = first;
      const int reps = tune_reps(first);
      for (int r = 0; r < reps; ++r) {
        restore();
        t = std::min(t, time_on_stream(ex, ev, run));
      }
    } catch (const Error& e) {
      if (e.status != ERR_INTERNAL) throw;
      continue;  // a configuration that cannot launch on this device
    }
    ++best.tried;
    if (best.tried == 1 || t < best.ms * 0.97) {
      best.ms = t;
      best.choice = c;
    }
  }
  restore();
  if (best.tried == 0) throw Error(ERR_INTERNAL, "autotuner: no candidate configuration could be launched");
  best.tuned = true;
  return best;
}

int dt_code(const Product& pr) { return (int)pr.problem.dtype; }

// ---- streamed host execution
//
// With A, B and D in host memory, a synchronous call spends most of its time
// on the host link: every operand is copied in, the kernels run, D is copied
// out. Split along the outermost column axis of the oriented product (the
// last folded axis of N'), chunk c of the output needs all of A' but only
// chunk c of B' (and writes chunk c of D), so the copy of B' chunk c + 1, the
// kernels of chunk c and the copy out of chunk c - 1 run at once on three
// streams. A' is copied and (for the split schemes) packed once.

// One copy of a chunk region: `rows` rows of `width` bytes, `pitch` bytes
// apart, starting `off` bytes from the operand's origin.
struct ChunkCopy {
  int64_t off;
  size_t width, rows, pitch;
};

// The copies that move exactly the elements of an operand whose chunk-axis
// index lies in [lo, hi). `axes` are the operand's other axes as (extent,
// stride); those with a stride below `sc` must fit inside one chunk-axis
// step, those above must each span the whole block below them (a nested
// layout), and every stride must be positive. The smallest outer axis gives
// the rows of one pitched copy, further outer axes are looped (at most 4096
// copies).
bool chunk_copies(const std::vector<std::pair<int64_t, int64_t>>& axes, int64_t sc, int64_t ec, int64_t lo,
                  int64_t hi, int64_t elem, std::vector<ChunkCopy>& out) {
  if (sc <= 0 || lo >= hi) return false;
  int64_t inner_max = 0;
  std::vector<std::pair<int64_t, int64_t>> outer;  // (stride, extent)
  for (const auto& a : axes) {
    if (a.first <= 1 || a.second == 0) continue;
    if (a.second < 0 || a.second == sc) return false;
    if (a.second < sc)
      inner_max += (a.first - 1) * a.second;
    else
      outer.push_back({a.second, a.first});
  }
  if (inner_max >= sc) return false;
  std::sort(outer.begin(), outer.end());
  int64_t reach = (ec - 1) * sc + inner_max;  // last offset of the block below the next outer axis
  for (const auto& o : outer) {
    if (o.first <= reach) return false;
    reach += (o.second - 1) * o.first;
  }
  const int64_t seg0 = lo * sc, seg_len = (hi - 1) * sc + inner_max + 1 - seg0;
  int64_t combos = 1;
  for (size_t i = 1; i < outer.size(); ++i) combos *= outer[i].second;
  if (combos > 4096) return false;
  for (int64_t c = 0; c < combos; ++c) {
    int64_t base = 0, rem = c;
    for (size_t i = 1; i < outer.size(); ++i) {
      base += (rem % outer[i].second) * outer[i].first;
      rem /= outer[i].second;
    }
    ChunkCopy cc;
    cc.off = (base + seg0) * elem;
    cc.width = (size_t)(seg_len * elem);
    cc.rows = outer.empty() ? 1 : (size_t)outer[0].second;
    cc.pitch = outer.empty() ? cc.width : (size_t)(outer[0].first * elem);
    out.push_back(cc);
  }
  return true;
}

// Runs the item streamed when it qualifies (see above): returns false, with
// nothing enqueued, when it does not.
bool enqueue_streamed(Product& pr, Executor& ex, Scalar alpha, const Item& it) {
  const Problem& p = pr.problem;
  const OrientedView& v = pr.view;
  const PlanStats& stt = pr.packed.stats;
  const int64_t elem = (int64_t)dtype_size(p.dtype);
  const int sx = v.swapped ? SA : SB;  // the operand that plays B'
  const int sy = v.swapped ? SB : SA;  // the operand that plays A'
  if (v.H > 65535) return false;
  const auto stride_in = [](const Axis& a, int slot) {
    return slot == SA ? a.sa : slot == SB ? a.sb : slot == SC ? a.sc : a.sd;
  };
  // One side of the product is chunked along its outermost axis (of D's N
  // columns, or of its M rows), the other operand is copied whole first; the
  // larger operand is the one chunked, so the kernels start after the smaller
  // copy and the copies out of D start early (C2: B' 64 MB whole, then A'
  // 128 MB in chunks of its outermost row axis).
  struct Side {
    bool rows = false;  // chunks of M (A' rows) instead of N (B' columns)
    const Axis* ca = nullptr;
    int64_t E = 0, inner = 0;
    int slot = SB;  // the chunked operand
    std::vector<int64_t> lo, hi;
    std::vector<std::vector<ChunkCopy>> xcp, dcp;
  };
  const auto plan_side = [&](bool rows, Side& sd) {
    const std::vector<Axis>& ax = rows ? (v.swapped ? stt.n_axes : stt.m_axes) : (v.swapped ? stt.m_axes : stt.n_axes);
    if (ax.empty()) return false;
    sd.rows = rows;
    sd.ca = &ax.back();
    sd.E = sd.ca->extent;
    sd.slot = rows ? sy : sx;
    if (sd.E < 2) return false;
    // Chunks that halve in size (E/2, E/4, ... down to about E/16, the rest
    // last): the call ends with the kernels and the copy out of the last
    // chunk only, so a small last chunk shortens that tail while the large
    // first ones keep the kernels efficient. Every chunk keeps at least 256
    // rows or columns.
    sd.inner = (rows ? v.M : v.N) / sd.E;
    std::vector<int64_t> bounds{0};
    while (bounds.back() < sd.E) {
      const int64_t left = sd.E - bounds.back();
      int64_t take = left / 2;
      if (take * 16 < sd.E || take * sd.inner < 256 || (left - take) * sd.inner < 256) take = left;
      bounds.push_back(bounds.back() + take);
    }
    const int nc = (int)bounds.size() - 1;
    if (nc < 2 || nc > 8) return false;
    const Axis* ca = sd.ca;
    const auto others = [&](int slot) {
      std::vector<std::pair<int64_t, int64_t>> out;
      for (const std::vector<Axis>* role : {&stt.m_axes, &stt.n_axes, &stt.k_axes, &stt.h_axes})
        for (const Axis& a : *role)
          if (&a != ca) out.push_back({a.extent, stride_in(a, slot)});
      return out;
    };
    sd.xcp.assign(nc, {});
    sd.dcp.assign(nc, {});
    sd.lo.assign(nc, 0);
    sd.hi.assign(nc, 0);
    for (int c = 0; c < nc; ++c) {
      sd.lo[c] = bounds[c];
      sd.hi[c] = bounds[c + 1];
      if (!chunk_copies(others(sd.slot), stride_in(*ca, sd.slot), sd.E, sd.lo[c], sd.hi[c], elem, sd.xcp[c]) ||
          !chunk_copies(others(SD), stride_in(*ca, SD), sd.E, sd.lo[c], sd.hi[c], elem, sd.dcp[c]))
        return false;
    }
    return true;
  };
  int64_t span_lo = 0;
  size_t bytes_x = 0, bytes_y = 0;
  span_bytes(p, sx, &span_lo, &bytes_x);
  span_bytes(p, sy, &span_lo, &bytes_y);
  // Kernel configuration per chunk (the plain path: one launch each, no
  // split-K); a side whose chunks would need split-K or the tiny-batch kernel
  // is not taken.
  const bool split = pr.scheme == Scheme::Bf16x3 || pr.scheme == Scheme::Bf16x6;
  if (!split && pr.scheme != Scheme::Plain) return false;
  std::vector<PlainChoice> pcs;
  size_t scratch = 0;
  const auto configure = [&](const Side& sd) {
    const int nc = (int)sd.lo.size();
    const auto cm = [&](int c) { return sd.rows ? (sd.hi[c] - sd.lo[c]) * sd.inner : v.M; };
    const auto cn = [&](int c) { return sd.rows ? v.N : (sd.hi[c] - sd.lo[c]) * sd.inner; };
    pcs.assign(nc, PlainChoice{});
    scratch = 0;
    if (split) {
      // The whole operand's planes (packed once), then room for the largest
      // chunk's planes.
      const dev::SplitLayout L = dev::split_layout((int)pr.scheme, v.M, v.N, v.K, v.H);
      int64_t mmax = 0, nmax = 0;
      for (int c = 0; c < nc; ++c) {
        mmax = std::max(mmax, cm(c));
        nmax = std::max(nmax, cn(c));
      }
      const dev::SplitLayout Lc = dev::split_layout((int)pr.scheme, mmax, nmax, v.K, v.H);
      const size_t whole_planes = sd.rows ? (size_t)L.planes * L.H * L.n_pad * L.k_pad * 2
                                          : (size_t)L.planes * L.H * L.m_pad * L.k_pad * 2;
      const size_t chunk_planes = sd.rows ? (size_t)Lc.planes * Lc.H * Lc.m_pad * Lc.k_pad * 2
                                          : (size_t)Lc.planes * Lc.H * Lc.n_pad * Lc.k_pad * 2;
      scratch = align_up(whole_planes, 256) + align_up(chunk_planes, 256) + dev::split_tail_bytes(L, ex.num_sms) + 1024;
      return true;
    }
    for (int c = 0; c < nc; ++c) {
      const int64_t mc = cm(c), ncols = cn(c);
      PlainChoice& pc = pcs[c];
      if (dev::use_tiny_batched(mc, ncols, v.K, v.H)) return false;
      dev::choose_plain_launch((int)p.dtype, pr.kernel_pin, mc, ncols, v.K, v.H, ex.num_sms, &pc.kernel, &pc.splits,
                               &pc.chunk);
      if (pc.splits > 1) return false;
      if (dev::is_packed_kernel(pc.kernel))
        scratch = std::max(scratch,
                           dev::packed_workspace_bytes(dev::packed_layout(pc.kernel, mc, ncols, v.K, v.H)) + 512);
    }
    return true;
  };
  Side sd;
  const bool prefer_rows = bytes_y > bytes_x;
  if (!(plan_side(prefer_rows, sd) && configure(sd)) && !(plan_side(!prefer_rows, sd) && configure(sd)))
    return false;
  const bool rows = sd.rows;
  const int nchunks = (int)sd.lo.size();
  const std::vector<int64_t>& lo = sd.lo;
  const std::vector<int64_t>& hi = sd.hi;
  const int64_t inner = sd.inner;
  const int chunked = sd.slot, whole = rows ? sx : sy;
  // Rows and columns of chunk c.
  const auto chunk_m = [&](int c) { return rows ? (hi[c] - lo[c]) * inner : v.M; };
  const auto chunk_n = [&](int c) { return rows ? v.N : (hi[c] - lo[c]) * inner; };

  // Workspace: the staged spans of A, B and D, then the kernels' scratch.
  Staged st[4];
  const void* origins[4] = {it.a, it.b, nullptr, it.d};
  size_t total = 0;
  for (int s : {SA, SB, SD}) {
    st[s].host = origins[s];
    st[s].staged = true;
    span_bytes(p, s, &st[s].lo_bytes, &st[s].bytes);
    total = align_up(total, 256) + st[s].bytes;
  }
  injected_failure_check(ex);
  char* ws = static_cast<char*>(ex.workspace(align_up(total, 256) + align_up(scratch, 256) + 1024));
  size_t off = 0;
  for (int s : {SA, SB, SD}) {
    off = align_up(off, 256);
    st[s].buf = ws + off;
    st[s].dev_origin = st[s].buf - st[s].lo_bytes;
    off += st[s].bytes;
  }
  char* scratch_ptr = reinterpret_cast<char*>(align_up((uintptr_t)(ws + off), 256));
  if (!ex.copy_in) check_cuda(cudaStreamCreateWithFlags(&ex.copy_in, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!ex.copy_out) check_cuda(cudaStreamCreateWithFlags(&ex.copy_out, cudaStreamNonBlocking), "cudaStreamCreate");
  while ((int)ex.stream_events.size() < 2 * nchunks + 3) {
    cudaEvent_t e;
    check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    ex.stream_events.push_back(e);
  }
  cudaEvent_t* ev = ex.stream_events.data();
  // The copy streams start behind everything already on the executor's stream.
  check_cuda(cudaEventRecord(ev[2 * nchunks + 2], ex.stream), "cudaEventRecord");
  check_cuda(cudaStreamWaitEvent(ex.copy_in, ev[2 * nchunks + 2], 0), "cudaStreamWaitEvent");
  check_cuda(cudaStreamWaitEvent(ex.copy_out, ev[2 * nchunks + 2], 0), "cudaStreamWaitEvent");

  // In: the whole operand, then the chunked one chunk by chunk.
  check_cuda(cudaMemcpyAsync(st[whole].buf, static_cast<const char*>(st[whole].host) + st[whole].lo_bytes,
                             st[whole].bytes, cudaMemcpyHostToDevice, ex.copy_in),
             "host-to-device copy");
  check_cuda(cudaEventRecord(ev[0], ex.copy_in), "cudaEventRecord");
  for (int c = 0; c < nchunks; ++c) {
    for (const ChunkCopy& cc : sd.xcp[c])
      check_cuda(cudaMemcpy2DAsync(st[chunked].dev_origin + cc.off, cc.pitch,
                                   static_cast<const char*>(st[chunked].host) + cc.off, cc.pitch, cc.width, cc.rows,
                                   cudaMemcpyHostToDevice, ex.copy_in),
                 "host-to-device chunk copy");
    check_cuda(cudaEventRecord(ev[1 + c], ex.copy_in), "cudaEventRecord");
  }

  // Kernels, chunk by chunk, on the executor's stream. The split schemes
  // pack the whole operand's planes once and each chunk's planes before its
  // GEMM.
  check_cuda(cudaStreamWaitEvent(ex.stream, ev[0], 0), "cudaStreamWaitEvent");
  const dev::GemmArgs g = build_args(pr, ex, alpha, Scalar{}, false, st[SA].dev_origin, st[SB].dev_origin, nullptr,
                                     st[SD].dev_origin);
  dev::SplitLayout L{};
  char* wp = scratch_ptr;  // the whole operand's planes
  char* cp = scratch_ptr;  // the current chunk's planes
  if (split) {
    L = dev::split_layout((int)pr.scheme, v.M, v.N, v.K, v.H);
    Timed t(ex, "split_pack");
    check_cuda(dev::launch_split_pack_f32(g, rows ? 1 : 0, L, wp, ex.stream), "split pack of the whole operand");
    cp = wp + align_up(rows ? (size_t)L.planes * L.H * L.n_pad * L.k_pad * 2 : (size_t)L.planes * L.H * L.m_pad * L.k_pad * 2,
                       256);
  }
  for (int c = 0; c < nchunks; ++c) {
    check_cuda(cudaStreamWaitEvent(ex.stream, ev[1 + c], 0), "cudaStreamWaitEvent");
    dev::GemmArgs gc = g;
    const int64_t x0 = lo[c] * inner;
    if (rows) {
      gc.M = chunk_m(c);
      gc.s.a_m += x0;
      gc.s.c_m += x0;
      gc.s.d_m += x0;
      gc.s.blk_a_m = (x0 % dev::SCATTER_BLOCK == 0) ? g.s.blk_a_m + x0 / dev::SCATTER_BLOCK : nullptr;
    } else {
      gc.N = chunk_n(c);
      gc.s.b_n += x0;
      gc.s.c_n += x0;
      gc.s.d_n += x0;
      gc.s.blk_b_n = (x0 % dev::SCATTER_BLOCK == 0) ? g.s.blk_b_n + x0 / dev::SCATTER_BLOCK : nullptr;
    }
    if (split) {
      const dev::SplitLayout Lc = dev::split_layout((int)pr.scheme, gc.M, gc.N, v.K, v.H);
      const size_t cbytes = rows ? (size_t)Lc.planes * Lc.H * Lc.m_pad * Lc.k_pad * 2
                                 : (size_t)Lc.planes * Lc.H * Lc.n_pad * Lc.k_pad * 2;
      char* tail = reinterpret_cast<char*>(align_up((uintptr_t)(cp + cbytes), 256));
      {
        Timed t(ex, "split_pack");
        check_cuda(dev::launch_split_pack_f32(gc, rows ? 0 : 1, Lc, cp, ex.stream), "split pack of a chunk");
      }
      Timed t(ex, pr.scheme == Scheme::Bf16x3 ? "tc_bf16x3_gemm" : "tc_bf16x6_gemm");
      check_cuda(dev::launch_tc_bf16_gemm(gc, Lc, rows ? cp : wp, rows ? wp : cp, (int)pr.scheme, ex.stream, tail),
                 "tcgen05 contraction launch");
    } else {
      launch_plain(pr, ex, gc, pcs[c], scratch_ptr, scratch);
    }
    check_cuda(cudaEventRecord(ev[1 + nchunks + c], ex.stream), "cudaEventRecord");
  }
  if (!split) {
    std::lock_guard<std::mutex> lk(pr.mu);
    pr.last = pcs[0];
    pr.last_source = (pr.kernel_pin || pr.split_pin) ? ChoiceSource::Pinned : ChoiceSource::Model;
    pr.executed = true;
  }

  // Out: D chunk by chunk as each is written; the executor's stream then
  // waits for the last copy, so draining it covers the whole call.
  for (int c = 0; c < nchunks; ++c) {
    check_cuda(cudaStreamWaitEvent(ex.copy_out, ev[1 + nchunks + c], 0), "cudaStreamWaitEvent");
    for (const ChunkCopy& cc : sd.dcp[c])
      check_cuda(cudaMemcpy2DAsync(const_cast<char*>(static_cast<const char*>(st[SD].host)) + cc.off, cc.pitch,
                                   st[SD].dev_origin + cc.off, cc.pitch, cc.width, cc.rows, cudaMemcpyDeviceToHost,
                                   ex.copy_out),
                 "device-to-host chunk copy");
  }
  check_cuda(cudaEventRecord(ev[2 * nchunks + 1], ex.copy_out), "cudaEventRecord");
  check_cuda(cudaStreamWaitEvent(ex.stream, ev[2 * nchunks + 1], 0), "cudaStreamWaitEvent");
  return true;
}

// Enqueue one item; returns whether host copies were involved (the caller
// must then drain the stream before returning to the host).
bool enqueue_item(Product& pr, Executor& ex, Scalar alpha, Scalar beta, const Item& it) {
  const Problem& p = pr.problem;
  if (p.out_empty) return false;
  const bool c_read = it.c != nullptr && !beta.is_zero();
  const bool output_only = p.k_empty || alpha.is_zero();
  if (output_only && c_read && it.c == it.d && p.c_matches_d && beta.is_one() && !pr.view.conj_c &&
      !pr.view.conj_d)
    return false;  // in-place identity update: nothing changes (plan/mod.rs:515-519)

  // Which operands are read / written, and where they live.
  const bool need_ab = !output_only;
  const bool in_place = c_read && it.c == it.d;
  Staged st[4];
  const void* origins[4] = {it.a, it.b, it.c, it.d};
  bool use[4] = {need_ab, need_ab, c_read && !in_place, true};
  size_t total = 0;
  for (int s = 0; s < 4; ++s) {
    if (!use[s] || p.spans[s].empty) continue;
    st[s].host = origins[s];
    if (classify(origins[s], ex.device) == Where::Device) {
      st[s].dev_origin = const_cast<char*>(static_cast<const char*>(origins[s]));
      continue;
    }
    st[s].staged = true;
    span_bytes(p, s, &st[s].lo_bytes, &st[s].bytes);
    total = align_up(total, 256) + st[s].bytes;
  }
  // Large contractions of host operands that write all of D and read no C
  // run streamed (copies in and out overlap the kernels chunk by chunk).
  if (ex.streaming && need_ab && !c_read && st[SA].staged && st[SB].staged && st[SD].staged && !pr.autotune &&
      pr.split_pin <= 1 && fully_written(pr) &&
      st[SA].bytes + st[SB].bytes + st[SD].bytes >= (size_t(32) << 20) && enqueue_streamed(pr, ex, alpha, it))
    return true;
  // The plain path's configuration: the pins, else (autotune) the executor's
  // tuning cache or a measurement now, else the model.
  PlainChoice pc{};
  ChoiceSource src = ChoiceSource::Model;
  bool tune = false;
  std::string key;
  if (pr.scheme == Scheme::Plain && !output_only) {
    pc = model_choice(pr, ex.num_sms);
    if (pr.kernel_pin || pr.split_pin) {
      src = ChoiceSource::Pinned;
    } else if (pr.autotune) {
      key = tune_key(pr, c_read);
      const auto hit = ex.tune.find(key);
      if (hit != ex.tune.end()) {
        // A loaded entry that does not fit this product (a stale or edited
        // file: another family's kernel, or K chunks that would skip part of
        // K) keeps the model's choice.
        if (choice_fits(hit->second.choice, pr)) {
          pc = hit->second.choice;
          src = hit->second.tuned ? ChoiceSource::Cached : ChoiceSource::Model;
        }
      } else {
        tune = true;
      }
    }
  }
  size_t scratch = output_only ? 0 : scheme_scratch(pr, pc, ex.num_sms);
  int64_t d_lo = 0;
  size_t d_bytes = 0, snap = 0;
  if (tune) {
    // Room for the largest candidate, and for a copy of D when the call reads it.
    size_t tune_scratch = scratch;
    for (const auto& c : plain_candidates(dt_code(pr), pr.view.M, pr.view.N, pr.view.K, pr.view.H, ex.num_sms))
      tune_scratch = std::max(tune_scratch, plain_scratch(c, pr));
    if (in_place) {
      span_bytes(p, SD, &d_lo, &d_bytes);
      snap = align_up(d_bytes, 256);
    }
    const size_t limit = std::min<size_t>(ex.ws_limit, size_t(4) << 30);
    if (align_up(total, 256) + tune_scratch + snap + 1024 > limit) {
      // Too large to measure within the workspace cap: keep the model's choice.
      tune = false;
      snap = 0;
      TuneEntry e;
      e.choice = pc;
      e.tuned = false;
      ex.tune[key] = e;
    } else {
      scratch = tune_scratch;
    }
  }
  char* ws = static_cast<char*>(ex.workspace(align_up(total, 256) + align_up(scratch, 256) + snap + 1024));
  size_t off = 0;
  for (int s = 0; s < 4; ++s) {
    if (!st[s].staged) continue;
    off = align_up(off, 256);
    st[s].buf = ws + off;
    st[s].dev_origin = st[s].buf - st[s].lo_bytes;
    off += st[s].bytes;
    const bool copy_in = s != SD || c_read || !fully_written(pr);
    if (copy_in)
      check_cuda(cudaMemcpyAsync(st[s].buf, static_cast<const char*>(st[s].host) + st[s].lo_bytes, st[s].bytes,
                                 cudaMemcpyHostToDevice, ex.stream),
                 "host-to-device copy");
  }
  char* scratch_ptr = ws + align_up(off, 256);
  char* snap_ptr = snap ? scratch_ptr + align_up(scratch, 256) : nullptr;

  const dev::GemmArgs g = build_args(pr, ex, alpha, beta, c_read, st[SA].dev_origin, st[SB].dev_origin,
                                     c_read ? (in_place ? st[SD].dev_origin : st[SC].dev_origin) : nullptr,
                                     st[SD].dev_origin);
  if (tune) {
    const TuneEntry e = autotune_plain(pr, ex, g, scratch_ptr, scratch, snap ? st[SD].dev_origin + d_lo : nullptr,
                                       snap_ptr, d_bytes);
    ex.tune[key] = e;
    pc = e.choice;
    src = ChoiceSource::Autotuned;
  }
  if (pr.scheme == Scheme::Plain && !output_only) {
    std::lock_guard<std::mutex> lk(pr.mu);
    pr.last = pc;
    pr.last_source = src;
    pr.executed = true;
  }
  launch_contraction(pr, ex, g, output_only, pc, scratch_ptr, scratch);

  if (st[SD].staged)
    check_cuda(cudaMemcpyAsync(const_cast<void*>(static_cast<const void*>(static_cast<const char*>(st[SD].host) +
                                                                          st[SD].lo_bytes)),
                               st[SD].buf, st[SD].bytes, cudaMemcpyDeviceToHost, ex.stream),
               "device-to-host copy");
  for (auto& s : st)
    if (s.staged) return true;
  return false;
}

}  // namespace

void execute_item(Product& pr, Executor& ex, Scalar alpha, Scalar beta, const Item& it) {
  NvtxRange range("tprims.execute_product");
  std::lock_guard<std::mutex> lk(ex.mu);
  DeviceGuard g(ex.device);
  const bool staged = enqueue_item(pr, ex, alpha, beta, it);
  if (ex.sync || staged) finish(ex);
}

namespace {

// Whether an item can join a grouped launch: plain scheme, a real contraction
// (not the output-only pass), every operand already in device memory.
bool groupable(Product& pr, Executor& ex, Scalar alpha, Scalar beta, const Item& it) {
  const Problem& p = pr.problem;
  if (pr.scheme != Scheme::Plain || p.out_empty || p.k_empty || alpha.is_zero()) return false;
  if (pr.view.H > 65535) return false;
  if (!pr.kernel_pin && dev::use_tiny_batched(pr.view.M, pr.view.N, pr.view.K, pr.view.H)) return false;
  if (pr.split_pin > 1) return false;  // the grouped kernel does not split K
  const bool c_read = it.c != nullptr && !beta.is_zero();
  const void* ptrs[4] = {it.a, it.b, c_read ? it.c : nullptr, it.d};
  for (const void* q : ptrs)
    if (q && classify(q, ex.device) != Where::Device) return false;
  return true;
}

uint64_t mix(uint64_t h, uint64_t v) {
  h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h;
}

// One grouped submission: descriptors for every groupable item, tiles in
// decreasing-K order, one persistent launch per kernel family; captured in a
// CUDA graph cached by the item list (plans, pointers and scalars), so a
// repeated list replays with one graph launch.
uint64_t list_key(int n, Product* const* plans, const Scalar* alpha, const Scalar* beta, const Item* items) {
  uint64_t key = 1469598103934665603ull;
  for (int i = 0; i < n; ++i) {
    const uint64_t f[7] = {plans[i]->uid,
                           (uint64_t)(uintptr_t)items[i].a,
                           (uint64_t)(uintptr_t)items[i].b,
                           (uint64_t)(uintptr_t)items[i].c,
                           (uint64_t)(uintptr_t)items[i].d,
                           (uint64_t)plans[i]->kernel_pin | ((uint64_t)plans[i]->autotune << 32),
                           ((uint64_t)plans[i]->scheme << 8) | (uint64_t)plans[i]->ozaki_slices};
    for (uint64_t v : f) key = mix(key, v);
    double sc[4] = {alpha[i].re, alpha[i].im, beta[i].re, beta[i].im};
    uint64_t bits[4];
    std::memcpy(bits, sc, sizeof(bits));
    for (uint64_t v : bits) key = mix(key, v);
  }
  return mix(key, (uint64_t)n);
}

// The device side of one grouped submission: descriptors of the items `idx`
// (each with its tile family under the list's tile `policy`), tiles in
// decreasing-K order within a family, one persistent launch per family.
struct GroupSet {
  void* buf = nullptr;  // descriptors, tile starts, claim counters
  std::vector<int> family;
  std::vector<size_t> item0, start0, count;
  char* counters = nullptr;
  char* starts = nullptr;
};

GroupSet build_group_set(Executor& ex, const std::vector<int>& idx, int policy, Product* const* plans,
                         const Scalar* alpha, const Scalar* beta, const Item* items) {
  std::map<int, std::vector<int>> by_family;
  for (int i : idx) by_family[grouped_family(*plans[i], policy)].push_back(i);
  // Families in decreasing order of work (padded tile volume): the first one
  // runs on the submitting stream and the others fill its tail.
  std::vector<std::pair<int, std::vector<int>>> fam(by_family.begin(), by_family.end());
  auto work = [&](const std::pair<int, std::vector<int>>& f) {
    int bm = 0, bn = 0;
    dev::plain_tile_shape(f.first, &bm, &bn);
    double w = 0;
    for (int i : f.second) {
      const Product& pr = *plans[i];
      w += (double)((pr.view.M + bm - 1) / bm * bm) * (double)((pr.view.N + bn - 1) / bn * bn) *
           (double)pr.view.K * (double)pr.view.H;
    }
    return w;
  };
  std::stable_sort(fam.begin(), fam.end(), [&](const auto& a, const auto& b) { return work(a) > work(b); });
  GroupSet gs;
  std::vector<dev::GroupItem> host_items;
  std::vector<int64_t> host_starts;
  for (auto& kv : fam) {
    std::vector<int>& list = kv.second;
    std::stable_sort(list.begin(), list.end(),
                     [&](int a, int b) { return plans[a]->view.K > plans[b]->view.K; });
    int bm = 0, bn = 0;
    dev::plain_tile_shape(kv.first, &bm, &bn);
    gs.family.push_back(kv.first);
    gs.item0.push_back(host_items.size());
    gs.start0.push_back(host_starts.size());
    gs.count.push_back(list.size());
    int64_t acc = 0;
    for (int i : list) {
      Product& pr = *plans[i];
      const bool c_read = items[i].c != nullptr && !beta[i].is_zero();
      dev::GroupItem gi{};
      gi.g = build_args(pr, ex, alpha[i], beta[i], c_read, static_cast<const char*>(items[i].a),
                        static_cast<const char*>(items[i].b),
                        c_read ? static_cast<const char*>(items[i].c) : nullptr, static_cast<char*>(items[i].d));
      gi.tiles_m = (pr.view.M + bm - 1) / bm;
      gi.tiles_n = (pr.view.N + bn - 1) / bn;
      host_items.push_back(gi);
      host_starts.push_back(acc);
      acc += gi.tiles_m * gi.tiles_n * pr.view.H;
    }
    host_starts.push_back(acc);
  }
  const size_t items_bytes = host_items.size() * sizeof(dev::GroupItem);
  const size_t starts_bytes = host_starts.size() * sizeof(int64_t);
  check_cuda(device_alloc(&gs.buf, align_up(items_bytes, 256) + align_up(starts_bytes, 256) + 256 * (gs.family.size() + 1)),
             "cudaMalloc(groups)");
  char* base = static_cast<char*>(gs.buf);
  // Stream-ordered copies, complete before any capture (see Product::scatters).
  gs.starts = base + align_up(items_bytes, 256);
  cudaError_t up = cudaMemcpyAsync(base, host_items.data(), items_bytes, cudaMemcpyHostToDevice, ex.stream);
  if (up == cudaSuccess)
    up = cudaMemcpyAsync(gs.starts, host_starts.data(), starts_bytes, cudaMemcpyHostToDevice, ex.stream);
  if (up == cudaSuccess) up = cudaStreamSynchronize(ex.stream);
  if (up != cudaSuccess) {
    cudaFree(gs.buf);
    check_cuda(up, "group descriptor upload");
  }
  gs.counters = gs.starts + align_up(starts_bytes, 256);
  for (int f : gs.family) {
    const cudaError_t e = dev::prepare_grouped(f);
    if (e != cudaSuccess) {
      cudaFree(gs.buf);
      check_cuda(e, "grouped kernel load");
    }
  }
  return gs;
}

// One persistent launch per family. With several families the first (the
// one with the most work, see build_group_set) runs on `st` and
// each other one on a side stream forked from `st` before it and joined back
// after; the persistent grids of the later families take SMs as the earlier
// ones' CTAs run out of tiles, instead of starting after their last tile.
cudaError_t launch_group_set(Executor& ex, const GroupSet& gs, cudaStream_t st) {
  const size_t nf = gs.family.size();
  auto launch = [&](size_t l, cudaStream_t s) {
    return dev::launch_grouped(gs.family[l], reinterpret_cast<dev::GroupItem*>(gs.buf) + gs.item0[l],
                               reinterpret_cast<int64_t*>(gs.starts) + gs.start0[l], (int)gs.count[l],
                               reinterpret_cast<unsigned long long*>(gs.counters + 256 * l), ex.status, ex.num_sms,
                               s);
  };
  if (nf <= 1) {
    cudaError_t e = cudaSuccess;
    for (size_t l = 0; l < nf && e == cudaSuccess; ++l) e = launch(l, st);
    return e;
  }
  ensure_side(ex, nf - 1, nf);
  cudaError_t e = cudaEventRecord(ex.family_events[0], st);
  for (size_t l = 1; l < nf && e == cudaSuccess; ++l) e = cudaStreamWaitEvent(ex.family_streams[l - 1], ex.family_events[0], 0);
  if (e == cudaSuccess) e = launch(0, st);
  for (size_t l = 1; l < nf && e == cudaSuccess; ++l) {
    e = launch(l, ex.family_streams[l - 1]);
    if (e == cudaSuccess) e = cudaEventRecord(ex.family_events[l], ex.family_streams[l - 1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ex.family_events[l], 0);
  }
  return e;
}

// A stable text key of a grouped list for the autotuner: the multiset of its
// items' tuning keys (FNV-1a over the sorted keys).
std::string list_signature(const std::vector<int>& idx, Product* const* plans, const Scalar* beta,
                           const Item* items) {
  std::vector<std::string> keys;
  keys.reserve(idx.size());
  for (int i : idx) keys.push_back(tune_key(*plans[i], items[i].c != nullptr && !beta[i].is_zero()));
  std::sort(keys.begin(), keys.end());
  uint64_t h = 1469598103934665603ull;
  for (const auto& k : keys) {
    for (unsigned char ch : k) {
      h ^= ch;
      h *= 1099511628211ull;
    }
    h ^= '|';
    h *= 1099511628211ull;
  }
  char buf[64];
  std::snprintf(buf, sizeof(buf), "list-%016llx-n%zu", (unsigned long long)h, idx.size());
  return buf;
}

// The tile policy of a grouped list: from the executor's tuning cache, or
// measured now (every distinct policy run directly, minimum over repetitions
// after a warm-up; policy 0, the model, kept unless another is 3 % faster).
// A list whose items read their own D (in-place accumulation) cannot be run
// repeatedly and keeps the model.
int list_policy(Executor& ex, const std::vector<int>& idx, Product* const* plans, const Scalar* alpha,
                const Scalar* beta, const Item* items) {
  const std::string sig = list_signature(idx, plans, beta, items);
  const auto hit = ex.list_tune.find(sig);
  if (hit != ex.list_tune.end()) return hit->second.policy;
  TuneEntry best;
  for (int i : idx)
    if (items[i].c != nullptr && !beta[i].is_zero() && items[i].c == items[i].d) {
      best.tuned = false;
      ex.list_tune[sig] = best;
      return 0;
    }
  ProfileOff off(ex);
  EventPair ev;
  std::vector<std::vector<int>> seen;
  for (int policy = 0; policy < GROUP_POLICIES; ++policy) {
    std::vector<int> fam;
    for (int i : idx) fam.push_back(grouped_family(*plans[i], policy));
    if (std::find(seen.begin(), seen.end(), fam) != seen.end()) continue;
    seen.push_back(fam);
    GroupSet gs = build_group_set(ex, idx, policy, plans, alpha, beta, items);
    double t = 0;
    try {
      const auto run = [&] { check_cuda(launch_group_set(ex, gs, ex.stream), "grouped launch"); };
      const double first = time_on_stream(ex, ev, run);
      t = first;
      const int reps = tune_reps(first);
      for (int r = 0; r < reps; ++r) t = std::min(t, time_on_stream(ex, ev, run));
    } catch (...) {
      cudaFree(gs.buf);
      throw;
    }
    cudaFree(gs.buf);
    ++best.tried;
    if (best.tried == 1 || t < best.ms * 0.97) {
      best.ms = t;
      best.policy = policy;
    }
  }
  best.tuned = true;
  ex.list_tune[sig] = best;
  return best.policy;
}

// Builds, captures and caches the graph of the grouped items `idx`; the
// entry also remembers the items that run individually (`single`).
Executor::Graph& capture_grouped(Executor& ex, uint64_t key, const std::vector<int>& idx,
                                 const std::vector<int>& single, int policy, Product* const* plans,
                                 const Scalar* alpha, const Scalar* beta, const Item* items) {
  GroupSet gs = build_group_set(ex, idx, policy, plans, alpha, beta, items);
  Executor::Graph gr;
  gr.single = single;
  gr.buf = gs.buf;
  // Capture on a private non-blocking stream (a capture on a stream that
  // synchronises with the legacy stream would make other threads' legacy-stream
  // work fail meanwhile); the graph is launched on the executor's stream.
  if (!ex.capture_stream) {
    const cudaError_t e = cudaStreamCreateWithFlags(&ex.capture_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      cudaFree(gr.buf);
      check_cuda(e, "cudaStreamCreate(capture)");
    }
  }
  // Side streams and events for concurrent family launches exist before the
  // capture starts (nothing is created while it runs).
  try {
    ensure_side(ex, gs.family.size(), gs.family.size() + 1);
  } catch (...) {
    cudaFree(gr.buf);
    throw;
  }
  const cudaError_t begin = cudaStreamBeginCapture(ex.capture_stream, cudaStreamCaptureModeThreadLocal);
  if (begin != cudaSuccess) {
    cudaFree(gr.buf);
    check_cuda(begin, "cudaStreamBeginCapture");
  }
  const cudaError_t cap = launch_group_set(ex, gs, ex.capture_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t end = cudaStreamEndCapture(ex.capture_stream, &graph);
  if (cap != cudaSuccess || end != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaFree(gr.buf);
    check_cuda(cap != cudaSuccess ? cap : end, "grouped launch capture");
  }
  cudaError_t inst = cudaGraphInstantiate(&gr.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) {
    cudaFree(gr.buf);
    check_cuda(inst, "cudaGraphInstantiate");
  }
  gr.last_use = ++ex.graph_clock;
  // Bounded cache: evict the least recently used graph.
  if (ex.graphs.size() >= 16) {
    auto victim = ex.graphs.begin();
    for (auto it = ex.graphs.begin(); it != ex.graphs.end(); ++it)
      if (it->second.last_use < victim->second.last_use) victim = it;
    drain(ex);
    cudaGraphExecDestroy(victim->second.exec);
    cudaFree(victim->second.buf);
    ex.graphs.erase(victim);
  }
  return ex.graphs.emplace(key, gr).first->second;
}

}  // namespace

namespace {

// The body of execute_items under the caller's lock and device guard: the
// grouped graph and the individual items are enqueued; returns whether a
// host operand was staged (the caller must then drain before reusing the
// workspace).
bool enqueue_items(Executor& ex, int n, Product* const* plans, const Scalar* alpha, const Scalar* beta,
                   const Item* items) {
  const uint64_t key = ex.grouping ? list_key(n, plans, alpha, beta, items) : 0;
  auto hit = ex.grouping ? ex.graphs.find(key) : ex.graphs.end();
  Executor::Graph* gr = nullptr;
  std::vector<int> single;
  if (hit != ex.graphs.end()) {
    gr = &hit->second;
    single = gr->single;
  } else {
    std::vector<int> grouped;
    for (int i = 0; i < n; ++i)
      (ex.grouping && groupable(*plans[i], ex, alpha[i], beta[i], items[i]) ? grouped : single).push_back(i);
    if (grouped.size() < 2) {
      single.insert(single.end(), grouped.begin(), grouped.end());
      grouped.clear();
    } else {
      bool tuned = true;
      for (int i : grouped) tuned = tuned && plans[i]->autotune && !plans[i]->kernel_pin;
      const int policy = tuned ? list_policy(ex, grouped, plans, alpha, beta, items) : 0;
      gr = &capture_grouped(ex, key, grouped, single, policy, plans, alpha, beta, items);
    }
  }
  bool staged = false;
  if (gr) {
    injected_failure_check(ex);
    Timed t(ex, "grouped");
    gr->last_use = ++ex.graph_clock;
    check_cuda(cudaGraphLaunch(gr->exec, ex.stream), "cudaGraphLaunch");
  }
  for (size_t j = 0; j < single.size(); ++j) {
    const int i = single[j];
    staged |= enqueue_item(*plans[i], ex, alpha[i], beta[i], items[i]);
    // A staged item's workspace is reused by the next item: drain between.
    if (staged && j + 1 < single.size()) finish(ex);
  }
  return staged;
}

}  // namespace

void execute_items(Executor& ex, int n, Product* const* plans, const Scalar* alpha, const Scalar* beta,
                   const Item* items) {
  NvtxRange range("tprims.contract_batched");
  std::lock_guard<std::mutex> lk(ex.mu);
  DeviceGuard g(ex.device);
  const bool staged = enqueue_items(ex, n, plans, alpha, beta, items);
  if (ex.sync || staged) finish(ex);
}

std::vector<int> balance_parts(const std::vector<double>& costs, const std::vector<int>& homes,
                               const std::vector<int>& part_devices) {
  const size_t n = costs.size();
  if (homes.size() != n) throw Error(ERR_INVALID_ARGUMENT, "one home device per item");
  if (part_devices.empty() && n > 0) throw Error(ERR_INVALID_ARGUMENT, "no parts to balance over");
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return costs[a] > costs[b]; });
  std::vector<double> load(part_devices.size(), 0.0);
  std::vector<int> part(n, -1);
  for (size_t i : order) {
    int best = -1;
    for (size_t q = 0; q < part_devices.size(); ++q)
      if ((homes[i] < 0 || part_devices[q] == homes[i]) && (best < 0 || load[q] < load[(size_t)best]))
        best = (int)q;
    if (best < 0)
      throw Error(ERR_DEVICE, "item " + std::to_string(i) + " lives on CUDA device " + std::to_string(homes[i]) +
                                  ", which no executor of the call serves");
    part[i] = best;
    load[(size_t)best] += costs[i];
  }
  return part;
}

void execute_items_sharded(Executor* const* exs, int n_exec, int n, Product* const* plans, const Scalar* alpha,
                           const Scalar* beta, const Item* items) {
  NvtxRange range("tprims.contract_batched_sharded");
  std::vector<double> costs(n);
  std::vector<int> homes(n, -1), devs(n_exec);
  for (int e = 0; e < n_exec; ++e) devs[e] = exs[e]->device;
  for (int i = 0; i < n; ++i) {
    costs[i] = plans[i]->problem.macs();
    cudaPointerAttributes at;
    if (items[i].d && cudaPointerGetAttributes(&at, items[i].d) == cudaSuccess && at.type == cudaMemoryTypeDevice)
      homes[i] = at.device;
    else
      cudaGetLastError();
  }
  const std::vector<int> part = balance_parts(costs, homes, devs);
  std::vector<std::vector<int>> idx(n_exec);
  for (int i = 0; i < n; ++i) idx[part[i]].push_back(i);
  // Enqueue every share first (the streams run side by side), then drain.
  for (int e = 0; e < n_exec; ++e) {
    if (idx[e].empty()) continue;
    std::vector<Product*> ps;
    std::vector<Scalar> al, be;
    std::vector<Item> its;
    for (int i : idx[e]) {
      ps.push_back(plans[i]);
      al.push_back(alpha[i]);
      be.push_back(beta[i]);
      its.push_back(items[i]);
    }
    Executor& ex = *exs[e];
    std::lock_guard<std::mutex> lk(ex.mu);
    DeviceGuard g(ex.device);
    if (enqueue_items(ex, (int)ps.size(), ps.data(), al.data(), be.data(), its.data())) finish(ex);
  }
  for (int e = 0; e < n_exec; ++e) {
    if (idx[e].empty() || !exs[e]->sync) continue;
    Executor& ex = *exs[e];
    std::lock_guard<std::mutex> lk(ex.mu);
    DeviceGuard g(ex.device);
    finish(ex);
  }
}

void execute_networks(Executor& ex, int n, Network* const* nets, const Scalar* alpha, const Scalar* beta,
                      const void* const* const* inputs, void* const* outs, void* const* workspaces) {
  NvtxRange range("tprims.execute_networks");
  std::lock_guard<std::mutex> lk(ex.mu);
  DeviceGuard g(ex.device);
  // Arenas of the intermediates: the caller's workspace or the network's own.
  std::vector<char*> base(n, nullptr);
  for (int i = 0; i < n; ++i) {
    Network& net = *nets[i];
    if (net.arena_bytes == 0) continue;
    if (workspaces && workspaces[i]) {
      if (classify(workspaces[i], ex.device) != Where::Device)
        throw Error(ERR_DEVICE, "network workspace " + std::to_string(i) + " is not device memory of the executor");
      base[i] = static_cast<char*>(workspaces[i]);
      continue;
    }
    std::lock_guard<std::mutex> nl(net.mu);
    void*& a = net.arena[ex.device];
    if (!a) check_cuda(device_alloc(&a, net.arena_bytes), "cudaMalloc(network arena)");
    base[i] = static_cast<char*>(a);
  }
  // Every step's operands, validated before anything runs (all-or-nothing).
  size_t max_steps = 0;
  for (int i = 0; i < n; ++i) max_steps = std::max(max_steps, nets[i]->steps.size());
  std::vector<std::vector<Item>> step_items(max_steps);
  for (int i = 0; i < n; ++i) {
    const Network& net = *nets[i];
    const int nin = (int)net.inputs.size();
    auto origin = [&](int id) -> const void* {
      if (id < nin) return inputs[i][id];
      return base[i] + net.steps[id - nin].offset;
    };
    for (size_t s = 0; s < net.steps.size(); ++s) {
      const NetworkStep& st = net.steps[s];
      void* d = st.last ? outs[i] : static_cast<void*>(base[i] + st.offset);
      const bool c_read = st.last && !beta[i].is_zero();
      const Item it{origin(st.a), origin(st.b), c_read ? d : nullptr, d};
      validate_item(*st.plan, it, !c_read);
      step_items[s].push_back(it);
    }
  }
  const Scalar one{1.0, 0.0}, zero{};
  for (size_t s = 0; s < max_steps; ++s) {
    std::vector<Product*> plans;
    std::vector<Scalar> al, be;
    size_t k = 0;
    for (int i = 0; i < n; ++i) {
      if (s >= nets[i]->steps.size()) continue;
      const NetworkStep& st = nets[i]->steps[s];
      plans.push_back(st.plan.get());
      al.push_back(st.last ? alpha[i] : one);
      be.push_back(st.last ? beta[i] : zero);
      ++k;
    }
    if (k == 0) continue;
    // Stream order keeps step s + 1 behind step s; a staged host operand's
    // workspace is reused by the next step, so that case drains first.
    if (enqueue_items(ex, (int)k, plans.data(), al.data(), be.data(), step_items[s].data())) finish(ex);
  }
  if (ex.sync) finish(ex);
}

namespace {

bool has_repeat(const std::vector<int64_t>& labels) {
  for (size_t i = 0; i < labels.size(); ++i)
    for (size_t j = i + 1; j < labels.size(); ++j)
      if (labels[i] == labels[j]) return true;
  return false;
}

// Zero every element of `op`'s layout at `origin` (device or host memory).
void zero_layout(Executor& ex, DType dt, const Operand& op, void* origin) {
  const Layout& l = op.layout;
  const size_t elem = dtype_size(dt);
  __int128 n = 1, lo = 0, hi = 0;
  for (size_t i = 0; i < l.rank(); ++i) {
    n *= l.dims[i];
    const __int128 reach = (__int128)(l.dims[i] - 1) * l.strides[i];
    if (reach < 0) lo += reach; else hi += reach;
  }
  if (n <= 0) return;
  const bool dense = n == hi - lo + 1;
  if (classify(origin, ex.device) == Where::Device) {
    char* base = static_cast<char*>(origin);
    Timed t(ex, "zero_fill");
    if (dense)
      check_cuda(cudaMemsetAsync(base + (int64_t)lo * (int64_t)elem, 0, (size_t)n * elem, ex.stream), "zero fill");
    else
      check_cuda(dev::launch_fill_zero(elem, origin, (int)l.rank(), l.dims.data(), l.strides.data(), ex.stream),
                 "zero fill launch");
    return;
  }
  // Host memory: the staged copy of this operand is taken after this fill.
  char* base = static_cast<char*>(origin);
  if (dense) {
    std::memset(base + (int64_t)lo * (int64_t)elem, 0, (size_t)n * elem);
    return;
  }
  std::vector<int64_t> idx(l.rank(), 0);
  for (__int128 t = 0; t < n; ++t) {
    int64_t off = 0;
    for (size_t a = 0; a < l.rank(); ++a) off += idx[a] * l.strides[a];
    std::memset(base + off * (int64_t)elem, 0, elem);
    for (size_t a = 0; a < l.rank(); ++a) {
      if (++idx[a] < l.dims[a]) break;
      idx[a] = 0;
    }
  }
}

}  // namespace

// Plan::vjp. With P = op_A(A), Q = op_B(B) and D = op_D(alpha P Q + ...), the
// cotangents follow the conjugate-Wirtinger convention (a real loss L, dX =
// dL/d conj(X)): grad_P = conj(alpha) op_D(dD) conj(Q), grad_Q = conj(alpha)
// conj(P) op_D(dD), and grad_A = op_A(grad_P), grad_B = op_B(grad_Q). Each is
// one contraction of the existing kernels over the original labels: dA takes
// A's labels as its output labels, so a repeated label of A writes the
// diagonal (the rest of dA is zeroed first).
void execute_vjp(Product& p, Executor& ex, Scalar alpha, const void* A, const void* B, const void* dD, void* dA,
                 void* dB) {
  NvtxRange range("tprims.vjp");
  const Problem& pb = p.problem;
  const bool ca = pb.a.conj, cb = pb.b.conj, cd = pb.d.conj;
  const bool cplx = dtype_complex(pb.dtype);
  {
    std::lock_guard<std::mutex> lk(p.mu);
    if (dA && !p.adj_a) {
      Operand x = pb.d, y = pb.b, out = pb.a;
      x.conj = cd != ca;
      y.conj = !(cb != ca);
      out.conj = false;
      p.adj_a.reset(new Product(Problem::from_labels(pb.dtype, x, y, CMode::Absent, out, out, pb.ld, pb.lb, false, {},
                                                     pb.la, false, true)));
    }
    if (dB && !p.adj_b) {
      Operand x = pb.a, y = pb.d, out = pb.b;
      x.conj = !(ca != cb);
      y.conj = cd != cb;
      out.conj = false;
      p.adj_b.reset(new Product(Problem::from_labels(pb.dtype, x, y, CMode::Absent, out, out, pb.la, pb.ld, false, {},
                                                     pb.lb, false, true)));
    }
  }
  if (dA) validate_item(*p.adj_a, Item{dD, B, nullptr, dA}, true);
  if (dB) validate_item(*p.adj_b, Item{A, dD, nullptr, dB}, true);
  std::lock_guard<std::mutex> lk(ex.mu);
  DeviceGuard g(ex.device);
  const Scalar conj_alpha{alpha.re, cplx ? -alpha.im : 0.0};
  const Scalar zero{};
  bool staged = false;
  if (dA) {
    if (has_repeat(pb.la)) zero_layout(ex, pb.dtype, pb.a, dA);
    staged |= enqueue_item(*p.adj_a, ex, ca ? alpha : conj_alpha, zero, Item{dD, B, nullptr, dA});
  }
  if (dB) {
    if (staged) finish(ex);  // the staged workspace is reused
    if (has_repeat(pb.lb)) zero_layout(ex, pb.dtype, pb.b, dB);
    staged |= enqueue_item(*p.adj_b, ex, cb ? alpha : conj_alpha, zero, Item{A, dD, nullptr, dB});
  }
  if (ex.sync || staged) finish(ex);
}

}  // namespace tprims
