// Split-precision f32 contraction (bf16x3 / bf16x6 on tcgen05) that allocates
// no device memory: for callers that cannot call cudaMalloc, such as code that
// runs inside a memory pool owned by someone else (a framework's caching
// allocator, a serving process that reserved all of HBM up front) or that must
// not synchronise the device the way cudaMalloc / cudaFree may.
//
// The scratch the split path needs (the device status word, the plan's 12
// scatter vectors and the packed BF16 planes of A' and B') lives in one
// fixed file-scope device array, g_noalloc_scratch, of NOALLOC_SCRATCH_BYTES.
// It is part of this library's device image, so every GPU that loads the
// library holds it until the process exits. Every call shares it and it keeps
// the last call's contents; calls whose work overlaps on the same GPU (from two
// streams or two host threads) race on it and produce wrong results.
#include <chrono>
#include <cuda.h>
#include <mutex>
#include <string>
#include <thread>

#include "kernels.cuh"
#include "runtime.hpp"

namespace tprims {

namespace {

// 64 MiB: enough for f32 contractions up to about M = N = K = 2048 at bf16x6
// (3 planes of both operands, 48 MiB) plus the scatter vectors.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;
constexpr size_t NOALLOC_STATUS_BYTES = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;

// Device memory. In host code this name is only a host-side stand-in for the
// symbol, never a device address: the host passes kernels the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Upper bound of the wait for the caller's stream to drain (the executor's
// default drain limit); a stream that has not drained by then is reported as
// TPRIMS_ERR_INTERNAL instead of blocking the caller forever.
constexpr int NOALLOC_DRAIN_LIMIT_S = 60;

std::mutex g_noalloc_mu;
void* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
CUcontext g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The current context through the runtime's driver entry point (no link
// against libcuda); null when it cannot be queried.
CUcontext current_context() {
  typedef CUresult (*GetCurrentFn)(CUcontext*);
  static GetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<GetCurrentFn>(p);
  });
  CUcontext c = nullptr;
  if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

// The device address of the scratch array on `device` (the current device).
// It is looked up once per device and context: cudaGetSymbolAddress may load
// this library's module on the device the first time, which is why the first
// call on a device should not happen during a stream capture. When the
// current context is no longer the one the address came from (the caller
// reset the device and a new primary context exists), it is looked up again.
unsigned char* scratch_on(int device) {
  if (device < 0 || device >= NOALLOC_MAX_DEVICES)
    throw Error(ERR_DEVICE, "no-allocation entry point: device " + std::to_string(device) + " out of range");
  const CUcontext ctx = current_context();
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device] || g_noalloc_ctx[device] != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw Error(ERR_DEVICE, std::string("no-allocation entry point: cudaGetSymbolAddress failed: ") +
                                  cudaGetErrorString(e));
    }
    g_noalloc_addr[device] = p;
    g_noalloc_ctx[device] = ctx;
  }
  return static_cast<unsigned char*>(g_noalloc_addr[device]);
}

// Waits for `stream` to drain, giving up after NOALLOC_DRAIN_LIMIT_S.
void drain_bounded(cudaStream_t stream) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaStreamQuery(stream);
    if (q == cudaSuccess) return;
    if (q != cudaErrorNotReady) check_cuda(q, "kernel execution");
    const auto waited = std::chrono::steady_clock::now() - t0;
    if (waited > std::chrono::seconds(NOALLOC_DRAIN_LIMIT_S))
      throw Error(ERR_INTERNAL, "no-allocation entry point: the stream did not drain within " +
                                    std::to_string(NOALLOC_DRAIN_LIMIT_S) + " s");
    if (waited > std::chrono::microseconds(200)) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

bool on_device(const void* p, int device) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == device;
}

}  // namespace

void execute_split_noalloc(Product& pr, cudaStream_t stream, Scalar alpha, Scalar beta, const Item& it) {
  if (pr.problem.dtype != DType::F32 || (pr.scheme != Scheme::Bf16x3 && pr.scheme != Scheme::Bf16x6))
    throw Error(ERR_UNSUPPORTED,
                "the no-allocation entry point runs f32 plans set to split precision (bf16x3 or bf16x6) only");
  const Problem& p = pr.problem;
  const OrientedView& v = pr.view;
  if (p.out_empty) return;
  const bool c_read = it.c != nullptr && !beta.is_zero();
  const bool output_only = p.k_empty || alpha.is_zero();

  int device = -1;
  check_cuda(cudaGetDevice(&device), "cudaGetDevice");
  const void* ptrs[4] = {output_only ? nullptr : it.a, output_only ? nullptr : it.b, c_read ? it.c : nullptr, it.d};
  const char* names[4] = {"A", "B", "C", "D"};
  for (int s = 0; s < 4; ++s)
    if (ptrs[s] && !p.spans[s].empty && !on_device(ptrs[s], device))
      throw Error(ERR_DEVICE, std::string("no-allocation entry point: operand ") + names[s] +
                                  " is not in the current device's memory (host operands would need a staging "
                                  "allocation)");

  // Scratch layout: [status word][12 scatter vectors][BF16 planes of A'][of B'].
  const std::vector<int64_t>* vs[12] = {&v.a_m, &v.a_k, &v.b_k, &v.b_n, &v.c_m, &v.c_n,
                                        &v.d_m, &v.d_n, &v.h_a, &v.h_b, &v.h_c, &v.h_d};
  size_t offs[12], nscat = 0;
  for (int i = 0; i < 12; ++i) {
    offs[i] = nscat;
    nscat += (vs[i]->size() + 1 + 3) & ~size_t(3);  // never empty, 32-byte multiples
  }
  const size_t scat_bytes = align256(nscat * sizeof(int64_t));
  const dev::SplitLayout L = dev::split_layout((int)pr.scheme, v.M, v.N, v.K, v.H);
  const size_t plane_bytes = output_only ? 0 : dev::split_workspace_bytes(L);
  const size_t need = NOALLOC_STATUS_BYTES + scat_bytes + align256(plane_bytes);
  if (need > NOALLOC_SCRATCH_BYTES)
    throw Error(ERR_SHAPE, "no-allocation entry point: this contraction needs " + std::to_string(need) +
                               " bytes of scratch; the fixed scratch array holds " +
                               std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes (64 MiB)");

  unsigned char* base = scratch_on(device);
  unsigned* status = reinterpret_cast<unsigned*>(base);
  int64_t* scat = reinterpret_cast<int64_t*>(base + NOALLOC_STATUS_BYTES);
  unsigned char* planes = base + NOALLOC_STATUS_BYTES + scat_bytes;

  // The status word must start at zero; the scatter vectors are rewritten for
  // this plan; the pack kernels write every byte of the planes, padding included.
  check_cuda(cudaMemsetAsync(status, 0, sizeof(unsigned), stream), "no-allocation status clear");
  for (int i = 0; i < 12; ++i)
    if (!vs[i]->empty())
      check_cuda(cudaMemcpyAsync(scat + offs[i], vs[i]->data(), vs[i]->size() * sizeof(int64_t),
                                 cudaMemcpyHostToDevice, stream),
                 "no-allocation scatter upload");

  dev::GemmArgs g{};
  g.s = dev::Scatters{scat + offs[0], scat + offs[1], scat + offs[2],  scat + offs[3],
                      scat + offs[4], scat + offs[5], scat + offs[6],  scat + offs[7],
                      scat + offs[8], scat + offs[9], scat + offs[10], scat + offs[11]};
  g.A = v.swapped ? it.b : it.a;
  g.B = v.swapped ? it.a : it.b;
  g.C = c_read ? it.c : nullptr;
  g.D = it.d;
  g.M = v.M;
  g.N = v.N;
  g.K = v.K;
  g.H = v.H;
  g.a_kfast = v.a_kfast;
  g.b_kfast = v.b_kfast;
  g.d_mfast = v.d_mfast;
  g.e.alpha_re = alpha.re;
  g.e.beta_re = beta.re;
  g.e.beta_zero = c_read ? 0 : 1;
  g.e.plain = (!c_read && alpha.is_one()) ? 1 : 0;
  g.status = status;

  if (output_only) {
    check_cuda(dev::launch_output_pass((int)p.dtype, g, stream), "output pass launch");
  } else {
    unsigned char* ap = planes;
    unsigned char* bp = ap + (size_t)L.planes * L.H * L.m_pad * L.k_pad * 2;
    check_cuda(dev::launch_split_pack_f32(g, 0, L, ap, stream), "split pack A");
    check_cuda(dev::launch_split_pack_f32(g, 1, L, bp, stream), "split pack B");
    check_cuda(dev::launch_tc_bf16_gemm(g, L, ap, bp, (int)pr.scheme, stream), "tcgen05 contraction launch");
  }

  // Synchronous: wait (bounded) for the stream to drain, then read the status
  // word back on the same, now idle, stream.
  drain_bounded(stream);
  unsigned word = 0;
  check_cuda(cudaMemcpyAsync(&word, status, sizeof(word), cudaMemcpyDeviceToHost, stream), "status read");
  check_cuda(cudaStreamSynchronize(stream), "status read");
  if (word & dev::STATUS_WAIT_TIMEOUT)
    throw Error(ERR_INTERNAL, "a kernel gave up on a bounded wait (device status word " + std::to_string(word) + ")");
  if (word != 0) throw Error(ERR_INTERNAL, "a kernel reported device status word " + std::to_string(word));
}

}  // namespace tprims
