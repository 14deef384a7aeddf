// Output-only pass: D = op_D(beta * op_C(C)) over the whole (batched) output.
//
// Used when alpha == 0 or a contracted extent is zero, where A and B are not
// read at all. It is the semantics of the reference's ElementPlan::output
// (crates/tprims-contract/src/strategy/elementwise.rs:210) and scale_only
// (crates/tprims-kernel/src/pack/writeback.rs:495-550): beta == 0 writes zeros
// without reading C. Memory-bound: one pass over D (and C), threads running
// along whichever output index is unit-stride.
#include <climits>

#include "device_common.cuh"

namespace tprims {
namespace dev {

template <class R, bool CPLX>
__global__ void output_pass_kernel(GemmArgs g) {
  using T = typename Elem<R, CPLX>::type;
  const int64_t total = g.M * g.N * g.H;
  const T* C = static_cast<const T*>(g.C);
  T* D = static_cast<T*>(g.D);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t m, n, h;
    if (g.d_mfast) {
      m = i % g.M;
      n = (i / g.M) % g.N;
      h = i / (g.M * g.N);
    } else {
      n = i % g.N;
      m = (i / g.N) % g.M;
      h = i / (g.M * g.N);
    }
    R vr = R(0), vi = R(0);
    if (!g.e.beta_zero) {
      R cr, ci;
      Elem<R, CPLX>::load(C + g.s.h_c[h] + g.s.c_m[m] + g.s.c_n[n], cr, ci);
      if (g.e.conj_c) ci = -ci;
      const R br = (R)g.e.beta_re, bi = (R)g.e.beta_im;
      if (CPLX) {
        vr = cr * br - ci * bi;
        vi = cr * bi + ci * br;
      } else {
        vr = cr * br;
      }
    }
    if (CPLX && g.e.conj_d) vi = -vi;
    Elem<R, CPLX>::store(D + g.s.h_d[h] + g.s.d_m[m] + g.s.d_n[n], vr, vi);
  }
}

cudaError_t launch_output_pass(int dtype, const GemmArgs& g, cudaStream_t st) {
  const int64_t total = g.M * g.N * g.H;
  if (total <= 0) return cudaSuccess;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  switch (dtype) {
    case 0: output_pass_kernel<float, false><<<blocks, 256, 0, st>>>(g); break;
    case 1: output_pass_kernel<double, false><<<blocks, 256, 0, st>>>(g); break;
    case 2: output_pass_kernel<float, true><<<blocks, 256, 0, st>>>(g); break;
    case 3: output_pass_kernel<double, true><<<blocks, 256, 0, st>>>(g); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Batches of tiny products (the all-batch / elementwise shapes: M N K <= 256,
// e.g. a Hadamard product with M = N = K = 1): one thread per output element,
// the batch index fastest (it is usually the unit-stride one), the K sum in
// registers, then the epilogue. A batch scatter vector that is an arithmetic
// sequence from 0 is replaced by its stride (INT64_MIN marks one that is not),
// so the kernel reads only operand data. HBM-bound: A, B (and C) read once, D written once.
template <class R, bool CPLX>
__global__ void __launch_bounds__(256) tiny_batched_kernel(GemmArgs g, TinyStrides hs) {
  using T = typename Elem<R, CPLX>::type;
  const int64_t total = g.M * g.N * g.H;
  const T* A = static_cast<const T*>(g.A);
  const T* B = static_cast<const T*>(g.B);
  const T* C = static_cast<const T*>(g.C);
  T* D = static_cast<T*>(g.D);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t h = i % g.H, mn = i / g.H, m = mn % g.M, n = mn / g.M;
    const int64_t ha = hs.a != INT64_MIN ? h * hs.a : g.s.h_a[h];
    const int64_t hb = hs.b != INT64_MIN ? h * hs.b : g.s.h_b[h];
    const int64_t hd = hs.d != INT64_MIN ? h * hs.d : g.s.h_d[h];
    const T* ar = A + ha + g.s.a_m[m];
    const T* bc = B + hb + g.s.b_n[n];
    R sr = R(0), si = R(0);
    for (int64_t k = 0; k < g.K; ++k) {
      R xr, xi, yr, yi;
      Elem<R, CPLX>::load(ar + g.s.a_k[k], xr, xi);
      Elem<R, CPLX>::load(bc + g.s.b_k[k], yr, yi);
      if (CPLX) {
        if (g.conj_a) xi = -xi;
        if (g.conj_b) yi = -yi;
        sr = fma(xr, yr, sr);
        sr = fma(-xi, yi, sr);
        si = fma(xr, yi, si);
        si = fma(xi, yr, si);
      } else {
        sr = fma(xr, yr, sr);
      }
    }
    const T* c = C + (g.e.beta_zero ? 0 : (hs.c != INT64_MIN ? h * hs.c : g.s.h_c[h]) + g.s.c_m[m] + g.s.c_n[n]);
    epilogue_store<R, CPLX>(g.e, sr, si, c, D + hd + g.s.d_m[m] + g.s.d_n[n]);
  }
}

cudaError_t launch_tiny_batched(int dtype, const GemmArgs& g, const TinyStrides& hs, int num_sms, cudaStream_t st) {
  const int64_t total = g.M * g.N * g.H;
  if (total <= 0) return cudaSuccess;
  const int64_t want = (total + 255) / 256;
  const unsigned blocks = (unsigned)(want < (int64_t)num_sms * 16 ? want : (int64_t)num_sms * 16);
  switch (dtype) {
    case 0: tiny_batched_kernel<float, false><<<blocks, 256, 0, st>>>(g, hs); break;
    case 1: tiny_batched_kernel<double, false><<<blocks, 256, 0, st>>>(g, hs); break;
    case 2: tiny_batched_kernel<float, true><<<blocks, 256, 0, st>>>(g, hs); break;
    case 3: tiny_batched_kernel<double, true><<<blocks, 256, 0, st>>>(g, hs); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Self-test of the bounded-wait path: one thread waits for a flag that nothing
// sets, gives up after `limit_ns` of %globaltimer, records the timeout in the
// status word and returns, exactly as the tensor-core kernels do when a
// barrier phase never completes. No fault, no trap: the context stays usable.
__global__ void bounded_wait_selftest_kernel(const volatile unsigned* flag, unsigned* status, uint64_t limit_ns) {
  if (threadIdx.x != 0) return;
  const uint64_t t0 = globaltimer_ns();
  while (*flag == 0u) {
    if (globaltimer_ns() - t0 > limit_ns) {
      atomicOr(status, STATUS_WAIT_TIMEOUT);
      return;
    }
  }
}

cudaError_t launch_wait_selftest(const unsigned* flag, unsigned* status, uint64_t limit_ns, cudaStream_t st) {
  bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(flag, status, limit_ns);
  return cudaGetLastError();
}

// Pipe-peak probes for roofline denominators: register-only chains of
// independent operations, no memory traffic. FP64: mma.sync m8n8k4 (DMMA,
// 512 flops per warp instruction); FP32: FFMA (2 flops per lane).
__global__ void __launch_bounds__(128) probe_dmma_kernel(double* sink, int iters) {
  double acc[8][2];
  double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(acc[i][0]), "+d"(acc[i][1])
                   : "d"(a), "d"(b));
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
  if (s == 12345.678) sink[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) probe_ffma_kernel(float* sink, int iters) {
  float acc[16];
  const float a = 1.0f + threadIdx.x * 1e-7f, b = 0.999f;
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = (float)i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = fmaf(acc[i], b, a);
  }
  float s = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) s += acc[i];
  if (s == 12345.678f) sink[threadIdx.x] = s;
}

cudaError_t launch_probe(int which, void* sink, int blocks, int iters, cudaStream_t st, double* flops) {
  if (which == 0) {
    probe_dmma_kernel<<<blocks, 128, 0, st>>>(static_cast<double*>(sink), iters);
    *flops = (double)blocks * 4 /*warps*/ * iters * 8 * 512.0;
  } else {
    probe_ffma_kernel<<<blocks, 256, 0, st>>>(static_cast<float*>(sink), iters);
    *flops = (double)blocks * 256 * iters * 16 * 2.0;
  }
  return cudaGetLastError();
}

// Zero every element a layout addresses (rank <= 16): the off-diagonal part of
// a cotangent whose operand has a repeated label.
struct FillLayout {
  int rank;
  int64_t dims[16];
  int64_t strides[16];
};

template <class W>
__global__ void fill_zero_kernel(W* base, FillLayout L, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = i, off = 0;
    for (int a = 0; a < L.rank; ++a) {
      off += (rem % L.dims[a]) * L.strides[a];
      rem /= L.dims[a];
    }
    base[off] = W{};
  }
}

struct W16 {
  double a, b;
};

cudaError_t launch_fill_zero(size_t elem, void* origin, int rank, const int64_t* dims, const int64_t* strides,
                             cudaStream_t st) {
  if (rank > 16) return cudaErrorInvalidValue;
  FillLayout L{};
  L.rank = rank;
  int64_t total = 1;
  for (int a = 0; a < rank; ++a) {
    L.dims[a] = dims[a];
    L.strides[a] = strides[a];
    total *= dims[a];
  }
  if (total <= 0) return cudaSuccess;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  switch (elem) {
    case 4: fill_zero_kernel<float><<<blocks, 256, 0, st>>>(static_cast<float*>(origin), L, total); break;
    case 8: fill_zero_kernel<double><<<blocks, 256, 0, st>>>(static_cast<double*>(origin), L, total); break;
    case 16: fill_zero_kernel<W16><<<blocks, 256, 0, st>>>(static_cast<W16*>(origin), L, total); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace tprims
