// Output-only pass: D = op_D(beta * op_C(C)) over the whole (batched) output.
//
// Used when alpha == 0 or a contracted extent is zero, where A and B are not
// read at all. It is the semantics of the reference's ElementPlan::output
// (crates/tprims-contract/src/strategy/elementwise.rs:210) and scale_only
// (crates/tprims-kernel/src/pack/writeback.rs:495-550): beta == 0 writes zeros
// without reading C. Memory-bound: one pass over D (and C), threads running
// along whichever output index is unit-stride.
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
