// Ozaki-style INT8 slice contraction for f64 / c64 on the sm_100a tensor cores.
//
// Each row of A' (and each column of B') gets a power-of-two scale 2^e with
// max |x| < 2^e over that row. The scaled value x 2^(8S-2-e) is rounded to
// the nearest integer T (|T| <= 2^(8S-2)), and T is written as S balanced
// base-256 digits, T = sum_t d_t 256^(S-1-t): the S-1 low digits in
// [-128, 127] (eight bits each, the whole INT8 range) and the top digit in
// [-64, 64]. So x = 2^e sum_t d_t 2^-(8t+6), to within half a unit of
// 2^(e-8S+2). Slice products d_t(A) . d_u(B) accumulate exactly in INT32 on
// the tensor cores (tcgen05.mma kind::i8); the pairs with t + u = g share the
// weight 2^-(8g+12) and therefore one accumulator. Only pairs with t + u < S
// are formed (S(S+1)/2 products), which drops terms below about 2^-8S of the
// row and column scales. The epilogue recombines the S accumulators in FP64
// (smallest weight first), applies the row and column scales, then alpha,
// beta and conjugation (the write-back of
// crates/tprims-kernel/src/pack/writeback.rs:311-486).
//
// Complex operands are embedded as one real problem of twice the rows and
// twice the depth: A' row 2r = [Re A_r, -Im A_r], row 2r+1 = [Im A_r, Re A_r],
// B' depth [Re B; Im B] (each depth half padded with zeros to a whole number
// of 64-deep k-blocks), so rows 2r and 2r+1 of the product are the real and
// imaginary parts of row r (the four real products of the planar method);
// adjacent TMEM lanes hold them and the epilogue pairs them with a shuffle.
//
// INT32 exactness needs (g+1) K 128^2 < 2^31 for every diagonal g; the host
// splits deeper contractions into K chunks that accumulate into D (the KC-slab
// rule of the reference, driver/tile.rs:312-350).
#include <climits>

#include "tc_common.cuh"

namespace tprims {
namespace dev {

namespace {

using namespace tc;

constexpr int OZ_BM = 128;
constexpr int OZ_BN = 64;
constexpr int OZ_BK = 64;  // depth unit of the slice planes' padding and of the host's K chunks
constexpr int OZ_SK = 64;  // INT8 depth of one ring stage: 64-byte rows (SWIZZLE_64B), two MMAs deep
constexpr int EXP_NONFINITE = INT_MAX;

__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  // D format S32 (2), A and B signed INT8 (1), K-major, N >> 3, M >> 4.
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// 2^k for k in [-1022, 1023], built from its bits.
__device__ __forceinline__ double oz_pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// 0x80 in each of the S-1 low bytes: U = T + bias holds the S-1 low balanced
// digits of T as d + 128 in its low bytes (each in [0, 255], so no carry
// crosses a byte) and the top digit, in two's complement, from byte S-1 up.
__host__ __device__ constexpr unsigned long long oz_bias(int S) {
  unsigned long long c = 0ull;
  for (int i = 0; i + 1 < S; ++i) c |= 0x80ull << (8 * i);
  return c;
}

// T = round(x 2^(8S-2-e)) for four values of one row with exponent e
// (|x| < 2^e): the product is exact in FP64 and |T| <= 2^(8S-2) <= 2^62. The
// scale is s1 * s2 (two factors only for rows so small that 8S-2-e is above
// 1023); e >= -1073 and e <= 1024 keep both exponents in the normal range. A
// non-finite row (its x are zeros) takes scale 1.
template <int S>
__device__ __forceinline__ void oz_round(const double (&x)[4], int e, long long (&t)[4]) {
  const int k = e == EXP_NONFINITE ? 0 : 8 * S - 2 - e;
  const bool two = k > 1023;
  const double s1 = oz_pow2(two ? 1000 : k);
  const double s2 = oz_pow2(two ? k - 1000 : 0);
#pragma unroll
  for (int q = 0; q < 4; ++q) t[q] = __double2ll_rn((x[q] * s1) * s2);
}

// The S slice words of four biased values U = T + bias (plane sl holds the
// digit of weight 256^(S-1-sl), one byte per value): byte i of each U, four
// gathered into one word by byte permutes, with the bias taken off the low
// digits by flipping their top bit ((d + 128) ^ 0x80 is d in two's
// complement).
template <int S>
__device__ __forceinline__ void oz_planes(const unsigned long long (&u)[4], uint32_t (&out)[8]) {
#pragma unroll
  for (int sl = 0; sl < S; ++sl) {
    const int i = S - 1 - sl;
    const uint32_t sel = (uint32_t)(i & 3) | ((uint32_t)(4 + (i & 3)) << 4);
    uint32_t w4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) w4[q] = i < 4 ? (uint32_t)u[q] : (uint32_t)(u[q] >> 32);
    const uint32_t p01 = __byte_perm(w4[0], w4[1], sel), p23 = __byte_perm(w4[2], w4[3], sel);
    const uint32_t w = __byte_perm(p01, p23, 0x5410);
    out[sl] = i < S - 1 ? w ^ 0x80808080u : w;
  }
}

template <int S>
__device__ inline void write_slices_t(const double (&x)[4], int e, int8_t* o, int64_t plane) {
  long long t[4];
  oz_round<S>(x, e, t);
  unsigned long long u[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) u[q] = (unsigned long long)t[q] + oz_bias(S);
  uint32_t w[8];
  oz_planes<S>(u, w);
#pragma unroll
  for (int sl = 0; sl < S; ++sl) *reinterpret_cast<uint32_t*>(o + sl * plane) = w[sl];
}

// The four embedded copies of a complex quad of A' (rows 2r and 2r+1, both
// depth halves: re, -im / im, re) from one rounding per part: re is stored
// twice, and the digits of -im are those of -T (bias - T), since a balanced
// digit -128 has no negation in INT8.
template <int S>
__device__ inline void write_slices_a_t(const double (&re)[4], const double (&im)[4], int e, int8_t* o0, int8_t* o1,
                                        int64_t kh, int64_t plane) {
  long long tr[4], ti[4];
  oz_round<S>(re, e, tr);
  oz_round<S>(im, e, ti);
  unsigned long long ur[4], ui[4], un[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    ur[q] = (unsigned long long)tr[q] + oz_bias(S);
    ui[q] = (unsigned long long)ti[q] + oz_bias(S);
    un[q] = oz_bias(S) - (unsigned long long)ti[q];
  }
  uint32_t wr[8], wi[8], wn[8];
  oz_planes<S>(ur, wr);
  oz_planes<S>(ui, wi);
  oz_planes<S>(un, wn);
#pragma unroll
  for (int sl = 0; sl < S; ++sl) {
    *reinterpret_cast<uint32_t*>(o0 + sl * plane) = wr[sl];
    *reinterpret_cast<uint32_t*>(o0 + kh + sl * plane) = wn[sl];
    *reinterpret_cast<uint32_t*>(o1 + sl * plane) = wi[sl];
    *reinterpret_cast<uint32_t*>(o1 + kh + sl * plane) = wr[sl];
  }
}

__device__ inline void write_slices_a(const double (&re)[4], const double (&im)[4], int e, int S, int8_t* o0,
                                      int8_t* o1, int64_t kh, int64_t plane) {
  switch (S) {
    case 4: write_slices_a_t<4>(re, im, e, o0, o1, kh, plane); break;
    case 5: write_slices_a_t<5>(re, im, e, o0, o1, kh, plane); break;
    case 6: write_slices_a_t<6>(re, im, e, o0, o1, kh, plane); break;
    case 7: write_slices_a_t<7>(re, im, e, o0, o1, kh, plane); break;
    default: write_slices_a_t<8>(re, im, e, o0, o1, kh, plane); break;
  }
}

__device__ inline void write_slices(const double (&x)[4], int e, int S, int8_t* o, int64_t plane) {
  switch (S) {
    case 4: write_slices_t<4>(x, e, o, plane); break;
    case 5: write_slices_t<5>(x, e, o, plane); break;
    case 6: write_slices_t<6>(x, e, o, plane); break;
    case 7: write_slices_t<7>(x, e, o, plane); break;
    default: write_slices_t<8>(x, e, o, plane); break;
  }
}

// Bit pattern of |x|: ordered like |x| for finite values, and every inf or
// NaN (of either part of a complex value) compares at or above 0x7ff0...0, so
// one integer max over a row finds both its largest magnitude and whether it
// holds a non-finite entry.
__device__ __forceinline__ unsigned long long mag_bits(double x) {
  return (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
}
__device__ __forceinline__ unsigned long long max_bits(unsigned long long a, unsigned long long b) {
  return a > b ? a : b;
}

// Per row (complex: per complex row) exponent e with max |x| < 2^e; a row with
// a non-finite entry gets EXP_NONFINITE. One CTA per 32 rows, looping over K.
template <bool CPLX>
__global__ void __launch_bounds__(256) ozaki_exp_kernel(const double* __restrict__ X, const int64_t* rows_scat,
                                                        const int64_t* k_scat, const int64_t* h_scat, int64_t nrows,
                                                        int64_t K, int64_t rows_pad, int kfast, int* __restrict__ out) {
  __shared__ unsigned long long rowmax[32];
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * 32, h = blockIdx.y;
  if (tid < 32) rowmax[tid] = 0ull;
  __syncthreads();
  const int64_t hoff = h_scat[h];
  unsigned long long local[8];
  int myrow[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    local[j] = 0ull;
    myrow[j] = kfast ? (tid / 64 + 4 * j) : (tid % 32);
  }
  for (int64_t k0 = 0; k0 < K; k0 += 64) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int rr = myrow[j];
      const int kk = kfast ? (tid % 64) : (tid / 32 + 8 * j);
      const int64_t r = r0 + rr, k = k0 + kk;
      if (r < nrows && k < K) {
        const double* e = X + (CPLX ? 2 : 1) * (hoff + rows_scat[r] + k_scat[k]);
        unsigned long long bits = mag_bits(e[0]);
        if (CPLX) bits = max_bits(bits, mag_bits(e[1]));
        if (bits > local[j]) local[j] = bits;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) atomicMax(&rowmax[myrow[j]], local[j]);
  __syncthreads();
  if (tid < 32 && r0 + tid < rows_pad) {
    const unsigned long long bits = rowmax[tid];
    int e = 0;
    if (bits >= 0x7ff0000000000000ull) e = EXP_NONFINITE;
    else if (bits != 0ull) frexp(__longlong_as_double((long long)bits), &e);
    out[h * rows_pad + r0 + tid] = e;
  }
}

// Gather + scale + slice of one 32-row x 64-k tile of a real operand, written
// K-major into planes[S][H][rows_pad][k_pad] (INT8), zero-padded. (Complex
// operands use ozaki_slice_c64_kernel.)
__global__ void __launch_bounds__(256) ozaki_slice_kernel(const double* __restrict__ X, const int64_t* rows_scat,
                                                          const int64_t* k_scat, const int64_t* h_scat,
                                                          const int* __restrict__ exps, int64_t nrows, int64_t K,
                                                          int64_t rows_pad, int64_t exp_pad, int64_t k_pad, int64_t H,
                                                          int kfast, int S, int8_t* __restrict__ out) {
  __shared__ double tile[32][65];
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 64, h = blockIdx.z;
  const int64_t hoff = h_scat[h];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int rr, kk;
    if (kfast) {
      rr = tid / 64 + 4 * j;
      kk = tid % 64;
    } else {
      rr = tid % 32;
      kk = tid / 32 + 8 * j;
    }
    const int64_t r = r0 + rr, k = k0 + kk;
    tile[rr][kk] = (r < nrows && k < K) ? X[hoff + rows_scat[r] + k_scat[k]] : 0.0;
  }
  __syncthreads();
  const int64_t plane = H * rows_pad * k_pad;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int p = tid + 256 * j;
    const int rr = p / 16, kq = (p % 16) * 4;
    const int64_t r = r0 + rr;
    const int e = (r < nrows) ? exps[h * exp_pad + r] : 0;
    double x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = (e == EXP_NONFINITE) ? 0.0 : tile[rr][kq + q];
    write_slices(x, e, S, out + (h * rows_pad + r) * k_pad + k0 + kq, plane);
  }
}

// Batch-innermost operands (the batch index has the smallest stride, as in a
// [batch, k, row] tensor stored batch-first): the same scan and slicing with
// the 32 lanes of a warp on 32 consecutive batch entries, so each warp load
// is one contiguous run.
template <bool CPLX>
__global__ void __launch_bounds__(256) ozaki_exp_hfast_kernel(const double* __restrict__ X, const int64_t* rows_scat,
                                                              const int64_t* k_scat, const int64_t* h_scat,
                                                              int64_t nrows, int64_t K, int64_t rows_pad, int64_t H,
                                                              int* __restrict__ out) {
  // One CTA per (row, 32 batch entries); the 8 warps split k and combine in
  // shared memory.
  __shared__ unsigned long long red[8][32];
  const int hl = threadIdx.x & 31, kp = threadIdx.x >> 5;
  const int64_t r = blockIdx.x, h = (int64_t)blockIdx.y * 32 + hl;
  unsigned long long best = 0ull;
  if (r < nrows && h < H) {
    const double* base = X + (CPLX ? 2 : 1) * (h_scat[h] + rows_scat[r]);
#pragma unroll 4
    for (int64_t k = kp; k < K; k += 8) {
      const double* e = base + (CPLX ? 2 : 1) * __ldg(k_scat + k);
      unsigned long long bits = mag_bits(e[0]);
      if (CPLX) bits = max_bits(bits, mag_bits(e[1]));
      if (bits > best) best = bits;
    }
  }
  red[kp][hl] = best;
  __syncthreads();
  if (kp == 0 && h < H && r < rows_pad) {
#pragma unroll
    for (int j = 1; j < 8; ++j) best = red[j][hl] > best ? red[j][hl] : best;
    int e = 0;
    if (best >= 0x7ff0000000000000ull) e = EXP_NONFINITE;
    else if (best != 0ull) frexp(__longlong_as_double((long long)best), &e);
    out[h * rows_pad + r] = e;
  }
}

// Slicing of one real row across 32 batch entries x 64 k: loads run along
// the batch index, the K-major plane rows are written 4 bytes per thread.
__global__ void __launch_bounds__(256) ozaki_slice_hfast_kernel(const double* __restrict__ X, const int64_t* rows_scat,
                                                                const int64_t* k_scat, const int64_t* h_scat,
                                                                const int* __restrict__ exps, int64_t nrows, int64_t K,
                                                                int64_t rows_pad, int64_t exp_pad, int64_t k_pad,
                                                                int64_t H, int S, int8_t* __restrict__ out) {
  __shared__ double tile[32][65];
  const int tid = threadIdx.x;
  const int64_t k0 = (int64_t)blockIdx.x * 64, r = blockIdx.y, h0 = (int64_t)blockIdx.z * 32;
  {
    const int hl = tid & 31;
    const int64_t h = h0 + hl;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int kk = (tid >> 5) + 8 * j;
      const int64_t k = k0 + kk;
      tile[hl][kk] = (h < H && r < nrows && k < K) ? X[h_scat[h] + rows_scat[r] + k_scat[k]] : 0.0;
    }
  }
  __syncthreads();
  const int64_t plane = H * rows_pad * k_pad;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int p = tid + 256 * j;
    const int hl = p / 16, kq = (p % 16) * 4;
    const int64_t h = h0 + hl;
    if (h >= H) continue;
    const int e = (r < nrows) ? exps[h * exp_pad + r] : 0;
    double x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = (e == EXP_NONFINITE) ? 0.0 : tile[hl][kq + q];
    write_slices(x, e, S, out + (h * rows_pad + r) * k_pad + k0 + kq, plane);
  }
}

// Complex batch-innermost slicing: one load of a complex element gives all of
// its embedded values (A': rows 2r and 2r+1, both depth halves; B': row n,
// both halves). One CTA per (complex row, 32 batch entries, 64 k).
template <int WHICH>
__global__ void __launch_bounds__(256) ozaki_slice_hfast_c64_kernel(
    const double* __restrict__ X, const int64_t* rows_scat, const int64_t* k_scat, const int64_t* h_scat,
    const int* __restrict__ exps, int64_t nrows, int64_t K, int64_t Kh, int64_t rows_pad, int64_t exp_pad,
    int64_t k_pad, int64_t H, int conj, int S, int8_t* __restrict__ out) {
  __shared__ double t_re[32][65], t_im[32][65];
  const int tid = threadIdx.x;
  const int64_t k0 = (int64_t)blockIdx.x * 64, r = blockIdx.y, h0 = (int64_t)blockIdx.z * 32;
  {
    const int hl = tid & 31;
    const int64_t h = h0 + hl;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int kk = (tid >> 5) + 8 * j;
      const int64_t k = k0 + kk;
      double re = 0.0, im = 0.0;
      if (h < H && r < nrows && k < K) {
        const double* e = X + 2 * (h_scat[h] + rows_scat[r] + k_scat[k]);
        re = e[0];
        im = conj ? -e[1] : e[1];
      }
      t_re[hl][kk] = re;
      t_im[hl][kk] = im;
    }
  }
  __syncthreads();
  const int64_t plane = H * rows_pad * k_pad;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int p = tid + 256 * j;
    const int hl = p / 16, kq = (p % 16) * 4;
    const int64_t h = h0 + hl;
    if (h >= H) continue;
    const int e = (r < nrows) ? exps[h * exp_pad + r] : 0;
    double re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool bad = e == EXP_NONFINITE;
      re[q] = bad ? 0.0 : t_re[hl][kq + q];
      im[q] = bad ? 0.0 : t_im[hl][kq + q];
    }
    if (WHICH == 0) {
      int8_t* o0 = out + (h * rows_pad + 2 * r) * k_pad + k0 + kq;
      write_slices_a(re, im, e, S, o0, o0 + k_pad, Kh, plane);
    } else {
      int8_t* o0 = out + (h * rows_pad + r) * k_pad + k0 + kq;
      write_slices(re, e, S, o0, plane);
      write_slices(im, e, S, o0 + Kh, plane);
    }
  }
}

// One pass over a batch-innermost operand: a CTA holds OZ_HB batch entries of
// one row, all of K, in shared memory, takes their exponents there and slices
// them, so the operand is read from HBM once instead of once by the scan and
// once by the slicing. Shared layout t[hl][swz(k)] with an odd row stride:
// the loads (16 lanes on 16 batch entries at one k) and the slicing reads (32
// lanes on 32 consecutive quads of k, one q at a time) both touch 16
// distinct 8-byte bank slots per half-warp. swz only permutes k inside its
// aligned group of four.
constexpr int OZ_HB = 16;

__device__ __forceinline__ int64_t oz_swz(int64_t k) { return k ^ ((k >> 4) & 3); }

__host__ __device__ inline int64_t oz_hfast_stride(int64_t K) { return (K + 3) / 4 * 4 + 1; }

template <bool CPLX, int WHICH>
__global__ void __launch_bounds__(256, 2) ozaki_pack_hfast_kernel(
    const double* __restrict__ X, const int64_t* rows_scat, const int64_t* k_scat, const int64_t* h_scat,
    int64_t nrows, int64_t crows, int64_t K, int64_t kw, int64_t rows_pad, int64_t exp_pad, int64_t k_pad,
    int64_t Kh, int64_t H, int conj, int S, int* __restrict__ exps, int8_t* __restrict__ out) {
  extern __shared__ double oz_t[];
  __shared__ unsigned long long red[256 / OZ_HB][OZ_HB];
  __shared__ int ex_s[OZ_HB];
  const int tid = threadIdx.x, hl = tid % OZ_HB, kp = tid / OZ_HB;
  const int64_t ks = oz_hfast_stride(K);
  double* t_re = oz_t;
  double* t_im = oz_t + OZ_HB * ks;
  // Batch groups vary fastest over the grid, so the CTAs resident together
  // read all the batch entries of their rows: every batch run of an operand
  // row is read at once, not the same part of each row by every SM (which
  // loaded some DRAM channels twice as much as others).
  const int64_t hgroups = (H + OZ_HB - 1) / OZ_HB;
  const int64_t r = (int64_t)blockIdx.x / hgroups, h0 = ((int64_t)blockIdx.x % hgroups) * OZ_HB;
  const bool live = r < nrows && h0 + hl < H;
  const double* base = X + (CPLX ? 2 : 1) * (live ? h_scat[h0 + hl] + rows_scat[r] : 0);
  unsigned long long best = 0ull;
  if (live) {
#pragma unroll 8
    for (int64_t k = kp; k < K; k += 256 / OZ_HB) {
      const double* e = base + (CPLX ? 2 : 1) * __ldg(k_scat + k);
      const double re = e[0];
      unsigned long long bits = mag_bits(re);
      const int64_t pos = hl * ks + oz_swz(k);
      t_re[pos] = re;
      if constexpr (CPLX) {
        const double im = e[1];
        bits = max_bits(bits, mag_bits(im));
        t_im[pos] = conj ? -im : im;
      }
      best = bits > best ? bits : best;
    }
  }
  red[kp][hl] = best;
  __syncthreads();
  if (tid < OZ_HB) {
    unsigned long long b = red[0][tid];
#pragma unroll
    for (int j = 1; j < 256 / OZ_HB; ++j) b = red[j][tid] > b ? red[j][tid] : b;
    int e = 0;
    if (b >= 0x7ff0000000000000ull) e = EXP_NONFINITE;
    else if (b != 0ull) frexp(__longlong_as_double((long long)b), &e);
    ex_s[tid] = e;
    if (h0 + tid < H && r < exp_pad) exps[(h0 + tid) * exp_pad + r] = e;
  }
  __syncthreads();
  if (r >= crows) return;
  const int64_t nq = kw / 4, plane = H * rows_pad * k_pad;
  for (int64_t it = tid; it < OZ_HB * nq; it += 256) {
    const int hh = (int)(it / nq);
    const int64_t kq = (it - hh * nq) * 4, h = h0 + hh;
    if (h >= H) break;
    const int e = ex_s[hh];
    double re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t k = kq + q;
      const bool in = k < K && e != EXP_NONFINITE && r < nrows;
      const int64_t pos = hh * ks + oz_swz(k);
      re[q] = in ? t_re[pos] : 0.0;
      if constexpr (CPLX) im[q] = in ? t_im[pos] : 0.0;
    }
    if constexpr (!CPLX) {
      write_slices(re, e, S, out + (h * rows_pad + r) * k_pad + kq, plane);
    } else if constexpr (WHICH == 0) {
      int8_t* o0 = out + (h * rows_pad + 2 * r) * k_pad + kq;
      write_slices_a(re, im, e, S, o0, o0 + k_pad, Kh, plane);
    } else {
      int8_t* o0 = out + (h * rows_pad + r) * k_pad + kq;
      write_slices(re, e, S, o0, plane);
      write_slices(im, e, S, o0 + Kh, plane);
    }
  }
}

// Shared memory of the one-pass kernel; it runs when two CTAs fit on an SM.
inline size_t oz_hfast_smem(bool cplx, int64_t K) { return (cplx ? 2 : 1) * OZ_HB * oz_hfast_stride(K) * 8; }
constexpr size_t OZ_HFAST_SMEM_MAX = 100 * 1024;

// Complex slicing for the general layouts (rows or k unit-stride): one load
// of a complex element writes all of its embedded values, as in the
// batch-innermost kernel above. One CTA per (32 complex rows, 64 k, batch
// entry); threads run along k when k is the unit-stride index.
template <int WHICH>
__global__ void __launch_bounds__(256) ozaki_slice_c64_kernel(
    const double* __restrict__ X, const int64_t* rows_scat, const int64_t* k_scat, const int64_t* h_scat,
    const int* __restrict__ exps, int64_t nrows, int64_t K, int64_t Kh, int64_t rows_pad, int64_t exp_pad,
    int64_t k_pad, int64_t H, int kfast, int conj, int S, int8_t* __restrict__ out) {
  __shared__ double t_re[32][65], t_im[32][65];
  const int tid = threadIdx.x;
  const int64_t k0 = (int64_t)blockIdx.x * 64, r0 = (int64_t)blockIdx.y * 32, h = blockIdx.z;
  const int64_t hoff = h_scat[h];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int rr, kk;
    if (kfast) {
      rr = tid / 64 + 4 * j;
      kk = tid % 64;
    } else {
      rr = tid % 32;
      kk = tid / 32 + 8 * j;
    }
    const int64_t r = r0 + rr, k = k0 + kk;
    double re = 0.0, im = 0.0;
    if (r < nrows && k < K) {
      const double* e = X + 2 * (hoff + rows_scat[r] + k_scat[k]);
      re = e[0];
      im = conj ? -e[1] : e[1];
    }
    t_re[rr][kk] = re;
    t_im[rr][kk] = im;
  }
  __syncthreads();
  const int64_t plane = H * rows_pad * k_pad;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int p = tid + 256 * j;
    const int rr = p / 16, kq = (p % 16) * 4;
    const int64_t r = r0 + rr;
    const int e = (r < nrows) ? exps[h * exp_pad + r] : 0;
    double re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool bad = e == EXP_NONFINITE;
      re[q] = bad ? 0.0 : t_re[rr][kq + q];
      im[q] = bad ? 0.0 : t_im[rr][kq + q];
    }
    if (WHICH == 0) {
      int8_t* o0 = out + (h * rows_pad + 2 * r) * k_pad + k0 + kq;
      write_slices_a(re, im, e, S, o0, o0 + k_pad, Kh, plane);
    } else {
      int8_t* o0 = out + (h * rows_pad + r) * k_pad + k0 + kq;
      write_slices(re, e, S, o0, plane);
      write_slices(im, e, S, o0 + Kh, plane);
    }
  }
}

template <int S>
struct OzCfg {
  static constexpr int A_TILE = OZ_BM * OZ_SK;  // bytes of one A plane tile
  static constexpr int B_TILE = OZ_BN * OZ_SK;
  // A and B slice tiles of a k-block live in two rings of their own: three A
  // stages when they fit beside two B stages, and a third B stage when it
  // fits too (six slices: 3 x 48 KB + 3 x 24 KB; seven: 3 x 56 KB + 2 x
  // 28 KB), so more operand bytes are in flight per SM than whole stages of
  // both operands allow.
  static constexpr int A_STAGE = S * A_TILE, B_STAGE = S * B_TILE;
  static constexpr int LIMIT = 222 * 1024;
  static constexpr int A_STAGES = (3 * A_STAGE + 2 * B_STAGE <= LIMIT) ? 3 : 2;
  static constexpr int B_STAGES = (A_STAGES * A_STAGE + 3 * B_STAGE <= LIMIT) ? 3 : 2;
  static constexpr int RING = A_STAGES * A_STAGE + B_STAGES * B_STAGE;
  static constexpr int BAR = (2 * A_STAGES + 2 * B_STAGES + 3) * 8 + 16;
  static constexpr int SMEM = 1024 + RING + BAR;
  static constexpr int TMEM_COLS = (S * OZ_BN <= 256) ? 256 : 512;
  static_assert(S * OZ_BN <= 512, "one INT32 accumulator per diagonal must fit in TMEM");
};

// Persistent: one CTA per SM walks the 128 x 64 tiles of the embedded product
// (tile = blockIdx.x, blockIdx.x + gridDim.x, ...; n fastest, then m, then
// batch), each over k-blocks [kb0, kb1). Warp 0: TMA producer, running ahead
// across tile boundaries through the stage ring; warp 1: TMEM owner and MMA
// issuer; warps 2-9: epilogue, two warps per TMEM lane quarter (warp % 4),
// one per 32-column half of the tile. The epilogue drains the S diagonal
// accumulators of a tile into FP64 registers, hands TMEM back (tmem_empty) and
// then scales and stores while the MMAs of the next tile run.
// Every mbarrier wait is bounded; a timeout sets STATUS_WAIT_TIMEOUT and the
// role stops, so the kernel always ends.
constexpr int OZ_THREADS = 320;
constexpr int OZ_EPI_WARPS = 8;
constexpr int OZ_EPI_COLS = OZ_BN / 2;  // columns per epilogue warp

// 2^e as a double for e in [-1022, 1023] (exact).
__device__ inline double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

template <int S, bool CPLX>
__global__ void __launch_bounds__(OZ_THREADS, 1)
ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g,
                  const int* __restrict__ exp_a, const int* __restrict__ exp_b, int64_t m_emb, int64_t m_pad,
                  int64_t n_pad, int64_t exp_a_pad, int kb0, int kb1) {
  using Cfg = OzCfg<S>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* ring_a = smem;
  uint8_t* ring_b = smem + Cfg::A_STAGES * Cfg::A_STAGE;
  uint64_t* full_a = reinterpret_cast<uint64_t*>(smem + Cfg::RING);
  uint64_t* empty_a = full_a + Cfg::A_STAGES;
  uint64_t* full_b = empty_a + Cfg::A_STAGES;
  uint64_t* empty_b = full_b + Cfg::B_STAGES;
  uint64_t* accf = empty_b + Cfg::B_STAGES;
  uint64_t* tmem_empty = accf + 1;
  uint64_t* mma_done = tmem_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  __shared__ uint32_t consumed_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nk = (kb1 - kb0) * (OZ_BK / OZ_SK);  // ring stages per tile
  const int64_t tiles_n = n_pad / OZ_BN, tiles_m = m_pad / OZ_BM;
  const int64_t ntiles = tiles_n * tiles_m * g.H;

  if (warp == 0 && lane == 0) {
    for (int i = 0; i < Cfg::A_STAGES; ++i) {
      mbar_init(&full_a[i], 1);
      mbar_init(&empty_a[i], 1);
    }
    for (int i = 0; i < Cfg::B_STAGES; ++i) {
      mbar_init(&full_b[i], 1);
      mbar_init(&empty_b[i], 1);
    }
    mbar_init(mma_done, 1);
    consumed_s = 0xffffffffu;
    mbar_init(accf, 1);
    mbar_init(tmem_empty, OZ_EPI_WARPS);  // one arrival per epilogue warp
    fence_barrier_init();
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  uint32_t issued_a = 0, issued_b = 0;  // k-blocks whose A / B tiles the producer issued
  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      bool alive = true;
      for (int64_t tile = blockIdx.x; alive && tile < ntiles; tile += gridDim.x) {
        const int64_t nt = tile % tiles_n, mt = (tile / tiles_n) % tiles_m, h = tile / (tiles_n * tiles_m);
        for (int i = 0; i < nk; ++i, ++it) {
          const int kx = kb0 * OZ_BK + i * OZ_SK;
          const int sa = (int)(it % Cfg::A_STAGES), sb = (int)(it % Cfg::B_STAGES);
          if (!mbar_wait(&empty_a[sa], ((it / Cfg::A_STAGES) & 1u) ^ 1u)) {
            atomicOr(g.status, STATUS_WAIT_TIMEOUT);
            alive = false;
            break;
          }
          mbar_arrive_expect_tx(&full_a[sa], (uint32_t)Cfg::A_STAGE);
#pragma unroll
          for (int p = 0; p < S; ++p)
            tma_load_2d(ring_a + sa * Cfg::A_STAGE + p * Cfg::A_TILE, &tmA, &full_a[sa], kx,
                        (int)((p * g.H + h) * m_pad + mt * OZ_BM));
          issued_a = it + 1;
          if (!mbar_wait(&empty_b[sb], ((it / Cfg::B_STAGES) & 1u) ^ 1u)) {
            atomicOr(g.status, STATUS_WAIT_TIMEOUT);
            alive = false;
            break;
          }
          mbar_arrive_expect_tx(&full_b[sb], (uint32_t)Cfg::B_STAGE);
#pragma unroll
          for (int p = 0; p < S; ++p)
            tma_load_2d(ring_b + sb * Cfg::B_STAGE + p * Cfg::B_TILE, &tmB, &full_b[sb], kx,
                        (int)((p * g.H + h) * n_pad + nt * OZ_BN));
          issued_b = it + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, j = 0;
      bool alive = true;
      for (int64_t tile = blockIdx.x; alive && tile < ntiles; tile += gridDim.x, ++j) {
        // The epilogue must have drained the previous tile's accumulators.
        if (!mbar_wait(tmem_empty, (j & 1u) ^ 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          break;
        }
        tc_fence_after();
        for (int i = 0; i < nk; ++i, ++it) {
          const int sa = (int)(it % Cfg::A_STAGES), sb = (int)(it % Cfg::B_STAGES);
          if (!mbar_wait(&full_a[sa], (it / Cfg::A_STAGES) & 1u) || !mbar_wait(&full_b[sb], (it / Cfg::B_STAGES) & 1u)) {
            atomicOr(g.status, STATUS_WAIT_TIMEOUT);
            alive = false;
            break;
          }
          tc_fence_after();
          const uint32_t abase = smem_u32(ring_a + sa * Cfg::A_STAGE);
          const uint32_t bbase = smem_u32(ring_b + sb * Cfg::B_STAGE);
          // A slice t meets B slices u = 0 .. S-1-t, whose diagonals t + u
          // are the consecutive TMEM column blocks from t * 64 on, and whose
          // tiles are consecutive 64-row blocks of one K-major operand in
          // the stage. So one MMA takes a run of up to four B slices (N up
          // to 256): S(S+1)/2 products in about 2S instructions, each
          // reading the A tile once for all the slices it meets. The t = 0
          // MMAs cover every diagonal and start them on the first k-block.
#pragma unroll
          for (int t = 0; t < S; ++t) {
            const uint64_t ad = sdesc_sw64(abase + t * Cfg::A_TILE);
#pragma unroll
            for (int u0 = 0; u0 < S - t; u0 += 4) {
              const int cnt = (S - t - u0) < 4 ? (S - t - u0) : 4;
              const uint32_t idesc = idesc_i8(OZ_BM, OZ_BN * cnt);
              const uint64_t bd = sdesc_sw64(bbase + u0 * Cfg::B_TILE);
#pragma unroll
              for (int kk = 0; kk < OZ_SK / 32; ++kk)
                umma_i8(tmem + (uint32_t)((t + u0) * OZ_BN), ad + 2 * kk, bd + 2 * kk, idesc,
                        (i | t | kk) != 0 ? 1u : 0u);
            }
          }
          umma_commit(&empty_a[sa]);
          umma_commit(&empty_b[sb]);
        }
        if (alive) umma_commit(accf);
      }
      // Every MMA issued has finished reading shared memory and writing TMEM
      // before the CTA ends (bounded); `consumed_s` tells the producer which
      // k-blocks' copies nobody waited for.
      umma_commit(mma_done);
      (void)mbar_wait(mma_done, 0u);
      consumed_s = it;
    }
  } else {
    const int lane_base = 32 * (warp & 3);
    const int col0 = OZ_EPI_COLS * ((warp - 2) >> 2);  // this warp's column half
    const uint32_t lane_addr = (uint32_t)lane_base << 16;
    using T = typename Elem<double, CPLX>::type;
    uint32_t j = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++j) {
      const int64_t nt = tile % tiles_n, mt = (tile / tiles_n) % tiles_m, h = tile / (tiles_n * tiles_m);
      const int64_t n0 = nt * OZ_BN + col0;
      // Column data of the tile, one column per lane (broadcast by shuffles in
      // the store loop), loaded before the accumulators are ready.
      const int64_t n_l = n0 + lane;
      const bool col_ok_l = n_l < g.N;
      const int en_r = __ldg(exp_b + h * n_pad + n_l);
      const int64_t dn_r = col_ok_l ? __ldg(g.s.d_n + n_l) : 0;
      const int64_t cn_r = (col_ok_l && !g.e.beta_zero) ? __ldg(g.s.c_n + n_l) : 0;
      const int64_t me = mt * OZ_BM + lane_base + lane;  // row of the embedded product
      const int64_t m = CPLX ? (me >> 1) : me;            // output row
      const bool row_ok = me < m_emb;
      const int em = row_ok ? __ldg(exp_a + h * exp_a_pad + m) : 0;
      const int64_t dm = row_ok ? __ldg(g.s.d_m + m) : 0;
      const int64_t cm = (row_ok && !g.e.beta_zero) ? __ldg(g.s.c_m + m) : 0;
      const T* Cb = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : __ldg(g.s.h_c + h)) + cm;
      T* Db = static_cast<T*>(g.D) + __ldg(g.s.h_d + h) + dm;

      if (!mbar_wait(accf, j & 1u)) {
        atomicOr(g.status, STATUS_WAIT_TIMEOUT);
        break;
      }
      tc_fence_after();
      // Drain: the S diagonals, smallest weight first, into FP64 (each term
      // is an exact power-of-two multiple of an INT32); both 16-column loads
      // of a diagonal are in flight together.
      double v[OZ_EPI_COLS];
#pragma unroll
      for (int jj = 0; jj < OZ_EPI_COLS; ++jj) v[jj] = 0.0;
#pragma unroll
      for (int gd = S - 1; gd >= 0; --gd) {
        uint32_t r[OZ_EPI_COLS / 16][16];
#pragma unroll
        for (int c = 0; c < OZ_EPI_COLS / 16; ++c)
          tmem_ld_32x32b_x16(tmem + lane_addr + (uint32_t)(gd * OZ_BN + col0 + c * 16), r[c]);
        tmem_ld_wait();
        const double w = pow2(-8 * gd - 12);
#pragma unroll
        for (int c = 0; c < OZ_EPI_COLS / 16; ++c)
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) v[c * 16 + jj] += (double)(int)r[c][jj] * w;
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_empty);

      // x = v 2^(em + en), rounded once (as ldexp would).
#pragma unroll
      for (int nn = 0; nn < OZ_EPI_COLS; ++nn) {
        const int64_t n = n0 + nn;
        const bool col_ok = n < g.N;
        const int en = __shfl_sync(0xffffffffu, en_r, nn);
        const int64_t dn = __shfl_sync(0xffffffffu, dn_r, nn);
        const int64_t cn = __shfl_sync(0xffffffffu, cn_r, nn);
        const int sc = em + en;
        double x;
        if (em == EXP_NONFINITE || en == EXP_NONFINITE) x = __longlong_as_double(0x7ff8000000000000ll);
        else if (sc >= -1022 && sc <= 1023) x = v[nn] * pow2(sc);
        else x = ldexp(v[nn], sc);
        if constexpr (CPLX) {
          const double other = __shfl_xor_sync(0xffffffffu, x, 1);
          if (row_ok && (lane & 1) == 0 && col_ok) epilogue_store<double, true>(g.e, x, other, Cb + cn, Db + dn);
        } else {
          if (row_ok && col_ok) epilogue_store<double, false>(g.e, x, 0.0, Cb + cn, Db + dn);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  // After a timeout: wait (bounded) for the copies still in flight into the
  // stages the MMA warp did not consume.
  if (warp == 0 && lane == 0 && consumed_s != 0xffffffffu) {
    for (uint32_t k = consumed_s; k < issued_a; ++k)
      (void)mbar_wait(&full_a[k % Cfg::A_STAGES], (k / Cfg::A_STAGES) & 1u);
    for (uint32_t k = consumed_s; k < issued_b; ++k)
      (void)mbar_wait(&full_b[k % Cfg::B_STAGES], (k / Cfg::B_STAGES) & 1u);
  }
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, Cfg::TMEM_COLS);
  }
}

template <int S, bool CPLX>
cudaError_t run_gemm(const GemmArgs& g, const OzakiLayout& L, const void* ap, const void* bp, const int* ea,
                     const int* eb, int kb0, int kb1, cudaStream_t st) {
  using Cfg = OzCfg<S>;
  CUtensorMap ma, mb;
  if (!make_map_2d(&ma, ap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L.k_pad, (int64_t)S * L.H * L.m_pad, OZ_SK, OZ_BM,
                   CU_TENSOR_MAP_SWIZZLE_64B))
    return cudaErrorInvalidValue;
  if (!make_map_2d(&mb, bp, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L.k_pad, (int64_t)S * L.H * L.n_pad, OZ_SK, OZ_BN,
                   CU_TENSOR_MAP_SWIZZLE_64B))
    return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(ozaki_gemm_kernel<S, CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t ntiles = (L.n_pad / OZ_BN) * (L.m_pad / OZ_BM) * L.H;
  const unsigned grid = (unsigned)(ntiles < sms ? ntiles : sms);
  ozaki_gemm_kernel<S, CPLX><<<grid, OZ_THREADS, Cfg::SMEM, st>>>(ma, mb, g, ea, eb, L.m_emb, L.m_pad, L.n_pad, L.exp_a_pad,
                                                           kb0, kb1);
  return cudaGetLastError();
}

template <bool CPLX>
cudaError_t gemm_dispatch(const GemmArgs& g, const OzakiLayout& L, const void* ap, const void* bp, const int* ea,
                          const int* eb, int kb0, int kb1, cudaStream_t st) {
  switch (L.slices) {
    case 4: return run_gemm<4, CPLX>(g, L, ap, bp, ea, eb, kb0, kb1, st);
    case 5: return run_gemm<5, CPLX>(g, L, ap, bp, ea, eb, kb0, kb1, st);
    case 6: return run_gemm<6, CPLX>(g, L, ap, bp, ea, eb, kb0, kb1, st);
    case 7: return run_gemm<7, CPLX>(g, L, ap, bp, ea, eb, kb0, kb1, st);
    case 8: return run_gemm<8, CPLX>(g, L, ap, bp, ea, eb, kb0, kb1, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

OzakiLayout ozaki_layout(int slices, bool cplx, int64_t M, int64_t N, int64_t K, int64_t H) {
  OzakiLayout L{};
  L.slices = slices;
  L.cplx = cplx ? 1 : 0;
  L.m_emb = cplx ? 2 * M : M;
  // Complex depth: real parts in [0, K), imaginary parts in [k_half, k_half + K).
  L.k_half = cplx ? (K + OZ_BK - 1) / OZ_BK * OZ_BK : K;
  L.k_emb = cplx ? 2 * L.k_half : K;
  L.m_pad = (L.m_emb + OZ_BM - 1) / OZ_BM * OZ_BM;
  L.n_pad = (N + OZ_BN - 1) / OZ_BN * OZ_BN;
  L.k_pad = (L.k_emb + OZ_BK - 1) / OZ_BK * OZ_BK;
  L.exp_a_pad = (M + 31) / 32 * 32 + 32;
  L.H = H;
  // INT32 exactness: S * k * 128^2 < 2^31 over one chunk of k-blocks.
  int64_t kmax = (((int64_t)1 << 31) - 1) / ((int64_t)slices * 128 * 128);
  L.kb_chunk = (int)(kmax / OZ_BK);
  if (L.kb_chunk < 1) L.kb_chunk = 1;
  return L;
}

size_t ozaki_workspace_bytes(const OzakiLayout& L) {
  const size_t pa = (size_t)L.slices * L.H * L.m_pad * L.k_pad;
  const size_t pb = (size_t)L.slices * L.H * L.n_pad * L.k_pad;
  const size_t ex = ((size_t)L.H * L.exp_a_pad + (size_t)L.H * L.n_pad) * 4;
  return pa + pb + ex + 4 * 256;
}

// Exponent scan + slicing of one operand (rows = M for A', N for B'), with the
// batch-innermost variants when the batch index has the smallest stride.
template <bool CPLX>
static void pack_operand(const double* X, const int64_t* rows_s, const int64_t* k_s, const int64_t* h_s, int64_t nrows,
                         int64_t K, const OzakiLayout& L, int64_t exp_pad, int64_t rows_pad,
                         int kfast, int hfast, int which, int conj, int* exps, int8_t* planes, cudaStream_t st) {
  const size_t one_pass = oz_hfast_smem(CPLX, K);
  // Complex rows: rows_pad / 2 for A' (two embedded rows each), rows_pad for B'.
  const int64_t crows = CPLX && which == 0 ? rows_pad / 2 : rows_pad;
  const int64_t rows = exp_pad > crows ? exp_pad : crows;
  const int64_t blocks = rows * ((L.H + OZ_HB - 1) / OZ_HB);
  if (hfast && one_pass <= OZ_HFAST_SMEM_MAX && blocks <= 0x7fffffff) {
    const dim3 grid((unsigned)blocks);
    const int64_t kw = CPLX ? L.k_half : L.k_pad;
    auto kern = which == 0 ? ozaki_pack_hfast_kernel<CPLX, 0> : ozaki_pack_hfast_kernel<CPLX, 1>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)one_pass);
    kern<<<grid, 256, one_pass, st>>>(X, rows_s, k_s, h_s, nrows, crows, K, kw, rows_pad, exp_pad, L.k_pad,
                                      L.k_half, L.H, conj, L.slices, exps, planes);
  } else if (hfast) {
    ozaki_exp_hfast_kernel<CPLX><<<dim3((unsigned)exp_pad, (unsigned)((L.H + 31) / 32)), 256, 0, st>>>(
        X, rows_s, k_s, h_s, nrows, K, exp_pad, L.H, exps);
    if constexpr (CPLX) {
      // Complex rows: rows_pad / 2 for A' (two embedded rows each), rows_pad for B'.
      const dim3 grid((unsigned)(L.k_half / 64), (unsigned)(which == 0 ? rows_pad / 2 : rows_pad),
                      (unsigned)((L.H + 31) / 32));
      if (which == 0)
        ozaki_slice_hfast_c64_kernel<0><<<grid, 256, 0, st>>>(X, rows_s, k_s, h_s, exps, nrows, K, L.k_half, rows_pad,
                                                               exp_pad, L.k_pad, L.H, conj, L.slices, planes);
      else
        ozaki_slice_hfast_c64_kernel<1><<<grid, 256, 0, st>>>(X, rows_s, k_s, h_s, exps, nrows, K, L.k_half, rows_pad,
                                                               exp_pad, L.k_pad, L.H, conj, L.slices, planes);
    } else {
      ozaki_slice_hfast_kernel<<<dim3((unsigned)(L.k_pad / 64), (unsigned)rows_pad, (unsigned)((L.H + 31) / 32)),
                                 256, 0, st>>>(X, rows_s, k_s, h_s, exps, nrows, K, rows_pad, exp_pad, L.k_pad, L.H,
                                               L.slices, planes);
    }
  } else {
    ozaki_exp_kernel<CPLX><<<dim3((unsigned)((nrows + 31) / 32), (unsigned)L.H), 256, 0, st>>>(
        X, rows_s, k_s, h_s, nrows, K, exp_pad, kfast, exps);
    if constexpr (CPLX) {
      // Complex rows: rows_pad / 2 for A' (two embedded rows each), rows_pad for B'.
      const int64_t crows = which == 0 ? rows_pad / 2 : rows_pad;
      const dim3 grid((unsigned)(L.k_half / 64), (unsigned)(crows / 32), (unsigned)L.H);
      if (which == 0)
        ozaki_slice_c64_kernel<0><<<grid, 256, 0, st>>>(X, rows_s, k_s, h_s, exps, nrows, K, L.k_half, rows_pad,
                                                         exp_pad, L.k_pad, L.H, kfast, conj, L.slices, planes);
      else
        ozaki_slice_c64_kernel<1><<<grid, 256, 0, st>>>(X, rows_s, k_s, h_s, exps, nrows, K, L.k_half, rows_pad,
                                                         exp_pad, L.k_pad, L.H, kfast, conj, L.slices, planes);
    } else {
      ozaki_slice_kernel<<<dim3((unsigned)(L.k_pad / 64), (unsigned)(rows_pad / 32), (unsigned)L.H), 256, 0, st>>>(
          X, rows_s, k_s, h_s, exps, nrows, K, rows_pad, exp_pad, L.k_pad, L.H, kfast, L.slices, planes);
    }
  }
}

cudaError_t launch_ozaki_pack(const GemmArgs& g, const OzakiLayout& L, void* ws, cudaStream_t st, cudaStream_t st_b) {
  int8_t* ap = static_cast<int8_t*>(ws);
  int8_t* bp = ap + (size_t)L.slices * L.H * L.m_pad * L.k_pad;
  int* ea = reinterpret_cast<int*>(bp + (size_t)L.slices * L.H * L.n_pad * L.k_pad);
  int* eb = ea + L.H * L.exp_a_pad;
  if (L.H > 65535) return cudaErrorInvalidConfiguration;
  const double* A = static_cast<const double*>(g.A);
  const double* B = static_cast<const double*>(g.B);
  // Row exponents of A (per complex row) and column exponents of B.
  if (L.cplx) {
    pack_operand<true>(A, g.s.a_m, g.s.a_k, g.s.h_a, g.M, g.K, L, L.exp_a_pad, L.m_pad, g.a_kfast, L.a_hfast,
                       0, g.conj_a, ea, ap, st);
    pack_operand<true>(B, g.s.b_n, g.s.b_k, g.s.h_b, g.N, g.K, L, L.n_pad, L.n_pad, g.b_kfast, L.b_hfast, 1,
                       g.conj_b, eb, bp, st_b);
  } else {
    pack_operand<false>(A, g.s.a_m, g.s.a_k, g.s.h_a, g.M, g.K, L, L.exp_a_pad, L.m_pad, g.a_kfast,
                        L.a_hfast, 0, 0, ea, ap, st);
    pack_operand<false>(B, g.s.b_n, g.s.b_k, g.s.h_b, g.N, g.K, L, L.n_pad, L.n_pad, g.b_kfast, L.b_hfast, 1, 0,
                        eb, bp, st_b);
  }
  return cudaGetLastError();
}

cudaError_t launch_ozaki_gemm(const GemmArgs& g, const OzakiLayout& L, const void* ws, int kb0, int kb1,
                              cudaStream_t st) {
  const int8_t* ap = static_cast<const int8_t*>(ws);
  const int8_t* bp = ap + (size_t)L.slices * L.H * L.m_pad * L.k_pad;
  const int* ea = reinterpret_cast<const int*>(bp + (size_t)L.slices * L.H * L.n_pad * L.k_pad);
  const int* eb = ea + L.H * L.exp_a_pad;
  if ((int64_t)L.slices * L.H * (L.m_pad > L.n_pad ? L.m_pad : L.n_pad) >= (int64_t)1 << 31)
    return cudaErrorInvalidValue;
  if (L.H > 65535) return cudaErrorInvalidConfiguration;
  if (L.cplx) return gemm_dispatch<true>(g, L, ap, bp, ea, eb, kb0, kb1, st);
  return gemm_dispatch<false>(g, L, ap, bp, ea, eb, kb0, kb1, st);
}

namespace {

// Tensor-pipe probe: one CTA per SM, one thread issuing `iters` dense
// 128 x 256 tcgen05.mma products (kind::i8 with K = 32, or kind::f16 BF16
// with K = 16) from one shared-memory operand pair into one TMEM accumulator,
// then a commit and a bounded wait. No memory traffic beyond the CTA's own
// shared memory: the measured rate is the pipe's.
__global__ void __launch_bounds__(128, 1) tc_probe_kernel(int int8, int iters, unsigned* status) {
  __shared__ __align__(1024) uint8_t ops[8192 + 16384];  // A: 128 rows x 64 B, B: 256 rows x 64 B
  __shared__ uint64_t bar;
  __shared__ uint32_t slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < (8192 + 16384) / 16; i += 128) reinterpret_cast<uint4*>(ops)[i] = make_uint4(0, 0, 0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    tmem_alloc(&slot, 256);
    tmem_relinquish();
  }
  if (tid == 32) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = slot;
  if (tid == 0) {
    const uint64_t ad = sdesc_sw64(smem_u32(ops)), bd = sdesc_sw64(smem_u32(ops + 8192));
    const uint32_t idesc = int8 ? idesc_i8(128, 256) : ((1u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) |
                                                         ((128u >> 4) << 24));
    for (int it = 0; it < iters; ++it) {
      const uint64_t k = (uint64_t)(2 * (it & 1));  // the two 32-byte K steps of the 64-byte rows
      if (int8)
        umma_i8(tmem, ad + k, bd + k, idesc, it > 0 ? 1u : 0u);
      else
        umma_bf16(tmem, ad + k, bd + k, idesc, it > 0 ? 1u : 0u);
    }
    umma_commit(&bar);
    if (!mbar_wait(&bar, 0)) atomicOr(status, STATUS_WAIT_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

}  // namespace

cudaError_t launch_tc_probe(int int8, int blocks, int iters, unsigned* status, cudaStream_t st, double* ops) {
  // Unused dynamic shared memory keeps one CTA per SM.
  constexpr int kPad = 160 * 1024;
  const cudaError_t e = cudaFuncSetAttribute(tc_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPad);
  if (e != cudaSuccess) return e;
  tc_probe_kernel<<<blocks, 128, kPad, st>>>(int8, iters, status);
  *ops = (double)blocks * iters * 2.0 * 128 * 256 * (int8 ? 32 : 16);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace tprims
