// Split-precision f32 contraction on the sm_100a tensor cores.
//
// f32 operands are split into BF16 planes, x = x0 + x1 (+ x2), and the
// product is accumulated in FP32 from a subset of the plane products:
//   bf16x3: x0*y0 + x0*y1 + x1*y0                       (2 planes, 3 products)
//   bf16x6: bf16x3 + x0*y2 + x1*y1 + x2*y0              (3 planes, 6 products)
// Each plane keeps the next 8 significant bits of the remainder, so bf16x6
// carries 24 bits (the f32 significand) and drops only terms below 2^-24 of
// the product; bf16x3 carries 16 bits.
//
// Two kernels:
//  * split_pack: gathers A' (or B') through its scatter vectors (the packing of
//    crates/tprims-kernel/src/pack/pack.rs:152-203, here into HBM once per
//    call), transposes through shared memory so that reads run along the
//    operand's unit-stride index and writes along k, splits, and writes the
//    planes K-major, zero-padded to whole tiles.
//  * tc_bf16_gemm: one CTA per 128 x BN output tile. Warp 0 issues TMA tile
//    loads (SWIZZLE_64B, 32 k per stage) into a multi-stage ring; warp 1 owns
//    the TMEM accumulators and issues tcgen05.mma kind::f16 (BF16 in, FP32
//    accumulate) from one thread; warps 2-9 drain the accumulators with
//    tcgen05.ld into FP32 registers (two-level accumulation, see below) and
//    apply the scatter epilogue D = op_D(alpha*acc + beta*C)
//    (pack/writeback.rs:311-486). Every mbarrier wait is bounded by
//    %globaltimer; a timeout sets a status bit and the kernel drains and
//    returns. No cluster, no multicast.
#include <cuda.h>
#include <cuda_bf16.h>

#include "tc_common.cuh"

namespace tprims {
namespace dev {

namespace {

using namespace tc;

constexpr int TC_BM = 128;
constexpr int TC_BK = 32;  // BF16 elements per stage row: 64 bytes = one SWIZZLE_64B atom

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void split3(float x, __nv_bfloat16& p0, __nv_bfloat16& p1, __nv_bfloat16& p2) {
  p0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(p0);
  p1 = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(p1);
  p2 = __float2bfloat16_rn(r2);
}

// Gather + split + K-major write of one 32-row x 64-k tile.
__global__ void __launch_bounds__(256) split_pack_kernel(const float* __restrict__ X, const int64_t* __restrict__ rows_scat,
                                                         const int64_t* __restrict__ k_scat,
                                                         const int64_t* __restrict__ h_scat,
                                                         const int64_t* __restrict__ rows_blk,
                                                         const int64_t* __restrict__ k_blk, int64_t nrows, int64_t K,
                                                         int64_t rows_pad, int64_t k_pad, int64_t H, int kfast,
                                                         int planes, __nv_bfloat16* __restrict__ out) {
  __shared__ float tile[32][65];
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.y * 32, k0 = (int64_t)blockIdx.x * 64, h = blockIdx.z;
  const float* base = X + h_scat[h];
  // A whole tile on regular blocks (32 rows; two 32-deep k blocks of one
  // arithmetic run): addressed from one base offset and two strides, with
  // float4 loads along a unit-stride fast index when aligned.
  int64_t rs = SCATTER_IRREGULAR, ks = SCATTER_IRREGULAR;
  if (rows_blk && k_blk && r0 + 32 <= nrows && k0 + 64 <= K) {
    rs = rows_blk[blockIdx.y];
    const int64_t k1 = k_blk[2 * blockIdx.x], k2 = k_blk[2 * blockIdx.x + 1];
    if (k1 != SCATTER_IRREGULAR && k1 == k2 && k_scat[k0 + 32] - k_scat[k0] == 32 * k1) ks = k1;
  }
  if (rs != SCATTER_IRREGULAR && ks != SCATTER_IRREGULAR) {
    const float* tb = base + rows_scat[r0] + k_scat[k0];
    const int64_t fs = kfast ? ks : rs, ss = kfast ? rs : ks;
    if (fs == 1 && (reinterpret_cast<uintptr_t>(tb) & 15) == 0 && (ss & 3) == 0) {
      // kfast: 16 threads per row (64 k); otherwise 8 threads per k column (32 rows).
      const int tpr = kfast ? 16 : 8;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int a0 = (tid % tpr) * 4, b = tid / tpr + j * (256 / tpr);
        const float4 v = __ldg(reinterpret_cast<const float4*>(tb + b * ss + a0));
        const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (kfast)
            tile[b][a0 + q] = e[q];
          else
            tile[a0 + q][b] = e[q];
        }
      }
    } else {
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
        tile[rr][kk] = __ldg(tb + rr * rs + kk * ks);
      }
    }
  } else {
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
      float v = 0.f;
      if (r < nrows && k < K) v = base[rows_scat[r] + k_scat[k]];
      tile[rr][kk] = v;
    }
  }
  __syncthreads();
  const int64_t plane_stride = H * rows_pad * k_pad;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int p = tid + 256 * j;
    const int rr = p / 32, kp = p % 32;
    __nv_bfloat16 a0, a1, a2, b0, b1, b2;
    split3(tile[rr][2 * kp], a0, a1, a2);
    split3(tile[rr][2 * kp + 1], b0, b1, b2);
    const int64_t off = (h * rows_pad + r0 + rr) * k_pad + k0 + 2 * kp;
    __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + off);
    o[0] = __halves2bfloat162(a0, b0);
    reinterpret_cast<__nv_bfloat162*>(out + plane_stride + off)[0] = __halves2bfloat162(a1, b1);
    if (planes > 2) reinterpret_cast<__nv_bfloat162*>(out + 2 * plane_stride + off)[0] = __halves2bfloat162(a2, b2);
  }
}

template <int S>
struct Pairs;
template <>
struct Pairs<2> {
  static constexpr int N = 3;
  __device__ static inline int a(int p) { return p == 2 ? 1 : 0; }
  __device__ static inline int b(int p) { return p == 1 ? 1 : 0; }
};
template <>
struct Pairs<3> {
  static constexpr int N = 6;
  // (0,0) (0,1) (1,0) (0,2) (1,1) (2,0)
  __device__ static inline int a(int p) { return p < 2 ? 0 : (p == 2 ? 1 : (p == 3 ? 0 : (p == 4 ? 1 : 2))); }
  __device__ static inline int b(int p) { return p == 0 ? 0 : (p == 1 ? 1 : (p == 2 ? 0 : (p == 3 ? 2 : (p == 4 ? 1 : 0)))); }
};

// Tile order: within a batch entry, tiles go in groups of TILE_GROUP_M m-tiles
// (the last group may be narrower); inside a group the m-tile is fastest, then
// the n-tile. A wave of 148 CTAs then covers a block of about 16 A row panels
// by 9 B column panels instead of 9 row panels by every column panel, so the
// B planes a wave reads stay in L2 for the next wave of the same group.
constexpr int TILE_GROUP_M = 16;

__host__ __device__ inline void tile_coords(int64_t tile, int64_t tiles_m, int64_t tiles_n, int64_t& h, int64_t& mt,
                                            int64_t& nt) {
  const int64_t per_h = tiles_m * tiles_n;
  h = tile / per_h;
  const int64_t t = tile % per_h;
  const int64_t group = t / (TILE_GROUP_M * tiles_n);
  const int64_t first_m = group * TILE_GROUP_M;
  const int64_t gm = tiles_m - first_m < TILE_GROUP_M ? tiles_m - first_m : TILE_GROUP_M;
  const int64_t local = t - group * TILE_GROUP_M * tiles_n;
  mt = first_m + local % gm;
  nt = local / gm;
}

template <int S, int BN>
struct TcCfg {
  static constexpr int A_TILE = TC_BM * TC_BK * 2;  // bytes of one A plane tile
  static constexpr int B_TILE = BN * TC_BK * 2;
  static constexpr int STAGE = S * (A_TILE + B_TILE);
  static constexpr int STAGES = (S == 3) ? 3 : 4;
  static constexpr int RING = STAGES * STAGE;
  static constexpr int SCAT = 2 * BN * 8;  // d_n, c_n of the tile
  static constexpr int BAR = (2 * STAGES + 3) * 8 + 16;
  static constexpr int SMEM = 1024 + RING + SCAT + BAR;
  static constexpr int EPI_WARPS = 8;  // two per TMEM lane quarter, each half of the columns
  static constexpr int THREADS = 64 + 32 * EPI_WARPS;
  static constexpr int COLS_PER_THREAD = BN / 2;
};

// Two-level accumulation. The tensor core's FP32 accumulate truncates, so its
// error grows with the number of MMA steps folded into one accumulator. The
// leading product x0*y0 therefore goes into a "main" TMEM accumulator that is
// restarted every CK k-blocks; the epilogue warps drain each chunk into FP32
// registers with round-to-nearest adds. The cross terms, 2^-8 smaller, go to
// a second ("corr") accumulator that lives for the whole K loop. TMEM columns:
// main [0, BN), corr [BN, 2 BN).
//
// Tail split: the grid is 1-D; CTAs [0, whole) own one tile each over all of
// K, and the last `tail` tiles (those that would run as a partly filled last
// wave) are split into `parts` K ranges of whole CK chunks, one CTA each. A
// tail CTA writes its FP32 sum to partial[(tail tile * parts + part) * TC_BM
// * BN + col * TC_BM + row] and split_tail_reduce_kernel adds the parts in
// order and applies the epilogue.
template <int S, int BN, int CK>
__global__ void __launch_bounds__(TcCfg<S, BN>::THREADS, 1)
tc_bf16_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g,
                    int64_t m_pad, int64_t n_pad, int64_t k_pad, int64_t whole, int parts, float* partial) {
  using Cfg = TcCfg<S, BN>;
  constexpr int CPT = Cfg::COLS_PER_THREAD;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* ring = smem;
  int64_t* dn_s = reinterpret_cast<int64_t*>(smem + Cfg::RING);
  int64_t* cn_s = dn_s + BN;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Cfg::RING + Cfg::SCAT);
  uint64_t* empty = full + Cfg::STAGES;
  uint64_t* main_full = empty + Cfg::STAGES;
  uint64_t* main_empty = main_full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(main_empty + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t tiles_n = n_pad / BN, tiles_m = m_pad / TC_BM;
  const int nk_all = (int)(k_pad / TC_BK);
  int64_t tile = blockIdx.x;
  int part = -1;  // -1: the whole K range
  int kb_lo = 0, kb_hi = nk_all;
  if ((int64_t)blockIdx.x >= whole) {
    const int64_t j = (int64_t)blockIdx.x - whole;
    tile = whole + j / parts;
    part = (int)(j % parts);
    const int per = ((nk_all + parts - 1) / parts + CK - 1) / CK * CK;  // whole chunks per part
    kb_lo = part * per;
    kb_hi = kb_lo + per < nk_all ? kb_lo + per : nk_all;
  }
  int64_t h, mt, nt;
  tile_coords(tile, tiles_m, tiles_n, h, mt, nt);
  const int64_t m0 = mt * TC_BM, n0 = nt * BN;
  const int nk = kb_hi - kb_lo;  // k-blocks of this CTA (>= 1)
  const int nchunks = (nk + CK - 1) / CK;

  if (warp == 0 && lane == 0) {
    for (int i = 0; i < Cfg::STAGES; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(main_full, 1);
    mbar_init(main_empty, Cfg::EPI_WARPS);
    fence_barrier_init();
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 2 * BN);
    tmem_relinquish();
  }
  if (warp >= 2) {
    for (int i = tid - 64; i < BN; i += 32 * Cfg::EPI_WARPS) {
      const int64_t n = n0 + i;
      const bool ok = n < g.N;
      dn_s[i] = ok ? g.s.d_n[n] : 0;
      cn_s[i] = ok ? g.s.c_n[n] : 0;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_main = tmem, tmem_corr = tmem + BN;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = 0; kb < nk; ++kb) {
        const int st = kb % Cfg::STAGES;
        const uint32_t round = (uint32_t)(kb / Cfg::STAGES);
        if (!mbar_wait(&empty[st], (round & 1u) ^ 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          break;
        }
        mbar_arrive_expect_tx(&full[st], (uint32_t)Cfg::STAGE);
        uint8_t* sbase = ring + st * Cfg::STAGE;
        const int kx = (kb_lo + kb) * TC_BK;
#pragma unroll
        for (int p = 0; p < S; ++p)
          tma_load_2d(sbase + p * Cfg::A_TILE, &tmA, &full[st], kx, (int)((p * g.H + h) * m_pad + m0));
#pragma unroll
        for (int p = 0; p < S; ++p)
          tma_load_2d(sbase + S * Cfg::A_TILE + p * Cfg::B_TILE, &tmB, &full[st], kx,
                      (int)((p * g.H + h) * n_pad + n0));
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t IDESC = idesc_bf16(TC_BM, BN);
      bool ok = true;
      for (int kb = 0; kb < nk && ok; ++kb) {
        const int st = kb % Cfg::STAGES;
        const uint32_t round = (uint32_t)(kb / Cfg::STAGES);
        if (!mbar_wait(&full[st], round & 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          break;
        }
        tc_fence_after();
        const uint32_t sbase = smem_u32(ring + st * Cfg::STAGE);
        // Cross terms first: they overlap the drain of the previous chunk.
#pragma unroll
        for (int p = 1; p < Pairs<S>::N; ++p) {
          const uint64_t ad = sdesc_sw64(sbase + Pairs<S>::a(p) * Cfg::A_TILE);
          const uint64_t bd = sdesc_sw64(sbase + S * Cfg::A_TILE + Pairs<S>::b(p) * Cfg::B_TILE);
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk)
            umma_bf16(tmem_corr, ad + 2 * kk, bd + 2 * kk, IDESC, (kb | (p - 1) | kk) != 0 ? 1u : 0u);
        }
        const int chunk = kb / CK, in_chunk = kb % CK;
        if (in_chunk == 0 && !mbar_wait(main_empty, ((uint32_t)chunk & 1u) ^ 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          ok = false;
        }
        tc_fence_after();
        {
          const uint64_t ad = sdesc_sw64(sbase);
          const uint64_t bd = sdesc_sw64(sbase + S * Cfg::A_TILE);
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk)
            umma_bf16(tmem_main, ad + 2 * kk, bd + 2 * kk, IDESC, (in_chunk | kk) != 0 ? 1u : 0u);
        }
        umma_commit(&empty[st]);
        if (in_chunk == CK - 1 || kb == nk - 1) umma_commit(main_full);
      }
      if (!ok) umma_commit(main_full);
    }
  } else {
    // Epilogue: warp w reads TMEM lanes 32*(w%4) .. +31 (tile rows) and half
    // of the columns; it keeps the running FP32 sum of its 128 outputs.
    const int lane_base = 32 * (warp & 3);
    const int col0 = ((warp - 2) >> 2) * CPT;
    const uint32_t lane_addr = (uint32_t)lane_base << 16;
    float run[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) run[j] = 0.f;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      if (!mbar_wait(main_full, (uint32_t)c & 1u)) {
        atomicOr(g.status, STATUS_WAIT_TIMEOUT);
        ok = false;
        break;
      }
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < CPT / 16; ++q) {
        uint32_t r[16];
        tmem_ld_32x32b_x16(tmem_main + lane_addr + (uint32_t)(col0 + 16 * q), r);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) run[16 * q + j] += __uint_as_float(r[j]);
      }
      tc_fence_before();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(main_empty)) : "memory");
    }
    const int64_t m = m0 + lane_base + lane;
    const bool mok = ok && m < g.M;
    const int64_t dm = mok ? g.s.d_m[m] : 0;
    const int64_t cm = (mok && !g.e.beta_zero) ? g.s.c_m[m] : 0;
    const float* Cb = static_cast<const float*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]) + cm;
    float* Db = static_cast<float*>(g.D) + g.s.h_d[h] + dm;
    float* Pb = part >= 0 ? partial + ((tile - whole) * parts + part) * (int64_t)(TC_BM * BN) + lane_base + lane
                          : nullptr;
    // The last main_full commit also covers every cross-term MMA.
#pragma unroll
    for (int q = 0; q < CPT / 16; ++q) {
      uint32_t r[16];
      tmem_ld_32x32b_x16(tmem_corr + lane_addr + (uint32_t)(col0 + 16 * q), r);
      tmem_ld_wait();
      if (part >= 0) {
        // Tail part: the raw FP32 sum, column-major in the tile (coalesced).
#pragma unroll
        for (int j = 0; j < 16; ++j) Pb[(col0 + 16 * q + j) * TC_BM] = run[16 * q + j] + __uint_as_float(r[j]);
      } else if (mok) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int nn = col0 + 16 * q + j;
          if (n0 + nn < g.N)
            epilogue_store<float, false>(g.e, run[16 * q + j] + __uint_as_float(r[j]), 0.f, Cb + cn_s[nn],
                                         Db + dn_s[nn]);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * BN);
  }
}

// Tail tiles: add the parts in order, then the epilogue through the scatter.
template <int BN>
__global__ void __launch_bounds__(256) split_tail_reduce_kernel(GemmArgs g, const float* __restrict__ partial,
                                                                int64_t whole, int parts, int64_t tail, int64_t m_pad,
                                                                int64_t n_pad) {
  const int64_t tiles_n = n_pad / BN, tiles_m = m_pad / TC_BM;
  const int64_t total = tail * TC_BM * BN;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = idx / (TC_BM * BN), within = idx % (TC_BM * BN);
    const int row = (int)(within % TC_BM), col = (int)(within / TC_BM);
    const int64_t tile = whole + t;
    int64_t h, mt, nt;
    tile_coords(tile, tiles_m, tiles_n, h, mt, nt);
    const int64_t m = mt * TC_BM + row, n = nt * BN + col;
    if (m >= g.M || n >= g.N) continue;
    float v = 0.f;
    for (int p = 0; p < parts; ++p) v += partial[(t * parts + p) * (int64_t)(TC_BM * BN) + within];
    const float* c = static_cast<const float*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h] + g.s.c_m[m] + g.s.c_n[n]);
    float* d = static_cast<float*>(g.D) + g.s.h_d[h] + g.s.d_m[m] + g.s.d_n[n];
    epilogue_store<float, false>(g.e, v, 0.f, c, d);
  }
}

// The tail split for a grid of `tiles` tiles on `sms` SMs (one CTA per SM):
// the tiles of a partly filled last wave are split into `parts` K ranges when
// that fills the wave better; parts = 1 means no split.
struct TailSplit {
  int64_t whole, tail;
  int parts;
};
inline TailSplit tail_split(int64_t tiles, int sms, int nk, int ck) {
  TailSplit t{tiles, 0, 1};
  const int64_t rem = tiles % sms;
  if (rem == 0 || tiles < sms) return t;  // full waves, or one partial wave of whole tiles
  int parts = (int)(sms / rem);
  parts = parts < 4 ? parts : 4;
  // Each part keeps at least two CK chunks and the last part is not empty.
  auto fits = [&](int p) {
    const int per = ((nk + p - 1) / p + ck - 1) / ck * ck;
    return nk >= p * 2 * ck && (p - 1) * per < nk;
  };
  while (parts > 1 && !fits(parts)) --parts;
  if (parts < 2) return t;
  t.whole = tiles - rem;
  t.tail = rem;
  t.parts = parts;
  return t;
}

template <int S, int BN, int CK>
cudaError_t run_tc(const GemmArgs& g, const SplitLayout& L, const void* ap, const void* bp, float* tail_partial,
                   cudaStream_t st) {
  using Cfg = TcCfg<S, BN>;
  CUtensorMap ma, mb;
  if (!make_map_2d(&ma, ap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, L.k_pad, (int64_t)S * L.H * L.m_pad, TC_BK, TC_BM))
    return cudaErrorInvalidValue;
  if (!make_map_2d(&mb, bp, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, L.k_pad, (int64_t)S * L.H * L.n_pad, TC_BK, BN))
    return cudaErrorInvalidValue;
  // Per call: the attribute belongs to the current device's context.
  cudaError_t e =
      cudaFuncSetAttribute(tc_bf16_gemm_kernel<S, BN, CK>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (L.n_pad / BN) * (L.m_pad / TC_BM) * L.H;
  TailSplit ts{tiles, 0, 1};
  if (tail_partial) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    ts = tail_split(tiles, sms, (int)(L.k_pad / TC_BK), CK);
  }
  const int64_t grid = ts.whole + ts.tail * ts.parts;
  tc_bf16_gemm_kernel<S, BN, CK><<<(unsigned)grid, Cfg::THREADS, Cfg::SMEM, st>>>(
      ma, mb, g, L.m_pad, L.n_pad, L.k_pad, ts.whole, ts.parts, tail_partial);
  e = cudaGetLastError();
  if (e != cudaSuccess || ts.tail == 0) return e;
  const int64_t elems = ts.tail * TC_BM * BN;
  const unsigned blocks = (unsigned)((elems + 255) / 256 < 4096 ? (elems + 255) / 256 : 4096);
  split_tail_reduce_kernel<BN><<<blocks, 256, 0, st>>>(g, tail_partial, ts.whole, ts.parts, ts.tail, L.m_pad,
                                                       L.n_pad);
  return cudaGetLastError();
}

}  // namespace

SplitLayout split_layout(int scheme, int64_t M, int64_t N, int64_t K, int64_t H) {
  SplitLayout L;
  L.planes = (scheme == 2) ? 3 : 2;
  L.m_pad = (M + TC_BM - 1) / TC_BM * TC_BM;
  L.n_pad = (N + 255) / 256 * 256;
  L.k_pad = (K + 63) / 64 * 64;
  L.H = H;
  return L;
}

size_t split_workspace_bytes(const SplitLayout& L) {
  return (size_t)L.planes * (size_t)L.H * (size_t)(L.m_pad + L.n_pad) * (size_t)L.k_pad * 2 + 256;
}

cudaError_t launch_split_pack_f32(const GemmArgs& g, int which, const SplitLayout& L, void* planes, cudaStream_t st) {
  const bool a = which == 0;
  const int64_t rows_pad = a ? L.m_pad : L.n_pad;
  dim3 grid((unsigned)(L.k_pad / 64), (unsigned)(rows_pad / 32), (unsigned)L.H);
  if (L.H > 65535 || rows_pad / 32 > 65535) return cudaErrorInvalidConfiguration;
  split_pack_kernel<<<grid, 256, 0, st>>>(static_cast<const float*>(a ? g.A : g.B), a ? g.s.a_m : g.s.b_n,
                                          a ? g.s.a_k : g.s.b_k, a ? g.s.h_a : g.s.h_b, a ? g.s.blk_a_m : g.s.blk_b_n,
                                          a ? g.s.blk_a_k : g.s.blk_b_k, a ? g.M : g.N, g.K, rows_pad,
                                          L.k_pad, L.H, a ? g.a_kfast : g.b_kfast, L.planes,
                                          static_cast<__nv_bfloat16*>(planes));
  return cudaGetLastError();
}

int split_tail_parts(const SplitLayout& L, int num_sms) {
  const int64_t tiles = (L.n_pad / 256) * (L.m_pad / TC_BM) * L.H;
  return tail_split(tiles, num_sms, (int)(L.k_pad / TC_BK), 4).parts;
}

size_t split_tail_bytes(const SplitLayout& L, int num_sms) {
  // At most one wave of tail parts (tail * parts <= num_sms) of 128 x 256 FP32.
  (void)L;
  return (size_t)num_sms * TC_BM * 256 * sizeof(float) + 256;
}

cudaError_t launch_tc_bf16_gemm(const GemmArgs& g, const SplitLayout& L, const void* ap, const void* bp, int scheme,
                                cudaStream_t st, void* tail_partial) {
  if ((int64_t)L.planes * L.H * (L.m_pad > L.n_pad ? L.m_pad : L.n_pad) >= (int64_t)1 << 31)
    return cudaErrorInvalidValue;
  if (L.H > 65535) return cudaErrorInvalidConfiguration;
  float* tp = static_cast<float*>(tail_partial);
  if (scheme == 2) return run_tc<3, 256, 4>(g, L, ap, bp, tp, st);
  return run_tc<2, 256, 4>(g, L, ap, bp, tp, st);
}

}  // namespace dev
}  // namespace tprims
