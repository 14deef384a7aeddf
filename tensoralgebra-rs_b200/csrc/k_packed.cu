// Packed plain families: a pack pass gathers each operand through its scatter
// vectors into dense panels, then a tile kernel streams the panels into
// shared memory with TMA tiled loads (cp.async.bulk.tensor, no multicast).
//
// This is the reference's own structure (pack panels, then run micro-kernels
// over them: crates/tprims-kernel/src/pack/pack.rs:152-270 and
// kernels/reference/scalar.rs:31-175) with the panels packed once per call for
// the whole operand. The pack reads each operand once, with threads along
// whichever index is unit-stride and a shared-memory transpose to the panel
// order, so the tile kernels never pay for a general-stride gather: every
// operand byte they read is a dense TMA box.
//
//  * simt_packed_kernel: FP32 FFMA, 128 x 128 tiles, 32-deep stages in a
//    4-stage TMA ring (one producer warp), eight compute warps with 8 x 8
//    outputs per thread; the running sums are restarted every 64 k and added
//    into the totals with round-to-nearest adds (FP32 error near
//    u (sqrt(64) + sqrt(K / 64))). Real f32, and c32 through the 1m embedding.
//  * dmma_packed_kernel: FP64 DMMA (mma.sync m16n8k8) on K-major panels whose
//    128-byte rows TMA swizzles (SWIZZLE_128B), so the fragment reads are free
//    of bank conflicts; real f64 (64 x 64 tiles) and c64 through 3m (three
//    planes, three accumulators, 64 x 32 tiles).
//
// Every mbarrier wait is bounded by %globaltimer; a timeout sets a status bit,
// the kernel stops, waits (again bounded) for its own copies in flight and
// returns.
#include <cuda.h>

#include <climits>

#include "tc_common.cuh"

namespace tprims {
namespace dev {

namespace {

using namespace tc;

// Tile order shared by the packed kernels: groups of 16 m-tiles, m fastest
// inside a group (a wave reuses the B panels of its group from L2).
__device__ inline void packed_tile_coords(int64_t tile, int64_t tiles_m, int64_t tiles_n, int64_t& h, int64_t& mt,
                                          int64_t& nt) {
  constexpr int64_t G = 16;
  const int64_t per_h = tiles_m * tiles_n;
  h = tile / per_h;
  const int64_t t = tile % per_h;
  const int64_t group = t / (G * tiles_n);
  const int64_t first_m = group * G;
  const int64_t gm = tiles_m - first_m < G ? tiles_m - first_m : G;
  const int64_t local = t - group * G * tiles_n;
  mt = first_m + local % gm;
  nt = local / gm;
}

// ------------------------------------------------------------------ pack pass

enum PackMode { PM_ROWS_FAST = 0, PM_K_FAST = 1, PM_1M_A = 2, PM_1M_B = 3, PM_3M = 4 };

struct PanelArgs {
  void* out;
  int64_t rows_pad, k_pad;  // panel extents (of the embedded real problem)
  int64_t plane_stride;     // elements between the planes of 3m
  int64_t H;
  // Block order over the 1-D grid of gx k-tiles x gy row-tiles x H batch
  // entries: batch fastest (hfast, for operands whose batch index has the
  // smallest stride, so CTAs resident together read neighbouring batch
  // entries of the same lines) or k fastest.
  int64_t gx = 0, gy = 0;
  int hfast = 0;
};

// One 32-row x 32-k tile of the source operand (rows = m for A', n for B'):
// loaded with the threads along the operand's unit-stride index, transposed
// through shared memory, written in the panel's order with zero padding.
//   PM_ROWS_FAST: panel [H][k_pad][rows_pad] (FFMA tiles read rows as float4)
//   PM_K_FAST:    panel [H][rows_pad][k_pad] (K-major for the DMMA tiles)
//   PM_3M:        three K-major planes: re, im, re + im
//   PM_1M_A:      [H][k_pad][rows_pad] of the 2M x 2K real embedding
//   PM_1M_B:      [H][k_pad][rows_pad] of the 2K x N real embedding
template <class R, bool CPLX, int MODE>
__global__ void __launch_bounds__(256) plain_pack_kernel(const typename Elem<R, CPLX>::type* __restrict__ X,
                                                         const int64_t* __restrict__ rows_scat,
                                                         const int64_t* __restrict__ k_scat,
                                                         const int64_t* __restrict__ h_scat,
                                                         const int64_t* __restrict__ rows_blk,
                                                         const int64_t* __restrict__ k_blk, int64_t nrows, int64_t K,
                                                         int kfast, int conj, PanelArgs o) {
  using T = typename Elem<R, CPLX>::type;
  __shared__ R tre[32][33];
  __shared__ R tim[CPLX ? 32 : 1][33];
  const int tid = threadIdx.x;
  int64_t bx, by, h;
  {
    const int64_t b = blockIdx.x;
    if (o.hfast) {
      h = b % o.H;
      bx = (b / o.H) % o.gx;
      by = b / o.H / o.gx;
    } else {
      bx = b % o.gx;
      by = (b / o.gx) % o.gy;
      h = b / o.gx / o.gy;
    }
  }
  const int64_t r0 = by * 32, k0 = bx * 32;
  const T* base = X + h_scat[h];
  // A whole tile on regular blocks of both vectors (block size 32 = the
  // tile): one base offset and two strides, 16-byte vectors along a
  // unit-stride fast index when aligned.
  int64_t rs = SCATTER_IRREGULAR, ks = SCATTER_IRREGULAR;
  if (rows_blk && k_blk && r0 + 32 <= nrows && k0 + 32 <= K) {
    rs = rows_blk[by];
    ks = k_blk[bx];
  }
  if (rs != SCATTER_IRREGULAR && ks != SCATTER_IRREGULAR) {
    const T* tb = base + rows_scat[r0] + k_scat[k0];
    const int64_t fs = kfast ? ks : rs, ss = kfast ? rs : ks;  // strides of the fast and the slow index
    constexpr int VEC = 16 / (int)sizeof(T);
    if (VEC > 1 && fs == 1 && (reinterpret_cast<uintptr_t>(tb) & 15) == 0 && ((ss * (int64_t)sizeof(T)) & 15) == 0) {
      constexpr int TPR = 32 / (VEC > 1 ? VEC : 1);  // threads per slow index
#pragma unroll
      for (int j = 0; j < 32 * TPR / 256; ++j) {
        const int a0 = (tid % TPR) * VEC, b = tid / TPR + j * (256 / TPR);
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(tb + b * ss + a0));
        const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
          R re, im;
          Elem<R, CPLX>::load(e + q, re, im);
          if (conj) im = -im;
          const int rr = kfast ? b : a0 + q, kk = kfast ? a0 + q : b;
          tre[rr][kk] = re;
          if (CPLX) tim[rr][kk] = im;
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int a = tid & 31, b = (tid >> 5) + 8 * j;
        R re, im;
        Elem<R, CPLX>::load(tb + a * fs + b * ss, re, im);
        if (conj) im = -im;
        const int rr = kfast ? b : a, kk = kfast ? a : b;
        tre[rr][kk] = re;
        if (CPLX) tim[rr][kk] = im;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int a = tid & 31, b = (tid >> 5) + 8 * j;
      const int rr = kfast ? b : a, kk = kfast ? a : b;
      const int64_t r = r0 + rr, k = k0 + kk;
      R re = R(0), im = R(0);
      if (r < nrows && k < K) {
        Elem<R, CPLX>::load(base + rows_scat[r] + k_scat[k], re, im);
        if (conj) im = -im;
      }
      tre[rr][kk] = re;
      if (CPLX) tim[rr][kk] = im;
    }
  }
  __syncthreads();
  R* out = static_cast<R*>(o.out);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int a = tid & 31, b = (tid >> 5) + 8 * j;
    if (MODE == PM_ROWS_FAST) {
      const int64_t r = r0 + a, k = k0 + b;
      if (k < o.k_pad && r < o.rows_pad) out[(h * o.k_pad + k) * o.rows_pad + r] = tre[a][b];
    } else if (MODE == PM_K_FAST || MODE == PM_3M) {
      const int64_t r = r0 + b, k = k0 + a;
      if (k < o.k_pad && r < o.rows_pad) {
        const int64_t off = (h * o.rows_pad + r) * o.k_pad + k;
        const R re = tre[b][a];
        if (MODE == PM_K_FAST) {
          out[off] = re;
        } else {
          const R im = tim[CPLX ? b : 0][a];
          out[off] = re;
          out[o.plane_stride + off] = im;
          out[2 * o.plane_stride + off] = re + im;
        }
      }
    } else if (MODE == PM_1M_A) {
      // Element (r, k) becomes rows 2r, 2r+1 at depths 2k (re, im) and 2k+1 (-im, re).
      const int64_t r = r0 + a, k = k0 + b;
      const R re = tre[a][b], im = tim[CPLX ? a : 0][b];
      if (2 * r + 1 < o.rows_pad) {
        if (2 * k < o.k_pad) {
          R* p = out + (h * o.k_pad + 2 * k) * o.rows_pad + 2 * r;
          p[0] = re;
          p[1] = im;
        }
        if (2 * k + 1 < o.k_pad) {
          R* p = out + (h * o.k_pad + 2 * k + 1) * o.rows_pad + 2 * r;
          p[0] = -im;
          p[1] = re;
        }
      }
    } else {  // PM_1M_B: element (n, k) becomes depths 2k (re) and 2k+1 (im) of column n
      const int64_t r = r0 + a, k = k0 + b;
      const R re = tre[a][b], im = tim[CPLX ? a : 0][b];
      if (r < o.rows_pad) {
        if (2 * k < o.k_pad) out[(h * o.k_pad + 2 * k) * o.rows_pad + r] = re;
        if (2 * k + 1 < o.k_pad) out[(h * o.k_pad + 2 * k + 1) * o.rows_pad + r] = im;
      }
    }
  }
}

// ------------------------------------------------------------ FFMA tile (f32)

// Tile shapes of the FFMA kernel: 128 rows x BN columns, 32-deep stages (one
// barrier wait and arrival per 32 k), 256 compute threads each with 8 rows x
// BN/16 columns (groups of four columns 64 apart), one producer warp. BN = 128
// runs one CTA per SM (168 registers), BN = 64 two (half the accumulators,
// twice the warps to hide latency). Running sums restart every FLUSH stages
// (64 k).
template <int BN>
struct SpCfg {
  static constexpr int BM = 128, BK = 32, STAGES = 4, FLUSH = 2;
  static constexpr int TN = BN / 16, CG = TN / 4;  // columns per thread, groups of four
  static constexpr int A = BK * BM * 4, B = BK * BN * 4, STAGE = A + B;
  static constexpr int COMPUTE = 256, THREADS = COMPUTE + 32;
  static constexpr int MINB = BN == 128 ? 1 : 2;
  static constexpr int SMEM = 1024 + STAGES * STAGE + (2 * BM + 2 * BN) * 8 + 2 * STAGES * 8 + 16;
};

// Packed pairs of FP32 values (sm_100 f32x2 arithmetic; each half rounds as
// its own IEEE operation).
__device__ __forceinline__ unsigned long long f32x2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f32x2_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f32x2_fma(unsigned long long a, unsigned long long b,
                                                        unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long f32x2_add(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Stores four consecutive rows of one column when D's rows are consecutive in
// memory and the address is 16-byte aligned (the reference's unit-stride
// write-back, pack/writeback.rs:426-486); returns false when it did not.
__device__ inline bool store4_f32(const Epilogue& e, float* d0, const int64_t* dm, float v0, float v1, float v2,
                                  float v3) {
  if (!e.beta_zero || dm[1] != dm[0] + 1 || dm[2] != dm[0] + 2 || dm[3] != dm[0] + 3 ||
      (reinterpret_cast<uintptr_t>(d0) & 15) != 0)
    return false;
  const float a = (float)e.alpha_re;
  float4 v = e.plain ? make_float4(v0, v1, v2, v3) : make_float4(v0 * a, v1 * a, v2 * a, v3 * a);
  *reinterpret_cast<float4*>(d0) = v;
  return true;
}

template <bool ONEM, int BN>
__global__ void __launch_bounds__(SpCfg<BN>::THREADS, SpCfg<BN>::MINB)
simt_packed_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g,
                   int64_t k_pad, int64_t tiles_m, int64_t tiles_n, int64_t kchunk, int splits) {
  using Cfg = SpCfg<BN>;
  constexpr int BM = Cfg::BM, BK = Cfg::BK, STAGES = Cfg::STAGES, TN = Cfg::TN, CG = Cfg::CG;
  using T = typename Elem<float, ONEM>::type;
  constexpr int EROWS = ONEM ? BM / 2 : BM;  // output rows per tile
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* ring = smem;
  int64_t* dm_s = reinterpret_cast<int64_t*>(smem + STAGES * Cfg::STAGE);
  int64_t* cm_s = dm_s + BM;
  int64_t* dn_s = cm_s + BM;
  int64_t* cn_s = dn_s + BN;
  uint64_t* full = reinterpret_cast<uint64_t*>(cn_s + BN);
  uint64_t* empty = full + STAGES;
  int* stop = reinterpret_cast<int*>(empty + STAGES);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t split = (int64_t)blockIdx.x % splits, tile = (int64_t)blockIdx.x / splits;
  int64_t h, mt, nt;
  packed_tile_coords(tile, tiles_m, tiles_n, h, mt, nt);
  const int64_t m0 = mt * BM, n0 = nt * BN, em0 = ONEM ? m0 / 2 : m0;
  const int64_t nkb_all = k_pad / BK;
  const int64_t kb_lo = kchunk ? split * (kchunk / BK) : 0;
  const int64_t kb_hi = kchunk ? min(nkb_all, kb_lo + kchunk / BK) : nkb_all;
  const int nk = (int)(kb_hi - kb_lo);

  if (warp == 8 && lane == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Cfg::COMPUTE / 32);
    }
    fence_barrier_init();
    *stop = nk;
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
  }
  if (tid < EROWS) {
    const int64_t m = em0 + tid;
    const bool ok = m < g.M;
    dm_s[tid] = ok ? g.s.d_m[m] : 0;
    cm_s[tid] = (ok && !g.e.beta_zero) ? g.s.c_m[m] : 0;
  }
  if (tid < BN) {
    const int64_t n = n0 + tid;
    const bool ok = n < g.N;
    dn_s[tid] = ok ? g.s.d_n[n] : 0;
    cn_s[tid] = (ok && !g.e.beta_zero) ? g.s.c_n[n] : 0;
  }
  __syncthreads();

  int issued = 0;
  if (warp == 8) {
    if (lane == 0) {
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES;
        const uint32_t round = (uint32_t)(i / STAGES);
        if (!mbar_wait(&empty[s], (round & 1u) ^ 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          break;
        }
        mbar_arrive_expect_tx(&full[s], (uint32_t)Cfg::STAGE);
        const int y = (int)(h * k_pad + (kb_lo + i) * BK);
        tma_load_2d(ring + s * Cfg::STAGE, &tmA, &full[s], (int)m0, y);
        tma_load_2d(ring + s * Cfg::STAGE + Cfg::A, &tmB, &full[s], (int)n0, y);
        issued = i + 1;
      }
    }
  } else {
    const int tx = tid & 15, ty = tid >> 4;
    // Accumulators in packed pairs of rows (fma.rn.f32x2: two IEEE FMAs per
    // instruction, half the issue slots of scalar FFMA): pair p holds rows
    // 2p and 2p + 1 of the thread's eight rows for one column.
    unsigned long long totp[4][TN], accp[4][TN];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        totp[p][j] = 0ull;
        accp[p][j] = 0ull;
      }
    for (int i = 0; i < nk; ++i) {
      const int s = i % STAGES;
      const uint32_t round = (uint32_t)(i / STAGES);
      if (!mbar_wait(&full[s], round & 1u)) {
        atomicOr(g.status, STATUS_WAIT_TIMEOUT);
        atomicMin(stop, i);
        break;
      }
      const float* As = reinterpret_cast<const float*>(ring + s * Cfg::STAGE);
      const float* Bs = reinterpret_cast<const float*>(ring + s * Cfg::STAGE + Cfg::A);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        const ulonglong2 a0 = *reinterpret_cast<const ulonglong2*>(As + kk * BM + tx * 4);
        const ulonglong2 a1 = *reinterpret_cast<const ulonglong2*>(As + kk * BM + 64 + tx * 4);
        const unsigned long long ap[4] = {a0.x, a0.y, a1.x, a1.y};
        unsigned long long bd[TN];  // each column value duplicated into both halves
#pragma unroll
        for (int c = 0; c < CG; ++c) {
          const float4 b = *reinterpret_cast<const float4*>(Bs + kk * BN + 64 * c + ty * 4);
          bd[4 * c] = f32x2_pack(b.x, b.x);
          bd[4 * c + 1] = f32x2_pack(b.y, b.y);
          bd[4 * c + 2] = f32x2_pack(b.z, b.z);
          bd[4 * c + 3] = f32x2_pack(b.w, b.w);
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int jj = 0; jj < TN; ++jj) accp[p][jj] = f32x2_fma(ap[p], bd[jj], accp[p][jj]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if ((i + 1) % Cfg::FLUSH == 0) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int jj = 0; jj < TN; ++jj) {
            totp[p][jj] = f32x2_add(totp[p][jj], accp[p][jj]);
            accp[p][jj] = 0ull;
          }
      }
    }
    float tot[8][TN];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int jj = 0; jj < TN; ++jj) f32x2_unpack(f32x2_add(totp[p][jj], accp[p][jj]), tot[2 * p][jj], tot[2 * p + 1][jj]);

    // Epilogue. Thread rows: tx*4 + [0,4) and 64 + tx*4 + [0,4); columns
    // 64 c + ty*4 + [0,4) for each group c.
    const T* Cb = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]);
    T* Db = static_cast<T*>(g.D) + g.s.h_d[h];
#pragma unroll
    for (int jj = 0; jj < TN; ++jj) {
      const int cc = 64 * (jj / 4) + ty * 4 + (jj % 4);
      const int64_t n = n0 + cc;
      if (n >= g.N) continue;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int rbase = half * 64 + tx * 4;  // real rows of the tile
        if constexpr (!ONEM) {
          const int64_t m = em0 + rbase;
          if (g.partial) {
            float* P = reinterpret_cast<float*>(g.partial) + ((split * g.H + h) * g.N + n) * g.M;
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (m + q < g.M) P[m + q] = tot[half * 4 + q][jj];
            continue;
          }
          if (m + 3 < g.M &&
              store4_f32(g.e, reinterpret_cast<float*>(Db) + dm_s[rbase] + dn_s[cc], dm_s + rbase,
                         tot[half * 4][jj], tot[half * 4 + 1][jj], tot[half * 4 + 2][jj], tot[half * 4 + 3][jj]))
            continue;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (m + q < g.M)
              epilogue_store<float, false>(g.e, tot[half * 4 + q][jj], 0.f,
                                           reinterpret_cast<const float*>(Cb) + cm_s[rbase + q] + cn_s[cc],
                                           reinterpret_cast<float*>(Db) + dm_s[rbase + q] + dn_s[cc]);
        } else {
          // Real rows 2p, 2p+1 are Re and Im of complex row p.
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int pr = rbase / 2 + q;
            const int64_t m = em0 + pr;
            if (m >= g.M) continue;
            const float re = tot[half * 4 + 2 * q][jj], im = tot[half * 4 + 2 * q + 1][jj];
            if (g.partial)
              Elem<float, true>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n) * g.M + m, re, im);
            else
              epilogue_store<float, true>(g.e, re, im, Cb + cm_s[pr] + cn_s[cc], Db + dm_s[pr] + dn_s[cc]);
          }
        }
      }
    }
  }

  __syncthreads();
  // Copies issued but not consumed (only after a timeout) land before exit.
  if (warp == 8 && lane == 0)
    for (int i = *stop; i < issued; ++i) (void)mbar_wait(&full[i % STAGES], (uint32_t)(i / STAGES) & 1u);
}

// ------------------------------------------------------------ DMMA tile (f64)

__device__ inline void dmma_m16n8k8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Element (row, k) of a 16-deep K-major tile of 128-byte rows as TMA's
// SWIZZLE_128B stores it: 16-byte chunk k/2 of row r sits at chunk
// (k/2) xor (r mod 8) (the tile base is 1024-byte aligned).
__device__ __forceinline__ int swz128(int row, int k) { return row * 16 + ((((k >> 1) ^ (row & 7)) << 1) | (k & 1)); }

template <bool THREE_M, int WM, int WN, int STAGES>
struct DpCfg {
  static constexpr int BM = 2 * WM, BN = 2 * WN, BK = 16;
  static constexpr int P = THREE_M ? 3 : 1;
  static constexpr int A_PL = BM * BK * 8, B_PL = BN * BK * 8;  // bytes of one plane tile
  static constexpr int STAGE = P * (A_PL + B_PL);
  static constexpr int SMEM = 1024 + STAGES * STAGE + (2 * BM + 2 * BN) * 8 + 2 * STAGES * 8 + 16;
  static constexpr int THREADS = 160;  // four compute warps (2 x 2) and a producer warp
};

// Persistent when the host sizes the grid below the work (MINB CTAs per
// SM): CTA c walks the work items c, c + gridDim.x, ... (a work item is one
// tile and one K split); with one CTA per work item the loop runs once. The producer warp runs through the stage ring
// across work-item boundaries, so the next tile's first stages load while
// the compute warps finish the current tile and write its epilogue; the
// tile's scatter vectors arrive by cp.async during its main loop. Two CTAs
// of one SM no longer start and end their tiles in step with empty
// pipelines in between.
// 8-byte asynchronous copy to shared memory; zero-filled (nothing read) when
// !ok.
__device__ __forceinline__ void cp_async8_zfill(void* smem, const void* gmem, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(ok ? 8 : 0)
               : "memory");
}

template <bool THREE_M, int WM, int WN, int STAGES, int MINB>
__global__ void __launch_bounds__(160, MINB)
dmma_packed_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g,
                   int64_t m_pad, int64_t n_pad, int64_t k_pad, int64_t tiles_m, int64_t tiles_n, int64_t kchunk,
                   int splits) {
  using Cfg = DpCfg<THREE_M, WM, WN, STAGES>;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, P = Cfg::P;
  constexpr int TI = WM / 16, TJ = WN / 8;
  using T = typename Elem<double, THREE_M>::type;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* ring = smem;
  int64_t* dm_s = reinterpret_cast<int64_t*>(smem + STAGES * Cfg::STAGE);
  int64_t* cm_s = dm_s + BM;
  int64_t* dn_s = cm_s + BM;
  int64_t* cn_s = dn_s + BN;
  uint64_t* full = reinterpret_cast<uint64_t*>(cn_s + BN);
  uint64_t* empty = full + STAGES;
  int* stop = reinterpret_cast<int*>(empty + STAGES);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t nwork = tiles_m * tiles_n * g.H * splits;
  const int64_t nkb_all = k_pad / BK;
  // Stages of one work item (its K split).
  auto k_range = [&](int64_t split, int64_t& lo) {
    lo = kchunk ? split * (kchunk / BK) : 0;
    const int64_t hi = kchunk ? min(nkb_all, lo + kchunk / BK) : nkb_all;
    return (int)(hi - lo);
  };

  if (warp == 4 && lane == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 4);
    }
    fence_barrier_init();
    *stop = INT_MAX;
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
  }
  __syncthreads();

  int issued = 0;
  if (warp == 4) {
    if (lane == 0) {
      bool alive = true;
      for (int64_t w = blockIdx.x; alive && w < nwork; w += gridDim.x) {
        int64_t h, mt, nt, kb_lo;
        packed_tile_coords(w / splits, tiles_m, tiles_n, h, mt, nt);
        const int nk = k_range(w % splits, kb_lo);
        for (int i = 0; i < nk; ++i) {
          const int s = issued % STAGES;
          const uint32_t round = (uint32_t)(issued / STAGES);
          if (!mbar_wait(&empty[s], (round & 1u) ^ 1u)) {
            atomicOr(g.status, STATUS_WAIT_TIMEOUT);
            alive = false;
            break;
          }
          mbar_arrive_expect_tx(&full[s], (uint32_t)Cfg::STAGE);
          uint8_t* sb = ring + s * Cfg::STAGE;
          const int x = (int)((kb_lo + i) * BK);
#pragma unroll
          for (int p = 0; p < P; ++p) {
            tma_load_2d(sb + p * Cfg::A_PL, &tmA, &full[s], x, (int)((p * g.H + h) * m_pad + mt * BM));
            tma_load_2d(sb + P * Cfg::A_PL + p * Cfg::B_PL, &tmB, &full[s], x, (int)((p * g.H + h) * n_pad + nt * BN));
          }
          ++issued;
        }
      }
    }
  } else {
    const int wm0 = (warp & 1) * WM, wn0 = (warp >> 1) * WN;
    const int fr = lane >> 2, fk = lane & 3;
    int it = 0;  // stages consumed
    bool alive = true;
    for (int64_t w = blockIdx.x; alive && w < nwork; w += gridDim.x) {
      const int64_t split = w % splits;
      int64_t h, mt, nt, kb_lo;
      packed_tile_coords(w / splits, tiles_m, tiles_n, h, mt, nt);
      const int nk = k_range(split, kb_lo);
      const int64_t m0 = mt * BM, n0 = nt * BN;
      // The previous tile's epilogue has read the scatter buffers; this
      // tile's entries then arrive while the main loop runs.
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (tid < BM) {
        const int64_t m = m0 + tid;
        const bool ok = m < g.M;
        const bool c_ok = ok && !g.e.beta_zero;
        cp_async8_zfill(dm_s + tid, g.s.d_m + (ok ? m : 0), ok);
        cp_async8_zfill(cm_s + tid, c_ok ? g.s.c_m + m : g.s.d_m, c_ok);
      }
      if (tid < BN) {
        const int64_t n = n0 + tid;
        const bool ok = n < g.N;
        const bool c_ok = ok && !g.e.beta_zero;
        cp_async8_zfill(dn_s + tid, g.s.d_n + (ok ? n : 0), ok);
        cp_async8_zfill(cn_s + tid, c_ok ? g.s.c_n + n : g.s.d_n, c_ok);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
      double acc[P][TI][TJ][4];
#pragma unroll
      for (int p = 0; p < P; ++p)
#pragma unroll
        for (int i = 0; i < TI; ++i)
#pragma unroll
          for (int j = 0; j < TJ; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][i][j][q] = 0.0;
      for (int kt = 0; kt < nk; ++kt, ++it) {
        const int s = it % STAGES;
        const uint32_t round = (uint32_t)(it / STAGES);
        if (!mbar_wait(&full[s], round & 1u)) {
          atomicOr(g.status, STATUS_WAIT_TIMEOUT);
          atomicMin(stop, it);
          alive = false;
          break;
        }
        const double* sA = reinterpret_cast<const double*>(ring + s * Cfg::STAGE);
        const double* sB = reinterpret_cast<const double*>(ring + s * Cfg::STAGE + P * Cfg::A_PL);
#pragma unroll
        for (int ks = 0; ks < BK / 8; ++ks) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const double* pA = sA + p * (Cfg::A_PL / 8);
            const double* pB = sB + p * (Cfg::B_PL / 8);
            double a[TI][4], b[TJ][2];
#pragma unroll
            for (int i = 0; i < TI; ++i)
#pragma unroll
              for (int q = 0; q < 4; ++q)
                a[i][q] = pA[swz128(wm0 + i * 16 + fr + 8 * (q & 1), ks * 8 + fk + 4 * (q >> 1))];
#pragma unroll
            for (int j = 0; j < TJ; ++j)
#pragma unroll
              for (int q = 0; q < 2; ++q) b[j][q] = pB[swz128(wn0 + j * 8 + fr, ks * 8 + fk + 4 * q)];
#pragma unroll
            for (int i = 0; i < TI; ++i)
#pragma unroll
              for (int j = 0; j < TJ; ++j) dmma_m16n8k8(acc[p][i][j], a[i], b[j]);
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
      }
      asm volatile("cp.async.wait_all;" ::: "memory");
      asm volatile("bar.sync 1, 128;" ::: "memory");  // every thread's scatter entries have landed
      // A wait that ran out in any compute warp ends all four (the flag was
      // set before the barrier).
      if (*reinterpret_cast<volatile int*>(stop) != INT_MAX) break;

      const T* Cb = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]);
      T* Db = static_cast<T*>(g.D) + g.s.h_d[h];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int rr = wm0 + i * 16 + fr + 8 * (q >> 1);
            const int cc = wn0 + j * 8 + fk * 2 + (q & 1);
            const int64_t m = m0 + rr, n = n0 + cc;
            if (m >= g.M || n >= g.N) continue;
            double re = acc[0][i][j][q], im = 0.0;
            if (THREE_M) {
              const double m1 = acc[0][i][j][q], m2 = acc[P > 1 ? 1 : 0][i][j][q], m3 = acc[P > 2 ? 2 : 0][i][j][q];
              re = m1 - m2;
              im = m3 - m1 - m2;
            }
            if (g.partial)
              Elem<double, THREE_M>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n) * g.M + m, re,
                                           im);
            else
              epilogue_store<double, THREE_M>(g.e, re, im, Cb + cm_s[rr] + cn_s[cc], Db + dm_s[rr] + dn_s[cc]);
          }
    }
  }

  __syncthreads();
  // After a timeout: wait (bounded) for the copies still in flight into the
  // stages nobody consumed.
  if (warp == 4 && lane == 0)
    for (int i = *stop; i < issued; ++i) (void)mbar_wait(&full[i % STAGES], (uint32_t)(i / STAGES) & 1u);
}

constexpr int DP_F64_STAGES = 4, DP_3M_STAGES = 3;
using DpF64 = DpCfg<false, 32, 32, DP_F64_STAGES>;
using Dp3M = DpCfg<true, 32, 16, DP_3M_STAGES>;

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

size_t elem_bytes_of(int kernel) {
  return (kernel == PLAIN_F64_PACKED_64x64 || kernel == PLAIN_C64_PACKED_3M_64x32) ? 8 : 4;
}

template <class R, bool CPLX, int MODE>
cudaError_t run_pack(const GemmArgs& g, int which, const PanelArgs& o, int64_t src_rows, int64_t src_k,
                     cudaStream_t st) {
  const int64_t gy = (src_rows + 31) / 32, gx = (src_k + 31) / 32;
  if (gx * gy * o.H > 0x7fffffff) return cudaErrorInvalidConfiguration;
  PanelArgs og = o;
  og.gx = gx;
  og.gy = gy;
  const dim3 grid((unsigned)(gx * gy * o.H));
  using T = typename Elem<R, CPLX>::type;
  const bool a = which == 0;
  plain_pack_kernel<R, CPLX, MODE><<<grid, 256, 0, st>>>(
      static_cast<const T*>(a ? g.A : g.B), a ? g.s.a_m : g.s.b_n, a ? g.s.a_k : g.s.b_k, a ? g.s.h_a : g.s.h_b,
      a ? g.s.blk_a_m : g.s.blk_b_n, a ? g.s.blk_a_k : g.s.blk_b_k, a ? g.M : g.N, g.K, a ? g.a_kfast : g.b_kfast,
      CPLX ? (a ? g.conj_a : g.conj_b) : 0, og);
  return cudaGetLastError();
}

// The FFMA tile over f32 panels: [H * k_pad] rows of m_pad (n_pad) floats,
// boxes of 16 rows x 128 (BN) floats.
template <bool ONEM, int BN>
cudaError_t run_simt_packed(const GemmArgs& g, const PackedLayout& L, const void* pa, const void* pb, int64_t splits,
                            cudaStream_t st) {
  using Cfg = SpCfg<BN>;
  if (L.H * L.k_pad >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  if (!make_map_2d(&ma, pa, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, L.m_pad, L.H * L.k_pad, Cfg::BM, Cfg::BK,
                   CU_TENSOR_MAP_SWIZZLE_NONE) ||
      !make_map_2d(&mb, pb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, L.n_pad, L.H * L.k_pad, BN, Cfg::BK,
                   CU_TENSOR_MAP_SWIZZLE_NONE))
    return cudaErrorInvalidValue;
  const int64_t tiles = (L.m_pad / Cfg::BM) * (L.n_pad / BN) * L.H;
  const int64_t kchunk = g.k_chunk ? (ONEM ? 2 * g.k_chunk : g.k_chunk) : 0;
  if (tiles * splits >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
  auto kern = simt_packed_kernel<ONEM, BN>;
  cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
  if (r != cudaSuccess) return r;
  kern<<<(unsigned)(tiles * splits), Cfg::THREADS, Cfg::SMEM, st>>>(ma, mb, g, L.k_pad, L.m_pad / Cfg::BM,
                                                                    L.n_pad / BN, kchunk, (int)splits);
  return cudaGetLastError();
}

}  // namespace

bool is_packed_kernel(int kernel) { return kernel >= PLAIN_F32_PACKED_128x128 && kernel <= PLAIN_C32_PACKED_1M_64x64; }

int packed_dtype(int kernel) {
  switch (kernel) {
    case PLAIN_F32_PACKED_128x128:
    case PLAIN_F32_PACKED_128x64: return 0;
    case PLAIN_F64_PACKED_64x64: return 1;
    case PLAIN_C32_PACKED_1M_64x128:
    case PLAIN_C32_PACKED_1M_64x64: return 2;
    case PLAIN_C64_PACKED_3M_64x32: return 3;
  }
  return -1;
}

PackedLayout packed_layout(int kernel, int64_t M, int64_t N, int64_t K, int64_t H) {
  PackedLayout L;
  L.kernel = kernel;
  L.H = H;
  switch (kernel) {
    case PLAIN_F32_PACKED_128x128:
    case PLAIN_F32_PACKED_128x64:
      L.m_pad = round_up(M, SpCfg<128>::BM);
      L.n_pad = round_up(N, kernel == PLAIN_F32_PACKED_128x128 ? 128 : 64);
      L.k_pad = round_up(K, SpCfg<128>::BK);
      break;
    case PLAIN_C32_PACKED_1M_64x128:
    case PLAIN_C32_PACKED_1M_64x64:
      L.m_pad = round_up(2 * M, SpCfg<128>::BM);
      L.n_pad = round_up(N, kernel == PLAIN_C32_PACKED_1M_64x128 ? 128 : 64);
      L.k_pad = round_up(2 * K, SpCfg<128>::BK);
      break;
    case PLAIN_F64_PACKED_64x64:
      L.m_pad = round_up(M, DpF64::BM);
      L.n_pad = round_up(N, DpF64::BN);
      L.k_pad = round_up(K, DpF64::BK);
      break;
    case PLAIN_C64_PACKED_3M_64x32:
      L.planes = 3;
      L.m_pad = round_up(M, Dp3M::BM);
      L.n_pad = round_up(N, Dp3M::BN);
      L.k_pad = round_up(K, Dp3M::BK);
      break;
    default:
      break;
  }
  return L;
}

size_t packed_workspace_bytes(const PackedLayout& L) {
  const size_t e = elem_bytes_of(L.kernel);
  const size_t a = (size_t)L.planes * L.H * L.m_pad * L.k_pad * e;
  const size_t b = (size_t)L.planes * L.H * L.n_pad * L.k_pad * e;
  return ((a + 255) & ~size_t(255)) + ((b + 255) & ~size_t(255)) + 256;
}

cudaError_t launch_packed_pack(const GemmArgs& g, const PackedLayout& L, void* panels, cudaStream_t st,
                               cudaStream_t st_b) {
  const size_t e = elem_bytes_of(L.kernel);
  const size_t a_bytes = (size_t)L.planes * L.H * L.m_pad * L.k_pad * e;
  char* pa = static_cast<char*>(panels);
  char* pb = pa + ((a_bytes + 255) & ~size_t(255));
  PanelArgs oa{pa, L.m_pad, L.k_pad, L.H * L.m_pad * L.k_pad, L.H};
  PanelArgs ob{pb, L.n_pad, L.k_pad, L.H * L.n_pad * L.k_pad, L.H};
  oa.hfast = L.a_hfast;
  ob.hfast = L.b_hfast;
  cudaError_t r;
  switch (L.kernel) {
    case PLAIN_F32_PACKED_128x128:
    case PLAIN_F32_PACKED_128x64:
      r = run_pack<float, false, PM_ROWS_FAST>(g, 0, oa, L.m_pad, L.k_pad, st);
      if (r != cudaSuccess) return r;
      return run_pack<float, false, PM_ROWS_FAST>(g, 1, ob, L.n_pad, L.k_pad, st_b);
    case PLAIN_C32_PACKED_1M_64x128:
    case PLAIN_C32_PACKED_1M_64x64:
      r = run_pack<float, true, PM_1M_A>(g, 0, oa, L.m_pad / 2, (L.k_pad + 1) / 2, st);
      if (r != cudaSuccess) return r;
      return run_pack<float, true, PM_1M_B>(g, 1, ob, L.n_pad, (L.k_pad + 1) / 2, st_b);
    case PLAIN_F64_PACKED_64x64:
      r = run_pack<double, false, PM_K_FAST>(g, 0, oa, L.m_pad, L.k_pad, st);
      if (r != cudaSuccess) return r;
      return run_pack<double, false, PM_K_FAST>(g, 1, ob, L.n_pad, L.k_pad, st_b);
    case PLAIN_C64_PACKED_3M_64x32:
      r = run_pack<double, true, PM_3M>(g, 0, oa, L.m_pad, L.k_pad, st);
      if (r != cudaSuccess) return r;
      return run_pack<double, true, PM_3M>(g, 1, ob, L.n_pad, L.k_pad, st_b);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_packed_gemm(const GemmArgs& g, const PackedLayout& L, const void* panels, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.H <= 0) return cudaSuccess;
  const size_t e = elem_bytes_of(L.kernel);
  const size_t a_bytes = (size_t)L.planes * L.H * L.m_pad * L.k_pad * e;
  const char* pa = static_cast<const char*>(panels);
  const char* pb = pa + ((a_bytes + 255) & ~size_t(255));
  const int64_t splits = g.k_chunk ? (g.K + g.k_chunk - 1) / g.k_chunk : 1;
  if (splits > 64) return cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  const bool onem = L.kernel == PLAIN_C32_PACKED_1M_64x128 || L.kernel == PLAIN_C32_PACKED_1M_64x64;
  if (L.kernel == PLAIN_F32_PACKED_128x128 || L.kernel == PLAIN_C32_PACKED_1M_64x128)
    return onem ? run_simt_packed<true, 128>(g, L, pa, pb, splits, st) : run_simt_packed<false, 128>(g, L, pa, pb, splits, st);
  if (L.kernel == PLAIN_F32_PACKED_128x64 || L.kernel == PLAIN_C32_PACKED_1M_64x64)
    return onem ? run_simt_packed<true, 64>(g, L, pa, pb, splits, st) : run_simt_packed<false, 64>(g, L, pa, pb, splits, st);
  // K-major f64 panels: [planes * H * rows_pad] rows of k_pad doubles; boxes
  // of BM (BN) rows x 16 doubles (128 bytes), SWIZZLE_128B.
  const bool three = L.kernel == PLAIN_C64_PACKED_3M_64x32;
  const int bm = three ? Dp3M::BM : DpF64::BM, bn = three ? Dp3M::BN : DpF64::BN;
  if ((int64_t)L.planes * L.H * (L.m_pad > L.n_pad ? L.m_pad : L.n_pad) >= ((int64_t)1 << 31))
    return cudaErrorInvalidValue;
  if (!make_map_2d(&ma, pa, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, L.k_pad, L.planes * L.H * L.m_pad, 16, bm,
                   CU_TENSOR_MAP_SWIZZLE_128B) ||
      !make_map_2d(&mb, pb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, L.k_pad, L.planes * L.H * L.n_pad, 16, bn,
                   CU_TENSOR_MAP_SWIZZLE_128B))
    return cudaErrorInvalidValue;
  const int64_t tiles = (L.m_pad / bm) * (L.n_pad / bn) * L.H;
  if (tiles * splits >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t work = tiles * splits;
  // Short work items (at most 64 stages: K per item up to 1024) run on a
  // persistent grid, where the next tile's loads hide the fill and the
  // epilogue (C3's 64 x 384^3: 0.85 -> 0.81 ms); longer ones keep one CTA per
  // work item, whose hardware scheduling balances SMs better (a persistent
  // grid measured 0.83 -> 0.76 of the FP64 pipe on a 4096^3 GEMM).
  const int64_t nk_item = (g.k_chunk ? g.k_chunk : L.k_pad) / 16;
  const bool persistent = nk_item <= 64;
  if (three) {
    auto kern = dmma_packed_kernel<true, 32, 16, DP_3M_STAGES, 2>;
    cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Dp3M::SMEM);
    if (r != cudaSuccess) return r;
    const unsigned grid = (unsigned)(persistent && work > 2 * sms ? 2 * sms : work);
    kern<<<grid, Dp3M::THREADS, Dp3M::SMEM, st>>>(ma, mb, g, L.m_pad, L.n_pad, L.k_pad, L.m_pad / bm, L.n_pad / bn,
                                                  g.k_chunk, (int)splits);
  } else {
    auto kern = dmma_packed_kernel<false, 32, 32, DP_F64_STAGES, 3>;
    cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, DpF64::SMEM);
    if (r != cudaSuccess) return r;
    const unsigned grid = (unsigned)(persistent && work > 3 * sms ? 3 * sms : work);
    kern<<<grid, DpF64::THREADS, DpF64::SMEM, st>>>(ma, mb, g, L.m_pad, L.n_pad, L.k_pad, L.m_pad / bm, L.n_pad / bn,
                                                    g.k_chunk, (int)splits);
  }
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace tprims
