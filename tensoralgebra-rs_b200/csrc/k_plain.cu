// Plain (drop-in precision) contraction kernels: one launch per contraction,
// one CTA per (batch, M tile, N tile), the whole K loop inside the CTA.
//
// The gather stage replaces the reference's packing (crates/tprims-kernel/src/
// pack/pack.rs:152-203): each K step reads A'[m, k] = A[h_a + a_m[m] + a_k[k]]
// and B'[k, n] through the scatter vectors straight into shared memory, with
// threads running along whichever index is unit-stride in memory, and folds
// conjugation into the sign of the imaginary plane. Real tiles stage the next
// K step in registers (TileGather); complex tiles and grouped f64 lists fill a
// ring of four shared-memory stages with cp.async (AsyncGather), which keeps
// three stages of global loads in flight. The register tile replaces
// the microkernels (kernels/reference/scalar.rs:31-175): FP32 FFMA for f32,
// FP64 DMMA (mma.sync m16n8k8) for f64, and four real products per complex MAC
// for c32/c64 (the planar method, writeback.rs:54-97 Planar). The epilogue is
// the scatter write-back (writeback.rs:311-486) applied once per element after
// the full K loop.
#include "device_common.cuh"

namespace tprims {
namespace dev {

namespace {

// Gather of one ROWS x BK tile (A': rows = m; B': rows = n) into registers,
// then into planar shared memory laid out [k][row]. Threads run along k when
// k is the unit-stride index (kfast) and along the rows otherwise, so each
// thread sees one fixed k (kfast) or one fixed row (otherwise) for all its
// PER elements. Its offsets are therefore one fixed value plus one value per
// element: kfast: the element's row offset (set once per tile, in var[]) plus
// the stage's k offset (fixed); otherwise: the row offset (fixed, set once)
// plus each element's k offset (var[], per stage). The k offsets of a stage
// are fetched one stage ahead of its elements (load_idx), so an element load
// never waits on the index load in front of it. INT64_MIN marks a row or k
// outside the operand (the element reads as zero).
template <class R, bool CPLX, int ROWS, int BK, int NT>
struct TileGather {
  using T = typename Elem<R, CPLX>::type;
  static constexpr int PER = ROWS * BK / NT;
  static_assert(ROWS * BK % NT == 0, "tile must split evenly over threads");
  static_assert(NT % BK == 0 && NT % ROWS == 0, "a thread keeps one k (kfast) or one row");
  R re[PER];
  R im[CPLX ? PER : 1];
  int64_t var[PER];  // kfast: row offsets; otherwise: k offsets of the next stage
  int64_t fixed;     // kfast: k offset of the next stage; otherwise: the row offset
  // k-fast operands: a warp covers RS rows x KQ consecutive k (the same
  // spread over the shared-memory banks as AsyncGather below).
  static constexpr int KQ = sizeof(R) == 4 ? 8 : 4, RS = 32 / KQ;
  static constexpr bool WIDE = BK % KQ == 0 && ROWS % RS == 0 && (NT / 32) % (BK / KQ) == 0;

  __device__ static inline void coords(int idx, int kfast, int& kk, int& rr) {
    if (kfast) {
      if constexpr (WIDE) {
        const int w = idx / 32, l = idx % 32;
        kk = (w % (BK / KQ)) * KQ + l % KQ;
        rr = (w / (BK / KQ)) * RS + l / KQ;
      } else {
        kk = idx % BK;
        rr = idx / BK;
      }
    } else {
      kk = idx / ROWS;
      rr = idx % ROWS;
    }
  }

  // Row offsets of this tile (rows_s: the tile's row scatter in shared memory).
  __device__ inline void init(const int64_t* rows_s, int64_t row0, int64_t nrows, int kfast, int tid) {
    if (kfast) {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        int kk, rr;
        coords(tid + j * NT, 1, kk, rr);
        var[j] = row0 + rr < nrows ? rows_s[rr] : INT64_MIN;
      }
    } else {
      int kk, rr;
      coords(tid, 0, kk, rr);
      fixed = row0 + rr < nrows ? rows_s[rr] : INT64_MIN;
    }
  }

  __device__ inline void load_idx(const int64_t* kscat, int64_t k0, int64_t K, int kfast, int tid) {
    if (kfast) {
      int kk, rr;
      coords(tid, 1, kk, rr);
      const int64_t k = k0 + kk;
      fixed = k < K ? __ldg(kscat + k) : INT64_MIN;
    } else {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        int kk, rr;
        coords(tid + j * NT, 0, kk, rr);
        const int64_t k = k0 + kk;
        var[j] = k < K ? __ldg(kscat + k) : INT64_MIN;
      }
    }
  }

  __device__ inline void load(const T* base, int conj) {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      R vr = R(0), vi = R(0);
      if (var[j] != INT64_MIN && fixed != INT64_MIN) {
        Elem<R, CPLX>::load(base + var[j] + fixed, vr, vi);
        if (conj) vi = -vi;
      }
      re[j] = vr;
      if (CPLX) im[j] = vi;
    }
  }

  __device__ inline void store(R* s_re, R* s_im, int stride, int kfast, int tid) const {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int kk, rr;
      coords(tid + j * NT, kfast, kk, rr);
      s_re[kk * stride + rr] = re[j];
      if (CPLX) s_im[kk * stride + rr] = im[j];
    }
  }
};

// ---------------------------------------------------------------- SIMT (FFMA)

// Each K tile is accumulated into a fresh register tile that is then added to
// the running total (round-to-nearest FADD), which keeps the FP32 rounding
// error of a deep K near u * (sqrt(BK) + sqrt(K / BK)) instead of u * sqrt(K).
template <class R, bool CPLX, int BM, int BN, int BK, int TM, int TN>
__device__ __forceinline__ void simt_tile(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                          int64_t split = 0) {
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int PAD = 4;
  constexpr int SA = BM + PAD, SB = BN + PAD;
  constexpr int NPL = CPLX ? 2 : 1;
  using T = typename Elem<R, CPLX>::type;

  __shared__ __align__(16) R As[2][NPL][BK * SA];
  __shared__ __align__(16) R Bs[2][NPL][BK * SB];
  __shared__ int64_t am_s[BM], bn_s[BN], dm_s[BM], cm_s[BM], dn_s[BN], cn_s[BN];

  const int tid = threadIdx.x;
  const int64_t m0 = mtile * BM, n0 = ntile * BN;

  for (int i = tid; i < BM; i += NT) {
    const int64_t m = m0 + i;
    const bool ok = m < g.M;
    am_s[i] = ok ? g.s.a_m[m] : 0;
    dm_s[i] = ok ? g.s.d_m[m] : 0;
    cm_s[i] = ok ? g.s.c_m[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int64_t n = n0 + i;
    const bool ok = n < g.N;
    bn_s[i] = ok ? g.s.b_n[n] : 0;
    dn_s[i] = ok ? g.s.d_n[n] : 0;
    cn_s[i] = ok ? g.s.c_n[n] : 0;
  }
  __syncthreads();

  const T* Ab = static_cast<const T*>(g.A) + g.s.h_a[h];
  const T* Bb = static_cast<const T*>(g.B) + g.s.h_b[h];

  TileGather<R, CPLX, BM, BK, NT> ga;
  TileGather<R, CPLX, BN, BK, NT> gb;

  constexpr int HM = TM / 2, HN = TN / 2;
  const int tx = tid % (BM / TM), ty = tid / (BM / TM);
  R tot_re[TM][TN], tot_im[CPLX ? TM : 1][CPLX ? TN : 1];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      tot_re[i][j] = R(0);
      if (CPLX) tot_im[i][j] = R(0);
    }

  // This CTA's K range (the whole of K unless split).
  const int64_t kb = g.k_chunk ? split * g.k_chunk : 0;
  const int64_t ke = g.k_chunk ? min(g.K, kb + g.k_chunk) : g.K;
  const int64_t nt = (ke - kb + BK - 1) / BK;
  ga.init(am_s, m0, g.M, g.a_kfast, tid);
  gb.init(bn_s, n0, g.N, g.b_kfast, tid);
  ga.load_idx(g.s.a_k, kb, ke, g.a_kfast, tid);
  gb.load_idx(g.s.b_k, kb, ke, g.b_kfast, tid);
  ga.load(Ab, g.conj_a);
  gb.load(Bb, g.conj_b);
  ga.store(As[0][0], As[0][NPL - 1], SA, g.a_kfast, tid);
  gb.store(Bs[0][0], Bs[0][NPL - 1], SB, g.b_kfast, tid);
  if (nt > 1) {
    ga.load_idx(g.s.a_k, kb + BK, ke, g.a_kfast, tid);
    gb.load_idx(g.s.b_k, kb + BK, ke, g.b_kfast, tid);
  }
  __syncthreads();

  for (int64_t t = 0; t < nt; ++t) {
    const int buf = (int)(t & 1);
    if (t + 1 < nt) {
      ga.load(Ab, g.conj_a);
      gb.load(Bb, g.conj_b);
    }
    R acc_re[TM][TN], acc_im[CPLX ? TM : 1][CPLX ? TN : 1];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        acc_re[i][j] = R(0);
        if (CPLX) acc_im[i][j] = R(0);
      }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      R ar[TM], br[TN], ai[CPLX ? TM : 1], bi[CPLX ? TN : 1];
#pragma unroll
      for (int i = 0; i < HM; ++i) {
        ar[i] = As[buf][0][kk * SA + tx * HM + i];
        ar[HM + i] = As[buf][0][kk * SA + BM / 2 + tx * HM + i];
        if (CPLX) {
          ai[i] = As[buf][NPL - 1][kk * SA + tx * HM + i];
          ai[HM + i] = As[buf][NPL - 1][kk * SA + BM / 2 + tx * HM + i];
        }
      }
#pragma unroll
      for (int j = 0; j < HN; ++j) {
        br[j] = Bs[buf][0][kk * SB + ty * HN + j];
        br[HN + j] = Bs[buf][0][kk * SB + BN / 2 + ty * HN + j];
        if (CPLX) {
          bi[j] = Bs[buf][NPL - 1][kk * SB + ty * HN + j];
          bi[HN + j] = Bs[buf][NPL - 1][kk * SB + BN / 2 + ty * HN + j];
        }
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          if (CPLX) {
            acc_re[i][j] = fma(ar[i], br[j], acc_re[i][j]);
            acc_re[i][j] = fma(-ai[i], bi[j], acc_re[i][j]);
            acc_im[i][j] = fma(ar[i], bi[j], acc_im[i][j]);
            acc_im[i][j] = fma(ai[i], br[j], acc_im[i][j]);
          } else {
            acc_re[i][j] = fma(ar[i], br[j], acc_re[i][j]);
          }
        }
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        tot_re[i][j] += acc_re[i][j];
        if (CPLX) tot_im[i][j] += acc_im[i][j];
      }
    if (t + 1 < nt) {
      ga.store(As[buf ^ 1][0], As[buf ^ 1][NPL - 1], SA, g.a_kfast, tid);
      gb.store(Bs[buf ^ 1][0], Bs[buf ^ 1][NPL - 1], SB, g.b_kfast, tid);
      if (t + 2 < nt) {
        ga.load_idx(g.s.a_k, kb + (t + 2) * BK, ke, g.a_kfast, tid);
        gb.load_idx(g.s.b_k, kb + (t + 2) * BK, ke, g.b_kfast, tid);
      }
    }
    __syncthreads();
  }

  const T* Cb = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]);
  T* Db = static_cast<T*>(g.D) + g.s.h_d[h];
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int rr = (i < HM) ? (tx * HM + i) : (BM / 2 + tx * HM + (i - HM));
    if (m0 + rr >= g.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int cc = (j < HN) ? (ty * HN + j) : (BN / 2 + ty * HN + (j - HN));
      if (n0 + cc >= g.N) continue;
      if (g.partial)
        Elem<R, CPLX>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n0 + cc) * g.M + m0 + rr,
                             tot_re[i][j], CPLX ? tot_im[i][j] : R(0));
      else
        epilogue_store<R, CPLX>(g.e, tot_re[i][j], CPLX ? tot_im[i][j] : R(0), Cb + cm_s[rr] + cn_s[cc],
                              Db + dm_s[rr] + dn_s[cc]);
    }
  }
}

// ---------------------------------------------------------------- FP64 DMMA

__device__ __forceinline__ uint32_t smem_addr_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// D (16 x 8) += A (16 x 8, row) B (8 x 8, col) in FP64. Fragments, with
// g = lane / 4 and t = lane % 4: a[r] = A[g + 8 (r % 2)][t + 4 (r / 2)],
// b[r] = B[t + 4 r][g], d[r] = D[g + 8 (r / 2)][2 t + r % 2].
__device__ inline void dmma_1688(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Asynchronous gather of one ROWS x BK FP64 tile (planar for complex) into a
// shared-memory stage: the same per-thread offsets as TileGather (one fixed
// offset and one per element), but each element goes straight from global to
// shared memory with cp.async (8 bytes; an element outside the operand is
// zero-filled by a zero source size), so several stages can be in flight
// without holding them in registers. Conjugation is applied when fragments
// are read.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_addr_u32(smem)), "l"(gmem),
               "r"(ok ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_addr_u32(smem)), "l"(gmem),
               "r"(ok ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_elem(double* smem, const double* gmem, bool ok) { cp_async8(smem, gmem, ok); }
__device__ __forceinline__ void cp_async_elem(float* smem, const float* gmem, bool ok) { cp_async4(smem, gmem, ok); }

template <class R, bool CPLX, int ROWS, int BK, int NT>
struct AsyncGather {
  using T = typename Elem<R, CPLX>::type;
  static constexpr int PER = ROWS * BK / NT;
  static_assert(ROWS * BK % NT == 0 && NT % BK == 0 && NT % ROWS == 0, "one k or one row per thread");
  int64_t var[PER];
  int64_t fixed;
  // k-fast operands: a warp covers RS rows x KQ consecutive k (32 bytes of
  // each row for 8-byte elements, 32 for 4-byte ones), so its cp.async
  // writes into the [k][row] stage (row stride = 4 mod 16 words) spread over
  // the banks; 32 lanes on 16 or 32 k of one row would land on a quarter of
  // them. The k of a thread stays the same across its PER elements.
  static constexpr int KQ = sizeof(R) == 4 ? 8 : 4, RS = 32 / KQ;
  static constexpr bool WIDE = BK % KQ == 0 && ROWS % RS == 0 && (NT / 32) % (BK / KQ) == 0;

  __device__ static inline void coords(int idx, int kfast, int& kk, int& rr) {
    if (kfast) {
      if constexpr (WIDE) {
        const int w = idx / 32, l = idx % 32;
        kk = (w % (BK / KQ)) * KQ + l % KQ;
        rr = (w / (BK / KQ)) * RS + l / KQ;
      } else {
        kk = idx % BK;
        rr = idx / BK;
      }
    } else {
      kk = idx / ROWS;
      rr = idx % ROWS;
    }
  }
  __device__ inline void init(const int64_t* rows_s, int64_t row0, int64_t nrows, int kfast, int tid) {
    if (kfast) {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        int kk, rr;
        coords(tid + j * NT, 1, kk, rr);
        var[j] = row0 + rr < nrows ? rows_s[rr] : INT64_MIN;
      }
    } else {
      int kk, rr;
      coords(tid, 0, kk, rr);
      fixed = row0 + rr < nrows ? rows_s[rr] : INT64_MIN;
    }
  }
  __device__ inline void load_idx(const int64_t* kscat, int64_t k0, int64_t K, int kfast, int tid) {
    if (kfast) {
      int kk, rr;
      coords(tid, 1, kk, rr);
      const int64_t k = k0 + kk;
      fixed = k < K ? __ldg(kscat + k) : INT64_MIN;
    } else {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        int kk, rr;
        coords(tid + j * NT, 0, kk, rr);
        const int64_t k = k0 + kk;
        var[j] = k < K ? __ldg(kscat + k) : INT64_MIN;
      }
    }
  }
  // The same from k offsets staged in shared memory (kscat_s[k - k_base]).
  __device__ inline void load_idx_s(const int64_t* kscat_s, int64_t k_base, int64_t k0, int64_t K, int kfast,
                                    int tid) {
    if (kfast) {
      int kk, rr;
      coords(tid, 1, kk, rr);
      const int64_t k = k0 + kk;
      fixed = k < K ? kscat_s[k - k_base] : INT64_MIN;
    } else {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        int kk, rr;
        coords(tid + j * NT, 0, kk, rr);
        const int64_t k = k0 + kk;
        var[j] = k < K ? kscat_s[k - k_base] : INT64_MIN;
      }
    }
  }
  // Copies of this thread's elements of the stage whose offsets are loaded.
  __device__ inline void issue(const T* base, R* s_re, R* s_im, int stride, int kfast, int tid) const {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int kk, rr;
      coords(tid + j * NT, kfast, kk, rr);
      const bool ok = var[j] != INT64_MIN && fixed != INT64_MIN;
      const T* src = ok ? base + var[j] + fixed : base;  // not read when !ok
      const R* d = reinterpret_cast<const R*>(src);
      cp_async_elem(s_re + kk * stride + rr, d, ok);
      if (CPLX) cp_async_elem(s_im + kk * stride + rr, d + 1, ok);
    }
  }
};

// Shape of the DMMA stage ring (dynamic shared memory, see dmma_tile).
template <bool CPLX, int WM, int WN, int BK, int STG = 4>
struct DmmaRing {
  static constexpr int BM = 2 * WM, BN = 2 * WN;
  static constexpr int SA = BM + 4, SB = BN + 4;  // strides = 4 (mod 16) doubles: conflict-free fragment reads
  static constexpr int NPL = CPLX ? 2 : 1;
  static constexpr int STAGES = STG;
  static constexpr int A_STAGE = NPL * BK * SA, B_STAGE = NPL * BK * SB;  // doubles
  static constexpr int BYTES = STAGES * (A_STAGE + B_STAGE) * 8;
};

// Asynchronous variant (used for complex): 4 warps in a 2x2 arrangement, each
// warp a WM x WN tile of 16x8 DMMA tiles, fed by a ring of STAGES
// shared-memory stages (dynamic shared memory of DmmaRing::BYTES) filled with
// cp.async.
template <bool CPLX, int WM, int WN, int BK, int STG = 4>
__device__ __forceinline__ void dmma_tile_async(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                          int64_t split = 0) {
  using Ring = DmmaRing<CPLX, WM, WN, BK, STG>;
  constexpr int BM = Ring::BM, BN = Ring::BN, NT = 128;
  constexpr int SA = Ring::SA, SB = Ring::SB;
  constexpr int NPL = Ring::NPL;
  constexpr int STAGES = Ring::STAGES;
  constexpr int TI = WM / 16, TJ = WN / 8;
  static_assert(WM % 16 == 0 && WN % 8 == 0 && BK % 8 == 0, "m16n8k8 fragments");
  using T = typename Elem<double, CPLX>::type;

  extern __shared__ __align__(16) double dmma_ring[];
  double(*As)[NPL][BK * SA] = reinterpret_cast<double(*)[NPL][BK * SA]>(dmma_ring);
  double(*Bs)[NPL][BK * SB] = reinterpret_cast<double(*)[NPL][BK * SB]>(dmma_ring + STAGES * Ring::A_STAGE);
  __shared__ int64_t am_s[BM], bn_s[BN], dm_s[BM], cm_s[BM], dn_s[BN], cn_s[BN];
  // A K range of at most KS is short: its k offsets are staged with the row
  // and column offsets, so no stage waits on a k-offset load before its
  // copies can be issued (each such load is a memory round trip).
  constexpr int KS = 64;
  __shared__ int64_t ak_s[KS], bk_s[KS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t m0 = mtile * BM, n0 = ntile * BN;
  const int wm0 = (warp & 1) * WM, wn0 = (warp >> 1) * WN;

  for (int i = tid; i < BM; i += NT) {
    const int64_t m = m0 + i;
    const bool ok = m < g.M;
    am_s[i] = ok ? g.s.a_m[m] : 0;
    dm_s[i] = ok ? g.s.d_m[m] : 0;
    cm_s[i] = ok ? g.s.c_m[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int64_t n = n0 + i;
    const bool ok = n < g.N;
    bn_s[i] = ok ? g.s.b_n[n] : 0;
    dn_s[i] = ok ? g.s.d_n[n] : 0;
    cn_s[i] = ok ? g.s.c_n[n] : 0;
  }
  // This CTA's K range (the whole of K unless split).
  const int64_t kb = g.k_chunk ? split * g.k_chunk : 0;
  const int64_t ke = g.k_chunk ? min(g.K, kb + g.k_chunk) : g.K;
  const bool kstaged = ke - kb <= KS;
  if (kstaged)
    for (int i = tid; i < ke - kb; i += NT) {
      ak_s[i] = g.s.a_k[kb + i];
      bk_s[i] = g.s.b_k[kb + i];
    }
  __syncthreads();

  const T* Ab = static_cast<const T*>(g.A) + g.s.h_a[h];
  const T* Bb = static_cast<const T*>(g.B) + g.s.h_b[h];
  AsyncGather<double, CPLX, BM, BK, NT> ga;
  AsyncGather<double, CPLX, BN, BK, NT> gb;

  // Complex tiles run 3m (kernels/reference/scalar.rs:136): cr = M1 = Ar Br,
  // cm = M2 = Ai Bi, ci = M3 = (Ar + Ai)(Br + Bi), the sums formed from the
  // fragments in registers; the epilogue takes (M1 - M2) + i (M3 - M1 - M2).
  double cr[TI][TJ][4], ci[CPLX ? TI : 1][CPLX ? TJ : 1][4], cm[CPLX ? TI : 1][CPLX ? TJ : 1][4];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        cr[i][j][q] = 0.0;
        if (CPLX) {
          ci[i][j][q] = 0.0;
          cm[i][j][q] = 0.0;
        }
      }

  const int64_t nt = (ke - kb + BK - 1) / BK;
  auto load_stage_idx = [&](int64_t k0) {
    if (kstaged) {
      ga.load_idx_s(ak_s, kb, k0, ke, g.a_kfast, tid);
      gb.load_idx_s(bk_s, kb, k0, ke, g.b_kfast, tid);
    } else {
      ga.load_idx(g.s.a_k, k0, ke, g.a_kfast, tid);
      gb.load_idx(g.s.b_k, k0, ke, g.b_kfast, tid);
    }
  };
  ga.init(am_s, m0, g.M, g.a_kfast, tid);
  gb.init(bn_s, n0, g.N, g.b_kfast, tid);
  // Prologue: stages 0 .. STAGES-2 in flight (one commit group each, empty
  // groups past the end keep the count uniform).
#pragma unroll
  for (int sidx = 0; sidx < STAGES - 1; ++sidx) {
    if (sidx < nt) {
      load_stage_idx(kb + sidx * BK);
      ga.issue(Ab, As[sidx][0], As[sidx][NPL - 1], SA, g.a_kfast, tid);
      gb.issue(Bb, Bs[sidx][0], Bs[sidx][NPL - 1], SB, g.b_kfast, tid);
    }
    cp_async_commit();
  }

  const double sa = g.conj_a ? -1.0 : 1.0, sb = g.conj_b ? -1.0 : 1.0;
  const int fr = lane >> 2, fk = lane & 3;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t tp = t + STAGES - 1;  // the stage issued in this iteration
    if (tp < nt) load_stage_idx(kb + tp * BK);
    cp_async_wait<STAGES - 2>();  // this thread's copies of stage t have landed
    __syncthreads();              // everyone's have; and stage t-1's buffer is free
    if (tp < nt) {
      const int pb = (int)(tp % STAGES);
      ga.issue(Ab, As[pb][0], As[pb][NPL - 1], SA, g.a_kfast, tid);
      gb.issue(Bb, Bs[pb][0], Bs[pb][NPL - 1], SB, g.b_kfast, tid);
    }
    cp_async_commit();
    const int buf = (int)(t % STAGES);
#pragma unroll
    for (int ks = 0; ks < BK / 8; ++ks) {
      double a_re[TI][4], b_re[TJ][2], a_im[CPLX ? TI : 1][4], a_sum[CPLX ? TI : 1][4], b_im[CPLX ? TJ : 1][2],
          b_sum[CPLX ? TJ : 1][2];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int idx = (ks * 8 + fk + 4 * (r >> 1)) * SA + wm0 + i * 16 + fr + 8 * (r & 1);
          a_re[i][r] = As[buf][0][idx];
          if (CPLX) {
            a_im[i][r] = sa * As[buf][NPL - 1][idx];
            a_sum[i][r] = a_re[i][r] + a_im[i][r];
          }
        }
#pragma unroll
      for (int j = 0; j < TJ; ++j)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int idx = (ks * 8 + fk + 4 * r) * SB + wn0 + j * 8 + fr;
          b_re[j][r] = Bs[buf][0][idx];
          if (CPLX) {
            b_im[j][r] = sb * Bs[buf][NPL - 1][idx];
            b_sum[j][r] = b_re[j][r] + b_im[j][r];
          }
        }
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) {
          dmma_1688(cr[i][j], a_re[i], b_re[j]);
          if (CPLX) {
            dmma_1688(cm[i][j], a_im[i], b_im[j]);
            dmma_1688(ci[i][j], a_sum[i], b_sum[j]);
          }
        }
    }
  }
  cp_async_wait<0>();  // no copy may still target the ring when the next tile starts

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
        if (m0 + rr >= g.M || n0 + cc >= g.N) continue;
        const double re = CPLX ? cr[i][j][q] - cm[i][j][q] : cr[i][j][q];
        const double im = CPLX ? ci[i][j][q] - cr[i][j][q] - cm[i][j][q] : 0.0;
        if (g.partial)
          Elem<double, CPLX>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n0 + cc) * g.M + m0 + rr,
                                    re, im);
        else
          epilogue_store<double, CPLX>(g.e, re, im, Cb + cm_s[rr] + cn_s[cc], Db + dm_s[rr] + dn_s[cc]);
      }
}

// ---------------------------------------------------------------- SIMT (FFMA), cp.async ring

// Shape of the FP32 stage ring (dynamic shared memory): planar [k][row]
// stages, rows padded by 4 floats.
template <bool CPLX, int BM, int BN, int BK>
struct SimtRing {
  static constexpr int SA = BM + 4, SB = BN + 4;
  static constexpr int NPL = CPLX ? 2 : 1;
  static constexpr int STAGES = 4;
  static constexpr int A_STAGE = NPL * BK * SA, B_STAGE = NPL * BK * SB;  // floats
  static constexpr int BYTES = STAGES * (A_STAGE + B_STAGE) * 4;
};

// FP32 register tile fed by a ring of STAGES shared-memory stages filled with
// cp.async (the gather of TileGather, without staging through registers), so
// the global loads of three stages are in flight behind the FFMA work. Each
// thread owns a TM x TN tile (two halves of TM/2 rows and TN/2 columns, so the
// fragment reads are vector loads without bank conflicts) and accumulates each
// BK-deep stage into a fresh register tile that is then added to the total
// (FP32 error near u * (sqrt(BK) + sqrt(K / BK))). CA / CB: conjugated A' / B'
// (complex only), folded into the signs of the FFMAs at compile time.
template <int BM, int BN>
struct TileScatters {
  int64_t am[BM], bn[BN], dm[BM], cm[BM], dn[BN], cn[BN];
};

template <bool CPLX, bool CA, bool CB, int BM, int BN, int BK, int TM, int TN>
__device__ __forceinline__ void simt_tile_async_body(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                                     int64_t split, TileScatters<BM, BN>& sc) {
  using R = float;
  using Ring = SimtRing<CPLX, BM, BN, BK>;
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int SA = Ring::SA, SB = Ring::SB, NPL = Ring::NPL, STAGES = Ring::STAGES;
  using T = typename Elem<R, CPLX>::type;

  extern __shared__ __align__(16) float simt_ring[];
  R(*As)[NPL][BK * SA] = reinterpret_cast<R(*)[NPL][BK * SA]>(simt_ring);
  R(*Bs)[NPL][BK * SB] = reinterpret_cast<R(*)[NPL][BK * SB]>(simt_ring + STAGES * Ring::A_STAGE);
  int64_t *am_s = sc.am, *bn_s = sc.bn, *dm_s = sc.dm, *cm_s = sc.cm, *dn_s = sc.dn, *cn_s = sc.cn;

  const int tid = threadIdx.x;
  const int64_t m0 = mtile * BM, n0 = ntile * BN;
  for (int i = tid; i < BM; i += NT) {
    const int64_t m = m0 + i;
    const bool ok = m < g.M;
    am_s[i] = ok ? g.s.a_m[m] : 0;
    dm_s[i] = ok ? g.s.d_m[m] : 0;
    cm_s[i] = ok ? g.s.c_m[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int64_t n = n0 + i;
    const bool ok = n < g.N;
    bn_s[i] = ok ? g.s.b_n[n] : 0;
    dn_s[i] = ok ? g.s.d_n[n] : 0;
    cn_s[i] = ok ? g.s.c_n[n] : 0;
  }
  __syncthreads();

  const T* Ab = static_cast<const T*>(g.A) + g.s.h_a[h];
  const T* Bb = static_cast<const T*>(g.B) + g.s.h_b[h];
  AsyncGather<R, CPLX, BM, BK, NT> ga;
  AsyncGather<R, CPLX, BN, BK, NT> gb;

  constexpr int HM = TM / 2, HN = TN / 2;
  const int tx = tid % (BM / TM), ty = tid / (BM / TM);
  R tot_re[TM][TN], tot_im[CPLX ? TM : 1][CPLX ? TN : 1];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      tot_re[i][j] = R(0);
      if (CPLX) tot_im[i][j] = R(0);
    }

  const int64_t kb = g.k_chunk ? split * g.k_chunk : 0;
  const int64_t ke = g.k_chunk ? min(g.K, kb + g.k_chunk) : g.K;
  const int64_t nt = (ke - kb + BK - 1) / BK;
  ga.init(am_s, m0, g.M, g.a_kfast, tid);
  gb.init(bn_s, n0, g.N, g.b_kfast, tid);
#pragma unroll
  for (int sidx = 0; sidx < STAGES - 1; ++sidx) {
    if (sidx < nt) {
      ga.load_idx(g.s.a_k, kb + sidx * BK, ke, g.a_kfast, tid);
      gb.load_idx(g.s.b_k, kb + sidx * BK, ke, g.b_kfast, tid);
      ga.issue(Ab, As[sidx][0], As[sidx][NPL - 1], SA, g.a_kfast, tid);
      gb.issue(Bb, Bs[sidx][0], Bs[sidx][NPL - 1], SB, g.b_kfast, tid);
    }
    cp_async_commit();
  }

  for (int64_t t = 0; t < nt; ++t) {
    const int64_t tp = t + STAGES - 1;
    if (tp < nt) {
      ga.load_idx(g.s.a_k, kb + tp * BK, ke, g.a_kfast, tid);
      gb.load_idx(g.s.b_k, kb + tp * BK, ke, g.b_kfast, tid);
    }
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    if (tp < nt) {
      const int pb = (int)(tp % STAGES);
      ga.issue(Ab, As[pb][0], As[pb][NPL - 1], SA, g.a_kfast, tid);
      gb.issue(Bb, Bs[pb][0], Bs[pb][NPL - 1], SB, g.b_kfast, tid);
    }
    cp_async_commit();
    const int buf = (int)(t % STAGES);
    R acc_re[TM][TN], acc_im[CPLX ? TM : 1][CPLX ? TN : 1];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        acc_re[i][j] = R(0);
        if (CPLX) acc_im[i][j] = R(0);
      }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      R ar[TM], br[TN], ai[CPLX ? TM : 1], bi[CPLX ? TN : 1];
#pragma unroll
      for (int i = 0; i < HM; ++i) {
        ar[i] = As[buf][0][kk * SA + tx * HM + i];
        ar[HM + i] = As[buf][0][kk * SA + BM / 2 + tx * HM + i];
        if (CPLX) {
          ai[i] = As[buf][NPL - 1][kk * SA + tx * HM + i];
          ai[HM + i] = As[buf][NPL - 1][kk * SA + BM / 2 + tx * HM + i];
        }
      }
#pragma unroll
      for (int j = 0; j < HN; ++j) {
        br[j] = Bs[buf][0][kk * SB + ty * HN + j];
        br[HN + j] = Bs[buf][0][kk * SB + BN / 2 + ty * HN + j];
        if (CPLX) {
          bi[j] = Bs[buf][NPL - 1][kk * SB + ty * HN + j];
          bi[HN + j] = Bs[buf][NPL - 1][kk * SB + BN / 2 + ty * HN + j];
        }
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          if (CPLX) {
            // (ar + i sa ai)(br + i sb bi), sa = -1 when A' is conjugated, sb likewise.
            acc_re[i][j] = fma(ar[i], br[j], acc_re[i][j]);
            acc_re[i][j] = fma((CA != CB) ? ai[i] : -ai[i], bi[j], acc_re[i][j]);
            acc_im[i][j] = fma(CB ? -ar[i] : ar[i], bi[j], acc_im[i][j]);
            acc_im[i][j] = fma(CA ? -ai[i] : ai[i], br[j], acc_im[i][j]);
          } else {
            acc_re[i][j] = fma(ar[i], br[j], acc_re[i][j]);
          }
        }
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        tot_re[i][j] += acc_re[i][j];
        if (CPLX) tot_im[i][j] += acc_im[i][j];
      }
  }
  cp_async_wait<0>();  // no copy may still target the ring when the next tile starts

  const T* Cb = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]);
  T* Db = static_cast<T*>(g.D) + g.s.h_d[h];
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int rr = (i < HM) ? (tx * HM + i) : (BM / 2 + tx * HM + (i - HM));
    if (m0 + rr >= g.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int cc = (j < HN) ? (ty * HN + j) : (BN / 2 + ty * HN + (j - HN));
      if (n0 + cc >= g.N) continue;
      if (g.partial)
        Elem<R, CPLX>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n0 + cc) * g.M + m0 + rr,
                             tot_re[i][j], CPLX ? tot_im[i][j] : R(0));
      else
        epilogue_store<R, CPLX>(g.e, tot_re[i][j], CPLX ? tot_im[i][j] : R(0), Cb + cm_s[rr] + cn_s[cc],
                              Db + dm_s[rr] + dn_s[cc]);
    }
  }
}

// The conjugation variant of a complex tile is chosen per tile.
template <bool CPLX, int BM, int BN, int BK, int TM, int TN>
__device__ __forceinline__ void simt_tile_async(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                                int64_t split = 0) {
  __shared__ TileScatters<BM, BN> sc;
  if (!CPLX || (!g.conj_a && !g.conj_b))
    simt_tile_async_body<CPLX, false, false, BM, BN, BK, TM, TN>(g, h, mtile, ntile, split, sc);
  else if (g.conj_a && !g.conj_b)
    simt_tile_async_body<CPLX, true, false, BM, BN, BK, TM, TN>(g, h, mtile, ntile, split, sc);
  else if (!g.conj_a)
    simt_tile_async_body<CPLX, false, true, BM, BN, BK, TM, TN>(g, h, mtile, ntile, split, sc);
  else
    simt_tile_async_body<CPLX, true, true, BM, BN, BK, TM, TN>(g, h, mtile, ntile, split, sc);
}

// Register-staged variant (used for real f64): 4 warps in a 2x2 arrangement,
// each warp a WM x WN tile of 16x8 DMMA tiles, two shared-memory stages, the
// next stage's elements held in registers (TileGather).
template <bool CPLX, int WM, int WN, int BK>
__device__ __forceinline__ void dmma_tile_regs(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                          int64_t split = 0) {
  constexpr int BM = 2 * WM, BN = 2 * WN, NT = 128;
  constexpr int SA = BM + 4, SB = BN + 4;  // strides = 4 (mod 16) doubles: conflict-free fragment reads
  constexpr int NPL = CPLX ? 2 : 1;
  constexpr int TI = WM / 16, TJ = WN / 8;
  static_assert(WM % 16 == 0 && WN % 8 == 0 && BK % 8 == 0, "m16n8k8 fragments");
  using T = typename Elem<double, CPLX>::type;

  __shared__ __align__(16) double As[2][NPL][BK * SA];
  __shared__ __align__(16) double Bs[2][NPL][BK * SB];
  __shared__ int64_t am_s[BM], bn_s[BN], dm_s[BM], cm_s[BM], dn_s[BN], cn_s[BN];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t m0 = mtile * BM, n0 = ntile * BN;
  const int wm0 = (warp & 1) * WM, wn0 = (warp >> 1) * WN;

  for (int i = tid; i < BM; i += NT) {
    const int64_t m = m0 + i;
    const bool ok = m < g.M;
    am_s[i] = ok ? g.s.a_m[m] : 0;
    dm_s[i] = ok ? g.s.d_m[m] : 0;
    cm_s[i] = ok ? g.s.c_m[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int64_t n = n0 + i;
    const bool ok = n < g.N;
    bn_s[i] = ok ? g.s.b_n[n] : 0;
    dn_s[i] = ok ? g.s.d_n[n] : 0;
    cn_s[i] = ok ? g.s.c_n[n] : 0;
  }
  __syncthreads();

  const T* Ab = static_cast<const T*>(g.A) + g.s.h_a[h];
  const T* Bb = static_cast<const T*>(g.B) + g.s.h_b[h];
  TileGather<double, CPLX, BM, BK, NT> ga;
  TileGather<double, CPLX, BN, BK, NT> gb;

  double cr[TI][TJ][4], ci[CPLX ? TI : 1][CPLX ? TJ : 1][4];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        cr[i][j][q] = 0.0;
        if (CPLX) ci[i][j][q] = 0.0;
      }

  // This CTA's K range (the whole of K unless split).
  const int64_t kb = g.k_chunk ? split * g.k_chunk : 0;
  const int64_t ke = g.k_chunk ? min(g.K, kb + g.k_chunk) : g.K;
  const int64_t nt = (ke - kb + BK - 1) / BK;
  ga.init(am_s, m0, g.M, g.a_kfast, tid);
  gb.init(bn_s, n0, g.N, g.b_kfast, tid);
  ga.load_idx(g.s.a_k, kb, ke, g.a_kfast, tid);
  gb.load_idx(g.s.b_k, kb, ke, g.b_kfast, tid);
  ga.load(Ab, g.conj_a);
  gb.load(Bb, g.conj_b);
  ga.store(As[0][0], As[0][NPL - 1], SA, g.a_kfast, tid);
  gb.store(Bs[0][0], Bs[0][NPL - 1], SB, g.b_kfast, tid);
  if (nt > 1) {
    ga.load_idx(g.s.a_k, kb + BK, ke, g.a_kfast, tid);
    gb.load_idx(g.s.b_k, kb + BK, ke, g.b_kfast, tid);
  }
  __syncthreads();

  const int fr = lane >> 2, fk = lane & 3;
  for (int64_t t = 0; t < nt; ++t) {
    const int buf = (int)(t & 1);
    if (t + 1 < nt) {
      ga.load(Ab, g.conj_a);
      gb.load(Bb, g.conj_b);
    }
#pragma unroll
    for (int ks = 0; ks < BK / 8; ++ks) {
      double a_re[TI][4], b_re[TJ][2], a_im[CPLX ? TI : 1][4], na_im[CPLX ? TI : 1][4], b_im[CPLX ? TJ : 1][2];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int idx = (ks * 8 + fk + 4 * (r >> 1)) * SA + wm0 + i * 16 + fr + 8 * (r & 1);
          a_re[i][r] = As[buf][0][idx];
          if (CPLX) {
            a_im[i][r] = As[buf][NPL - 1][idx];
            na_im[i][r] = -a_im[i][r];
          }
        }
#pragma unroll
      for (int j = 0; j < TJ; ++j)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int idx = (ks * 8 + fk + 4 * r) * SB + wn0 + j * 8 + fr;
          b_re[j][r] = Bs[buf][0][idx];
          if (CPLX) b_im[j][r] = Bs[buf][NPL - 1][idx];
        }
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) {
          dmma_1688(cr[i][j], a_re[i], b_re[j]);
          if (CPLX) {
            dmma_1688(cr[i][j], na_im[i], b_im[j]);
            dmma_1688(ci[i][j], a_re[i], b_im[j]);
            dmma_1688(ci[i][j], a_im[i], b_re[j]);
          }
        }
    }
    if (t + 1 < nt) {
      ga.store(As[buf ^ 1][0], As[buf ^ 1][NPL - 1], SA, g.a_kfast, tid);
      gb.store(Bs[buf ^ 1][0], Bs[buf ^ 1][NPL - 1], SB, g.b_kfast, tid);
      if (t + 2 < nt) {
        ga.load_idx(g.s.a_k, kb + (t + 2) * BK, ke, g.a_kfast, tid);
        gb.load_idx(g.s.b_k, kb + (t + 2) * BK, ke, g.b_kfast, tid);
      }
    }
    __syncthreads();
  }

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
        if (m0 + rr >= g.M || n0 + cc >= g.N) continue;
        if (g.partial)
          Elem<double, CPLX>::store(static_cast<T*>(g.partial) + ((split * g.H + h) * g.N + n0 + cc) * g.M + m0 + rr,
                                    cr[i][j][q], CPLX ? ci[i][j][q] : 0.0);
        else
          epilogue_store<double, CPLX>(g.e, cr[i][j][q], CPLX ? ci[i][j][q] : 0.0, Cb + cm_s[rr] + cn_s[cc],
                                     Db + dm_s[rr] + dn_s[cc]);
      }
}

// The DMMA tile body: measured on B200, the cp.async ring is faster for the
// planar complex tiles and the register-staged path for real f64.
template <bool CPLX, int WM, int WN, int BK>
__device__ __forceinline__ void dmma_tile(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile,
                                          int64_t split = 0) {
  if constexpr (CPLX)
    dmma_tile_async<CPLX, WM, WN, BK>(g, h, mtile, ntile, split);
  else
    dmma_tile_regs<CPLX, WM, WN, BK>(g, h, mtile, ntile, split);
}

// Dynamic shared memory of a DMMA tile body.
template <bool CPLX, int WM, int WN, int BK>
constexpr int dmma_dyn_smem() {
  return CPLX ? DmmaRing<CPLX, WM, WN, BK>::BYTES : 0;
}

// Tile t of a one-launch contraction: N tile fastest, then M tile, then
// z = split * H + h. A 1-D grid (looping when there are more tiles than
// CTAs), so neither the batch count nor the M tile count is limited to the
// 65535 of a grid's y and z dimensions.
__device__ __forceinline__ void tile_coords(int64_t t, int64_t tn, int64_t tm, int64_t& nt, int64_t& mt,
                                            int64_t& z) {
  nt = t % tn;
  mt = (t / tn) % tm;
  z = t / (tn * tm);
}

template <class R, bool CPLX, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1) simt_gemm_kernel(GemmArgs g) {
  const int64_t tn = (g.N + BN - 1) / BN, tm = (g.M + BM - 1) / BM;
  const int64_t total = tn * tm * g.H * (g.k_chunk ? (g.K + g.k_chunk - 1) / g.k_chunk : 1);
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int64_t nt, mt, z;
    tile_coords(t, tn, tm, nt, mt, z);
    simt_tile<R, CPLX, BM, BN, BK, TM, TN>(g, z % g.H, mt, nt, z / g.H);
    __syncthreads();  // the next tile rewrites the shared scatter arrays
  }
}

template <bool CPLX, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), 1) simt_ring_gemm_kernel(GemmArgs g) {
  const int64_t tn = (g.N + BN - 1) / BN, tm = (g.M + BM - 1) / BM;
  const int64_t total = tn * tm * g.H * (g.k_chunk ? (g.K + g.k_chunk - 1) / g.k_chunk : 1);
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int64_t nt, mt, z;
    tile_coords(t, tn, tm, nt, mt, z);
    simt_tile_async<CPLX, BM, BN, BK, TM, TN>(g, z % g.H, mt, nt, z / g.H);
    __syncthreads();  // the next tile rewrites the shared scatter arrays
  }
}

// Three CTAs per SM (at most 170 registers a thread): twelve warps to hide the
// gather and shared-memory latency around the DMMA pipe; two for the tall
// complex tile, whose three 3m accumulators need the registers.
template <bool CPLX, int WM, int WN, int BK>
__global__ void __launch_bounds__(128, (CPLX && WM == 64) ? 2 : 3) dmma_gemm_kernel(GemmArgs g) {
  constexpr int BM = 2 * WM, BN = 2 * WN;
  const int64_t tn = (g.N + BN - 1) / BN, tm = (g.M + BM - 1) / BM;
  const int64_t total = tn * tm * g.H * (g.k_chunk ? (g.K + g.k_chunk - 1) / g.k_chunk : 1);
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int64_t nt, mt, z;
    tile_coords(t, tn, tm, nt, mt, z);
    dmma_tile<CPLX, WM, WN, BK>(g, z % g.H, mt, nt, z / g.H);
    __syncthreads();  // the next tile rewrites the shared scatter arrays
  }
}

// Persistent grouped kernel over a heterogeneous list (contract_batched): the
// tiles of all items form one queue, in the order of `tile_start` (items
// sorted by decreasing cost on the host, so the longest tiles go first); each
// CTA claims the next tile with an atomic counter, copies the item's
// arguments to shared memory and runs the same tile body as the one-item
// kernels. Claiming never waits. The kernel checks itself: a claim loop longer
// than the queue, a run past a %globaltimer limit, or an item / tile index out
// of range sets STATUS_BAD_ARGUMENT (or STATUS_WAIT_TIMEOUT) in the status
// word and ends the CTA.
template <class Tile, int NT>
__global__ void __launch_bounds__(NT, Tile::MIN_BLOCKS) grouped_kernel(const GroupItem* __restrict__ items,
                                                     const int64_t* __restrict__ tile_start, int nitems,
                                                     unsigned long long* counter, unsigned* status) {
  __shared__ __align__(16) GemmArgs sg;
  __shared__ long long claimed;
  __shared__ int item_s;
  __shared__ int stop;
  __shared__ int sg_item;  // the item whose arguments `sg` holds
  if (threadIdx.x == 0) sg_item = -1;
  const int64_t total = tile_start[nitems];
  const uint64_t t_start = globaltimer_ns();
  constexpr uint64_t LIMIT_NS = 60000000000ull;  // 60 s for one grouped launch
  // The claim of the next tile is issued before the current tile runs (its
  // result is first used after the tile), so the atomic's round trip overlaps
  // the tile instead of adding to it.
  long long next = 0;
  if (threadIdx.x == 0) next = (long long)atomicAdd(counter, 1ull);
  for (int64_t iter = 0;; ++iter) {
    if (threadIdx.x < 32) {
      // Find the item whose tile range holds the claimed tile (the last index
      // with tile_start <= claimed) by a 32-way search across the warp: each
      // round probes 32 evenly spaced entries at once, so a list of n items
      // costs about log32(n) dependent loads instead of log2(n).
      const int lane = threadIdx.x;
      const long long c = __shfl_sync(0xffffffffu, next, 0);
      int lo = 0, hi = nitems - 1;
      while (lo < hi) {
        const int step = (hi - lo + 32) / 32;
        const int pos = lo + lane * step;
        const bool le = pos <= hi && tile_start[pos] <= c;
        const unsigned m = __ballot_sync(0xffffffffu, le) | 1u;  // tile_start[lo] <= c holds for lo
        lo += (31 - __clz(m)) * step;
        hi = min(hi, lo + step - 1);
      }
      if (lane == 0) {
        stop = 0;
        claimed = c;
        item_s = lo;
      }
    }
    if (threadIdx.x == 0) {
      const int lo = item_s;
      if (claimed < total) {
        const int64_t local = claimed - tile_start[lo];
        const int64_t nt = items[lo].tiles_m * items[lo].tiles_n * items[lo].g.H;
        if (lo < 0 || lo >= nitems || local < 0 || local >= nt || iter > total) {
          atomicOr(status, STATUS_BAD_ARGUMENT);
          stop = 1;
        } else if (globaltimer_ns() - t_start > LIMIT_NS) {
          atomicOr(status, STATUS_WAIT_TIMEOUT);
          stop = 1;
        }
      }
    }
    __syncthreads();
    const long long t = claimed;
    if (t >= total || stop) break;
    if (threadIdx.x == 0) next = (long long)atomicAdd(counter, 1ull);
    const int it = item_s;
    if (it != sg_item) {  // uniform: both values were written before the barrier above
      const int4* src = reinterpret_cast<const int4*>(&items[it].g);
      int4* dst = reinterpret_cast<int4*>(&sg);
      for (int w = threadIdx.x; w < (int)(sizeof(GemmArgs) / 16); w += NT) dst[w] = src[w];
      __syncthreads();
      if (threadIdx.x == 0) sg_item = it;
    }
    const int64_t local = t - tile_start[it];
    const int64_t tn = items[it].tiles_n, tm = items[it].tiles_m;
    // Tile coordinates (batch, row tile, column tile); 32-bit divisions when
    // the item's tile counts fit, as they do for any realistic item.
    int64_t th, tmi, tni;
    if (local < 0x7fffffff && tm * tn < 0x7fffffff) {
      const uint32_t l = (uint32_t)local, per = (uint32_t)(tm * tn), n32 = (uint32_t)tn;
      const uint32_t hq = l / per, r = l - hq * per, mq = r / n32;
      th = hq;
      tmi = mq;
      tni = r - mq * n32;
    } else {
      th = local / (tm * tn);
      tmi = (local / tn) % tm;
      tni = local % tn;
    }
    Tile::run(sg, th, tmi, tni);
    __syncthreads();
  }
}

template <class R, bool CPLX, int BM, int BN, int BK, int TM, int TN>
struct SimtTileOp {
  static constexpr int NT = (BM / TM) * (BN / TN);
  static constexpr int SMEM = 0;
  static constexpr int MIN_BLOCKS = 1;
  __device__ static void run(const GemmArgs& g, int64_t h, int64_t mt, int64_t nt) {
    simt_tile<R, CPLX, BM, BN, BK, TM, TN>(g, h, mt, nt);
  }
};
template <bool CPLX, int BM, int BN, int BK, int TM, int TN>
struct SimtRingTileOp {
  static constexpr int NT = (BM / TM) * (BN / TN);
  static constexpr int SMEM = SimtRing<CPLX, BM, BN, BK>::BYTES;
  static constexpr int MIN_BLOCKS = 1;
  __device__ static void run(const GemmArgs& g, int64_t h, int64_t mt, int64_t nt) {
    simt_tile_async<CPLX, BM, BN, BK, TM, TN>(g, h, mt, nt);
  }
};
template <bool CPLX, int WM, int WN, int BK, int STG = 4, int MINB = (WM == 64 ? 2 : 3)>
struct DmmaTileOp {
  // Grouped lists (many short-K tiles) take the cp.async ring for real f64 too.
  static constexpr int NT = 128;
  static constexpr int SMEM = DmmaRing<CPLX, WM, WN, BK, STG>::BYTES;
  static constexpr int MIN_BLOCKS = MINB;  // the tall tile's ring needs 86 KB
  __device__ static void run(const GemmArgs& g, int64_t h, int64_t mt, int64_t nt) {
    dmma_tile_async<CPLX, WM, WN, BK, STG>(g, h, mt, nt);
  }
};

// Short-K f64 tile of grouped lists (K <= 64, N <= BN; grouped only): 128
// rows x BN columns with the whole K extent in one shared-memory stage (one
// round of cp.async through the scatter vectors, whose k offsets are staged
// with the row and column offsets), then FP64 FMAs from registers, 4 rows x
// BN/8 columns per thread with rows 32 apart, so each warp store covers 32
// consecutive rows of D. One barrier per tile and no fragment bookkeeping:
// far fewer instructions per output than a DMMA tile spends on these shapes
// (step 2 of the C4 updates, K = N <= 64), and 256 threads with two CTAs per
// SM to hide the latency of a tile's single load round. BN = 16, 32 or 64
// keeps the padding of narrow outputs at most 2x.
template <int BN, int KM>
struct SkinnyRing {
  static constexpr int BM = 128, KMAX = KM, SA = BM + 4, SB = BN + 4;
  static constexpr int BYTES = KMAX * (SA + SB) * 8;
};

template <int BN, int KM>
__device__ __forceinline__ void skinny_tile(const GemmArgs& g, int64_t h, int64_t mtile, int64_t ntile) {
  using Ring = SkinnyRing<BN, KM>;
  constexpr int BM = Ring::BM, KMAX = Ring::KMAX, SA = Ring::SA, SB = Ring::SB, NT = 256;
  constexpr int TN = BN / 8;  // columns per thread: 8 column groups, one per warp
  extern __shared__ __align__(16) double skinny_ring[];
  double* As = skinny_ring;              // [k][row], row stride SA
  double* Bs = skinny_ring + KMAX * SA;  // [k][col], row stride SB
  __shared__ int64_t am_s[BM], dm_s[BM], cm_s[BM], bn_s[BN], dn_s[BN], cn_s[BN], ak_s[KMAX], bk_s[KMAX];
  const int tid = threadIdx.x;
  const int64_t m0 = mtile * BM, n0 = ntile * BN;
  const int64_t K = g.K < KMAX ? g.K : KMAX;  // the host routes only K <= KMAX here
  for (int i = tid; i < BM; i += NT) {
    const int64_t m = m0 + i;
    const bool ok = m < g.M;
    am_s[i] = ok ? g.s.a_m[m] : 0;
    dm_s[i] = ok ? g.s.d_m[m] : 0;
    cm_s[i] = (ok && !g.e.beta_zero) ? g.s.c_m[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int64_t n = n0 + i;
    const bool ok = n < g.N;
    bn_s[i] = ok ? g.s.b_n[n] : 0;
    dn_s[i] = ok ? g.s.d_n[n] : 0;
    cn_s[i] = (ok && !g.e.beta_zero) ? g.s.c_n[n] : 0;
  }
  for (int i = tid; i < K; i += NT) {
    ak_s[i] = g.s.a_k[i];
    bk_s[i] = g.s.b_k[i];
  }
  __syncthreads();
  {
    // All copies issued back to back, 16 k at a time (few offsets held in
    // registers); elements past K or past the operand's rows are zero-filled.
    constexpr int KB = 16;
    AsyncGather<double, false, BM, KB, NT> ga;
    AsyncGather<double, false, BN, KB, NT> gb;
    ga.init(am_s, m0, g.M, g.a_kfast, tid);
    gb.init(bn_s, n0, g.N, g.b_kfast, tid);
    const double* Ab = static_cast<const double*>(g.A) + g.s.h_a[h];
    const double* Bb = static_cast<const double*>(g.B) + g.s.h_b[h];
    for (int64_t k0 = 0; k0 < K; k0 += KB) {
      ga.load_idx_s(ak_s, 0, k0, K, g.a_kfast, tid);
      gb.load_idx_s(bk_s, 0, k0, K, g.b_kfast, tid);
      ga.issue(Ab, As + k0 * SA, As + k0 * SA, SA, g.a_kfast, tid);
      gb.issue(Bb, Bs + k0 * SB, Bs + k0 * SB, SB, g.b_kfast, tid);
    }
    cp_async_commit();
    cp_async_wait<0>();
  }
  __syncthreads();
  const int tx = tid & 31, ty = tid >> 5;
  double acc[4][TN];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;
  for (int k = 0; k < K; ++k) {
    double a[4], b[TN];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = As[k * SA + tx + 32 * i];
#pragma unroll
    for (int j = 0; j < TN; ++j) b[j] = Bs[k * SB + ty * TN + j];  // the same for the whole warp
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
  const double* Cb = static_cast<const double*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h]);
  double* Db = static_cast<double*>(g.D) + g.s.h_d[h];
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const int cc = ty * TN + j;
    if (n0 + cc >= g.N) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rr = tx + 32 * i;
      if (m0 + rr < g.M)
        epilogue_store<double, false>(g.e, acc[i][j], 0.0, Cb + cm_s[rr] + cn_s[cc], Db + dm_s[rr] + dn_s[cc]);
    }
  }
}

// KM = 64 takes K <= 64 at two CTAs per SM; KM = 32 (K <= 32, most of the
// C4 step-2 items) halves the A stage and runs three CTAs per SM (four with
// 16 columns, whose accumulators leave room in 64 registers). Occupancy is
// what these tiles need: their one load round per tile is latency.
template <int BN, int KM>
struct SkinnyTileOp {
  static constexpr int NT = 256;
  static constexpr int SMEM = SkinnyRing<BN, KM>::BYTES;
  static constexpr int MIN_BLOCKS = KM == 32 ? (BN == 16 ? 4 : 3) : 2;
  __device__ static void run(const GemmArgs& g, int64_t h, int64_t mt, int64_t nt) {
    skinny_tile<BN, KM>(g, h, mt, nt);
  }
};

template <int BM, int BN>
dim3 grid_for(const GemmArgs& g) {
  const int64_t splits = g.k_chunk ? (g.K + g.k_chunk - 1) / g.k_chunk : 1;
  const int64_t total = ((g.N + BN - 1) / BN) * ((g.M + BM - 1) / BM) * g.H * splits;
  return dim3((unsigned)(total < 0x7fffffff ? total : 0x7fffffff));
}

}  // namespace

const char* plain_kernel_name(int k) {
  switch (k) {
    case PLAIN_F32_SIMT_128x128: return "sm100.f32.simt.128x128x16";
    case PLAIN_F32_SIMT_64x64: return "sm100.f32.simt.64x64x16";
    case PLAIN_F64_DMMA_64x64: return "sm100.f64.dmma884.64x64x16";
    case PLAIN_F64_DMMA_32x32: return "sm100.f64.dmma884.32x32x16";
    case PLAIN_C32_SIMT_64x64: return "sm100.c32.simt.ring.planar.64x64x16";
    case PLAIN_C64_DMMA_64x32: return "sm100.c64.dmma884.3m.64x32x8";
    case PLAIN_C64_DMMA_32x32: return "sm100.c64.dmma884.3m.32x32x8";
    case PLAIN_F64_DMMA_128x32: return "sm100.f64.dmma884.128x32x16";
    case PLAIN_C64_DMMA_128x32: return "sm100.c64.dmma884.3m.128x32x8";
    case PLAIN_F32_PACKED_128x128: return "sm100.f32.simt.tma.packed.128x128x32";
    case PLAIN_C32_PACKED_1M_64x128: return "sm100.c32.simt.tma.1m.64x128x32";
    case PLAIN_F64_PACKED_64x64: return "sm100.f64.dmma884.tma.packed.64x64x16";
    case PLAIN_C64_PACKED_3M_64x32: return "sm100.c64.dmma884.tma.3m.64x32x16";
    case PLAIN_F32_PACKED_128x64: return "sm100.f32.simt.tma.packed.128x64x32";
    case PLAIN_C32_PACKED_1M_64x64: return "sm100.c32.simt.tma.1m.64x64x32";
    case PLAIN_F64_SKINNY_128x32: return "sm100.f64.fma.skinny.128x32xk64";
    case PLAIN_F64_SKINNY_128x64: return "sm100.f64.fma.skinny.128x64xk64";
    case PLAIN_F64_SKINNY_128x16: return "sm100.f64.fma.skinny.128x16xk64";
    case PLAIN_F64_SKINNY_128x16_K32: return "sm100.f64.fma.skinny.128x16xk32";
    case PLAIN_F64_SKINNY_128x32_K32: return "sm100.f64.fma.skinny.128x32xk32";
  }
  return "auto";
}

// Whether the packed families can take a shape: the pack grid's limits (batch
// and row tiles of 32 in a grid dimension) and the TMA maps' 32-bit rows.
bool packed_fits(int kernel, int64_t M, int64_t N, int64_t K, int64_t H) {
  const PackedLayout L = packed_layout(kernel, M, N, K, H);
  const int64_t rows = L.m_pad > L.n_pad ? L.m_pad : L.n_pad;
  return H <= 65535 && rows / 32 <= 65535 && (int64_t)L.planes * H * rows < ((int64_t)1 << 31) &&
         H * L.k_pad < ((int64_t)1 << 31) && K > 0;
}

int choose_plain_kernel(int dtype, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms) {
  auto tiles = [&](int bm, int bn) { return ((M + bm - 1) / bm) * ((N + bn - 1) / bn) * H; };
  // At least a full wave of packed tiles and some depth: the pack pass (one
  // read and one write of each operand) is then small beside the tiles' work.
  static const int packed[4] = {PLAIN_F32_PACKED_128x128, PLAIN_F64_PACKED_64x64, PLAIN_C32_PACKED_1M_64x64,
                                PLAIN_C64_PACKED_3M_64x32};
  {
    const int pk = packed[dtype & 3];
    int bm = 0, bn = 0;
    plain_tile_shape(pk, &bm, &bn);
    if (K >= 64 && tiles(bm, bn) >= num_sms && packed_fits(pk, M, N, K, H)) return pk;
  }
  switch (dtype) {
    case 0: return tiles(128, 128) >= num_sms ? PLAIN_F32_SIMT_128x128 : PLAIN_F32_SIMT_64x64;
    case 1: return tiles(64, 64) >= num_sms ? PLAIN_F64_DMMA_64x64 : PLAIN_F64_DMMA_32x32;
    case 2: return PLAIN_C32_SIMT_64x64;
    case 3: return tiles(64, 32) >= num_sms ? PLAIN_C64_DMMA_64x32 : PLAIN_C64_DMMA_32x32;
  }
  return PLAIN_AUTO;
}

int choose_grouped_kernel(int dtype, int64_t M, int64_t N, int64_t K) {
  // In a grouped launch the list fills the GPU, so the tile is chosen for
  // reuse and padding alone: the large tile unless it wastes much more of its
  // area on padding than the small one.
  static const int large[4] = {PLAIN_F32_SIMT_128x128, PLAIN_F64_DMMA_64x64, PLAIN_C32_SIMT_64x64,
                               PLAIN_C64_DMMA_64x32};
  static const int small[4] = {PLAIN_F32_SIMT_64x64, PLAIN_F64_DMMA_32x32, PLAIN_C32_SIMT_64x64,
                               PLAIN_C64_DMMA_32x32};
  auto util = [&](int k) {
    int bm = 0, bn = 0;
    plain_tile_shape(k, &bm, &bn);
    const double padded = (double)((M + bm - 1) / bm * bm) * (double)((N + bn - 1) / bn * bn);
    return (double)M * (double)N / padded;
  };
  // Short-K f64 items (K <= 64, N <= 64, some rows): the skinny FMA tile.
  if (dtype == 1 && K <= 32 && N <= 32 && M >= 128)
    return N <= 16 ? PLAIN_F64_SKINNY_128x16_K32 : PLAIN_F64_SKINNY_128x32_K32;
  if (dtype == 1 && K <= 64 && N <= 64 && M >= 128)
    return N <= 16 ? PLAIN_F64_SKINNY_128x16 : N <= 32 ? PLAIN_F64_SKINNY_128x32 : PLAIN_F64_SKINNY_128x64;
  const int L = large[dtype & 3], S = small[dtype & 3];
  const int best = util(L) >= 0.8 * util(S) ? L : S;
  // Narrow outputs (N <= 32) of many rows: the tall 128 x 32 tile amortises
  // each tile's fixed cost (scatter loads, epilogue) over four times the rows.
  if ((dtype == 1 || dtype == 3) && N <= 32 && M >= 256) {
    const int T = dtype == 1 ? PLAIN_F64_DMMA_128x32 : PLAIN_C64_DMMA_128x32;
    if (util(T) >= 0.9 * util(best)) return T;
  }
  return best;
}

void choose_plain_launch(int dtype, int pinned, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms, int* kernel,
                         int* splits, int64_t* k_chunk) {
  auto tiles = [&](int k) {
    int bm = 0, bn = 0;
    plain_tile_shape(k, &bm, &bn);
    return ((M + bm - 1) / bm) * ((N + bn - 1) / bn) * H;
  };
  static const int large[4] = {PLAIN_F32_SIMT_128x128, PLAIN_F64_DMMA_64x64, PLAIN_C32_SIMT_64x64,
                               PLAIN_C64_DMMA_64x32};
  static const int packed[4] = {PLAIN_F32_PACKED_128x128, PLAIN_F64_PACKED_64x64, PLAIN_C32_PACKED_1M_64x64,
                                PLAIN_C64_PACKED_3M_64x32};
  *splits = 1;
  *k_chunk = 0;
  const int64_t min_chunk = 512;  // K per split
  // Deep contractions split along K take the packed family when it fits.
  const int big = packed_fits(packed[dtype & 3], M, N, K, H) ? packed[dtype & 3] : large[dtype & 3];
  const int k = pinned ? pinned : big;
  const int64_t t = tiles(k);
  // Packed tiles stream their K range through a TMA ring, so shorter chunks
  // (at least 128 deep) still keep the pipe busy: a moderately deep
  // contraction with less than a wave of tiles splits too.
  const int64_t chunk_min = is_packed_kernel(k) ? 128 : min_chunk;
  if (t < num_sms && K >= 2 * chunk_min) {
    int64_t s = (2 * num_sms + t - 1) / t;
    s = s < K / chunk_min ? s : K / chunk_min;
    s = s < 64 ? s : 64;
    if (s > 1) {
      const int64_t chunk = ((K + s - 1) / s + 63) / 64 * 64;  // whole 64-deep blocks
      *kernel = k;
      *splits = (int)((K + chunk - 1) / chunk);
      *k_chunk = chunk;
      return;
    }
  }
  *kernel = pinned ? pinned : choose_plain_kernel(dtype, M, N, K, H, num_sms);
}

namespace {

// Split-K reduce: one thread per output element (m fastest), partials summed
// in split order, then the alpha/beta/conjugation epilogue through the scatter.
template <class R, bool CPLX>
__global__ void __launch_bounds__(256) splitk_reduce_kernel(GemmArgs g, int splits) {
  using T = typename Elem<R, CPLX>::type;
  const int64_t total = g.H * g.M * g.N;
  const T* P = static_cast<const T*>(g.partial);
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = idx % g.M, n = (idx / g.M) % g.N, h = idx / (g.M * g.N);
    R sr = R(0), si = R(0);
    for (int sp = 0; sp < splits; ++sp) {
      R vr, vi;
      Elem<R, CPLX>::load(P + ((sp * g.H + h) * g.N + n) * g.M + m, vr, vi);
      sr += vr;
      si += vi;
    }
    const T* c = static_cast<const T*>(g.C) + (g.e.beta_zero ? 0 : g.s.h_c[h] + g.s.c_m[m] + g.s.c_n[n]);
    T* d = static_cast<T*>(g.D) + g.s.h_d[h] + g.s.d_m[m] + g.s.d_n[n];
    epilogue_store<R, CPLX>(g.e, sr, si, c, d);
  }
}

}  // namespace

cudaError_t launch_splitk_reduce(int dtype, const GemmArgs& g, int splits, cudaStream_t st) {
  const int64_t total = g.H * g.M * g.N;
  if (total <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (total + 255) / 256;
  const unsigned blocks = (unsigned)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
  switch (dtype) {
    case 0: splitk_reduce_kernel<float, false><<<blocks, 256, 0, st>>>(g, splits); break;
    case 1: splitk_reduce_kernel<double, false><<<blocks, 256, 0, st>>>(g, splits); break;
    case 2: splitk_reduce_kernel<float, true><<<blocks, 256, 0, st>>>(g, splits); break;
    case 3: splitk_reduce_kernel<double, true><<<blocks, 256, 0, st>>>(g, splits); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

namespace {
template <bool CPLX, int WM, int WN, int BK>
cudaError_t launch_dmma(const GemmArgs& g, cudaStream_t st) {
  constexpr int bytes = dmma_dyn_smem<CPLX, WM, WN, BK>();
  if (bytes > 0) {
    const cudaError_t e =
        cudaFuncSetAttribute(dmma_gemm_kernel<CPLX, WM, WN, BK>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  dmma_gemm_kernel<CPLX, WM, WN, BK><<<grid_for<2 * WM, 2 * WN>(g), 128, bytes, st>>>(g);
  return cudaGetLastError();
}
}  // namespace

namespace {
template <bool CPLX, int BM, int BN, int BK, int TM, int TN>
cudaError_t launch_simt_ring(const GemmArgs& g, cudaStream_t st) {
  constexpr int bytes = SimtRing<CPLX, BM, BN, BK>::BYTES;
  const cudaError_t e = cudaFuncSetAttribute(simt_ring_gemm_kernel<CPLX, BM, BN, BK, TM, TN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  simt_ring_gemm_kernel<CPLX, BM, BN, BK, TM, TN><<<grid_for<BM, BN>(g), (BM / TM) * (BN / TN), bytes, st>>>(g);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_plain_gemm(int dtype, int kernel, const GemmArgs& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.H <= 0) return cudaSuccess;
  switch (kernel) {
    case PLAIN_F32_SIMT_128x128:
      if (dtype != 0) return cudaErrorInvalidValue;
      simt_gemm_kernel<float, false, 128, 128, 16, 8, 8><<<grid_for<128, 128>(g), 256, 0, st>>>(g);
      break;
    case PLAIN_F32_SIMT_64x64:
      if (dtype != 0) return cudaErrorInvalidValue;
      simt_gemm_kernel<float, false, 64, 64, 16, 4, 4><<<grid_for<64, 64>(g), 256, 0, st>>>(g);
      break;
    case PLAIN_C32_SIMT_64x64:
      if (dtype != 2) return cudaErrorInvalidValue;
      return launch_simt_ring<true, 64, 64, 16, 4, 4>(g, st);
    case PLAIN_F64_DMMA_64x64:
      if (dtype != 1) return cudaErrorInvalidValue;
      return launch_dmma<false, 32, 32, 16>(g, st);
    case PLAIN_F64_DMMA_32x32:
      if (dtype != 1) return cudaErrorInvalidValue;
      return launch_dmma<false, 16, 16, 16>(g, st);
    case PLAIN_C64_DMMA_64x32:
      if (dtype != 3) return cudaErrorInvalidValue;
      return launch_dmma<true, 32, 16, 8>(g, st);
    case PLAIN_C64_DMMA_32x32:
      if (dtype != 3) return cudaErrorInvalidValue;
      return launch_dmma<true, 16, 16, 8>(g, st);
    case PLAIN_F64_DMMA_128x32:
      if (dtype != 1) return cudaErrorInvalidValue;
      return launch_dmma<false, 64, 16, 16>(g, st);
    case PLAIN_C64_DMMA_128x32:
      if (dtype != 3) return cudaErrorInvalidValue;
      return launch_dmma<true, 64, 16, 8>(g, st);
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

void plain_tile_shape(int kernel, int* bm, int* bn) {
  switch (kernel) {
    case PLAIN_F32_SIMT_128x128: *bm = 128; *bn = 128; return;
    case PLAIN_F32_SIMT_64x64: *bm = 64; *bn = 64; return;
    case PLAIN_C32_SIMT_64x64: *bm = 64; *bn = 64; return;
    case PLAIN_F64_DMMA_64x64: *bm = 64; *bn = 64; return;
    case PLAIN_F64_DMMA_32x32: *bm = 32; *bn = 32; return;
    case PLAIN_C64_DMMA_64x32: *bm = 64; *bn = 32; return;
    case PLAIN_C64_DMMA_32x32: *bm = 32; *bn = 32; return;
    case PLAIN_F64_DMMA_128x32: *bm = 128; *bn = 32; return;
    case PLAIN_C64_DMMA_128x32: *bm = 128; *bn = 32; return;
    case PLAIN_F32_PACKED_128x128: *bm = 128; *bn = 128; return;
    case PLAIN_C32_PACKED_1M_64x128: *bm = 64; *bn = 128; return;
    case PLAIN_F64_PACKED_64x64: *bm = 64; *bn = 64; return;
    case PLAIN_C64_PACKED_3M_64x32: *bm = 64; *bn = 32; return;
    case PLAIN_F32_PACKED_128x64: *bm = 128; *bn = 64; return;
    case PLAIN_C32_PACKED_1M_64x64: *bm = 64; *bn = 64; return;
    case PLAIN_F64_SKINNY_128x32: *bm = 128; *bn = 32; return;
    case PLAIN_F64_SKINNY_128x64: *bm = 128; *bn = 64; return;
    case PLAIN_F64_SKINNY_128x16: *bm = 128; *bn = 16; return;
    case PLAIN_F64_SKINNY_128x16_K32: *bm = 128; *bn = 16; return;
    case PLAIN_F64_SKINNY_128x32_K32: *bm = 128; *bn = 32; return;
  }
  *bm = *bn = 0;
}

namespace {

// Resident CTAs per SM of each grouped kernel (occupancy of the built code),
// filled before any capture by prepare_grouped: the persistent grid must not
// exceed what can be resident at once, or the CTAs beyond it start only when
// others have drained the queue.
int g_grouped_per_sm[24] = {};

template <class Op>
cudaError_t grouped_prepare_op(int kernel) {
  if (Op::SMEM > 0) {
    const cudaError_t a =
        cudaFuncSetAttribute(grouped_kernel<Op, Op::NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, Op::SMEM);
    if (a != cudaSuccess) return a;
  }
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, grouped_kernel<Op, Op::NT>, Op::NT, Op::SMEM);
  if (e != cudaSuccess) return e;
  g_grouped_per_sm[kernel] = n > 0 ? n : 1;
  return cudaSuccess;
}

template <class Op>
void grouped_launch_op(int kernel, const GroupItem* items, const int64_t* tile_start, int nitems,
                       unsigned long long* counter, unsigned* status, int num_sms, cudaStream_t st) {
  const int per_sm = g_grouped_per_sm[kernel] > 0 ? g_grouped_per_sm[kernel] : 1;
  grouped_kernel<Op, Op::NT><<<num_sms * per_sm, Op::NT, Op::SMEM, st>>>(items, tile_start, nitems, counter, status);
}

using GSimtF32L = SimtTileOp<float, false, 128, 128, 16, 8, 8>;
using GSimtF32S = SimtTileOp<float, false, 64, 64, 16, 4, 4>;
using GSimtC32 = SimtRingTileOp<true, 64, 64, 16, 4, 4>;
// The f64 64 x 64 list tile runs three 16-deep stages (52 KB) and four CTAs
// per SM (128 registers), trading a stage for a fourth CTA: list tiles are
// short-K and latency-bound.
using GDmmaF64L = DmmaTileOp<false, 32, 32, 16, 3, 4>;
// The 32 x 32 list tiles fit five CTAs per SM in 96 registers.
using GDmmaF64S = DmmaTileOp<false, 16, 16, 16, 4, 5>;
using GDmmaC64L = DmmaTileOp<true, 32, 16, 8>;
using GDmmaC64S = DmmaTileOp<true, 16, 16, 8, 4, 5>;
using GDmmaF64T = DmmaTileOp<false, 64, 16, 16>;
using GDmmaC64T = DmmaTileOp<true, 64, 16, 8>;
using GSkinny32 = SkinnyTileOp<32, 64>;
using GSkinny64 = SkinnyTileOp<64, 64>;
using GSkinny16 = SkinnyTileOp<16, 64>;
using GSkinny16s = SkinnyTileOp<16, 32>;
using GSkinny32s = SkinnyTileOp<32, 32>;

}  // namespace

// Loads the family's grouped kernel (module loading is lazy) and records its
// occupancy, so that the launch inside a stream capture needs neither.
cudaError_t prepare_grouped(int kernel) {
  switch (kernel) {
    case PLAIN_F32_SIMT_128x128: return grouped_prepare_op<GSimtF32L>(kernel);
    case PLAIN_F32_SIMT_64x64: return grouped_prepare_op<GSimtF32S>(kernel);
    case PLAIN_C32_SIMT_64x64: return grouped_prepare_op<GSimtC32>(kernel);
    case PLAIN_F64_DMMA_64x64: return grouped_prepare_op<GDmmaF64L>(kernel);
    case PLAIN_F64_DMMA_32x32: return grouped_prepare_op<GDmmaF64S>(kernel);
    case PLAIN_C64_DMMA_64x32: return grouped_prepare_op<GDmmaC64L>(kernel);
    case PLAIN_C64_DMMA_32x32: return grouped_prepare_op<GDmmaC64S>(kernel);
    case PLAIN_F64_DMMA_128x32: return grouped_prepare_op<GDmmaF64T>(kernel);
    case PLAIN_C64_DMMA_128x32: return grouped_prepare_op<GDmmaC64T>(kernel);
    case PLAIN_F64_SKINNY_128x32: return grouped_prepare_op<GSkinny32>(kernel);
    case PLAIN_F64_SKINNY_128x64: return grouped_prepare_op<GSkinny64>(kernel);
    case PLAIN_F64_SKINNY_128x16: return grouped_prepare_op<GSkinny16>(kernel);
    case PLAIN_F64_SKINNY_128x16_K32: return grouped_prepare_op<GSkinny16s>(kernel);
    case PLAIN_F64_SKINNY_128x32_K32: return grouped_prepare_op<GSkinny32s>(kernel);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_grouped(int kernel, const GroupItem* items, const int64_t* tile_start, int nitems,
                           unsigned long long* counter, unsigned* status, int num_sms, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  if (nitems <= 0) return cudaSuccess;
  switch (kernel) {
    case PLAIN_F32_SIMT_128x128:
      grouped_launch_op<GSimtF32L>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F32_SIMT_64x64:
      grouped_launch_op<GSimtF32S>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_C32_SIMT_64x64:
      grouped_launch_op<GSimtC32>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_DMMA_64x64:
      grouped_launch_op<GDmmaF64L>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_DMMA_32x32:
      grouped_launch_op<GDmmaF64S>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_C64_DMMA_64x32:
      grouped_launch_op<GDmmaC64L>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_C64_DMMA_32x32:
      grouped_launch_op<GDmmaC64S>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_DMMA_128x32:
      grouped_launch_op<GDmmaF64T>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_C64_DMMA_128x32:
      grouped_launch_op<GDmmaC64T>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_SKINNY_128x32:
      grouped_launch_op<GSkinny32>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_SKINNY_128x64:
      grouped_launch_op<GSkinny64>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_SKINNY_128x16:
      grouped_launch_op<GSkinny16>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_SKINNY_128x16_K32:
      grouped_launch_op<GSkinny16s>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    case PLAIN_F64_SKINNY_128x32_K32:
      grouped_launch_op<GSkinny32s>(kernel, items, tile_start, nitems, counter, status, num_sms, st);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace tprims
