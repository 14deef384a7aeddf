// Device-side interface shared by the host runtime and the kernels.
//
// Every kernel reads its operands through the oriented scatter vectors of a
// plan: element (h, m, k) of A' lives at A + h_a[h] + a_m[m] + a_k[k], element
// (h, k, n) of B' at B + h_b[h] + b_k[k] + b_n[n], and element (h, m, n) of the
// output at D + h_d[h] + d_m[m] + d_n[n] (likewise C). Offsets are in elements
// of the storage type. The reference packs panels through the same vectors
// (crates/tprims-kernel/src/pack/pack.rs:152-203) and writes back through them
// (pack/writeback.rs:311-486).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tprims {
namespace dev {

// Block scatters of the operand vectors (the reference's block scatter,
// crates/tprims-kernel/src/pack/scatter.rs:148-171, IRREGULAR sentinel :43):
// entry j of blk_x is the common difference of x[32 j .. 32 j + 31] (0 for a
// one-entry block) or SCATTER_IRREGULAR when the block is not an arithmetic
// run. A pack pass whose 32-row x 32-k tile sits on regular blocks of both of
// its vectors addresses the tile from one base offset and two strides (no
// per-element index loads), and loads 16-byte vectors along a unit-stride
// run. Null when absent (the kernels then read the scatter vectors); the
// struct is an aggregate, so an initializer list of the first 12 vectors (or
// value-initialization) leaves them null.
constexpr int SCATTER_BLOCK = 32;
constexpr int64_t SCATTER_IRREGULAR = INT64_MIN;

struct Scatters {
  const int64_t *a_m, *a_k, *b_k, *b_n, *c_m, *c_n, *d_m, *d_n, *h_a, *h_b, *h_c, *h_d;
  const int64_t *blk_a_m, *blk_a_k, *blk_b_k, *blk_b_n;
};

// D = op_D(alpha * acc + beta * op_C(C)); beta_zero means C is never read.
struct Epilogue {
  double alpha_re, alpha_im, beta_re, beta_im;
  int beta_zero;  // C not read
  int plain;      // alpha == 1, beta == 0, no conj on D: store acc as is
  int conj_c, conj_d;
};

// Bits of the device status word an executor owns. A kernel that gives up on a
// bounded wait or meets an inconsistent argument sets a bit and returns; the
// host turns a non-zero word into an error status.
enum : unsigned {
  STATUS_WAIT_TIMEOUT = 1u,
  STATUS_BAD_ARGUMENT = 2u,
};

struct GemmArgs {
  Scatters s;
  const void* A;
  const void* B;
  const void* C;
  void* D;
  int64_t M, N, K, H;
  int conj_a, conj_b;
  int a_kfast, b_kfast, d_mfast;
  Epilogue e;
  unsigned* status;
  // Split-K: each K chunk of k_chunk (a multiple of the tile depth; 0 = all
  // of K) is one CTA's range; with `partial` set, tiles write their raw
  // accumulators to partial[((split * H + h) * N + n) * M + m] and a reduce
  // pass applies the epilogue.
  int64_t k_chunk;
  void* partial;
};

// Kernel families of the plain (drop-in) path.
enum PlainKernel : int {
  PLAIN_AUTO = 0,
  PLAIN_F32_SIMT_128x128 = 1,
  PLAIN_F32_SIMT_64x64 = 2,
  PLAIN_F64_DMMA_64x64 = 3,
  PLAIN_F64_DMMA_32x32 = 4,
  PLAIN_C32_SIMT_64x64 = 5,
  PLAIN_C64_DMMA_64x32 = 6,
  PLAIN_C64_DMMA_32x32 = 7,
  PLAIN_F64_DMMA_128x32 = 8,  // tall tiles for N <= 32 (grouped lists)
  PLAIN_C64_DMMA_128x32 = 9,
  // Packed families: a pack pass writes dense panels, a TMA-fed tile reads them
  // (single launches only, never inside a grouped list).
  PLAIN_F32_PACKED_128x128 = 10,
  PLAIN_C32_PACKED_1M_64x128 = 11,  // 1m: the complex product as a 2M x N x 2K real one
  PLAIN_F64_PACKED_64x64 = 12,
  PLAIN_C64_PACKED_3M_64x32 = 13,   // 3m: three real products per complex MAC
  PLAIN_F32_PACKED_128x64 = 14,     // half-width FFMA tiles, two CTAs per SM
  PLAIN_C32_PACKED_1M_64x64 = 15,
  PLAIN_LAST = 15,  // the last family a caller can pin
  // Short-K f64 tiles (K <= 64) of grouped lists only: chosen by the model for
  // a list item, never pinned or used by single launches.
  PLAIN_F64_SKINNY_128x32 = 16,
  PLAIN_F64_SKINNY_128x64 = 17,
  PLAIN_F64_SKINNY_128x16 = 18,
  PLAIN_F64_SKINNY_128x16_K32 = 19,  // K <= 32: half the A stage, three CTAs per SM
  PLAIN_F64_SKINNY_128x32_K32 = 20,
};

// dtype: 0 f32, 1 f64, 2 c32, 3 c64 (TAPP numbering).
cudaError_t launch_output_pass(int dtype, const GemmArgs& g, cudaStream_t st);
cudaError_t launch_plain_gemm(int dtype, int kernel, const GemmArgs& g, cudaStream_t st);
static_assert(sizeof(GemmArgs) % 16 == 0, "grouped kernels copy GemmArgs in 16-byte words");

// One item of a grouped launch: its arguments and its tile grid.
struct GroupItem {
  GemmArgs g;
  int64_t tiles_m, tiles_n;
};
// CTA tile of a plain kernel family.
void plain_tile_shape(int kernel, int* bm, int* bn);
// Persistent grouped launch over `nitems` items whose tiles are numbered by the
// prefix `tile_start[0..nitems]` (device arrays); `counter` is reset here.
cudaError_t prepare_grouped(int kernel);
cudaError_t launch_grouped(int kernel, const GroupItem* items, const int64_t* tile_start, int nitems,
                           unsigned long long* counter, unsigned* status, int num_sms, cudaStream_t st);
// Register-only pipe probes (0: FP64 DMMA, 1: FP32 FFMA); *flops = work launched.
cudaError_t launch_probe(int which, void* sink, int blocks, int iters, cudaStream_t st, double* flops);
// Tensor-pipe probe (one CTA per SM): dense 128 x 256 tcgen05.mma products,
// kind::i8 (int8 = 1) or BF16 kind::f16 (int8 = 0); *ops = work launched.
cudaError_t launch_tc_probe(int int8, int blocks, int iters, unsigned* status, cudaStream_t st, double* ops);
// Bounded wait on a flag that stays zero: sets STATUS_WAIT_TIMEOUT after limit_ns.
cudaError_t launch_wait_selftest(const unsigned* flag, unsigned* status, uint64_t limit_ns, cudaStream_t st);
// Zero every element of a strided layout (origin = element of index 0).
cudaError_t launch_fill_zero(size_t elem, void* origin, int rank, const int64_t* dims, const int64_t* strides,
                             cudaStream_t st);
const char* plain_kernel_name(int kernel);
// The family the autotuner would pick for a shape (no launch).
int choose_plain_kernel(int dtype, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms);
// Batches of tiny products: per-operand batch strides when the batch scatter
// vector is an arithmetic sequence from 0, else INT64_MIN (the vector is read).
struct TinyStrides {
  int64_t a, b, c, d;
};
// Whether a shape takes the tiny batched kernel (M N K <= 256 and a batch of
// at least 64).
inline bool use_tiny_batched(int64_t M, int64_t N, int64_t K, int64_t H) {
  return M * N * K <= 256 && H >= 64;
}
cudaError_t launch_tiny_batched(int dtype, const GemmArgs& g, const TinyStrides& hs, int num_sms, cudaStream_t st);

// Family of an item inside a grouped launch (the list fills the GPU).
int choose_grouped_kernel(int dtype, int64_t M, int64_t N, int64_t K);
// One-launch choice with split-K: the family (or `pinned`) and the number of
// K chunks (1 = no split). Deep contractions with fewer large tiles than SMs
// take the large tile and split K so that about two CTAs run per SM.
void choose_plain_launch(int dtype, int pinned, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms, int* kernel,
                         int* splits, int64_t* k_chunk);
// Sum of the split-K partials (fixed order) and the epilogue into D.
cudaError_t launch_splitk_reduce(int dtype, const GemmArgs& g, int splits, cudaStream_t st);

// ---- packed plain families (pack pass + TMA-fed tiles) ----------------------
//
// The operands are first gathered through their scatter vectors into dense
// panels (the reference's packed panels, crates/tprims-kernel/src/pack/
// pack.rs:152-270, once per call for the whole operand), then a tile kernel
// streams the panels into shared memory with TMA tiled loads:
//   f32:     A' as [H][k_pad][m_pad], B' as [H][k_pad][n_pad] (rows fastest);
//            FFMA, 128 x 128 tiles.
//   c32 1m:  the complex product as a real one of 2M x N x 2K (the reference's
//            induced 1m method, kernels/reference/induced.rs:67): A' element
//            (m, k) becomes the real 2 x 2 block [[re, -im], [im, re]] at rows
//            2m, 2m+1 and depths 2k, 2k+1; B' element (k, n) the pair [re; im]
//            at depths 2k, 2k+1; output rows 2m, 2m+1 are Re and Im of row m.
//   f64:     A' as [H][m_pad][k_pad], B' as [H][n_pad][k_pad] (k fastest,
//            128-byte rows swizzled by TMA); DMMA, 64 x 64 tiles.
//   c64 3m:  three planes per operand, [re, im, re + im] (pack/pack.rs:70-72,
//            conjugation folded into the signs), three DMMA products M1 = Ar Br,
//            M2 = Ai Bi, M3 = (Ar + Ai)(Br + Bi) recombined as
//            (M1 - M2) + i (M3 - M1 - M2) (kernels/reference/scalar.rs:136,
//            pack/writeback.rs:86-92); 64 x 32 tiles.
// Split-K (k_chunk, partial) works as in the direct kernels.
struct PackedLayout {
  int kernel = 0;
  int planes = 1;
  int64_t m_pad = 0, n_pad = 0, k_pad = 0;  // of the (embedded) real problem
  int64_t H = 0;
  // The pack pass walks batch entries fastest for an operand whose batch
  // index has the smallest stride (set by the caller; the layout is the same).
  int a_hfast = 0, b_hfast = 0;
};
bool is_packed_kernel(int kernel);
// The dtype (TAPP numbering) a packed family computes in.
int packed_dtype(int kernel);
// Whether a packed family can take a shape (grid and TMA coordinate limits).
bool packed_fits(int kernel, int64_t M, int64_t N, int64_t K, int64_t H);
PackedLayout packed_layout(int kernel, int64_t M, int64_t N, int64_t K, int64_t H);
size_t packed_workspace_bytes(const PackedLayout& L);
// Pack both operands into `panels` (packed_workspace_bytes of device memory).
// A' on `st`, B' on `st_b` (the same stream or one the caller joins back).
cudaError_t launch_packed_pack(const GemmArgs& g, const PackedLayout& L, void* panels, cudaStream_t st,
                               cudaStream_t st_b);
// The tile kernel over the panels (with the epilogue, or split-K partials).
cudaError_t launch_packed_gemm(const GemmArgs& g, const PackedLayout& L, const void* panels, cudaStream_t st);

// ---- split precision (tensor cores) ----------------------------------------

// Layout of the packed split operands: planes[S][H][rows_pad][k_pad] BF16,
// k contiguous (K-major), zero-padded to the tile multiples.
struct SplitLayout {
  int planes;       // S: 2 (hi/lo) or 3 (hi/mid/lo)
  int64_t m_pad, n_pad, k_pad;
  int64_t H;
};

// Pack A' (rows = M) and B' (rows = N) into BF16 planes. `which` 0 = A', 1 = B'.
cudaError_t launch_split_pack_f32(const GemmArgs& g, int which, const SplitLayout& L, void* planes,
                                  cudaStream_t st);
// The tcgen05 GEMM over packed planes, with the scatter epilogue.
// npairs/pairs: the list of (a_plane, b_plane) products accumulated.
// With `tail_partial` (split_tail_bytes of device memory), the tiles of a
// partly filled last wave are split along K and reduced by a second kernel.
cudaError_t launch_tc_bf16_gemm(const GemmArgs& g, const SplitLayout& L, const void* a_planes, const void* b_planes,
                                int scheme, cudaStream_t st, void* tail_partial = nullptr);
size_t split_tail_bytes(const SplitLayout& L, int num_sms);
// K parts of the tail tiles for `num_sms` SMs (1 = no tail split).
int split_tail_parts(const SplitLayout& L, int num_sms);
// Bytes of packed workspace a split scheme needs.
size_t split_workspace_bytes(const SplitLayout& L);
SplitLayout split_layout(int scheme, int64_t M, int64_t N, int64_t K, int64_t H);

// ---- Ozaki INT8 slices (f64 / c64 on tensor cores) -------------------------

struct OzakiLayout {
  int slices;      // S: 7-bit slices per operand; S(S+1)/2 slice products
  int cplx;        // complex operands embedded as a real problem (2M rows, 2K depth)
  int64_t m_emb;   // rows of the embedded A'
  int64_t k_emb;   // depth of the embedded product
  int64_t k_half;  // complex: offset of the imaginary half of the depth (K rounded up to 64)
  int64_t m_pad, n_pad, k_pad;
  int64_t exp_a_pad;  // row stride of the A exponent array
  int64_t H;
  int kb_chunk;    // k-blocks per launch that keep INT32 accumulation exact
  int a_hfast = 0, b_hfast = 0;  // batch index has the smallest stride: batch-innermost packing
};
OzakiLayout ozaki_layout(int slices, bool cplx, int64_t M, int64_t N, int64_t K, int64_t H);
size_t ozaki_workspace_bytes(const OzakiLayout& L);
// Exponent scan and slicing of A' and B' into the workspace.
// A' on `st`, B' on `st_b` (the same stream or one the caller joins back).
cudaError_t launch_ozaki_pack(const GemmArgs& g, const OzakiLayout& L, void* ws, cudaStream_t st, cudaStream_t st_b);
// Slice products over k-blocks [kb0, kb1) with the recombining epilogue.
cudaError_t launch_ozaki_gemm(const GemmArgs& g, const OzakiLayout& L, const void* ws, int kb0, int kb1,
                              cudaStream_t st);

}  // namespace dev
}  // namespace tprims
