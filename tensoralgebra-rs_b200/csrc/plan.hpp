// Packed-plan analysis: a validated Problem seen as a batched matrix product
// over scatter vectors, plus the choices this engine makes on top of it
// (orientation, precision scheme, kernel family).
//
// The analysis follows crates/tprims-contract/src/plan/analysis.rs:197-321:
// per role, drop extent-1 axes, stable-sort (M, N, H by |stride in D|, K by
// |stride in A|, with the other input as tie-break), fold neighbours whose
// strides are compatible in all four operands, then build one mixed-radix
// scatter vector per (operand, role) (crates/tprims-kernel/src/pack/
// scatter.rs:70). The orientation rule is plan/orientation.rs:196-230 with the
// GPU's row block: a warp of 32 rows must land inside one unit-stride run of D.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "problem.hpp"

namespace tprims {

struct Axis {
  int64_t extent;
  int64_t sa, sb, sc, sd;
};

// Sentinel of a block-scatter entry whose run is not an arithmetic progression.
constexpr int64_t IRREGULAR = INT64_MIN;

std::vector<int64_t> build_scatter(const std::vector<int64_t>& extents, const std::vector<int64_t>& strides);
std::vector<int64_t> build_block_scatter(const std::vector<int64_t>& scat, size_t blk);
// (run length, stride) when the scatter is a concatenation of equal maximal
// arithmetic runs; {0,0} with ok=false otherwise.
bool run_structure(const std::vector<int64_t>& scat, size_t* len, int64_t* stride);
double regular_fraction(const std::vector<int64_t>& block_scatter);

struct PlanStats {
  int64_t m = 0, n = 0, k = 0, batch = 0;
  std::vector<Axis> m_axes, n_axes, k_axes, h_axes;
  bool is_pure_gemm = false;
};

struct PackedPlan {
  std::vector<int64_t> a_m, a_k, b_k, b_n, c_m, c_n, d_m, d_n, h_a, h_b, h_c, h_d;
  size_t d_m_run_len = 0, d_n_run_len = 0;
  int64_t d_m_run_stride = 0, d_n_run_stride = 0;
  bool conj_a = false, conj_b = false, conj_c = false, conj_d = false;
  PlanStats stats;

  static PackedPlan from_problem(const Problem& p);
  // plan/orientation.rs:196-230 (Orient::Rule): whether to compute D^T = B^T A^T.
  bool transposes_gemm(size_t mr) const;
};

// Precision schemes (TPRIMS_PREC_* of the C header).
enum class Scheme : int { Plain = 0, Bf16x3 = 1, Bf16x6 = 2, OzakiInt8 = 3 };

// The matrix view the kernels see after orientation: A' (M'xK), B' (KxN'),
// C'/D' (M'xN'), all through scatter vectors, batched over H.
struct OrientedView {
  bool swapped = false;
  int64_t M = 0, N = 0, K = 0, H = 0;
  std::vector<int64_t> a_m, a_k, b_k, b_n, c_m, c_n, d_m, d_n, h_a, h_b, h_c, h_d;
  bool conj_a = false, conj_b = false, conj_c = false, conj_d = false;
  // Which index is the faster one in memory for each operand (gather hints).
  bool a_kfast = false, b_kfast = true, d_mfast = true, c_mfast = true;
};

// The kernels' view of a packed plan; the scatter vectors move out of `pk`
// (which keeps its statistics and run structure).
OrientedView orient(PackedPlan& pk, bool swap);
// The packed plan's 12 scatter vectors (a_m, a_k, b_k, b_n, c_m, c_n, d_m,
// d_n, h_a, h_b, h_c, h_d) as they were before orientation, read from the view.
std::vector<const std::vector<int64_t>*> unorient(const OrientedView& v);

}  // namespace tprims
