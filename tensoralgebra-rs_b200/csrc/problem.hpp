// Host-side description of one binary contraction and its lowering to roles.
//
// D = op_D(alpha * sum_K op_A(A) * op_B(B) + beta * op_C(C)) over strided
// f32 / f64 / c32 / c64 operands. This file holds the validated metadata only
// (no pointers, no device state). The rules are those of the reference's
// lowering (crates/tprims-contract/src/api/validate.rs:207-308): repeated labels
// collapse onto a diagonal with summed strides, a label present in one input
// only becomes a K axis with a zero stride in the other input, an output-only
// label is refused, spans are checked for overflow and D must be injective.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace tprims {

// Status codes of the C ABI (crates/tprims-capi/src/status.rs:13-43).
enum Status : int {
  OK = 0,
  ERR_INVALID_ARGUMENT = 1,
  ERR_SHAPE = 2,
  ERR_DTYPE = 3,
  ERR_DEVICE = 4,
  ERR_READ_ONLY = 5,
  ERR_ALIASED = 6,
  ERR_WOULD_MATERIALIZE = 7,
  ERR_NUMERICAL = 8,
  BUSY = 9,
  ERR_WOULD_DEADLOCK = 10,
  ERR_PANIC = 12,
  ERR_INTERNAL = 13,
  ERR_LABELS = 14,
  ERR_UNSUPPORTED = 15,
};

// Every failure inside the library is thrown as this and turned into a status
// plus a thread-local message at the C boundary.
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

enum class DType : int { F32 = 0, F64 = 1, C32 = 2, C64 = 3 };
inline size_t dtype_size(DType t) {
  switch (t) {
    case DType::F32: return 4;
    case DType::F64: return 8;
    case DType::C32: return 8;
    case DType::C64: return 16;
  }
  return 0;
}
inline bool dtype_complex(DType t) { return t == DType::C32 || t == DType::C64; }
inline bool dtype_double(DType t) { return t == DType::F64 || t == DType::C64; }
const char* dtype_name(DType t);

// Extents, signed element strides and the element offset of index (0,..,0).
struct Layout {
  std::vector<int64_t> dims;
  std::vector<int64_t> strides;
  int64_t offset = 0;
  size_t rank() const { return dims.size(); }
};

struct Operand {
  Layout layout;
  bool conj = false;
};

// How the beta*op_C(C) term is supplied (api/problem.rs CSpec).
enum class CMode { Absent, Output, Separate };

// Operand slots, in the order the strides of a role axis are stored.
enum Slot { SA = 0, SB = 1, SC = 2, SD = 3 };

// One reduced logical axis with its (diagonal-summed) stride in A, B, C, D.
struct RoleAxis {
  int64_t label;
  int64_t extent;
  int64_t stride[4];
  bool in_a, in_b;
};

// Addressed element range of an operand, inclusive, relative to its storage.
struct Span {
  bool empty = true;
  __int128 lo = 0, hi = 0;
};

struct Problem {
  DType dtype = DType::F64;
  Operand a, b, c, d;  // c mirrors d unless cmode == Separate
  CMode cmode = CMode::Absent;
  bool op_c_conj = false;
  std::vector<RoleAxis> m, n, k, h;  // first-appearance order
  Span spans[4];
  bool c_matches_d = true;
  bool k_empty = false;
  bool out_empty = false;
  // The labels the problem was described with (synthetic ones for dot_general);
  // the adjoint contractions of Plan::vjp are built from them.
  std::vector<int64_t> la, lb, lc, ld;

  // Problem::from_labels (api/problem.rs:370). `lc` is used only for
  // CMode::Separate; `has_c_labels` says whether C labels were given at all.
  static Problem from_labels(DType dtype, const Operand& a, const Operand& b, CMode cmode, const Operand& c,
                             const Operand& d, const std::vector<int64_t>& la, const std::vector<int64_t>& lb,
                             bool has_c_labels, const std::vector<int64_t>& lc, const std::vector<int64_t>& ld,
                             bool output_conj_c = false, bool d_is_operand_layout = false);

  // Problem::from_dot_general (api/problem.rs:396) with DotGeneral::validate
  // (api/dot_general.rs:82). D must have extents [lhs_free, rhs_free, batch].
  static Problem from_dot_general(DType dtype, const Operand& a, const Operand& b, const Operand& d,
                                  const std::vector<int64_t>& lhs_contract, const std::vector<int64_t>& rhs_contract,
                                  const std::vector<int64_t>& lhs_batch, const std::vector<int64_t>& rhs_batch);

  bool all_batch() const { return m.empty() && n.empty() && k.empty(); }
  // Multiply-accumulates of one execution (the product of every reduced extent).
  double macs() const;
};

// Layout from signed C values (LayoutSpec::from_signed, api/problem.rs).
Layout layout_from_signed(const int64_t* dims, const int64_t* strides, int rank, int64_t offset);

// Whether distinct indices of a layout address distinct elements (the
// conservative sorted-stride test of validate.rs:122).
bool layout_injective(const std::vector<int64_t>& dims, const std::vector<int64_t>& strides);

}  // namespace tprims
