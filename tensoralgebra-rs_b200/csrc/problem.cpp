// Lowering of labels and dot_general descriptions into a validated Problem.
// Restates the checks of crates/tprims-contract/src/api/validate.rs (order and
// error classes) and api/dot_general.rs, with the C-ABI status mapping of
// crates/tprims-capi/src/abi.rs:97-113 applied at the throw site.
#include "problem.hpp"

#include <algorithm>
#include <cstdlib>
#include <limits>

namespace tprims {

const char* dtype_name(DType t) {
  switch (t) {
    case DType::F32: return "f32";
    case DType::F64: return "f64";
    case DType::C32: return "c32";
    case DType::C64: return "c64";
  }
  return "?";
}

namespace {

[[noreturn]] void overflow(const char* what) { throw Error(ERR_SHAPE, std::string(what) + " overflows"); }

// A label of one operand after repeated labels collapsed onto their diagonal.
struct Mode {
  int64_t label;
  int64_t extent;
  int64_t stride;
};

const char* slot_name(int s) {
  static const char* names[4] = {"A", "B", "C", "D"};
  return names[s];
}

// validate.rs:47 (reduce): label count, extent agreement of repeated labels,
// checked stride sums, and a checked product of the distinct extents.
std::vector<Mode> collapse(int slot, const Layout& l, const std::vector<int64_t>& labels) {
  if (l.rank() != labels.size()) {
    throw Error(ERR_LABELS, std::string(slot_name(slot)) + " has " + std::to_string(l.rank()) + " modes but " +
                                std::to_string(labels.size()) + " labels");
  }
  std::vector<Mode> out;
  __int128 product = 1;
  for (size_t ax = 0; ax < labels.size(); ++ax) {
    const int64_t e = l.dims[ax], s = l.strides[ax];
    auto it = std::find_if(out.begin(), out.end(), [&](const Mode& m) { return m.label == labels[ax]; });
    if (it != out.end()) {
      if (it->extent != e) {
        throw Error(ERR_SHAPE, "label " + std::to_string(labels[ax]) + " has extent " + std::to_string(e) +
                                   " where " + std::to_string(it->extent) + " was already seen");
      }
      __int128 sum = (__int128)it->stride + s;
      if (sum > std::numeric_limits<int64_t>::max() || sum < std::numeric_limits<int64_t>::min())
        overflow("repeated-label stride sum");
      it->stride = (int64_t)sum;
    } else {
      product *= e;
      if (product > std::numeric_limits<int64_t>::max()) overflow("extent product");
      out.push_back({labels[ax], e, s});
    }
  }
  return out;
}

// validate.rs:96 (span_of): the addressed element range, overflow-checked in
// bytes against the largest signed pointer offset.
Span span_of(DType dtype, const Layout& l) {
  Span sp;
  const __int128 elem = (__int128)dtype_size(dtype);
  __int128 lo = l.offset, hi = l.offset;
  for (size_t i = 0; i < l.rank(); ++i) {
    if (l.dims[i] == 0) return sp;  // empty
    __int128 reach = (__int128)(l.dims[i] - 1) * l.strides[i];
    if (reach < 0) lo += reach; else hi += reach;
  }
  const __int128 limit = (__int128)std::numeric_limits<int64_t>::max();
  __int128 alo = lo < 0 ? -lo : lo;
  if (alo * elem > limit || (hi + 1) * elem > limit) overflow("address range");
  sp.empty = false;
  sp.lo = lo;
  sp.hi = hi;
  return sp;
}

// validate.rs:122 (injective): sort axes of extent > 1 by |stride|; each stride
// must clear the reach of the smaller ones.
bool injective_modes(std::vector<std::pair<int64_t, int64_t>> axes /* extent, stride */) {
  for (auto& a : axes)
    if (a.first == 0) return true;
  std::vector<std::pair<__int128, __int128>> v;  // (|stride|, extent)
  for (auto& a : axes)
    if (a.first > 1) v.push_back({(__int128)(a.second < 0 ? -(__int128)a.second : (__int128)a.second), a.first});
  std::stable_sort(v.begin(), v.end(), [](auto& x, auto& y) { return x.first < y.first; });
  __int128 reach = 1;
  for (auto& a : v) {
    if (a.first < reach) return false;
    reach = a.first * a.second;
  }
  return true;
}

struct LabelRow {
  int64_t id;
  int64_t extent;
  int64_t strides[4];
  bool in[4];
};

// validate.rs:169 (merge): one table of labels with their strides per operand.
void merge(std::vector<LabelRow>& table, const std::vector<Mode>& modes, int slot) {
  for (const Mode& m : modes) {
    auto it = std::find_if(table.begin(), table.end(), [&](const LabelRow& r) { return r.id == m.label; });
    if (it == table.end()) {
      LabelRow r{m.label, m.extent, {0, 0, 0, 0}, {false, false, false, false}};
      table.push_back(r);
      it = table.end() - 1;
    } else if (it->extent != m.extent) {
      throw Error(ERR_SHAPE, "label " + std::to_string(m.label) + " has extent " + std::to_string(m.extent) +
                                 " where " + std::to_string(it->extent) + " was already seen");
    }
    it->strides[slot] = m.stride;
    it->in[slot] = true;
  }
}

}  // namespace

Layout layout_from_signed(const int64_t* dims, const int64_t* strides, int rank, int64_t offset) {
  Layout l;
  l.offset = offset;
  for (int i = 0; i < rank; ++i) {
    if (dims[i] < 0)
      throw Error(ERR_SHAPE, "axis " + std::to_string(i) + " has the negative extent " + std::to_string(dims[i]));
    l.dims.push_back(dims[i]);
    l.strides.push_back(strides[i]);
  }
  return l;
}

bool layout_injective(const std::vector<int64_t>& dims, const std::vector<int64_t>& strides) {
  std::vector<std::pair<int64_t, int64_t>> axes;
  for (size_t i = 0; i < dims.size(); ++i) axes.push_back({dims[i], strides[i]});
  return injective_modes(axes);
}

double Problem::macs() const {
  double p = 1;
  for (auto* role : {&m, &n, &k, &h})
    for (auto& ax : *role) p *= (double)ax.extent;
  return p;
}

Problem Problem::from_labels(DType dtype, const Operand& a, const Operand& b, CMode cmode, const Operand& c,
                             const Operand& d, const std::vector<int64_t>& la, const std::vector<int64_t>& lb,
                             bool has_c_labels, const std::vector<int64_t>& lc, const std::vector<int64_t>& ld,
                             bool output_conj_c, bool d_is_operand_layout) {
  if ((cmode == CMode::Separate) != has_c_labels)
    throw Error(ERR_LABELS, "a separate C needs C labels, and only a separate C may carry them");
  Problem p;
  p.dtype = dtype;
  p.a = a;
  p.b = b;
  p.d = d;
  p.cmode = cmode;
  p.c = (cmode == CMode::Separate) ? c : d;
  p.la = la;
  p.lb = lb;
  p.lc = (cmode == CMode::Separate) ? lc : ld;
  p.ld = ld;
  p.op_c_conj = (cmode == CMode::Separate) ? c.conj : (cmode == CMode::Output ? output_conj_c : false);
  p.c.conj = p.op_c_conj;

  auto ra = collapse(SA, a.layout, la);
  auto rb = collapse(SB, b.layout, lb);
  auto rd = collapse(SD, d.layout, ld);
  std::vector<Mode> rc = (cmode == CMode::Separate) ? collapse(SC, c.layout, lc) : rd;

  std::vector<LabelRow> table;
  merge(table, ra, SA);
  merge(table, rb, SB);
  merge(table, rc, SC);
  merge(table, rd, SD);
  for (auto& r : table)
    if (r.in[SC] != r.in[SD]) throw Error(ERR_LABELS, "C and D carry different label sets");

  for (auto& r : table) {
    RoleAxis ax{r.id, r.extent, {r.strides[0], r.strides[1], r.strides[2], r.strides[3]}, r.in[SA], r.in[SB]};
    const bool ia = r.in[SA], ib = r.in[SB], id = r.in[SD];
    if (ia && ib && id) p.h.push_back(ax);
    else if (ia && !ib && id) p.m.push_back(ax);
    else if (!ia && ib && id) p.n.push_back(ax);
    else if (!id) p.k.push_back(ax);  // contracted, or isolated in one input (a reduction)
    else
      throw Error(ERR_UNSUPPORTED, "label " + std::to_string(r.id) + " appears only in the output (a broadcast)");
  }

  p.spans[SA] = span_of(dtype, a.layout);
  p.spans[SB] = span_of(dtype, b.layout);
  p.spans[SC] = span_of(dtype, p.c.layout);
  p.spans[SD] = span_of(dtype, d.layout);

  {
    // The conservative sorted-stride test runs on the collapsed output modes
    // (validate.rs:122). An adjoint output that is an input operand's own
    // layout restricted to a diagonal (Plan::vjp) is injective whenever that
    // layout is, which is what is checked for it instead.
    std::vector<std::pair<int64_t, int64_t>> axes;
    if (d_is_operand_layout)
      for (size_t i = 0; i < d.layout.rank(); ++i) axes.push_back({d.layout.dims[i], d.layout.strides[i]});
    else
      for (auto& md : rd) axes.push_back({md.extent, md.stride});
    if (!injective_modes(axes))
      throw Error(ERR_ALIASED, "D addresses an element more than once (zero or overlapping strides)");
  }

  if (cmode == CMode::Separate) {
    bool same = c.layout.offset == d.layout.offset;
    for (auto& md : rd) {
      bool found = false;
      for (auto& mc : rc)
        if (mc.label == md.label && mc.stride == md.stride) found = true;
      same = same && found;
    }
    p.c_matches_d = same;
  } else {
    p.c_matches_d = true;
  }
  p.k_empty = std::any_of(p.k.begin(), p.k.end(), [](const RoleAxis& x) { return x.extent == 0; });
  p.out_empty = false;
  for (auto* role : {&p.m, &p.n, &p.h})
    for (auto& x : *role)
      if (x.extent == 0) p.out_empty = true;
  return p;
}

Problem Problem::from_dot_general(DType dtype, const Operand& a, const Operand& b, const Operand& d,
                                  const std::vector<int64_t>& lc, const std::vector<int64_t>& rc,
                                  const std::vector<int64_t>& lbt, const std::vector<int64_t>& rbt) {
  if (lc.size() != rc.size())
    throw Error(ERR_INVALID_ARGUMENT, "the contracting axis lists of A (" + std::to_string(lc.size()) + ") and B (" +
                                          std::to_string(rc.size()) + ") differ in length");
  if (lbt.size() != rbt.size())
    throw Error(ERR_INVALID_ARGUMENT, "the batch axis lists of A (" + std::to_string(lbt.size()) + ") and B (" +
                                          std::to_string(rbt.size()) + ") differ in length");
  auto free_axes = [](const char* name, size_t rank, const std::vector<int64_t>& con,
                      const std::vector<int64_t>& bat) {
    std::vector<bool> seen(rank, false);
    for (const auto* list : {&con, &bat})
      for (int64_t x : *list) {
        if (x < 0 || (size_t)x >= rank)
          throw Error(ERR_INVALID_ARGUMENT, std::string(name) + " axis " + std::to_string(x) +
                                                " is out of range for rank " + std::to_string(rank));
        if (seen[x]) throw Error(ERR_INVALID_ARGUMENT, std::string(name) + " axis " + std::to_string(x) + " is listed twice");
        seen[x] = true;
      }
    std::vector<int64_t> f;
    for (size_t i = 0; i < rank; ++i)
      if (!seen[i]) f.push_back((int64_t)i);
    return f;
  };
  const auto& ad = a.layout.dims;
  const auto& bd = b.layout.dims;
  auto lfree = free_axes("A", ad.size(), lc, lbt);
  auto rfree = free_axes("B", bd.size(), rc, rbt);
  auto check_pair = [&](int64_t l, int64_t r) {
    if (ad[l] != bd[r])
      throw Error(ERR_SHAPE, "A axis " + std::to_string(l) + " has extent " + std::to_string(ad[l]) + " but B axis " +
                                 std::to_string(r) + " has " + std::to_string(bd[r]));
  };
  for (size_t i = 0; i < lc.size(); ++i) check_pair(lc[i], rc[i]);
  for (size_t i = 0; i < lbt.size(); ++i) check_pair(lbt[i], rbt[i]);
  std::vector<int64_t> out;
  for (auto x : lfree) out.push_back(ad[x]);
  for (auto x : rfree) out.push_back(bd[x]);
  for (auto x : lbt) out.push_back(ad[x]);
  if (out != d.layout.dims) throw Error(ERR_SHAPE, "D's extents are not [lhs_free, rhs_free, batch]");

  // Synthetic labels: batch pairs 0..nb-1, contracted pairs nb..nb+nc-1, then
  // the free axes of A and B in order (problem.rs:411-441).
  const int64_t nb = (int64_t)lbt.size(), nc = (int64_t)lc.size();
  std::vector<int64_t> la(ad.size(), 0), lb(bd.size(), 0), ld;
  int64_t next = nb + nc;
  for (auto x : lfree) { la[x] = next; ld.push_back(next); ++next; }
  for (auto x : rfree) { lb[x] = next; ld.push_back(next); ++next; }
  for (int64_t p = 0; p < nb; ++p) { la[lbt[p]] = p; lb[rbt[p]] = p; ld.push_back(p); }
  for (int64_t p = 0; p < nc; ++p) { la[lc[p]] = nb + p; lb[rc[p]] = nb + p; }
  return from_labels(dtype, a, b, CMode::Output, d, d, la, lb, false, {}, ld, false);
}

}  // namespace tprims
