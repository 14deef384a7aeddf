// Scatter vectors, folding and orientation (see plan.hpp for the reference
// files each part restates).
#include "plan.hpp"

#include <algorithm>
#include <cstdlib>

namespace tprims {

namespace {

uint64_t uabs(int64_t x) { return x < 0 ? (uint64_t)0 - (uint64_t)x : (uint64_t)x; }

Axis axis_of(const RoleAxis& r) {
  return Axis{r.extent, r.stride[SA], r.stride[SB], r.stride[SC], r.stride[SD]};
}

// Neighbouring axes merge when the next one's stride is the previous one's
// stride times its extent in every operand at once (analysis.rs:299).
std::vector<Axis> fold(const std::vector<Axis>& in) {
  std::vector<Axis> out;
  for (const Axis& ax : in) {
    if (!out.empty()) {
      Axis& p = out.back();
      if (ax.sa == p.sa * p.extent && ax.sb == p.sb * p.extent && ax.sc == p.sc * p.extent &&
          ax.sd == p.sd * p.extent) {
        p.extent *= ax.extent;
        continue;
      }
    }
    out.push_back(ax);
  }
  return out;
}

template <class Key>
std::vector<Axis> role_axes(const std::vector<RoleAxis>& role, Key key) {
  std::vector<Axis> axes;
  for (auto& r : role)
    if (r.extent != 1) axes.push_back(axis_of(r));
  std::stable_sort(axes.begin(), axes.end(), [&](const Axis& x, const Axis& y) { return key(x) < key(y); });
  return fold(axes);
}

template <class Pick>
std::vector<int64_t> scatter_for(const std::vector<Axis>& axes, Pick pick) {
  std::vector<int64_t> e, s;
  for (auto& a : axes) {
    e.push_back(a.extent);
    s.push_back(pick(a));
  }
  return build_scatter(e, s);
}

int64_t run_stride(const int64_t* v, size_t n) {
  if (n <= 1) return 0;
  int64_t s = v[1] - v[0];
  for (size_t i = 1; i + 1 < n; ++i)
    if (v[i + 1] - v[i] != s) return IRREGULAR;
  return s;
}

// The smaller |stride| of the leading run of a scatter (its fastest direction
// in memory); a length-1 scatter counts as infinitely slow.
uint64_t lead_stride(const std::vector<int64_t>& v) {
  if (v.size() < 2) return UINT64_MAX;
  return uabs(v[1] - v[0]);
}

}  // namespace

std::vector<int64_t> build_scatter(const std::vector<int64_t>& extents, const std::vector<int64_t>& strides) {
  int64_t total = 1;
  for (auto e : extents) total *= e;
  std::vector<int64_t> out;
  if (total <= 0) return out;
  out.resize((size_t)total);
  if (extents.empty()) {
    out[0] = 0;
    return out;
  }
  // Mixed-radix odometer, fastest axis first (scatter.rs:70): the fastest
  // axis is written as one arithmetic run per position of the outer axes,
  // and only the outer axes step the odometer.
  const int64_t e0 = extents[0], s0 = strides[0];
  std::vector<int64_t> ctr(extents.size(), 0);
  int64_t base = 0;
  int64_t* o = out.data();
  for (int64_t i = 0; i < total; i += e0) {
    for (int64_t j = 0; j < e0; ++j) o[i + j] = base + j * s0;
    for (size_t d = 1; d < extents.size(); ++d) {
      base += strides[d];
      if (++ctr[d] < extents[d]) break;
      base -= strides[d] * extents[d];
      ctr[d] = 0;
    }
  }
  return out;
}

std::vector<int64_t> build_block_scatter(const std::vector<int64_t>& scat, size_t blk) {
  std::vector<int64_t> out;
  for (size_t lo = 0; lo < scat.size(); lo += blk) {
    size_t hi = std::min(lo + blk, scat.size());
    out.push_back(run_stride(scat.data() + lo, hi - lo));
  }
  return out;
}

bool run_structure(const std::vector<int64_t>& scat, size_t* len_out, int64_t* stride_out) {
  *len_out = 0;
  *stride_out = 0;
  if (scat.size() < 2) return false;
  const int64_t s = scat[1] - scat[0];
  size_t len = scat.size();
  for (size_t i = 0; i + 1 < scat.size(); ++i)
    if (scat[i + 1] - scat[i] != s) {
      len = i + 1;
      break;
    }
  if (len < 2 || scat.size() % len != 0) return false;
  for (size_t i = 0; i + 1 < scat.size(); ++i) {
    const bool boundary = (i + 1) % len == 0;
    const int64_t step = scat[i + 1] - scat[i];
    if (!boundary && step != s) return false;
    if (boundary && step == s) return false;  // runs would be longer than measured
  }
  *len_out = len;
  *stride_out = s;
  return true;
}

double regular_fraction(const std::vector<int64_t>& bs) {
  if (bs.empty()) return 1.0;
  size_t reg = 0;
  for (auto v : bs)
    if (v != IRREGULAR) ++reg;
  return (double)reg / (double)bs.size();
}

PackedPlan PackedPlan::from_problem(const Problem& p) {
  PackedPlan pk;
  auto m_ax = role_axes(p.m, [](const Axis& x) { return std::make_pair(uabs(x.sd), uabs(x.sa)); });
  auto n_ax = role_axes(p.n, [](const Axis& x) { return std::make_pair(uabs(x.sd), uabs(x.sb)); });
  auto k_ax = role_axes(p.k, [](const Axis& x) { return std::make_pair(uabs(x.sa), uabs(x.sb)); });
  auto h_ax = role_axes(p.h, [](const Axis& x) { return std::make_pair(uabs(x.sd), uabs(x.sa)); });
  for (auto* axes : {&m_ax, &n_ax, &k_ax, &h_ax}) {
    __int128 len = 1;
    for (auto& a : *axes) {
      len *= a.extent;
      if (len * 8 > (__int128)INT64_MAX) throw Error(ERR_SHAPE, "role extent product overflows");
    }
  }
  pk.a_m = scatter_for(m_ax, [](const Axis& x) { return x.sa; });
  pk.a_k = scatter_for(k_ax, [](const Axis& x) { return x.sa; });
  pk.b_k = scatter_for(k_ax, [](const Axis& x) { return x.sb; });
  pk.b_n = scatter_for(n_ax, [](const Axis& x) { return x.sb; });
  pk.c_m = scatter_for(m_ax, [](const Axis& x) { return x.sc; });
  pk.c_n = scatter_for(n_ax, [](const Axis& x) { return x.sc; });
  pk.d_m = scatter_for(m_ax, [](const Axis& x) { return x.sd; });
  pk.d_n = scatter_for(n_ax, [](const Axis& x) { return x.sd; });
  pk.h_a = scatter_for(h_ax, [](const Axis& x) { return x.sa; });
  pk.h_b = scatter_for(h_ax, [](const Axis& x) { return x.sb; });
  pk.h_c = scatter_for(h_ax, [](const Axis& x) { return x.sc; });
  pk.h_d = scatter_for(h_ax, [](const Axis& x) { return x.sd; });
  pk.stats.m = (int64_t)pk.d_m.size();
  pk.stats.n = (int64_t)pk.d_n.size();
  pk.stats.k = (int64_t)pk.a_k.size();
  pk.stats.batch = (int64_t)pk.h_d.size();
  pk.stats.is_pure_gemm = m_ax.size() <= 1 && n_ax.size() <= 1 && k_ax.size() <= 1 && h_ax.empty();
  pk.stats.m_axes = m_ax;
  pk.stats.n_axes = n_ax;
  pk.stats.k_axes = k_ax;
  pk.stats.h_axes = h_ax;
  if (!run_structure(pk.d_m, &pk.d_m_run_len, &pk.d_m_run_stride)) {
    pk.d_m_run_len = pk.d_m.size();
    pk.d_m_run_stride = 0;
  }
  if (!run_structure(pk.d_n, &pk.d_n_run_len, &pk.d_n_run_stride)) {
    pk.d_n_run_len = pk.d_n.size();
    pk.d_n_run_stride = 0;
  }
  pk.conj_a = p.a.conj;
  pk.conj_b = p.b.conj;
  pk.conj_c = p.op_c_conj;
  pk.conj_d = p.d.conj;
  return pk;
}

bool PackedPlan::transposes_gemm(size_t mr) const {
  // 1. prefer the arm whose row block lies inside one unit-stride run of D.
  const bool ab = d_m_run_stride == 1 && d_m_run_len >= mr;
  const bool ba = d_n_run_stride == 1 && d_n_run_len >= mr;
  if (ab != ba) return ba;
  if (ab) return false;
  // 2. an arm that cannot fill a row block loses; otherwise the shorter run
  //    takes the row role.
  const size_t m_rows = d_m.size(), n_rows = d_n.size();
  if ((m_rows >= mr) != (n_rows >= mr)) return n_rows >= mr;
  return d_n_run_len < d_m_run_len;
}

OrientedView orient(PackedPlan& pk, bool swap) {
  OrientedView v;
  v.swapped = swap;
  // The vectors move into the view (they are the plan's largest part); the
  // packed plan keeps its statistics, and unorient() gives the vectors back.
  if (!swap) {
    v.a_m = std::move(pk.a_m); v.a_k = std::move(pk.a_k); v.b_k = std::move(pk.b_k); v.b_n = std::move(pk.b_n);
    v.c_m = std::move(pk.c_m); v.c_n = std::move(pk.c_n); v.d_m = std::move(pk.d_m); v.d_n = std::move(pk.d_n);
    v.h_a = std::move(pk.h_a); v.h_b = std::move(pk.h_b);
    v.conj_a = pk.conj_a; v.conj_b = pk.conj_b;
  } else {
    // D^T = B^T A^T: B plays A's role and the output's row/column scatters swap.
    v.a_m = std::move(pk.b_n); v.a_k = std::move(pk.b_k); v.b_k = std::move(pk.a_k); v.b_n = std::move(pk.a_m);
    v.c_m = std::move(pk.c_n); v.c_n = std::move(pk.c_m); v.d_m = std::move(pk.d_n); v.d_n = std::move(pk.d_m);
    v.h_a = std::move(pk.h_b); v.h_b = std::move(pk.h_a);
    v.conj_a = pk.conj_b; v.conj_b = pk.conj_a;
  }
  v.h_c = std::move(pk.h_c);
  v.h_d = std::move(pk.h_d);
  v.conj_c = pk.conj_c;
  v.conj_d = pk.conj_d;
  v.M = (int64_t)v.d_m.size();
  v.N = (int64_t)v.d_n.size();
  v.K = (int64_t)v.a_k.size();
  v.H = (int64_t)v.h_d.size();
  v.a_kfast = lead_stride(v.a_k) < lead_stride(v.a_m);
  v.b_kfast = lead_stride(v.b_k) < lead_stride(v.b_n);
  v.d_mfast = lead_stride(v.d_m) <= lead_stride(v.d_n);
  v.c_mfast = lead_stride(v.c_m) <= lead_stride(v.c_n);
  return v;
}

std::vector<const std::vector<int64_t>*> unorient(const OrientedView& v) {
  if (!v.swapped)
    return {&v.a_m, &v.a_k, &v.b_k, &v.b_n, &v.c_m, &v.c_n, &v.d_m, &v.d_n, &v.h_a, &v.h_b, &v.h_c, &v.h_d};
  return {&v.b_n, &v.b_k, &v.a_k, &v.a_m, &v.c_n, &v.c_m, &v.d_n, &v.d_m, &v.h_b, &v.h_a, &v.h_c, &v.h_d};
}

}  // namespace tprims
