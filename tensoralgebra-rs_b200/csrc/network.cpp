// Planning of N-ary contraction networks (see network.hpp); execution is in
// runtime.cpp (execute_networks), next to the grouped submission it uses.
#include "network.hpp"

#include <algorithm>
#include <cmath>
#include <set>
#include <sstream>

namespace tprims {

namespace {

std::vector<int64_t> unique_labels(const std::vector<int64_t>& l) {
  std::vector<int64_t> u;
  for (int64_t x : l)
    if (std::find(u.begin(), u.end(), x) == u.end()) u.push_back(x);
  return u;
}

bool has(const std::vector<int64_t>& v, int64_t x) { return std::find(v.begin(), v.end(), x) != v.end(); }

// Labels of the result of contracting `la` with `lb` when `keep` holds every
// label still needed (other operands and the output): free labels of the
// first operand, free labels of the second, then the shared ones.
std::vector<int64_t> step_result(const std::vector<int64_t>& la, const std::vector<int64_t>& lb,
                                 const std::set<int64_t>& keep) {
  const std::vector<int64_t> ua = unique_labels(la), ub = unique_labels(lb);
  std::vector<int64_t> out;
  for (int64_t x : ua)
    if (!has(ub, x) && keep.count(x)) out.push_back(x);
  for (int64_t x : ub)
    if (!has(ua, x) && keep.count(x)) out.push_back(x);
  for (int64_t x : ua)
    if (has(ub, x) && keep.count(x)) out.push_back(x);
  return out;
}

std::set<int64_t> needed_elsewhere(const std::vector<std::vector<int64_t>>& cur, size_t i, size_t j,
                                   const std::vector<int64_t>& out) {
  std::set<int64_t> keep(out.begin(), out.end());
  for (size_t k = 0; k < cur.size(); ++k)
    if (k != i && k != j) keep.insert(cur[k].begin(), cur[k].end());
  return keep;
}

Layout dense_layout(const std::vector<int64_t>& dims) {
  Layout l;
  l.dims = dims;
  int64_t s = 1;
  for (int64_t d : dims) {
    l.strides.push_back(s);
    s *= std::max<int64_t>(d, 1);
  }
  return l;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

std::vector<std::pair<int, int>> greedy_path(const std::vector<std::vector<int64_t>>& labels,
                                             const std::vector<int64_t>& out_labels,
                                             const std::map<int64_t, int64_t>& extents) {
  std::vector<std::vector<int64_t>> cur;
  for (const auto& l : labels) cur.push_back(unique_labels(l));
  std::vector<std::pair<int, int>> path;
  auto prod = [&](const std::vector<int64_t>& ls) {
    double p = 1;
    for (int64_t x : ls) p *= (double)extents.at(x);
    return p;
  };
  while (cur.size() > 1) {
    size_t bi = 0, bj = 1;
    bool best_shared = false;
    double best_macs = INFINITY, best_size = INFINITY;
    for (size_t i = 0; i < cur.size(); ++i)
      for (size_t j = i + 1; j < cur.size(); ++j) {
        bool shared = false;
        for (int64_t x : cur[i]) shared = shared || has(cur[j], x);
        std::vector<int64_t> uni = cur[i];
        for (int64_t x : cur[j])
          if (!has(uni, x)) uni.push_back(x);
        const double macs = prod(uni);
        const double size = prod(step_result(cur[i], cur[j], needed_elsewhere(cur, i, j, out_labels)));
        const bool better = (shared && !best_shared) ||
                            (shared == best_shared &&
                             (macs < best_macs || (macs == best_macs && size < best_size)));
        if (better) {
          bi = i;
          bj = j;
          best_shared = shared;
          best_macs = macs;
          best_size = size;
        }
      }
    std::vector<int64_t> res = step_result(cur[bi], cur[bj], needed_elsewhere(cur, bi, bj, out_labels));
    path.push_back({(int)bi, (int)bj});
    cur.erase(cur.begin() + bj);
    cur.erase(cur.begin() + bi);
    cur.push_back(res);
  }
  return path;
}

Network* Network::create(DType dtype, std::vector<NetworkOperand> inputs, NetworkOperand output,
                         std::vector<std::pair<int, int>> path) {
  const int n = (int)inputs.size();
  if (n < 2) throw Error(ERR_UNSUPPORTED, "a network needs at least two input tensors");
  if (output.op.conj) throw Error(ERR_UNSUPPORTED, "a conjugated network output is not supported");
  // One extent per label, consistent over every operand (repeated labels of
  // one operand included).
  std::map<int64_t, int64_t> ext;
  auto note = [&](const NetworkOperand& o, const std::string& what) {
    if (o.labels.size() != o.op.layout.rank())
      throw Error(ERR_LABELS, what + ": " + std::to_string(o.labels.size()) + " labels for " +
                                  std::to_string(o.op.layout.rank()) + " modes");
    for (size_t k = 0; k < o.labels.size(); ++k) {
      const auto it = ext.find(o.labels[k]);
      if (it == ext.end()) ext[o.labels[k]] = o.op.layout.dims[k];
      else if (it->second != o.op.layout.dims[k])
        throw Error(ERR_SHAPE, what + ": label " + std::to_string(o.labels[k]) + " has extent " +
                                   std::to_string(o.op.layout.dims[k]) + ", elsewhere " + std::to_string(it->second));
    }
  };
  for (int i = 0; i < n; ++i) note(inputs[i], "input " + std::to_string(i));
  {
    std::set<int64_t> in_labels;
    for (const auto& o : inputs) in_labels.insert(o.labels.begin(), o.labels.end());
    for (int64_t x : output.labels)
      if (!in_labels.count(x))
        throw Error(ERR_UNSUPPORTED, "output label " + std::to_string(x) + " appears in no input (a broadcast)");
  }
  note(output, "output");

  std::unique_ptr<Network> net(new Network());
  net->dtype = dtype;
  net->inputs = std::move(inputs);
  net->output = std::move(output);
  std::vector<std::vector<int64_t>> labs;
  for (const auto& o : net->inputs) labs.push_back(o.labels);
  if (path.empty()) {
    path = greedy_path(labs, net->output.labels, ext);
    net->greedy = true;
  }
  if ((int)path.size() != n - 1)
    throw Error(ERR_INVALID_ARGUMENT, "a path of " + std::to_string(path.size()) + " steps for " +
                                          std::to_string(n) + " inputs (needs " + std::to_string(n - 1) + ")");
  net->path = path;

  // Walk the path over operand ids.
  std::vector<int> cur(n);
  for (int i = 0; i < n; ++i) cur[i] = i;
  std::vector<std::vector<int64_t>> cur_labels = labs;
  size_t off = 0;
  for (size_t s = 0; s < path.size(); ++s) {
    int i = path[s].first, j = path[s].second;
    const int m = (int)cur.size();
    if (i < 0 || j < 0 || i >= m || j >= m || i == j)
      throw Error(ERR_INVALID_ARGUMENT, "path step " + std::to_string(s) + " (" + std::to_string(i) + ", " +
                                            std::to_string(j) + ") with " + std::to_string(m) + " operands left");
    NetworkStep st;
    st.a = cur[i];
    st.b = cur[j];
    st.la = cur_labels[i];
    st.lb = cur_labels[j];
    st.last = s + 1 == path.size();
    if (st.last) {
      st.labels = net->output.labels;
      st.dims = net->output.op.layout.dims;
    } else {
      st.labels = step_result(st.la, st.lb, needed_elsewhere(cur_labels, (size_t)i, (size_t)j, net->output.labels));
      for (int64_t x : st.labels) st.dims.push_back(ext.at(x));
      int64_t elems = 1;
      for (int64_t d : st.dims) elems *= d;
      st.bytes = (size_t)elems * dtype_size(dtype);
      st.offset = off;
      off += align256(st.bytes);
    }
    auto operand_of = [&](int id) {
      if (id < n) return net->inputs[id].op;
      Operand o;
      o.layout = dense_layout(net->steps[id - n].dims);
      return o;
    };
    const Operand oa = operand_of(st.a), ob = operand_of(st.b);
    Operand od;
    if (st.last) od = net->output.op;
    else od.layout = dense_layout(st.dims);
    const Problem p = Problem::from_labels(dtype, oa, ob, CMode::Separate, od, od, st.la, st.lb, true, st.labels,
                                           st.labels);
    st.plan.reset(new Product(p));
    const std::vector<int64_t> res_labels = st.labels;
    if (i < j) std::swap(i, j);
    cur.erase(cur.begin() + i);
    cur.erase(cur.begin() + j);
    cur_labels.erase(cur_labels.begin() + i);
    cur_labels.erase(cur_labels.begin() + j);
    cur.push_back(n + (int)s);
    cur_labels.push_back(res_labels);
    net->steps.push_back(std::move(st));
  }
  net->arena_bytes = off;
  return net.release();
}

Network::~Network() {
  for (auto& kv : arena)
    if (kv.second) cudaFree(kv.second);
}

double Network::macs() const {
  double t = 0;
  for (const auto& s : steps) t += s.plan->problem.macs();
  return t;
}

std::string Network::report() const {
  std::ostringstream o;
  auto list = [&](const std::vector<int64_t>& v) {
    std::ostringstream q;
    q << "[";
    for (size_t i = 0; i < v.size(); ++i) q << (i ? "," : "") << v[i];
    q << "]";
    return q.str();
  };
  o << "{\"dtype\":\"" << dtype_name(dtype) << "\",\"inputs\":" << inputs.size() << ",\"greedy_path\":"
    << (greedy ? "true" : "false") << ",\"path\":[";
  for (size_t i = 0; i < path.size(); ++i)
    o << (i ? "," : "") << "[" << path[i].first << "," << path[i].second << "]";
  o << "],\"arena_bytes\":" << arena_bytes << ",\"macs\":" << macs() << ",\"steps\":[";
  for (size_t i = 0; i < steps.size(); ++i) {
    const NetworkStep& s = steps[i];
    o << (i ? "," : "") << "{\"a\":" << s.a << ",\"b\":" << s.b << ",\"labels_a\":" << list(s.la)
      << ",\"labels_b\":" << list(s.lb) << ",\"labels\":" << list(s.labels) << ",\"dims\":" << list(s.dims)
      << ",\"last\":" << (s.last ? "true" : "false") << ",\"offset\":" << s.offset
      << ",\"macs\":" << s.plan->problem.macs() << ",\"plan\":" << s.plan->report() << "}";
  }
  o << "]}";
  return o.str();
}

}  // namespace tprims
