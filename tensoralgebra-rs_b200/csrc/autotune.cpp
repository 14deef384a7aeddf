// The autotuner's host side: Problem signatures, candidate launch
// configurations, the model's default choice and the persisted cache.
//
// The reference freezes a kernel family and its blocking at plan time from an
// analytical model of the CPU caches (crates/tprims-contract/src/resolve.rs:42,
// crates/tprims-kernel/src/blocking/model.rs:220). On the GPU the equivalent
// free parameters are the tile family, split-K and (for lists) the tile policy
// of a grouped launch; the model in k_plain.cu picks them from wave counts and
// padding, and the autotuner replaces the model by measurement: the first
// execution of a signature on an executor times every candidate on the
// executor's stream (runtime.cpp) and the executor keeps the fastest, keyed by
// the signature, for every later execution of any plan with that signature.
//
// Cache file (text, one entry per line, fields separated by single spaces):
//   tprims-b200-tune 1 <sm count> <device name with '_' for spaces>
//   single <signature> <kernel> <splits> <chunk> <tiny> <tuned> <ms> <tried>
//   list <signature> <policy> <tuned> <ms> <tried>
// Signatures hold no spaces. Entries made on a device of another kind (SM
// count or name) are skipped on load, since their timings do not transfer.
#include <algorithm>
#include <cstdio>
#include <sstream>

#include "runtime.hpp"

namespace tprims {

namespace {

const char* scheme_tag(Scheme s) {
  switch (s) {
    case Scheme::Plain: return "plain";
    case Scheme::Bf16x3: return "bf16x3";
    case Scheme::Bf16x6: return "bf16x6";
    case Scheme::OzakiInt8: return "ozaki";
  }
  return "?";
}

void axes_tag(std::ostringstream& o, char role, const std::vector<Axis>& ax) {
  o << role << "=";
  for (size_t i = 0; i < ax.size(); ++i) {
    if (i) o << ",";
    o << ax[i].extent << ":" << ax[i].sa << ":" << ax[i].sb << ":" << ax[i].sc << ":" << ax[i].sd;
  }
  o << ";";
}

std::string device_tag(const Executor& ex) {
  std::string n = ex.device_name.empty() ? std::string("unknown") : ex.device_name;
  for (auto& c : n)
    if (c == ' ' || c == '\t' || c == '\n') c = '_';
  return n;
}

// The single-launch tile families of each dtype (direct, then packed).
const int kFamilies[4][4] = {
    {dev::PLAIN_F32_SIMT_128x128, dev::PLAIN_F32_SIMT_64x64, dev::PLAIN_F32_PACKED_128x128,
     dev::PLAIN_F32_PACKED_128x64},
    {dev::PLAIN_F64_DMMA_64x64, dev::PLAIN_F64_DMMA_32x32, dev::PLAIN_F64_DMMA_128x32, dev::PLAIN_F64_PACKED_64x64},
    {dev::PLAIN_C32_SIMT_64x64, dev::PLAIN_C32_PACKED_1M_64x128, dev::PLAIN_C32_PACKED_1M_64x64, 0},
    {dev::PLAIN_C64_DMMA_64x32, dev::PLAIN_C64_DMMA_32x32, dev::PLAIN_C64_DMMA_128x32, dev::PLAIN_C64_PACKED_3M_64x32}};

}  // namespace

std::string problem_signature(const Product& p) {
  // The folded axes fix every offset the kernels compute (extents and the
  // strides of A, B, C, D per role); with the dtype, the orientation and the
  // conjugation of each operand they fix the work of every launch.
  std::ostringstream o;
  const PlanStats& st = p.packed.stats;
  o << dtype_name(p.problem.dtype) << ";";
  axes_tag(o, 'm', st.m_axes);
  axes_tag(o, 'n', st.n_axes);
  axes_tag(o, 'k', st.k_axes);
  axes_tag(o, 'h', st.h_axes);
  o << "cj=" << p.view.conj_a << p.view.conj_b << p.view.conj_c << p.view.conj_d << ";sw=" << p.view.swapped;
  return o.str();
}

std::string tune_key(const Product& p, bool c_read) {
  return p.signature + ";" + scheme_tag(p.scheme) + ";c=" + (c_read ? "1" : "0");
}

std::vector<PlainChoice> plain_candidates(int dtype, int64_t M, int64_t N, int64_t K, int64_t H, int num_sms) {
  std::vector<PlainChoice> out;
  // The model's choice first (ties go to it).
  {
    PlainChoice m;
    if (dev::use_tiny_batched(M, N, K, H)) {
      m.tiny = true;
    } else {
      dev::choose_plain_launch(dtype, 0, M, N, K, H, num_sms, &m.kernel, &m.splits, &m.chunk);
    }
    out.push_back(m);
  }
  auto add = [&](const PlainChoice& c) {
    for (const auto& o : out)
      if (o == c) return;
    out.push_back(c);
  };
  if (dev::use_tiny_batched(M, N, K, H)) {
    PlainChoice t;
    t.tiny = true;
    add(t);
  }
  for (int f : kFamilies[dtype & 3]) {
    if (!f || (dev::is_packed_kernel(f) && !dev::packed_fits(f, M, N, K, H))) continue;
    PlainChoice c;
    c.kernel = f;
    add(c);
    int bm = 0, bn = 0;
    dev::plain_tile_shape(f, &bm, &bn);
    const int64_t tiles = ((M + bm - 1) / bm) * ((N + bn - 1) / bn) * H;
    // Split-K in whole 64-deep blocks, at least 128 deep, at most four CTAs
    // per SM in flight.
    for (int64_t s = 2; s <= 64; s *= 2) {
      const int64_t chunk = ((K + s - 1) / s + 63) / 64 * 64;
      const int64_t parts = (K + chunk - 1) / chunk;
      if (chunk < 128 || parts < 2) break;
      if (tiles * parts > 4 * (int64_t)num_sms) break;
      PlainChoice sc;
      sc.kernel = f;
      sc.splits = (int)parts;
      sc.chunk = chunk;
      add(sc);
    }
  }
  return out;
}

PlainChoice model_choice(const Product& p, int num_sms) {
  const OrientedView& v = p.view;
  const int dt = (int)p.problem.dtype;
  PlainChoice c;
  if (!p.kernel_pin && !p.split_pin && dev::use_tiny_batched(v.M, v.N, v.K, v.H)) {
    c.tiny = true;
    return c;
  }
  if (p.split_pin > 0) {
    c.kernel = p.kernel_pin ? p.kernel_pin : dev::choose_plain_kernel(dt, v.M, v.N, v.K, v.H, num_sms);
    if (p.split_pin > 1 && v.K > 1) {
      const int64_t chunk = std::max<int64_t>(64, ((v.K + p.split_pin - 1) / p.split_pin + 63) / 64 * 64);
      const int64_t parts = (v.K + chunk - 1) / chunk;
      if (parts > 1) {
        c.splits = (int)parts;
        c.chunk = chunk;
      }
    }
    return c;
  }
  dev::choose_plain_launch(dt, p.kernel_pin, v.M, v.N, v.K, v.H, num_sms, &c.kernel, &c.splits, &c.chunk);
  return c;
}

size_t plain_scratch(const PlainChoice& c, const Product& p) {
  if (c.tiny) return 0;
  size_t s = 0;
  if (dev::is_packed_kernel(c.kernel))
    s += dev::packed_workspace_bytes(dev::packed_layout(c.kernel, p.view.M, p.view.N, p.view.K, p.view.H)) + 512;
  if (c.splits > 1) s += (size_t)c.splits * p.view.H * p.view.M * p.view.N * dtype_size(p.problem.dtype) + 256;
  return s;
}

bool choice_fits(const PlainChoice& c, const Product& p) {
  const int64_t M = p.view.M, N = p.view.N, K = p.view.K, H = p.view.H;
  if (c.tiny) return dev::use_tiny_batched(M, N, K, H) && c.splits == 1;
  bool fam_ok = false;
  for (int f : kFamilies[(int)p.problem.dtype & 3]) fam_ok = fam_ok || (f != 0 && f == c.kernel);
  if (!fam_ok || c.splits < 1) return false;
  if (dev::is_packed_kernel(c.kernel) && !dev::packed_fits(c.kernel, M, N, K, H)) return false;
  if (c.splits == 1) return c.chunk == 0 || c.chunk >= K;
  return c.chunk > 0 && c.chunk % 64 == 0 && (K + c.chunk - 1) / c.chunk == c.splits;
}

int grouped_family(const Product& p, int policy) {
  // A packed family pinned on the plan serves its single launches; inside a
  // grouped list the item takes a direct family.
  if (p.kernel_pin && !dev::is_packed_kernel(p.kernel_pin)) return p.kernel_pin;
  const int dt = (int)p.problem.dtype;
  static const int large[4] = {dev::PLAIN_F32_SIMT_128x128, dev::PLAIN_F64_DMMA_64x64, dev::PLAIN_C32_SIMT_64x64,
                               dev::PLAIN_C64_DMMA_64x32};
  static const int small[4] = {dev::PLAIN_F32_SIMT_64x64, dev::PLAIN_F64_DMMA_32x32, dev::PLAIN_C32_SIMT_64x64,
                               dev::PLAIN_C64_DMMA_32x32};
  switch (policy) {
    case 1: return large[dt & 3];
    case 2: return small[dt & 3];
    case 3:
      if ((dt == 1 || dt == 3) && p.view.N <= 32)
        return dt == 1 ? dev::PLAIN_F64_DMMA_128x32 : dev::PLAIN_C64_DMMA_128x32;
      break;
    default: break;
  }
  return dev::choose_grouped_kernel(dt, p.view.M, p.view.N, p.view.K);
}

std::string choice_name(const PlainChoice& c, int dtype) {
  if (c.tiny) return std::string("sm100.") + dtype_name((DType)dtype) + ".tiny-batched";
  std::string s = dev::plain_kernel_name(c.kernel);
  if (c.splits > 1) s += "+splitk" + std::to_string(c.splits);
  return s;
}

std::string tuning_text(const Executor& ex) {
  std::ostringstream o;
  o.precision(17);
  o << "tprims-b200-tune 1 " << ex.num_sms << " " << device_tag(ex) << "\n";
  for (const auto& kv : ex.tune) {
    const TuneEntry& e = kv.second;
    o << "single " << kv.first << " " << e.choice.kernel << " " << e.choice.splits << " " << e.choice.chunk << " "
      << (e.choice.tiny ? 1 : 0) << " " << (e.tuned ? 1 : 0) << " " << e.ms << " " << e.tried << "\n";
  }
  for (const auto& kv : ex.list_tune) {
    const TuneEntry& e = kv.second;
    o << "list " << kv.first << " " << e.policy << " " << (e.tuned ? 1 : 0) << " " << e.ms << " " << e.tried << "\n";
  }
  return o.str();
}

TuningFile parse_tuning_text(const std::string& text) {
  std::istringstream in(text);
  std::string line;
  if (!std::getline(in, line)) throw Error(ERR_INVALID_ARGUMENT, "tuning cache: empty file");
  std::istringstream h(line);
  std::string magic;
  int version = 0;
  TuningFile tf;
  if (!(h >> magic >> version >> tf.sms >> tf.device) || magic != "tprims-b200-tune")
    throw Error(ERR_INVALID_ARGUMENT, "tuning cache: not a tprims-b200-tune file");
  if (version != 1) throw Error(ERR_UNSUPPORTED, "tuning cache: version " + std::to_string(version) + " (expected 1)");
  int lineno = 1;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.empty()) continue;
    std::istringstream f(line);
    std::string kind, sig;
    TuneEntry e;
    int tiny = 0, tuned = 0;
    bool ok = static_cast<bool>(f >> kind >> sig);
    if (ok && kind == "single") {
      ok = static_cast<bool>(f >> e.choice.kernel >> e.choice.splits >> e.choice.chunk >> tiny >> tuned >> e.ms >>
                             e.tried);
      ok = ok && (tiny != 0 || (e.choice.kernel >= 1 && e.choice.kernel <= dev::PLAIN_LAST)) &&
           e.choice.splits >= 1 && e.choice.splits <= 64 && e.choice.chunk >= 0 &&
           (e.choice.splits == 1 || e.choice.chunk > 0);
    } else if (ok && kind == "list") {
      ok = static_cast<bool>(f >> e.policy >> tuned >> e.ms >> e.tried);
      ok = ok && e.policy >= 0 && e.policy < GROUP_POLICIES;
    } else {
      ok = false;
    }
    std::string extra;
    if (!ok || (f >> extra)) throw Error(ERR_INVALID_ARGUMENT, "tuning cache: malformed line " + std::to_string(lineno));
    e.choice.tiny = tiny != 0;
    e.tuned = tuned != 0;
    (kind == "single" ? tf.singles : tf.lists)[sig] = e;
  }
  return tf;
}

void load_tuning_text(Executor& ex, const std::string& text) {
  const TuningFile tf = parse_tuning_text(text);  // all-or-nothing: a malformed file adds nothing
  if (tf.sms != ex.num_sms || tf.device != device_tag(ex)) return;  // measured on another kind of device
  for (auto& kv : tf.singles) ex.tune[kv.first] = kv.second;
  for (auto& kv : tf.lists) ex.list_tune[kv.first] = kv.second;
}

std::string tuning_json(const Executor& ex) {
  std::ostringstream o;
  o << "{\"device\":\"" << device_tag(ex) << "\",\"sms\":" << ex.num_sms << ",\"single\":{";
  bool first = true;
  for (const auto& kv : ex.tune) {
    if (!first) o << ",";
    first = false;
    const PlainChoice& c = kv.second.choice;
    const std::string fam =
        c.tiny ? std::string("tiny-batched")
               : std::string(dev::plain_kernel_name(c.kernel)) + (c.splits > 1 ? "+splitk" + std::to_string(c.splits) : "");
    o << "\"" << kv.first << "\":{\"family\":\"" << fam << "\",\"kernel\":" << kv.second.choice.kernel
      << ",\"splits\":" << kv.second.choice.splits << ",\"tiny\":" << (kv.second.choice.tiny ? "true" : "false")
      << ",\"tuned\":" << (kv.second.tuned ? "true" : "false") << ",\"ms\":" << kv.second.ms
      << ",\"tried\":" << kv.second.tried << "}";
  }
  o << "},\"list\":{";
  first = true;
  for (const auto& kv : ex.list_tune) {
    if (!first) o << ",";
    first = false;
    o << "\"" << kv.first << "\":{\"policy\":" << kv.second.policy << ",\"tuned\":"
      << (kv.second.tuned ? "true" : "false") << ",\"ms\":" << kv.second.ms << ",\"tried\":" << kv.second.tried << "}";
  }
  o << "}}";
  return o.str();
}

}  // namespace tprims
