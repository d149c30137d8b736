// search_api.cpp -- the Go search API mirror (search_api.h) over the C ABI.
#include "search_api.h"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <random>

namespace z80opt {

namespace {

std::mutex g_mu;
z80b_ctx* g_ctx = nullptr;

[[noreturn]] void raise(int st, const char* what) {
  std::string m = std::string(what) + ": " + z80b_status_string(st);
  if (g_ctx) m += std::string(" (") + z80b_last_error(g_ctx) + ")";
  throw Error(st, m);
}

void check(int st, const char* what) {
  if (st != Z80B_OK) raise(st, what);
}

std::vector<uint32_t> pack(const Seq& s) {
  std::vector<uint32_t> w(s.size());
  for (size_t i = 0; i < s.size(); i++) w[i] = s[i].packed();
  return w;
}

Seq unpack(const uint32_t* w, int n) {
  Seq s(static_cast<size_t>(n));
  for (int i = 0; i < n; i++) s[size_t(i)] = Instruction::unpack(w[i]);
  return s;
}

result::Rule to_rule(const z80b_rule& r) {
  result::Rule o;
  o.Source = unpack(r.src, r.src_len);
  o.Replacement = unpack(r.rep, r.rep_len);
  o.BytesSaved = r.bytes_saved;
  o.CyclesSaved = r.cycles_saved;
  o.DeadFlags = uint8_t(r.dead_flags);
  o.DeadRegs = uint8_t(r.dead_regs);
  return o;
}

// One z80b_search over packed targets (stride words each); rules appended
// to `table` in target order.
void run_job(const std::vector<uint32_t>& targets, const std::vector<uint8_t>& lens, uint32_t stride,
             int maxCand, search::FlagMask dead, uint32_t mode, result::Table* table, search::Stats* stats) {
  const uint32_t n = uint32_t(lens.size());
  if (n == 0) return;
  z80b_job job{};
  job.targets = targets.data();
  job.target_lens = lens.data();
  job.n_targets = n;
  job.target_stride = stride;
  job.max_cand_len = uint32_t(maxCand);
  job.global_dead_flags = dead;
  job.mode = mode;
  job.path = Z80B_PATH_BATCHED;
  std::vector<z80b_rule> out(size_t(n) * 2 + 16);
  uint64_t nr = 0;
  z80b_stats st{};
  int s = z80b_search(context(), &job, out.data(), out.size(), &nr, &st);
  if (s == Z80B_ECAPACITY && nr > out.size()) {
    out.resize(nr);
    st = z80b_stats{};
    s = z80b_search(context(), &job, out.data(), out.size(), &nr, &st);
  }
  check(s, "z80b_search");
  for (uint64_t i = 0; i < nr; i++) table->Add(to_rule(out[i]));
  if (stats) {
    stats->targets += st.targets;
    stats->checks += st.checks;
    stats->checked += st.checked_ref;
    stats->rules += st.rules;
    stats->device_ms += st.device_ms;
  }
}

// The unpruned targets of one length over the 8-bit list, in
// EnumerateSequences8 order, or a seeded sample of them by index.
void collect_targets(int len, uint64_t sample, uint64_t seed, std::vector<uint32_t>* out, uint64_t* count) {
  std::vector<uint32_t> pool(4531);
  pool.resize(z80b_pool8(pool.data(), uint32_t(pool.size())));
  const uint64_t total = z80b_enumerate(pool.data(), uint32_t(pool.size()), uint32_t(len), nullptr, 0);
  std::vector<uint32_t> all(total * uint64_t(len));
  z80b_enumerate(pool.data(), uint32_t(pool.size()), uint32_t(len), all.data(), total);
  if (sample == 0 || sample >= total) {
    *out = std::move(all);
    *count = total;
    return;
  }
  // Floyd's algorithm: `sample` distinct indices, then index order.
  std::mt19937_64 rng(seed);
  std::vector<uint64_t> pick;
  pick.reserve(sample);
  std::vector<uint8_t> taken(total, 0);
  for (uint64_t j = total - sample; j < total; j++) {
    uint64_t t = std::uniform_int_distribution<uint64_t>(0, j)(rng);
    if (taken[t]) t = j;
    taken[t] = 1;
    pick.push_back(t);
  }
  std::sort(pick.begin(), pick.end());
  out->resize(sample * uint64_t(len));
  for (uint64_t i = 0; i < sample; i++)
    std::memcpy(out->data() + i * uint64_t(len), all.data() + pick[i] * uint64_t(len), 4u * uint32_t(len));
  *count = sample;
}

result::Table run_lengths(int maxTarget, int maxCand, search::FlagMask dead, uint32_t mode, uint64_t sample,
                          uint64_t seed, bool verbose, search::Stats* stats) {
  result::Table table;
  for (int len = 2; len <= maxTarget; len++) {
    std::vector<uint32_t> t;
    uint64_t n = 0;
    collect_targets(len, sample, seed, &t, &n);
    if (verbose) std::printf("=== Searching target length %d ===\n  Generated %llu target sequences (after pruning)\n",
                             len, (unsigned long long)n);
    // jobs of at most 4M targets keep the per-job device buffers modest
    const uint64_t chunk = 1u << 22;
    for (uint64_t lo = 0; lo < n; lo += chunk) {
      const uint64_t hi = std::min(n, lo + chunk);
      std::vector<uint32_t> part(t.begin() + long(lo * uint64_t(len)), t.begin() + long(hi * uint64_t(len)));
      std::vector<uint8_t> lens(hi - lo, uint8_t(len));
      run_job(part, lens, uint32_t(len), maxCand, dead, mode, &table, stats);
    }
    if (verbose) std::printf("  Found: %zu\n", table.Len());
  }
  return table;
}

}  // namespace

z80b_ctx* context() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    z80b_ctx* c = nullptr;
    int s = z80b_init(0, &c);
    if (s != Z80B_OK) throw Error(s, std::string("z80b_init: ") + z80b_status_string(s));
    g_ctx = c;
  }
  return g_ctx;
}

namespace inst {
int SeqByteSize(const Seq& s) {
  int b = 0;
  for (const auto& i : s) {
    int size = 0;
    z80b_op_info(i.op, nullptr, 0, &size, nullptr, nullptr, nullptr, nullptr);
    b += size;
  }
  return b;
}
int SeqTStates(const Seq& s) {
  int t = 0;
  for (const auto& i : s) {
    int ts = 0;
    z80b_op_info(i.op, nullptr, 0, nullptr, &ts, nullptr, nullptr, nullptr);
    t += ts;
  }
  return t;
}
std::string Disassemble(const Instruction& i) { return DisasmSeq(Seq{i}); }
std::string DisasmSeq(const Seq& s) {
  const auto w = pack(s);
  char buf[256];
  if (z80b_disasm_seq(w.data(), uint32_t(w.size()), buf, sizeof buf) < 0) return "?";
  return buf;
}
}  // namespace inst

namespace result {
std::vector<Rule> Table::Rules() const {
  std::vector<Rule> r = rules_;
  std::stable_sort(r.begin(), r.end(), [](const Rule& a, const Rule& b) {
    if (a.BytesSaved != b.BytesSaved) return a.BytesSaved > b.BytesSaved;
    return a.CyclesSaved > b.CyclesSaved;
  });
  return r;
}
std::string DeadFlagDesc(uint8_t mask) {
  char buf[64];
  z80b_dead_flag_desc(mask, buf, sizeof buf);
  return buf;
}
void WriteJSON(std::FILE* f, const std::vector<Rule>& rules) {
  std::vector<z80b_rule> rr(rules.size());
  for (size_t i = 0; i < rules.size(); i++) {
    z80b_rule& o = rr[i];
    std::memset(&o, 0, sizeof o);
    o.src_len = int32_t(rules[i].Source.size());
    o.rep_len = int32_t(rules[i].Replacement.size());
    for (int k = 0; k < o.src_len && k < 4; k++) o.src[k] = rules[i].Source[size_t(k)].packed();
    for (int k = 0; k < o.rep_len && k < 4; k++) o.rep[k] = rules[i].Replacement[size_t(k)].packed();
    o.bytes_saved = rules[i].BytesSaved;
    o.cycles_saved = rules[i].CyclesSaved;
    o.dead_flags = rules[i].DeadFlags;
  }
  const long long n = z80b_rules_json(rr.data(), rr.size(), nullptr, 0);
  if (n < 0) throw Error(Z80B_EINVAL, "WriteJSON: rule with a bad instruction");
  std::string s(size_t(n) + 1, '\0');
  z80b_rules_json(rr.data(), rr.size(), &s[0], s.size());
  std::fwrite(s.data(), 1, size_t(n), f);
}
}  // namespace result

namespace search {

result::Table Run(const Config& cfg, Stats* stats) {
  const int maxCand = cfg.MaxCandLen > 0 ? cfg.MaxCandLen : cfg.MaxTargetLen - 1;
  return run_lengths(cfg.MaxTargetLen, maxCand, cfg.DeadFlags, Z80B_MODE_FIRST, cfg.SampleTargets, cfg.Seed,
                     cfg.Verbose, stats);
}

static bool single(const Seq& target, int maxCandLen, FlagMask dead, result::Rule* out) {
  if (target.empty() || target.size() > 4) throw Error(Z80B_EINVAL, "target length must be 1..4");
  result::Table t;
  const auto w = pack(target);
  run_job(w, {uint8_t(target.size())}, uint32_t(target.size()), maxCandLen, dead, Z80B_MODE_FIRST, &t, nullptr);
  const auto rules = t.Rules();
  if (rules.empty()) return false;
  if (out) *out = rules[0];
  return true;
}

bool SearchSingle(const Seq& target, int maxCandLen, bool, result::Rule* out) {
  return single(target, maxCandLen, DeadNone, out);
}

bool SearchSingleMasked(const Seq& target, int maxCandLen, FlagMask deadFlags, bool, result::Rule* out) {
  return single(target, maxCandLen, deadFlags, out);
}

std::vector<uint8_t> ExhaustiveCheckBatch(const std::vector<Seq>& targets, const std::vector<Seq>& cands,
                                          FlagMask deadFlags) {
  const size_t n = targets.size();
  if (cands.size() != n) throw Error(Z80B_EINVAL, "ExhaustiveCheckBatch: size mismatch");
  std::vector<uint8_t> pass(n, 0);
  if (n == 0) return pass;
  const uint32_t stride = 4;
  std::vector<uint32_t> tw(n * stride, 0), cw(n * stride, 0);
  std::vector<uint8_t> tl(n), cl(n), dd(n, deadFlags), fd(n);
  for (size_t i = 0; i < n; i++) {
    if (targets[i].empty() || targets[i].size() > 4 || cands[i].empty() || cands[i].size() > 3)
      throw Error(Z80B_EINVAL, "ExhaustiveCheckBatch: sequence lengths 1..4 (target), 1..3 (candidate)");
    tl[i] = uint8_t(targets[i].size());
    cl[i] = uint8_t(cands[i].size());
    for (size_t k = 0; k < targets[i].size(); k++) tw[i * stride + k] = targets[i][k].packed();
    for (size_t k = 0; k < cands[i].size(); k++) cw[i * stride + k] = cands[i][k].packed();
  }
  // the library takes bounded batches; split long lists
  const size_t chunk = 1u << 20;
  for (size_t lo = 0; lo < n; lo += chunk) {
    const size_t m = std::min(n - lo, chunk);
    check(z80b_verify_pairs(context(), tw.data() + lo * stride, tl.data() + lo, cw.data() + lo * stride, cl.data() + lo,
                            stride, uint32_t(m), dd.data() + lo, 4u, pass.data() + lo, fd.data() + lo),
          "z80b_verify_pairs");
  }
  return pass;
}

bool ExhaustiveCheck(const Seq& target, const Seq& cand) {
  return ExhaustiveCheckBatch({target}, {cand}, DeadNone)[0] != 0;
}
bool ExhaustiveCheckMasked(const Seq& target, const Seq& cand, FlagMask deadFlags) {
  return ExhaustiveCheckBatch({target}, {cand}, deadFlags)[0] != 0;
}

bool ShouldPrune(const Seq& s) {
  const auto w = pack(s);
  return z80b_should_prune(w.data(), uint32_t(w.size())) == 1;
}

bool ParseAssembly(const std::string& text, Seq* out) {
  uint32_t buf[64];
  const int n = z80b_parse_assembly(text.c_str(), buf, 64);
  if (n < 0 || n > 64) return false;
  *out = unpack(buf, n);
  return true;
}

bool ParseDeadFlags(const std::string& text, FlagMask* out) {
  uint32_t m = 0;
  if (z80b_parse_dead_flags(text.c_str(), &m) != Z80B_OK) return false;
  *out = FlagMask(m);
  return true;
}

}  // namespace search

namespace gpu {
result::Table SearchGPU(const SearchConfig& cfg) {
  return run_lengths(cfg.MaxTargetLen, 1, cfg.DeadFlags, Z80B_MODE_ALL, cfg.SampleTargets, cfg.Seed, cfg.Verbose,
                     nullptr);
}
}  // namespace gpu

namespace mul {
std::vector<Result> FindAll(int pool, uint8_t b, uint8_t c, uint8_t f, int minLen, int maxLen,
                            const std::vector<int>& ks, z80b_mul_stats* stats) {
  std::vector<int32_t> kk(ks.begin(), ks.end());
  std::vector<z80b_mul_result> out(kk.size());
  z80b_mul_stats st{};
  check(z80b_mul_search(context(), pool, b, c, f, minLen, maxLen, kk.data(), uint32_t(kk.size()), out.data(), &st),
        "z80b_mul_search");
  if (stats) *stats = st;
  int n = 0, maxl = 0;
  const char* names[32] = {};
  z80b_mul_pool(pool, &n, &maxl, names, nullptr, 32);
  std::vector<Result> res(kk.size());
  for (size_t i = 0; i < kk.size(); i++) {
    res[i].K = out[i].k;
    res[i].Found = out[i].found != 0;
    res[i].Length = out[i].length;
    res[i].TStates = out[i].tstates;
    for (int j = 0; j < out[i].length; j++) res[i].Ops.push_back(names[out[i].ops[j]]);
  }
  return res;
}

void WriteJSON(std::FILE* f, const std::vector<Result>& results) {
  // encoding/json with SetIndent("", "  ") (cmd/mulopt/main.go:336-350)
  std::vector<const Result*> found;
  for (const auto& r : results)
    if (r.Found) found.push_back(&r);
  if (found.empty()) {
    std::fprintf(f, "null\n");
    return;
  }
  std::fprintf(f, "[\n");
  for (size_t i = 0; i < found.size(); i++) {
    const Result& r = *found[i];
    std::fprintf(f, "  {\n    \"k\": %d,\n    \"ops\": [\n", r.K);
    for (size_t j = 0; j < r.Ops.size(); j++)
      std::fprintf(f, "      \"%s\"%s\n", r.Ops[j].c_str(), j + 1 < r.Ops.size() ? "," : "");
    std::fprintf(f, "    ],\n    \"length\": %d,\n    \"tstates\": %d\n  }%s\n", r.Length, r.TStates,
                 i + 1 < found.size() ? "," : "");
  }
  std::fprintf(f, "]\n");
}
}  // namespace mul

}  // namespace z80opt
