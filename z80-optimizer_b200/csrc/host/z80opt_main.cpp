// z80opt -- command-line front end of the candidate-verification path
// (cmd/z80opt/main.go and cmd/mulopt/main.go) on libz80b200.so.
//
//   z80opt enumerate [--max-target N] [--output FILE] [--dead-flags M] [--gpu]
//                    [--workers N] [-v] [--sample N] [--seed S]
//                    [--first-op-start M] [--first-op-end N] [--jsonl FILE] [--no-exhaust]
//                    [--targets-out FILE]
//   z80opt target "ASM : ASM ..." [--max-candidate N] [--dead-flags M] [-v]
//   z80opt verify-jsonl FILE [--dead-flags M] [-v]
//   z80opt mulopt [--pool mulopt|wide21|fast14|cuda21] [--max-len N] [--min-len N]
//                 [--k K] [--json] [--init B,C,F] [--resume FILE]
//   z80opt export FILE [-f go|peephole] [--output OUT] [--var NAME]
//
// Output text follows the reference commands.  --sample/--seed (search a
// seeded uniform sample of the targets), --first-op-start/--first-op-end
// (shard by the first instruction's index), --jsonl (stream rules as JSON
// lines) and --no-exhaust (with --gpu: MidCheck survivors without the
// ExhaustiveCheck tier), after cuda/z80_search_v2.cu, and --pool/--init are
// extensions, and
// so is `export`'s output (the reference command prints a placeholder line):
// result.WriteGoCode text, or the generated source of the peephole table
// package.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "search_api.h"

using namespace z80opt;

namespace {

struct Args {
  std::vector<std::string> pos;
  std::vector<std::pair<std::string, std::string>> opt;
  bool has(const char* k) const {
    for (auto& o : opt)
      if (o.first == k) return true;
    return false;
  }
  std::string get(const char* k, const char* def) const {
    for (auto& o : opt)
      if (o.first == k) return o.second;
    return def;
  }
  long num(const char* k, long def) const {
    const std::string v = get(k, "");
    return v.empty() ? def : std::strtol(v.c_str(), nullptr, 0);
  }
};

Args parse(int argc, char** argv, const std::vector<std::string>& flags) {
  Args a;
  for (int i = 0; i < argc; i++) {
    std::string s = argv[i];
    if (s == "-v") s = "--verbose";
    if (s == "-f") s = "--format";
    if (s == "-o") s = "--output";
    // Go's flag package (cmd/mulopt) also takes long flags with one dash
    if (s.size() > 2 && s[0] == '-' && s[1] != '-' && !(s[1] >= '0' && s[1] <= '9')) s = "-" + s;
    if (s.rfind("--", 0) == 0) {
      const size_t eq = s.find('=');
      std::string k = s.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
      bool is_flag = false;
      for (auto& f : flags) is_flag = is_flag || f == k;
      if (eq != std::string::npos) a.opt.push_back({k, s.substr(eq + 1)});
      else if (is_flag) a.opt.push_back({k, "1"});
      else if (i + 1 < argc) a.opt.push_back({k, argv[++i]});
      else a.opt.push_back({k, ""});
    } else {
      a.pos.push_back(s);
    }
  }
  return a;
}

search::FlagMask dead_flags(const Args& a) {
  search::FlagMask m = 0;
  if (!search::ParseDeadFlags(a.get("dead-flags", "none"), &m))
    throw Error(Z80B_EINVAL, "invalid dead-flags value: " + a.get("dead-flags", "none"));
  return m;
}

// One rule as a JSON line, in cuda/z80_search_v2.cu's emit_jsonl form
// (z80_search_v2.cu:923-942).
void write_jsonl(std::FILE* f, const result::Rule& r) {
  auto esc = [](const std::string& t) {
    std::string o;
    for (char c : t) {
      if (c == '"' || c == '\\') o += '\\';
      o += c;
    }
    return o;
  };
  std::fprintf(f,
               "{\"source_asm\":\"%s\",\"replacement_asm\":\"%s\",\"source_bytes\":%d,\"replacement_bytes\":%d,"
               "\"bytes_saved\":%d,\"cycles_saved\":%d",
               esc(inst::DisasmSeq(r.Source)).c_str(), esc(inst::DisasmSeq(r.Replacement)).c_str(),
               inst::SeqByteSize(r.Source), inst::SeqByteSize(r.Replacement), r.BytesSaved, r.CyclesSaved);
  if (r.DeadFlags) std::fprintf(f, ",\"dead_flags\":\"0x%02X\"", r.DeadFlags);
  std::fputs("}\n", f);
}

int cmd_enumerate(const Args& a) {
  const search::FlagMask dead = dead_flags(a);
  const int maxTarget = int(a.num("max-target", 2));
  const bool gpu = a.has("gpu"), verbose = a.has("verbose");
  const int first0 = int(a.num("first-op-start", 0)), first1 = int(a.num("first-op-end", -1));
  const bool noExhaust = a.has("no-exhaust");
  if (noExhaust && !gpu) throw Error(Z80B_EINVAL, "--no-exhaust needs --gpu (all-hits mode)");
  if (maxTarget < 2 || maxTarget > 3) throw Error(Z80B_EINVAL, "--max-target must be 2 or 3");
  std::FILE* jl = nullptr;
  uint64_t streamed = 0;
  search::RuleSink sink;
  const std::string jpath = a.get("jsonl", "");
  if (!jpath.empty()) {
    jl = std::fopen(jpath.c_str(), "w");
    if (!jl) throw Error(Z80B_EINVAL, "cannot create " + jpath);
    sink = [&](const result::Rule& r) {
      write_jsonl(jl, r);
      streamed++;
    };
  }
  // --targets-out FILE: every searched target as a JSON array of packed words
  std::FILE* tf = nullptr;
  search::TargetSink tsink;
  const std::string tpath = a.get("targets-out", "");
  if (!tpath.empty()) {
    tf = std::fopen(tpath.c_str(), "w");
    if (!tf) throw Error(Z80B_EINVAL, "cannot create " + tpath);
    tsink = [&](const std::vector<uint32_t>& w, int len, uint64_t n) {
      for (uint64_t i = 0; i < n; i++) {
        std::fputc('[', tf);
        for (int k = 0; k < len; k++) std::fprintf(tf, k ? ",%u" : "%u", w[size_t(i) * size_t(len) + size_t(k)]);
        std::fputs("]\n", tf);
      }
    };
  }
  std::printf("Z80 Superoptimizer\n");
  std::printf("  Max target length: %d\n", maxTarget);
  std::printf("  Target instructions: 4531 per position (8-bit only)\n");
  std::printf("  Mode: %s\n", gpu ? "B200 (all hits, pkg/gpu semantics)" : "B200 (first found, pkg/search semantics)");
  if (dead) std::printf("  Dead flags: 0x%02X (%s)\n", dead, result::DeadFlagDesc(dead).c_str());
  std::printf("\n");
  std::vector<result::Rule> rules;
  if (gpu) {
    gpu::SearchConfig c;
    c.MaxTargetLen = maxTarget;
    c.Verbose = verbose;
    c.DeadFlags = dead;
    c.SampleTargets = uint64_t(a.num("sample", 0));
    c.Seed = uint64_t(a.num("seed", 0));
    c.FirstOpStart = first0;
    c.FirstOpEnd = first1;
    c.NoExhaust = noExhaust;
    c.Sink = sink;
    c.Targets = tsink;
    rules = gpu::SearchGPU(c).Rules();
  } else {
    search::Config c;
    c.MaxTargetLen = maxTarget;
    c.NumWorkers = int(a.num("workers", 0));
    c.Verbose = verbose;
    c.DeadFlags = dead;
    c.SampleTargets = uint64_t(a.num("sample", 0));
    c.Seed = uint64_t(a.num("seed", 0));
    c.FirstOpStart = first0;
    c.FirstOpEnd = first1;
    c.Sink = sink;
    c.Targets = tsink;
    rules = search::Run(c).Rules();
  }
  if (tf) std::fclose(tf);
  if (jl) {
    std::fclose(jl);
    std::printf("\nFound %llu optimizations (streamed to %s)\n", (unsigned long long)streamed, jpath.c_str());
    return 0;
  }
  std::printf("\nFound %zu optimizations\n", rules.size());
  const std::string out = a.get("output", "");
  if (!out.empty()) {
    std::FILE* f = std::fopen(out.c_str(), "w");
    if (!f) throw Error(Z80B_EINVAL, "cannot create " + out);
    result::WriteJSON(f, rules);
    std::fclose(f);
    std::printf("Written to %s\n", out.c_str());
  }
  return 0;
}

int cmd_target(const Args& a) {
  if (a.pos.empty()) throw Error(Z80B_EINVAL, "target: an instruction sequence is required");
  std::string input;
  for (size_t i = 0; i < a.pos.size(); i++) input += (i ? " " : "") + a.pos[i];
  Seq seq;
  if (!search::ParseAssembly(input, &seq)) throw Error(Z80B_EINVAL, "failed to parse: " + input);
  std::printf("Target: %s (%d bytes, %d T-states)\n", input.c_str(), inst::SeqByteSize(seq), inst::SeqTStates(seq));
  int maxCand = int(a.num("max-candidate", 4));
  if (maxCand > 2) {
    std::fprintf(stderr, "note: candidates are searched up to 2 instructions (requested %d)\n", maxCand);
    maxCand = 2;
  }
  if (maxCand > int(seq.size()) - 1) maxCand = int(seq.size()) - 1 > 0 ? int(seq.size()) - 1 : 1;
  const search::FlagMask dead = dead_flags(a);
  result::Rule r;
  const bool found = dead ? search::SearchSingleMasked(seq, maxCand, dead, a.has("verbose"), &r)
                          : search::SearchSingle(seq, maxCand, a.has("verbose"), &r);
  if (!found) {
    std::printf("No shorter replacement found.\n");
    return 0;
  }
  std::printf("Replacement: %s (-%d bytes, -%d cycles)", inst::DisasmSeq(r.Replacement).c_str(), r.BytesSaved,
              r.CyclesSaved);
  if (r.DeadFlags) std::printf(" [dead flags 0x%02X: %s]", r.DeadFlags, result::DeadFlagDesc(r.DeadFlags).c_str());
  std::printf("\n");
  return 0;
}

// The value of a JSON string field in a one-object line ("" and false when
// absent or malformed).
bool json_field(const std::string& line, const char* key, std::string* out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = line.find(k);
  if (p == std::string::npos) {
    out->clear();
    return true;  // absent: the zero value, as encoding/json leaves it
  }
  p += k.size();
  while (p < line.size() && (line[p] == ' ' || line[p] == '\t')) p++;
  if (p >= line.size() || line[p] != ':') return false;
  p++;
  while (p < line.size() && (line[p] == ' ' || line[p] == '\t')) p++;
  if (p >= line.size() || line[p] != '"') return false;
  std::string v;
  for (p++; p < line.size(); p++) {
    char c = line[p];
    if (c == '"') {
      *out = v;
      return true;
    }
    if (c == '\\') {
      if (++p >= line.size()) return false;
      switch (line[p]) {
        case 'n': v += '\n'; break;
        case 't': v += '\t'; break;
        case 'r': v += '\r'; break;
        case 'b': v += '\b'; break;
        case 'f': v += '\f'; break;
        case 'u': {
          if (p + 4 >= line.size()) return false;
          const unsigned cp = unsigned(std::strtoul(line.substr(p + 1, 4).c_str(), nullptr, 16));
          if (cp < 0x80) v += char(cp);
          else return false;  // assembly text is ASCII
          p += 4;
        } break;
        default: v += line[p];
      }
    } else {
      v += c;
    }
  }
  return false;
}

// verifyJSONL (cmd/z80opt/main.go:399-476), with every parsed rule checked
// in one batched ExhaustiveCheck on the device.
int cmd_verify_jsonl(const Args& a) {
  if (a.pos.empty()) throw Error(Z80B_EINVAL, "verify-jsonl: a file is required");
  const search::FlagMask dead = dead_flags(a);
  const bool verbose = a.has("verbose");
  std::ifstream in(a.pos[0]);
  if (!in) throw Error(Z80B_EINVAL, "cannot open " + a.pos[0]);
  struct Item {
    int line;
    std::string src, rep;
  };
  std::vector<Item> items;
  std::vector<Seq> ts, cs;
  int total = 0, skipped = 0;
  std::string line;
  while (std::getline(in, line)) {
    const size_t b = line.find_first_not_of(" \t\r\n"), e = line.find_last_not_of(" \t\r\n");
    if (b == std::string::npos) continue;
    line = line.substr(b, e - b + 1);
    total++;
    std::string src, rep;
    if (line.front() != '{' || line.back() != '}' || !json_field(line, "source_asm", &src) ||
        !json_field(line, "replacement_asm", &rep)) {
      std::fprintf(stderr, "  [%d] JSON parse error: malformed object\n", total);
      skipped++;
      continue;
    }
    Seq s, r;
    if (!search::ParseAssembly(src, &s) || s.empty() || s.size() > 4) {
      std::fprintf(stderr, "  [%d] Cannot parse source \"%s\"\n", total, src.c_str());
      skipped++;
      continue;
    }
    if (!search::ParseAssembly(rep, &r) || r.empty() || r.size() > 3) {
      std::fprintf(stderr, "  [%d] Cannot parse replacement \"%s\"\n", total, rep.c_str());
      skipped++;
      continue;
    }
    items.push_back({total, src, rep});
    ts.push_back(s);
    cs.push_back(r);
  }
  const std::vector<uint8_t> ok = search::ExhaustiveCheckBatch(ts, cs, dead);
  int passed = 0, failed = 0;
  for (size_t i = 0; i < items.size(); i++) {
    if (ok[i]) {
      passed++;
      if (verbose) std::printf("  [%d] PASS: %s -> %s\n", items[i].line, items[i].src.c_str(), items[i].rep.c_str());
    } else {
      failed++;
      std::printf("  [%d] FAIL: %s -> %s\n", items[i].line, items[i].src.c_str(), items[i].rep.c_str());
    }
  }
  std::printf("\nVerification complete: %d total, %d passed, %d failed, %d skipped\n", total, passed, failed, skipped);
  if (failed > 0) {
    std::fprintf(stderr, "Error: %d rules failed verification\n", failed);
    return 1;
  }
  return 0;
}

int cmd_mulopt(const Args& a) {
  const std::string pn = a.get("pool", "mulopt");
  int pool = -1;
  if (pn == "mulopt") pool = Z80B_MULPOOL_MULOPT;
  if (pn == "wide21") pool = Z80B_MULPOOL_WIDE21;
  if (pn == "fast14") pool = Z80B_MULPOOL_FAST14;
  if (pn == "cuda21") pool = Z80B_MULPOOL_CUDA21;
  if (pool < 0) throw Error(Z80B_EINVAL, "unknown pool " + pn);
  unsigned b = 0, c = 0, f = 0;
  const std::string init = a.get("init", "");
  if (!init.empty() && std::sscanf(init.c_str(), "%i,%i,%i", &b, &c, &f) != 3)
    throw Error(Z80B_EINVAL, "--init wants B,C,F");
  const int maxLen = int(a.num("max-len", 8)), minLen = int(a.num("min-len", 1));
  const int k = int(a.num("k", 0));
  // -resume (cmd/mulopt/main.go:238-256,283-302): constants solved in an
  // earlier -json output are kept and not searched again
  std::vector<mul::Result> prev;
  const std::string resume = a.get("resume", "");
  if (!resume.empty()) {
    std::ifstream in(resume, std::ios::binary);
    if (!in) {
      std::fprintf(stderr, "Error reading resume file: cannot open %s\n", resume.c_str());
      return 1;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    try {
      prev = mul::ReadJSON(ss.str());
    } catch (const Error& e) {
      std::fprintf(stderr, "Error parsing resume file: %s\n", e.what());
      return 1;
    }
    for (const auto& r : prev)
      if (r.K < 2 || r.K > 255) {
        std::fprintf(stderr, "Error parsing resume file: constant %d outside 2..255\n", r.K);
        return 1;
      }
    std::fprintf(stderr, "Resumed %zu previous results\n", prev.size());
  }
  std::vector<int> ks;
  std::vector<int> pre(256, -1);  // index into prev of a pre-solved constant
  for (size_t i = 0; i < prev.size(); i++) pre[size_t(prev[i].K)] = int(i);
  if (k > 0) ks.push_back(k);
  else
    for (int i = 2; i <= 255; i++)
      if (pre[size_t(i)] < 0) ks.push_back(i);
  int n = 0, ml = 0;
  z80b_mul_pool(pool, &n, &ml, nullptr, nullptr, 0);
  int skipped = 0;
  for (int i = 2; i <= 255; i++) skipped += pre[size_t(i)] >= 0;
  if (k > 0) std::fprintf(stderr, "Searching for mul×%d (len %d..%d, %d ops)...\n", k, minLen, maxLen, n);
  else
    std::fprintf(stderr, "Searching len %d..%d, %zu constants to check (%d pre-solved)\n", minLen, maxLen, ks.size(),
                 skipped);
  z80b_mul_stats st{};
  std::vector<mul::Result> found;
  if (!ks.empty()) found = mul::FindAll(pool, uint8_t(b), uint8_t(c), uint8_t(f), minLen, maxLen, ks, &st);
  std::vector<mul::Result> res;
  if (k > 0) {
    res = found;
  } else {
    // 2..255 in order: pre-solved entries as loaded, the rest as searched
    size_t j = 0;
    for (int i = 2; i <= 255; i++) {
      if (pre[size_t(i)] >= 0) {
        res.push_back(prev[size_t(pre[size_t(i)])]);
        res.back().K = i;
      } else {
        res.push_back(found[j++]);
      }
    }
  }
  if (k > 0) {
    if (!res[0].Found) {
      std::fprintf(stderr, "No sequence found for ×%d within length %d\n", k, maxLen);
      return 1;
    }
    if (a.has("json")) {
      // a single object (encoding/json SetIndent("", "  "))
      std::printf("{\n  \"k\": %d,\n  \"ops\": [\n", res[0].K);
      for (size_t j = 0; j < res[0].Ops.size(); j++)
        std::printf("    \"%s\"%s\n", res[0].Ops[j].c_str(), j + 1 < res[0].Ops.size() ? "," : "");
      std::printf("  ],\n  \"length\": %d,\n  \"tstates\": %d\n}\n", res[0].Length, res[0].TStates);
    } else {
      std::printf("×%d: [", k);
      for (size_t j = 0; j < res[0].Ops.size(); j++) std::printf("%s%s", j ? " " : "", res[0].Ops[j].c_str());
      std::printf("] (%d insts, %dT)\n", res[0].Length, res[0].TStates);
    }
    return 0;
  }
  int solved = 0;
  for (auto& r : res) solved += r.Found;
  std::fprintf(stderr, "Done: %d/254 constants solved (%.1f ms on the device)\n", solved, st.device_ms);
  if (a.has("json")) {
    mul::WriteJSON(stdout, res);
  } else {
    for (auto& r : res) {
      if (!r.Found) continue;
      std::string ops = "[";
      for (size_t j = 0; j < r.Ops.size(); j++) ops += (j ? " " : "") + r.Ops[j];
      ops += "]";
      std::printf("×%3d: %-80s (%d insts, %dT)\n", r.K, ops.c_str(), r.Length, r.TStates);
    }
    for (auto& r : res)
      if (!r.Found) std::printf("×%3d: NOT FOUND (max %d)\n", r.K, maxLen);
  }
  return 0;
}

// export (cmd/z80opt/main.go:173-201): a rules JSON file (result.WriteJSON
// form) written as Go code.  -f go: result.WriteGoCode (pkg/result/
// output.go:95-125), the rules parsed back from their assembly with the
// reference's parser (which, like the reference's, does not take 16-bit
// immediates: such a rule is an error); -f peephole:
// the generated table package of pkg/peephole/rules.go, keyed by source
// assembly in file order (--var names the table, default Top500).  Needs no
// device.
int cmd_export(const Args& a) {
  if (a.pos.size() != 1) throw Error(Z80B_EINVAL, "export: exactly one rules file is required");
  std::FILE* in = std::fopen(a.pos[0].c_str(), "rb");
  if (!in) throw Error(Z80B_EINVAL, "cannot open " + a.pos[0]);
  std::vector<result::JSONRule> js;
  try {
    js = result::ReadJSON(in);
  } catch (...) {
    std::fclose(in);
    throw;
  }
  std::fclose(in);
  const std::string format = a.get("format", "go");
  if (format != "go" && format != "peephole") throw Error(Z80B_EINVAL, "unknown format: " + format);
  std::FILE* out = stdout;
  const std::string path = a.get("output", "");
  if (!path.empty()) {
    out = std::fopen(path.c_str(), "wb");
    if (!out) throw Error(Z80B_EINVAL, "cannot create " + path);
  }
  if (format == "go") {
    std::vector<result::Rule> rules;
    rules.reserve(js.size());
    for (const auto& j : js) rules.push_back(result::FromJSON(j));
    result::WriteGoCode(out, rules);
  } else {
    std::vector<std::pair<std::string, peephole::Rule>> entries;
    entries.reserve(js.size());
    for (const auto& j : js) entries.push_back({j.SourceASM, peephole::Rule{j.ReplacementASM, j.CyclesSaved, j.BytesSaved}});
    std::string from = a.pos[0];
    const size_t slash = from.find_last_of('/');
    if (slash != std::string::npos) from = from.substr(slash + 1);
    peephole::WriteTable(out, entries, from, a.get("var", "Top500"));
  }
  if (out != stdout) std::fclose(out);
  return 0;
}

void usage() {
  std::fprintf(stderr,
               "usage: z80opt enumerate|target|verify-jsonl|mulopt|export [flags]\n"
               "  enumerate    --max-target N --output FILE --dead-flags none|undoc|all|0xNN --gpu -v\n"
               "               --sample N --seed S --first-op-start M --first-op-end N --jsonl FILE --no-exhaust\n"
               "               --targets-out FILE\n"
               "  target       \"ASM : ASM\" --max-candidate N\n"
               "  verify-jsonl FILE --dead-flags M -v\n"
               "  mulopt       --pool mulopt|wide21|fast14|cuda21 --max-len N --k K --json --resume FILE\n"
               "  export       FILE -f go|peephole --output OUT --var NAME\n");
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return 2;
  }
  const std::string cmd = argv[1];
  const Args a = parse(argc - 2, argv + 2, {"verbose", "gpu", "json", "no-exhaust"});
  try {
    if (cmd == "enumerate") return cmd_enumerate(a);
    if (cmd == "target") return cmd_target(a);
    if (cmd == "verify-jsonl") return cmd_verify_jsonl(a);
    if (cmd == "mulopt") return cmd_mulopt(a);
    if (cmd == "export") return cmd_export(a);
    usage();
    return 2;
  } catch (const Error& e) {
    std::fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
}
