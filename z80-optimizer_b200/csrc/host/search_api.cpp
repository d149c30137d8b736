// search_api.cpp -- the Go search API mirror (search_api.h) over the C ABI.
#include "search_api.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstring>
#include <fstream>
#include <mutex>
#include <random>
#include <sstream>
#include <thread>
#include <unordered_set>

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

// A JSON value, as much of JSON as rule files need (RFC 8259 grammar).
struct JVal {
  enum Kind { kNull, kBool, kNum, kStr, kArr, kObj } k = kNull;
  bool b = false;
  double num = 0;
  bool integral = false;  // a number without fraction or exponent that fits in long long
  long long i = 0;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
};

class JParser {
 public:
  explicit JParser(const std::string& t) : t_(t) {}
  JVal parse() {
    JVal v = value(0);
    ws();
    if (p_ != t_.size()) fail("data after the top-level value");
    return v;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;

  [[noreturn]] void fail(const char* what) const {
    throw Error(Z80B_EINVAL, std::string("ReadJSON: ") + what + " at byte " + std::to_string(p_));
  }
  bool at(char c) const { return p_ < t_.size() && t_[p_] == c; }
  void ws() {
    while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t' || t_[p_] == '\n' || t_[p_] == '\r')) p_++;
  }
  bool word(const char* w) {
    const size_t n = std::strlen(w);
    if (t_.compare(p_, n, w) != 0) return false;
    p_ += n;
    return true;
  }
  JVal value(int depth) {
    if (depth > 256) fail("nesting too deep");
    ws();
    if (p_ >= t_.size()) fail("unexpected end of input");
    JVal v;
    const char c = t_[p_];
    if (c == '{') {
      p_++;
      v.k = JVal::kObj;
      ws();
      if (at('}')) {
        p_++;
        return v;
      }
      for (;;) {
        ws();
        if (!at('"')) fail("expected an object key");
        std::string key = str();
        ws();
        if (!at(':')) fail("expected ':'");
        p_++;
        v.obj.emplace_back(std::move(key), value(depth + 1));
        ws();
        if (at(',')) {
          p_++;
          continue;
        }
        if (at('}')) {
          p_++;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      p_++;
      v.k = JVal::kArr;
      ws();
      if (at(']')) {
        p_++;
        return v;
      }
      for (;;) {
        v.arr.push_back(value(depth + 1));
        ws();
        if (at(',')) {
          p_++;
          continue;
        }
        if (at(']')) {
          p_++;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.k = JVal::kStr;
      v.s = str();
      return v;
    }
    if (word("true")) {
      v.k = JVal::kBool;
      v.b = true;
      return v;
    }
    if (word("false")) {
      v.k = JVal::kBool;
      return v;
    }
    if (word("null")) return v;
    return number();
  }
  unsigned hex4() {
    if (p_ + 4 > t_.size()) fail("short \\u escape");
    unsigned v = 0;
    for (int k = 0; k < 4; k++) {
      const char h = t_[p_++];
      v <<= 4;
      if (h >= '0' && h <= '9') v |= unsigned(h - '0');
      else if (h >= 'a' && h <= 'f') v |= unsigned(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= unsigned(h - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  static void utf8(std::string& o, unsigned cp) {
    if (cp < 0x80) {
      o += char(cp);
    } else if (cp < 0x800) {
      o += char(0xC0 | (cp >> 6));
      o += char(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      o += char(0xE0 | (cp >> 12));
      o += char(0x80 | ((cp >> 6) & 0x3F));
      o += char(0x80 | (cp & 0x3F));
    } else {
      o += char(0xF0 | (cp >> 18));
      o += char(0x80 | ((cp >> 12) & 0x3F));
      o += char(0x80 | ((cp >> 6) & 0x3F));
      o += char(0x80 | (cp & 0x3F));
    }
  }
  std::string str() {
    p_++;  // opening quote
    std::string out;
    while (p_ < t_.size()) {
      const char c = t_[p_++];
      if (c == '"') return out;
      if (static_cast<unsigned char>(c) < 0x20) fail("control character in a string");
      if (c != '\\') {
        out += c;
        continue;
      }
      if (p_ >= t_.size()) break;
      const char e = t_[p_++];
      switch (e) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          unsigned cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00) {  // a surrogate pair, else U+FFFD
            const size_t save = p_;
            if (word("\\u")) {
              const unsigned lo = hex4();
              if (lo >= 0xDC00 && lo < 0xE000) {
                cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
              } else {
                cp = 0xFFFD;
                p_ = save;
              }
            } else {
              cp = 0xFFFD;
            }
          } else if (cp >= 0xDC00 && cp < 0xE000) {
            cp = 0xFFFD;
          }
          utf8(out, cp);
          break;
        }
        default: fail("bad escape in a string");
      }
    }
    fail("unterminated string");
  }
  JVal number() {
    const size_t b = p_;
    bool integral = true;
    if (at('-')) p_++;
    if (at('0')) {
      p_++;
    } else if (p_ < t_.size() && t_[p_] >= '1' && t_[p_] <= '9') {
      while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) p_++;
    } else {
      fail("invalid value");
    }
    if (at('.')) {
      integral = false;
      p_++;
      if (!(p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_])))) fail("bad number");
      while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) p_++;
    }
    if (at('e') || at('E')) {
      integral = false;
      p_++;
      if (at('+') || at('-')) p_++;
      if (!(p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_])))) fail("bad number");
      while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) p_++;
    }
    JVal v;
    v.k = JVal::kNum;
    const std::string text = t_.substr(b, p_ - b);
    v.num = std::strtod(text.c_str(), nullptr);
    if (integral) {
      errno = 0;
      char* end = nullptr;
      v.i = std::strtoll(text.c_str(), &end, 10);
      v.integral = errno == 0;
    }
    return v;
  }
};

// Go %q of a string (strconv.Quote): printable ASCII as is, quote and
// backslash escaped, the rest as escapes.
std::string go_quote(const std::string& s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    if (c == '"' || c == '\\') {
      o += '\\';
      o += char(c);
    } else if (c >= 0x20 && c < 0x7F) {
      o += char(c);
    } else if (c == '\n') {
      o += "\\n";
    } else if (c == '\t') {
      o += "\\t";
    } else if (c == '\r') {
      o += "\\r";
    } else {
      char buf[8];
      std::snprintf(buf, sizeof buf, "\\x%02x", c);
      o += buf;
    }
  }
  return o + "\"";
}

std::string read_all(std::FILE* f) {
  std::string t;
  char buf[65536];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) t.append(buf, n);
  return t;
}

bool key_is(const std::string& key, const char* tag) {
  const size_t n = std::strlen(tag);
  if (key.size() != n) return false;
  for (size_t i = 0; i < n; i++)
    if (std::tolower(static_cast<unsigned char>(key[i])) != std::tolower(static_cast<unsigned char>(tag[i])))
      return false;
  return true;
}

void json_string_field(const JVal& v, std::string* out, const char* key) {
  if (v.k == JVal::kNull) return;
  if (v.k != JVal::kStr) throw Error(Z80B_EINVAL, std::string("ReadJSON: field ") + key + " is not a string");
  *out = v.s;
}

void json_int_field(const JVal& v, int* out, const char* key) {
  if (v.k == JVal::kNull) return;
  if (v.k != JVal::kNum || !v.integral || v.i < INT_MIN || v.i > INT_MAX)
    throw Error(Z80B_EINVAL, std::string("ReadJSON: field ") + key + " is not an integer in range");
  *out = int(v.i);
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
             int maxCand, search::FlagMask dead, uint32_t mode, uint32_t flags,
             const std::function<void(const result::Rule&)>& emit, search::Stats* stats) {
  const uint32_t n = uint32_t(lens.size());
  if (n == 0) return;
  z80b_job job{};
  job.flags = flags;
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
  for (uint64_t i = 0; i < nr; i++) emit(to_rule(out[i]));
  if (stats) {
    stats->targets += st.targets;
    stats->checks += st.checks;
    stats->checked += st.checked_ref;
    stats->rules += st.rules;
    stats->device_ms += st.device_ms;
  }
}

// What run_lengths searches: target lengths 2..maxTarget (each over the
// first-instruction range, whole or sampled) as first-found or all-hits
// jobs of at most 4M targets.
struct RunSpec {
  int maxTarget = 2, maxCand = 1;
  search::FlagMask dead = 0;
  uint32_t mode = Z80B_MODE_FIRST, flags = 0;
  uint64_t sample = 0, seed = 0;
  bool verbose = false;
  int first0 = 0, first1 = -1;
  search::RuleSink sink;
  search::TargetSink targets;
};

result::Table run_lengths(const RunSpec& r, search::Stats* stats) {
  result::Table table;
  const std::function<void(const result::Rule&)> emit =
      r.sink ? r.sink : std::function<void(const result::Rule&)>([&](const result::Rule& x) { table.Add(x); });
  for (int len = 2; len <= r.maxTarget; len++) {
    if (r.verbose) std::printf("=== Searching target length %d ===\n", len);
    uint64_t n = 0;
    // jobs of at most 4M targets keep the per-job device buffers modest
    search::EnumerateTargets(len, r.first0, r.first1, r.sample, r.seed, 1u << 22,
                             [&](const std::vector<uint32_t>& w, uint64_t m) {
                               n += m;
                               if (r.targets) r.targets(w, len, m);
                               const std::vector<uint8_t> lens(m, uint8_t(len));
                               run_job(w, lens, uint32_t(len), r.maxCand, r.dead, r.mode, r.flags, emit, stats);
                             });
    if (r.verbose) {
      std::printf("  Generated %llu target sequences (after pruning)\n", (unsigned long long)n);
      if (!r.sink) std::printf("  Found: %zu\n", table.Len());
    }
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

std::vector<JSONRule> ReadJSON(const std::string& text) {
  const JVal top = JParser(text).parse();
  std::vector<JSONRule> out;
  if (top.k == JVal::kNull) return out;
  if (top.k != JVal::kArr) throw Error(Z80B_EINVAL, "ReadJSON: the top-level value is not an array");
  for (const JVal& e : top.arr) {
    JSONRule r;
    if (e.k == JVal::kNull) {
      out.push_back(r);
      continue;
    }
    if (e.k != JVal::kObj) throw Error(Z80B_EINVAL, "ReadJSON: an array element is not an object");
    for (const auto& kv : e.obj) {
      const std::string& k = kv.first;
      if (key_is(k, "source_asm")) json_string_field(kv.second, &r.SourceASM, "source_asm");
      else if (key_is(k, "replacement_asm")) json_string_field(kv.second, &r.ReplacementASM, "replacement_asm");
      else if (key_is(k, "source_bytes")) json_int_field(kv.second, &r.SourceBytes, "source_bytes");
      else if (key_is(k, "replacement_bytes")) json_int_field(kv.second, &r.ReplacementBytes, "replacement_bytes");
      else if (key_is(k, "bytes_saved")) json_int_field(kv.second, &r.BytesSaved, "bytes_saved");
      else if (key_is(k, "cycles_saved")) json_int_field(kv.second, &r.CyclesSaved, "cycles_saved");
      else if (key_is(k, "dead_flags")) json_string_field(kv.second, &r.DeadFlags, "dead_flags");
      else if (key_is(k, "dead_flag_desc")) json_string_field(kv.second, &r.DeadFlagDesc, "dead_flag_desc");
    }
    out.push_back(r);
  }
  return out;
}

std::vector<JSONRule> ReadJSON(std::FILE* f) { return ReadJSON(read_all(f)); }

Rule FromJSON(const JSONRule& j) {
  Rule r;
  if (!search::ParseAssembly(j.SourceASM, &r.Source) || r.Source.empty())
    throw Error(Z80B_EINVAL, "cannot parse source assembly: " + j.SourceASM);
  if (!j.ReplacementASM.empty() && !search::ParseAssembly(j.ReplacementASM, &r.Replacement))
    throw Error(Z80B_EINVAL, "cannot parse replacement assembly: " + j.ReplacementASM);
  r.BytesSaved = j.BytesSaved;
  r.CyclesSaved = j.CyclesSaved;
  if (!j.DeadFlags.empty()) {
    char* end = nullptr;
    const unsigned long m = std::strtoul(j.DeadFlags.c_str(), &end, 16);
    if (*end != '\0' || m > 0xFF) throw Error(Z80B_EINVAL, "bad dead_flags: " + j.DeadFlags);
    r.DeadFlags = uint8_t(m);
  }
  return r;
}

void WriteGoCode(std::FILE* f, const std::vector<Rule>& rules) {
  auto seq_text = [](const Seq& s) { return s.empty() ? std::string() : inst::DisasmSeq(s); };
  auto go_slice = [](const Seq& s) {
    std::string o;
    for (size_t i = 0; i < s.size(); i++) {
      if (i) o += ", ";
      o += go_quote(inst::Disassemble(s[i]));
    }
    return o;
  };
  std::fputs("// Code generated by z80opt. DO NOT EDIT.\n\npackage optimizer\n\n"
             "// Z80OptRules contains peephole optimization rules discovered by the superoptimizer.\n"
             "var Z80OptRules = []PeepholeRule{\n",
             f);
  for (const Rule& r : rules) {
    const std::string src = seq_text(r.Source), rep = seq_text(r.Replacement);
    if (r.DeadFlags)
      std::fprintf(f, "\t// %s -> %s (-%d bytes, -%d cycles) [dead: %s]\n", src.c_str(), rep.c_str(), r.BytesSaved,
                   r.CyclesSaved, DeadFlagDesc(r.DeadFlags).c_str());
    else
      std::fprintf(f, "\t// %s -> %s (-%d bytes, -%d cycles)\n", src.c_str(), rep.c_str(), r.BytesSaved,
                   r.CyclesSaved);
    std::fprintf(f, "\t{\n\t\tMatch: []string{%s},\n\t\tReplace: []string{%s},\n", go_slice(r.Source).c_str(),
                 go_slice(r.Replacement).c_str());
    if (r.DeadFlags) std::fprintf(f, "\t\tDeadFlags: 0x%02X, // %s\n", r.DeadFlags, DeadFlagDesc(r.DeadFlags).c_str());
    std::fputs("\t},\n", f);
  }
  std::fputs("}\n", f);
}
}  // namespace result

namespace peephole {
const Rule* Lookup(const Table& t, const std::string& source) {
  const auto it = t.find(source);
  return it == t.end() ? nullptr : &it->second;
}

Table LoadRules(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error(Z80B_EINVAL, "LoadRules: cannot open " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  const JVal top = JParser(ss.str()).parse();
  Table t;
  if (top.k == JVal::kNull) return t;
  if (top.k != JVal::kArr) throw Error(Z80B_EINVAL, "LoadRules: the top-level value is not an array");
  for (const JVal& e : top.arr) {
    if (e.k == JVal::kNull) {
      t[""] = Rule{};
      continue;
    }
    if (e.k != JVal::kObj) throw Error(Z80B_EINVAL, "LoadRules: an array element is not an object");
    std::string src;
    Rule r;
    for (const auto& kv : e.obj) {
      if (key_is(kv.first, "source")) json_string_field(kv.second, &src, "source");
      else if (key_is(kv.first, "replacement")) json_string_field(kv.second, &r.Replacement, "replacement");
      else if (key_is(kv.first, "cycles_saved")) json_int_field(kv.second, &r.CyclesSaved, "cycles_saved");
      else if (key_is(kv.first, "bytes_saved")) json_int_field(kv.second, &r.BytesSaved, "bytes_saved");
    }
    t[src] = r;
  }
  return t;
}

void WriteTable(std::FILE* f, const std::vector<std::pair<std::string, Rule>>& entries, const std::string& from,
                const std::string& var_name) {
  std::fprintf(f,
               "// Code generated from %s. DO NOT EDIT.\n"
               "package peephole\n\n"
               "import (\n\t\"encoding/json\"\n\t\"os\"\n)\n\n"
               "// Rule is a peephole replacement: the replacement assembly and what it saves.\n"
               "type Rule struct {\n\tReplacement string\n\tCyclesSaved int\n\tBytesSaved  int\n}\n\n"
               "// %s maps source assembly to its replacement.\n"
               "var %s = map[string]Rule{\n",
               from.c_str(), var_name.c_str(), var_name.c_str());
  for (const auto& e : entries)
    std::fprintf(f, "\t%s: {%s, %d, %d},\n", go_quote(e.first).c_str(), go_quote(e.second.Replacement).c_str(),
                 e.second.CyclesSaved, e.second.BytesSaved);
  std::fprintf(f,
               "}\n\n"
               "// Lookup returns the replacement recorded for source, or nil.\n"
               "func Lookup(source string) *Rule {\n"
               "\tr, ok := %s[source]\n"
               "\tif !ok {\n\t\treturn nil\n\t}\n"
               "\treturn &r\n"
               "}\n\n"
               "// LoadRules reads a JSON array of {\"source\", \"replacement\", \"cycles_saved\",\n"
               "// \"bytes_saved\"} objects into a table; a later source replaces an earlier one.\n"
               "func LoadRules(path string) (map[string]Rule, error) {\n"
               "\traw, err := os.ReadFile(path)\n"
               "\tif err != nil {\n\t\treturn nil, err\n\t}\n"
               "\tvar in []struct {\n"
               "\t\tSource      string `json:\"source\"`\n"
               "\t\tReplacement string `json:\"replacement\"`\n"
               "\t\tCyclesSaved int    `json:\"cycles_saved\"`\n"
               "\t\tBytesSaved  int    `json:\"bytes_saved\"`\n"
               "\t}\n"
               "\tif err := json.Unmarshal(raw, &in); err != nil {\n\t\treturn nil, err\n\t}\n"
               "\tt := make(map[string]Rule, len(in))\n"
               "\tfor _, e := range in {\n"
               "\t\tt[e.Source] = Rule{Replacement: e.Replacement, CyclesSaved: e.CyclesSaved, BytesSaved: e.BytesSaved}\n"
               "\t}\n"
               "\treturn t, nil\n"
               "}\n",
               var_name.c_str());
}
}  // namespace peephole

namespace search {

result::Table Run(const Config& cfg, Stats* stats) {
  const int maxCand = cfg.MaxCandLen > 0 ? cfg.MaxCandLen : cfg.MaxTargetLen - 1;
  RunSpec r;
  r.maxTarget = cfg.MaxTargetLen;
  r.maxCand = maxCand;
  r.dead = cfg.DeadFlags;
  r.mode = Z80B_MODE_FIRST;
  r.sample = cfg.SampleTargets;
  r.seed = cfg.Seed;
  r.verbose = cfg.Verbose;
  r.first0 = cfg.FirstOpStart;
  r.first1 = cfg.FirstOpEnd;
  r.sink = cfg.Sink;
  r.targets = cfg.Targets;
  return run_lengths(r, stats);
}

static bool single(const Seq& target, int maxCandLen, FlagMask dead, result::Rule* out) {
  if (target.empty() || target.size() > 4) throw Error(Z80B_EINVAL, "target length must be 1..4");
  result::Table t;
  const auto w = pack(target);
  run_job(w, {uint8_t(target.size())}, uint32_t(target.size()), maxCandLen, dead, Z80B_MODE_FIRST, 0,
          [&](const result::Rule& x) { t.Add(x); }, nullptr);
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

uint8_t FlagDiff(const Seq& target, const Seq& cand) {
  if (target.empty() || target.size() > 4 || cand.empty() || cand.size() > 3)
    throw Error(Z80B_EINVAL, "FlagDiff: sequence lengths 1..4 (target), 1..3 (candidate)");
  uint32_t tw[4] = {0, 0, 0, 0}, cw[4] = {0, 0, 0, 0};
  for (size_t k = 0; k < target.size(); k++) tw[k] = target[k].packed();
  for (size_t k = 0; k < cand.size(); k++) cw[k] = cand[k].packed();
  const uint8_t tl = uint8_t(target.size()), cl = uint8_t(cand.size());
  uint8_t bits = 0, fd = 0;
  check(z80b_verify_pairs(context(), tw, &tl, cw, &cl, 4, 1, nullptr, 1u, &bits, &fd), "z80b_verify_pairs");
  return fd;
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

void EnumerateTargets(int len, int firstStart, int firstEnd, uint64_t sample, uint64_t seed, uint64_t batch,
                      const std::function<void(const std::vector<uint32_t>&, uint64_t)>& fn) {
  if (len < 1 || len > 3) throw Error(Z80B_EINVAL, "EnumerateTargets: lengths 1..3");
  if (batch == 0) throw Error(Z80B_EINVAL, "EnumerateTargets: batch must be positive");
  std::vector<uint32_t> pool(4531);
  pool.resize(z80b_pool8(pool.data(), uint32_t(pool.size())));
  const uint64_t P = pool.size();
  const uint64_t lo = uint64_t(std::max(0, firstStart));
  const uint64_t hi = firstEnd < 0 ? P : std::min<uint64_t>(P, uint64_t(firstEnd));
  if (lo >= hi) return;
  const uint64_t per_first = len == 1 ? 1 : (len == 2 ? P : P * P);
  const uint64_t L = uint64_t(len);
  auto seq_at = [&](uint64_t raw, uint32_t* w) {  // raw index within the range
    uint64_t rest = raw;
    for (int k = len - 1; k >= 1; k--) {
      w[k] = pool[rest % P];
      rest /= P;
    }
    w[0] = pool[lo + rest];
  };
  {
    const uint32_t one = pool[0];  // builds the library's tables before any threads
    (void)z80b_should_prune(&one, 1);
  }
  // the unpruned sequences of one first instruction, in order (length 3:
  // the second instruction's range split over threads)
  auto of_first = [&](uint64_t i0, std::vector<uint32_t>* out) {
    out->clear();
    const uint64_t nth =
        len == 3 ? std::max<uint64_t>(1, std::min<uint64_t>(32, std::thread::hardware_concurrency())) : 1;
    std::vector<std::vector<uint32_t>> part(nth);
    auto work = [&](uint64_t t) {
      const uint64_t a = per_first * t / nth, b = per_first * (t + 1) / nth;
      uint32_t w[3];
      for (uint64_t r = a; r < b; r++) {
        seq_at((i0 - lo) * per_first + r, w);
        if (z80b_should_prune(w, uint32_t(len)) == 0) part[t].insert(part[t].end(), w, w + len);
      }
    };
    if (nth == 1) {
      work(0);
    } else {
      std::vector<std::thread> th;
      for (uint64_t t = 0; t < nth; t++) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    for (auto& v : part) out->insert(out->end(), v.begin(), v.end());
  };
  std::vector<uint32_t> buf;
  uint64_t nbuf = 0;
  auto push = [&](const uint32_t* w, uint64_t n) {
    while (n) {
      const uint64_t take = std::min(n, batch - nbuf);
      buf.insert(buf.end(), w, w + take * L);
      nbuf += take;
      w += take * L;
      n -= take;
      if (nbuf == batch) {
        fn(buf, nbuf);
        buf.clear();
        nbuf = 0;
      }
    }
  };
  if (sample == 0 || len < 3) {
    // every unpruned sequence of the range (and, for a sample of length 1
    // or 2, Floyd's algorithm over their indices, kept in index order)
    std::vector<uint32_t> all, one;
    for (uint64_t i0 = lo; i0 < hi; i0++) {
      of_first(i0, &one);
      if (sample == 0) push(one.data(), one.size() / L);
      else all.insert(all.end(), one.begin(), one.end());
    }
    if (sample) {
      const uint64_t total = all.size() / L;
      if (sample >= total) {
        push(all.data(), total);
      } else {
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
        for (uint64_t t : pick) push(all.data() + t * L, 1);
      }
    }
  } else {
    // length 3, sampled: distinct raw indices of the range drawn uniformly
    // until `sample` unpruned ones are in hand (uniform over the unpruned
    // sequences), then delivered in index order
    const uint64_t raw = (hi - lo) * per_first;
    if (sample > raw / 2)
      throw Error(Z80B_EINVAL, "EnumerateTargets: a sample above half the range; enumerate the range whole");
    std::mt19937_64 rng(seed);
    std::unordered_set<uint64_t> seen;
    std::vector<uint64_t> pick;
    pick.reserve(sample);
    uint32_t w[3];
    while (pick.size() < sample && seen.size() < raw) {
      const uint64_t t = std::uniform_int_distribution<uint64_t>(0, raw - 1)(rng);
      if (!seen.insert(t).second) continue;
      seq_at(t, w);
      if (z80b_should_prune(w, 3) == 0) pick.push_back(t);
    }
    std::sort(pick.begin(), pick.end());
    for (uint64_t t : pick) {
      seq_at(t, w);
      push(w, 1);
    }
  }
  if (nbuf) fn(buf, nbuf);
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
  RunSpec r;
  r.maxTarget = cfg.MaxTargetLen;
  r.maxCand = 1;
  r.dead = cfg.DeadFlags;
  r.mode = Z80B_MODE_ALL;
  r.flags = cfg.NoExhaust ? Z80B_JOB_NO_EXHAUSTIVE : 0u;
  r.sample = cfg.SampleTargets;
  r.seed = cfg.Seed;
  r.verbose = cfg.Verbose;
  r.first0 = cfg.FirstOpStart;
  r.first1 = cfg.FirstOpEnd;
  r.sink = cfg.Sink;
  r.targets = cfg.Targets;
  return run_lengths(r, nullptr);
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
std::vector<Result> ReadJSON(const std::string& text) {
  const JVal top = JParser(text).parse();
  std::vector<Result> out;
  if (top.k == JVal::kNull) return out;
  if (top.k != JVal::kArr) throw Error(Z80B_EINVAL, "mulopt results: the top-level value is not an array");
  for (const JVal& e : top.arr) {
    if (e.k == JVal::kNull) continue;
    if (e.k != JVal::kObj) throw Error(Z80B_EINVAL, "mulopt results: an array element is not an object");
    Result r;
    r.Found = true;
    for (const auto& kv : e.obj) {
      if (key_is(kv.first, "k")) json_int_field(kv.second, &r.K, "k");
      else if (key_is(kv.first, "length")) json_int_field(kv.second, &r.Length, "length");
      else if (key_is(kv.first, "tstates")) json_int_field(kv.second, &r.TStates, "tstates");
      else if (key_is(kv.first, "ops")) {
        if (kv.second.k == JVal::kNull) continue;
        if (kv.second.k != JVal::kArr) throw Error(Z80B_EINVAL, "mulopt results: ops is not an array");
        for (const JVal& o : kv.second.arr) {
          std::string op;
          json_string_field(o, &op, "ops");
          r.Ops.push_back(op);
        }
      }
    }
    out.push_back(r);
  }
  return out;
}
}  // namespace mul

}  // namespace z80opt
