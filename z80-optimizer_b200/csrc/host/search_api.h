// search_api.h -- C++ host mirror of the reference's Go search API for the
// candidate-verification path, on top of libz80b200.so's C ABI.
//
//   search::Config, Run, SearchSingle, SearchSingleMasked   pkg/search/search.go:13-110
//   search::ExhaustiveCheck[Masked]                        pkg/search/verifier.go:159,642
//   search::ShouldPrune, EnumerateSequences8 order         pkg/search/pruner.go, enumerator.go
//   gpu::SearchConfig, SearchGPU                           pkg/gpu/search.go:13-199
//   result::Rule, Table, WriteJSON, DeadFlagDesc           pkg/result/table.go, output.go
//   result::JSONRule, ReadJSON, WriteGoCode                pkg/result/output.go:12-22,86-141
//   peephole::Rule, Lookup, LoadRules, WriteTable          pkg/peephole/rules.go
//   mul::FindAll (findOptimal for many K)                  cmd/mulopt/main.go:186-229
//
// Errors that the Go code returns as `error` are thrown as search::Error
// (status and the library's message).  Every call runs on one lazily created
// process-wide device context; there is no CPU fallback.
#pragma once
#include <cstdint>
#include <cstdio>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "z80b200.h"

namespace z80opt {

struct Instruction {
  uint16_t op = 0;
  uint16_t imm = 0;
  uint32_t packed() const { return uint32_t(op) | uint32_t(imm) << 16; }
  static Instruction unpack(uint32_t w) { return {uint16_t(w & 0xFFFF), uint16_t(w >> 16)}; }
};
using Seq = std::vector<Instruction>;

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
  int status;
};

namespace inst {
int SeqByteSize(const Seq& s);
int SeqTStates(const Seq& s);
std::string Disassemble(const Instruction& i);
std::string DisasmSeq(const Seq& s);  // " : "-joined (pkg/search/worker.go:273-282)
}  // namespace inst

namespace result {
struct Rule {
  Seq Source, Replacement;
  int BytesSaved = 0, CyclesSaved = 0;
  uint8_t DeadFlags = 0;
  uint8_t DeadRegs = 0;  // extension: dead-register mask (bit0..5 = B,C,D,E,H,L)
};
// result.Table (pkg/result/table.go:20-57): Rules() sorted by bytes saved,
// then cycles saved, both descending.
class Table {
 public:
  void Add(const Rule& r) { rules_.push_back(r); }
  size_t Len() const { return rules_.size(); }
  std::vector<Rule> Rules() const;

 private:
  std::vector<Rule> rules_;
};
std::string DeadFlagDesc(uint8_t mask);
void WriteJSON(std::FILE* f, const std::vector<Rule>& rules);

// The JSON form of a rule (output.go:12-22); DeadFlags is "%02X" or empty.
struct JSONRule {
  std::string SourceASM, ReplacementASM;
  int SourceBytes = 0, ReplacementBytes = 0, BytesSaved = 0, CyclesSaved = 0;
  std::string DeadFlags, DeadFlagDesc;
};
// ReadJSON (output.go:86-93): a JSON array of rule objects.  Keys match the
// struct tags case-insensitively and unknown keys are skipped, as
// encoding/json does; malformed input throws Error(Z80B_EINVAL).
std::vector<JSONRule> ReadJSON(std::FILE* f);
std::vector<JSONRule> ReadJSON(const std::string& text);
// Back from the JSON form: the assembly parsed into instructions and the
// dead-flag mask from its hex text (the reference has no such parse-back;
// throws Error(Z80B_EINVAL) on text that does not parse).
Rule FromJSON(const JSONRule& j);
// WriteGoCode (output.go:95-125): the rules as MinZ PeepholeRule entries.
void WriteGoCode(std::FILE* f, const std::vector<Rule>& rules);
}  // namespace result

// The generated peephole table package (pkg/peephole/rules.go): a map from
// the source assembly to its replacement.
namespace peephole {
struct Rule {
  std::string Replacement;
  int CyclesSaved = 0, BytesSaved = 0;
};
using Table = std::map<std::string, Rule>;
// Lookup (rules.go:522-527): the replacement of a source sequence, or null.
const Rule* Lookup(const Table& t, const std::string& source);
// LoadRules (rules.go:529-550): [{"source", "replacement", "cycles_saved",
// "bytes_saved"}]; a later entry for the same source replaces an earlier one.
Table LoadRules(const std::string& path);
// Writes the Go source of the table package, entries in the given order
// (the layout of rules.go: the Rule type, the table under `var_name`,
// Lookup and LoadRules); `from` names the rule file in the header line.
void WriteTable(std::FILE* f, const std::vector<std::pair<std::string, Rule>>& entries, const std::string& from,
                const std::string& var_name = "Top500");
}  // namespace peephole

namespace search {
using FlagMask = uint8_t;
constexpr FlagMask DeadNone = 0x00, DeadUndoc = 0x28, DeadAll = 0xFF;

// Receives each rule as soon as its batch of targets is done (Run and
// SearchGPU then return an empty table): the form for enumerations whose
// rule sets do not fit in memory.
using RuleSink = std::function<void(const result::Rule&)>;
// Receives every batch of targets before it is searched: `n` sequences of
// `len` packed words each (extension; records exactly which targets a
// sampled or sharded enumeration searched).
using TargetSink = std::function<void(const std::vector<uint32_t>& words, int len, uint64_t n)>;

struct Config {
  int MaxTargetLen = 2;  // targets of length 2..MaxTargetLen
  int MaxCandLen = 0;    // 0: MaxTargetLen - 1
  int NumWorkers = 0;    // accepted for compatibility; the device runs every target
  bool Verbose = false;
  FlagMask DeadFlags = DeadNone;
  // Extension: draw a seeded uniform sample of this many targets per length
  // (by enumeration index) instead of all of them; 0 = all.
  uint64_t SampleTargets = 0;
  uint64_t Seed = 0;
  // Extension (cuda/z80_search_v2.cu --first-op-start/--first-op-end): only
  // targets whose first instruction has an index in [FirstOpStart,
  // FirstOpEnd) of the 8-bit list; -1 = to the end.  Disjoint ranges shard
  // an enumeration over processes or GPUs.
  int FirstOpStart = 0, FirstOpEnd = -1;
  RuleSink Sink;  // extension, see RuleSink
  TargetSink Targets;  // extension, see TargetSink
};

struct Stats {  // accumulated over Run's jobs
  uint64_t targets = 0, checks = 0, checked = 0, rules = 0;
  double device_ms = 0;
};

result::Table Run(const Config& cfg, Stats* stats = nullptr);
bool SearchSingle(const Seq& target, int maxCandLen, bool verbose, result::Rule* out);
bool SearchSingleMasked(const Seq& target, int maxCandLen, FlagMask deadFlags, bool verbose, result::Rule* out);
bool ExhaustiveCheck(const Seq& target, const Seq& cand);
bool ExhaustiveCheckMasked(const Seq& target, const Seq& cand, FlagMask deadFlags);
// Batched form of the two above: verdict per pair (the verify-jsonl path).
std::vector<uint8_t> ExhaustiveCheckBatch(const std::vector<Seq>& targets, const std::vector<Seq>& cands,
                                          FlagMask deadFlags);
// FlagDiff (verifier.go:658-673), computed on the device: the flag bits in
// which target and candidate differ over the QuickCheck vectors (0 when a
// register differs).  With ExhaustiveCheck[Masked] it is what the STOKE
// search (pkg/stoke/search.go:108-117) asks of the verifier.
uint8_t FlagDiff(const Seq& target, const Seq& cand);
bool ShouldPrune(const Seq& s);
bool ParseAssembly(const std::string& text, Seq* out);      // cmd/z80opt/main.go:325-397
bool ParseDeadFlags(const std::string& text, FlagMask* out);  // cmd/z80opt/main.go:305-322

// The unpruned sequences of `len` instructions over the 8-bit list whose
// first instruction has an index in [firstStart, firstEnd) (-1: to the
// end), in EnumerateSequences8 order (pkg/search/enumerator.go:14-60), or a
// seeded uniform sample of `sample` of them (0: all; drawn by index among
// the unpruned ones, delivered in index order).  Delivered in batches of at
// most `batch` sequences: packed words, `len` per sequence.  Lengths 1..3;
// nothing is held beyond one batch and one first instruction's sequences,
// so length 3 (93 billion sequences) can be walked range by range.
void EnumerateTargets(int len, int firstStart, int firstEnd, uint64_t sample, uint64_t seed, uint64_t batch,
                      const std::function<void(const std::vector<uint32_t>& words, uint64_t n)>& fn);
}  // namespace search

namespace gpu {
struct SearchConfig {
  int MaxTargetLen = 2;
  bool Verbose = false;
  search::FlagMask DeadFlags = search::DeadNone;
  uint64_t SampleTargets = 0;  // extension, as in search::Config
  uint64_t Seed = 0;
  int FirstOpStart = 0, FirstOpEnd = -1;  // extension, as in search::Config
  // Extension (cuda/z80_search_v2.cu --no-exhaust): every MidCheck survivor
  // is reported, without the ExhaustiveCheck tier.
  bool NoExhaust = false;
  search::RuleSink Sink;  // extension, as in search::Config
  search::TargetSink Targets;  // extension, as in search::Config
};
result::Table SearchGPU(const SearchConfig& cfg);
}  // namespace gpu

namespace mul {
struct Result {
  int K = 0;
  bool Found = false;
  int Length = 0, TStates = 0;
  std::vector<std::string> Ops;
};
// findOptimal for every constant of ks (2..255) over `pool` (Z80B_MULPOOL_*).
std::vector<Result> FindAll(int pool, uint8_t b, uint8_t c, uint8_t f, int minLen, int maxLen,
                            const std::vector<int>& ks, z80b_mul_stats* stats = nullptr);
void WriteJSON(std::FILE* f, const std::vector<Result>& results);  // cmd/mulopt -json
// The -json output read back (cmd/mulopt/main.go:238-256, the -resume file):
// every entry found, keys as in MulResult; throws Error(Z80B_EINVAL) on
// malformed input.
std::vector<Result> ReadJSON(const std::string& text);
}  // namespace mul

// The process-wide device context (created on first use).
z80b_ctx* context();

}  // namespace z80opt
