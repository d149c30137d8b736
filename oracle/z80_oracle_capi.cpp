// C entry points of the oracle for the Python tests and the CPU-baseline leg
// of bench.py (test infrastructure only; the product never loads this).
// Instructions cross this boundary packed as uint32 op | imm << 16, the
// packing of the reference's GPU bridge (pkg/gpu/cuda.go:310).
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <thread>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "z80_oracle.h"
#include "z80_oracle_mulopt.h"

using namespace orc;

extern "C" {

struct orc_state {  // 12 bytes, C layout
  uint8_t A, F, B, C, D, E, H, L;
  uint16_t SP;
  uint8_t M, pad;
};
struct orc_rule {
  uint32_t src[4];
  uint32_t rep[4];
  int32_t src_len, rep_len, bytes_saved, cycles_saved, dead_flags, target_index, dead_regs;
};

static inline Instruction unpack(uint32_t w) { return {uint16_t(w & 0xFFFF), uint16_t(w >> 16)}; }
static inline uint32_t pack(Instruction i) { return uint32_t(i.op) | (uint32_t(i.imm) << 16); }
static std::vector<Instruction> seqOf(const uint32_t* s, int n) {
  std::vector<Instruction> v(size_t(n > 0 ? n : 0));
  for (int i = 0; i < n; i++) v[size_t(i)] = unpack(s[i]);
  return v;
}
static State toS(const orc_state& s) { return State{s.A, s.F, s.B, s.C, s.D, s.E, s.H, s.L, s.SP, s.M}; }
static orc_state fromS(const State& s) { return orc_state{s.A, s.F, s.B, s.C, s.D, s.E, s.H, s.L, s.SP, s.M, 0}; }
static int copyStr(const std::string& s, char* buf, int cap) {
  if (cap > 0) {
    size_t n = std::min(size_t(cap - 1), s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return int(s.size());
}

int orc_op_count() { return OpCodeCount; }
int orc_init() { Init(); return 0; }

int orc_catalog(int op, char* mnem, int cap, uint8_t* enc, int* nenc, int* tstates, int* bytesize) {
  Init();
  if (op < 0 || op >= OpCodeCount) return -1;
  const Info& in = Catalog[op];
  copyStr(in.mnemonic, mnem, cap);
  for (int i = 0; i < in.nbytes; i++) enc[i] = in.bytes[i];
  *nenc = in.nbytes;
  *tstates = in.tstates;
  *bytesize = ByteSize(uint16_t(op));
  return 0;
}
int orc_op_name(int op, char* buf, int cap) { return copyStr(OpName(uint16_t(op)), buf, cap); }
int orc_has_imm(int op) { return HasImmediate(uint16_t(op)); }
int orc_has_imm16(int op) { return HasImm16(uint16_t(op)); }
int orc_op_reads(int op) { return OpReads(uint16_t(op)); }
int orc_op_writes(int op) { return OpWrites(uint16_t(op)); }

int orc_disasm_seq(const uint32_t* seq, int n, char* buf, int cap) {
  Init();
  return copyStr(DisasmSeq(seqOf(seq, n)), buf, cap);
}

int orc_exec(orc_state* st, int op, int imm) {
  Init();
  State s = toS(*st);
  int t = Exec(s, uint16_t(op), uint16_t(imm));
  *st = fromS(s);
  return t;
}
void orc_exec_seq(const orc_state* in, const uint32_t* seq, int n, orc_state* out) {
  Init();
  auto v = seqOf(seq, n);
  *out = fromS(ExecSeq(toS(*in), v.data(), n));
}

int orc_quickcheck(const uint32_t* t, int tn, const uint32_t* c, int cn, int dead) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return QuickCheckMasked(tv.data(), tn, cv.data(), cn, FlagMask(dead));
}
int orc_midcheck(const uint32_t* t, int tn, const uint32_t* c, int cn, int dead) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return MidCheckMasked(tv.data(), tn, cv.data(), cn, FlagMask(dead));
}
int orc_exhaustive(const uint32_t* t, int tn, const uint32_t* c, int cn, int dead) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return ExhaustiveCheckMasked(tv.data(), tn, cv.data(), cn, FlagMask(dead));
}
int orc_exhaustive_regs(const uint32_t* t, int tn, const uint32_t* c, int cn, int dead, int dregs) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return ExhaustiveCheckMaskedRegs(tv.data(), tn, cv.data(), cn, FlagMask(dead), uint8_t(dregs));
}
unsigned long long orc_exhaustive_states(const uint32_t* t, int tn, const uint32_t* c, int cn) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return ExhaustiveStates(tv.data(), tn, cv.data(), cn);
}
int orc_flagdiff(const uint32_t* t, int tn, const uint32_t* c, int cn) {
  Init();
  auto tv = seqOf(t, tn), cv = seqOf(c, cn);
  return FlagDiff(tv.data(), tn, cv.data(), cn);
}
void orc_fingerprint(const uint32_t* seq, int n, uint8_t* out80) {
  Init();
  auto v = seqOf(seq, n);
  Fingerprint(v.data(), n, out80);
}
int orc_should_prune(const uint32_t* seq, int n) {
  Init();
  auto v = seqOf(seq, n);
  return ShouldPrune(v.data(), n);
}
// EnumerateSequences8's order (pkg/search/enumerator.go:319-345: an odometer
// with position 0 most significant) over an arbitrary instruction pool,
// keeping the sequences ShouldPrune (pruner.go:7-27) lets through.  Writes up
// to cap sequences of n words to out and returns how many exist.
long long orc_enumerate_pool(const uint32_t* pool, int npool, int n, uint32_t* out, long long cap) {
  Init();
  if (n < 1 || n > 4 || npool < 1) return 0;
  std::vector<Instruction> P(static_cast<size_t>(npool));
  for (int i = 0; i < npool; i++) P[size_t(i)] = unpack(pool[i]);
  std::vector<int> idx(size_t(n), 0);
  std::vector<Instruction> seq(size_t(n), P[0]);
  long long k = 0;
  while (true) {
    if (!ShouldPrune(seq.data(), n)) {
      if (k < cap)
        for (int j = 0; j < n; j++) out[size_t(k) * size_t(n) + size_t(j)] = pack(seq[size_t(j)]);
      k++;
    }
    int p = n - 1;
    while (p >= 0) {
      if (++idx[size_t(p)] < npool) {
        seq[size_t(p)] = P[size_t(idx[size_t(p)])];
        break;
      }
      idx[size_t(p)] = 0;
      seq[size_t(p)] = P[0];
      p--;
    }
    if (p < 0) break;
  }
  return k;
}

int orc_instructions8(uint32_t* out, int cap) {
  const auto& p = Instructions8();
  for (int i = 0; i < int(p.size()) && i < cap; i++) out[i] = pack(p[size_t(i)]);
  return int(p.size());
}
// Indices (enumeration order) of the 8-bit instructions passing
// QuickCheckMasked against a target; writes up to cap, returns the count.
int orc_qc_survivors(const uint32_t* t, int tn, int dead, uint32_t* out, int cap) {
  Init();
  auto tv = seqOf(t, tn);
  const auto& pool = Instructions8();
  int k = 0;
  for (size_t i = 0; i < pool.size(); i++) {
    if (QuickCheckMasked(tv.data(), tn, &pool[i], 1, FlagMask(dead))) {
      if (k < cap) out[k] = uint32_t(i);
      k++;
    }
  }
  return k;
}

void orc_test_vectors(orc_state* qc8, orc_state* mid32) {
  for (int i = 0; i < 8; i++) qc8[i] = fromS(TestVectors[i]);
  for (int i = 0; i < 32; i++) mid32[i] = fromS(MidCheckVectors[i]);
}

static void toRule(const Rule& r, int ti, orc_rule* o) {
  std::memset(o, 0, sizeof *o);
  o->src_len = int(r.Source.size());
  o->rep_len = int(r.Replacement.size());
  for (size_t i = 0; i < r.Source.size() && i < 4; i++) o->src[i] = pack(r.Source[i]);
  for (size_t i = 0; i < r.Replacement.size() && i < 4; i++) o->rep[i] = pack(r.Replacement[i]);
  o->bytes_saved = r.BytesSaved;
  o->cycles_saved = r.CyclesSaved;
  o->dead_flags = r.DeadFlags;
  o->target_index = ti;
  o->dead_regs = r.DeadRegs;
}

// Targets: n sequences, stride 4 words, lengths in lens[].  Rules come out
// grouped by target index (deterministic order).  Returns the rule count or
// -1 if cap is too small.
long long orc_search_timed(const uint32_t* seqs, const int* lens, int n, int maxCandLen, int dead, int workers,
                           orc_rule* out, long long cap, unsigned long long* checked, double* secs,
                           double target_budget);
long long orc_search(const uint32_t* seqs, const int* lens, int n, int maxCandLen, int dead,
                     int workers, orc_rule* out, long long cap, unsigned long long* checked) {
  return orc_search_timed(seqs, lens, n, maxCandLen, dead, workers, out, cap, checked, nullptr, 0);
}

// orc_search that also reports, per target, the CPU time of its worker
// thread spent on that target (secs[i], seconds; secs may be NULL).  The sum
// over targets divided by the worker count is the wall time of a perfectly
// balanced pool, which a large target set approaches; a small sample's wall
// time is instead set by its slowest target.  With target_budget > 0 a
// target whose ExhaustiveCheck sweeps run past that many CPU seconds is
// abandoned: secs[i] = -1 and none of its rules or its `checked` count are
// reported (a bounded CPU sample; the tail it leaves out is counted by the
// caller from the -1 entries).
long long orc_search_timed(const uint32_t* seqs, const int* lens, int n, int maxCandLen, int dead, int workers,
                           orc_rule* out, long long cap, unsigned long long* checked, double* secs,
                           double target_budget) {
  Init();
  std::vector<std::vector<Instruction>> tg(size_t(n > 0 ? n : 0));
  for (int i = 0; i < n; i++) tg[size_t(i)] = seqOf(seqs + size_t(i) * 4, lens[i]);
  // Run per target so rules can be tagged with their target index.
  std::vector<std::vector<Rule>> per(tg.size());
  std::vector<SearchStats> st(tg.size());
  if (workers <= 0) workers = 1;
  std::vector<std::thread> th;
  std::atomic<size_t> next{0};
  for (int w = 0; w < workers; w++)
    th.emplace_back([&] {
      size_t i;
      while ((i = next.fetch_add(1)) < tg.size()) {
        timespec a{}, b{};
        if (secs) clock_gettime(CLOCK_THREAD_CPUTIME_ID, &a);
        if (target_budget > 0) SetSweepBudget(target_budget);
        ProcessTask(tg[i].data(), int(tg[i].size()), maxCandLen, FlagMask(dead), per[i], &st[i]);
        const bool abandoned = target_budget > 0 && SweepBudgetSpent();
        SetSweepBudget(0);
        if (abandoned) {
          per[i].clear();
          st[i] = SearchStats{};
        }
        if (secs) {
          clock_gettime(CLOCK_THREAD_CPUTIME_ID, &b);
          secs[i] = abandoned ? -1.0 : double(b.tv_sec - a.tv_sec) + 1e-9 * double(b.tv_nsec - a.tv_nsec);
        }
      }
    });
  for (auto& t : th) t.join();
  long long k = 0;
  unsigned long long ch = 0;
  for (size_t i = 0; i < per.size(); i++) {
    ch += st[i].checked;
    for (auto& r : per[i]) {
      if (k >= cap) return -1;
      toRule(r, int(i), &out[k++]);
    }
  }
  if (checked) *checked = ch;
  return k;
}

// orc_search with per-target dead flags and dead registers (extension);
// dead / dregs may be NULL (0 for every target).
long long orc_search_ext(const uint32_t* seqs, const int* lens, int n, int maxCandLen, const uint8_t* dead,
                         const uint8_t* dregs, int workers, orc_rule* out, long long cap, unsigned long long* checked) {
  Init();
  std::vector<std::vector<Instruction>> tg(size_t(n > 0 ? n : 0));
  for (int i = 0; i < n; i++) tg[size_t(i)] = seqOf(seqs + size_t(i) * 4, lens[i]);
  std::vector<std::vector<Rule>> per(tg.size());
  std::vector<SearchStats> st(tg.size());
  if (workers <= 0) workers = 1;
  std::vector<std::thread> th;
  std::atomic<size_t> next{0};
  for (int w = 0; w < workers; w++)
    th.emplace_back([&] {
      size_t i;
      while ((i = next.fetch_add(1)) < tg.size())
        ProcessTaskExt(tg[i].data(), int(tg[i].size()), maxCandLen, FlagMask(dead ? dead[i] : 0),
                       uint8_t(dregs ? dregs[i] : 0), per[i], &st[i]);
    });
  for (auto& t : th) t.join();
  long long k = 0;
  unsigned long long ch = 0;
  for (size_t i = 0; i < per.size(); i++) {
    ch += st[i].checked;
    for (auto& r : per[i]) {
      if (k >= cap) return -1;
      toRule(r, int(i), &out[k++]);
    }
  }
  if (checked) *checked = ch;
  return k;
}

long long orc_search_gpu(const uint32_t* seqs, const int* lens, int n, const uint32_t* cands,
                         int ncand, int dead, orc_rule* out, long long cap) {
  Init();
  auto cv = seqOf(cands, ncand);
  long long k = 0;
  for (int i = 0; i < n; i++) {
    auto t = seqOf(seqs + size_t(i) * 4, lens[i]);
    std::vector<Rule> rules;
    SearchGPUTarget(t.data(), lens[i], cv, FlagMask(dead), rules);
    for (auto& r : rules) {
      if (k >= cap) return -1;
      toRule(r, i, &out[k++]);
    }
  }
  return k;
}

int orc_write_json(const orc_rule* rules, int n, char* buf, int cap) {
  Init();
  std::vector<Rule> v(size_t(n > 0 ? n : 0));
  for (int i = 0; i < n; i++) {
    v[size_t(i)].Source = seqOf(rules[i].src, rules[i].src_len);
    v[size_t(i)].Replacement = seqOf(rules[i].rep, rules[i].rep_len);
    v[size_t(i)].BytesSaved = rules[i].bytes_saved;
    v[size_t(i)].CyclesSaved = rules[i].cycles_saved;
    v[size_t(i)].DeadFlags = uint8_t(rules[i].dead_flags);
  }
  return copyStr(WriteJSON(v), buf, cap);
}
int orc_dead_flag_desc(int mask, char* buf, int cap) { return copyStr(DeadFlagDesc(uint8_t(mask)), buf, cap); }
int orc_parse_dead_flags(const char* s, int* out) {
  FlagMask m;
  if (!ParseDeadFlags(s, &m)) return 0;
  *out = m;
  return 1;
}
int orc_parse_assembly(const char* text, uint32_t* out, int cap) {
  std::vector<Instruction> v;
  if (!ParseAssembly(text, &v)) return -1;
  for (size_t i = 0; i < v.size() && int(i) < cap; i++) out[i] = pack(v[i]);
  return int(v.size());
}

int orc_mul_find(int k, int minLen, int maxLen, int b, int c, int f, int* len, int* tstates, int* ops) {
  MulResult r;
  if (!MulFindOptimal(uint8_t(k), minLen, maxLen, MulInit{uint8_t(b), uint8_t(c), uint8_t(f)}, &r)) return 0;
  *len = r.length;
  *tstates = r.tstates;
  for (int i = 0; i < r.length; i++) ops[i] = r.ops[size_t(i)];
  return 1;
}
int orc_mul_run(const int* seq, int n, int x, int b, int c, int f) {
  return MulRun(seq, n, uint8_t(x), MulInit{uint8_t(b), uint8_t(c), uint8_t(f)});
}
int orc_mul_tstates(int i) { return MulOpTStates(i); }

// Pool-generic forms (pool ids of z80_oracle_mulopt.h).
int orc_mul_pool_size(int pool) { return MulPoolSize(pool); }
int orc_mul_find_pool(int pool, int k, int minLen, int maxLen, int b, int c, int f, int* len, int* tstates,
                      int* ops) {
  MulResult r;
  if (!MulFindOptimalPool(pool, uint8_t(k), minLen, maxLen, MulInit{uint8_t(b), uint8_t(c), uint8_t(f)}, &r))
    return 0;
  *len = r.length;
  *tstates = r.tstates;
  for (int i = 0; i < r.length; i++) ops[i] = r.ops[size_t(i)];
  return 1;
}
int orc_mul_run_pool(int pool, const int* seq, int n, int x, int b, int c, int f) {
  return MulRunPool(pool, seq, n, uint8_t(x), MulInit{uint8_t(b), uint8_t(c), uint8_t(f)});
}
int orc_mul_tstates_pool(int pool, int i) { return MulOpTStatesPool(pool, i); }
const char* orc_mul_op_name(int pool, int i) { return MulOpName(pool, i); }

}  // extern "C"
