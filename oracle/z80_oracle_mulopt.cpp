// Constant-multiply search model (oracle; test infrastructure only).
//
// Restates cmd/mulopt/main.go:186-229 (findOptimal: shortest length first,
// then minimum T-states, first sequence in odometer order wins ties) and
// main.go:142-160 (testSequence: quick reject on x = 1, 2, 3, then all 256 x)
// for four instruction pools:
//  * kMulPoolReference -- cmd/mulopt's own 14 ops with its MulState model
//    (main.go:25-127: A, B, carry and shadows A', B', carry', all zero but A);
//  * kMulPoolFast, kMulPoolCuda -- the 14 and 21 ops of the reference's CUDA
//    searchers (cuda/z80_mulopt_fast.cu, cuda/z80_mulopt.cu), same model;
//  * kMulPoolWide -- the 21-op pool of the constant-multiply workload, whose
//    instructions follow pkg/cpu.Exec, plus EX AF,AF' as the swap of
//    main.go:85-87; B, C, F start from the caller's values, A', F' at 0.
// The reference pools take B and the carry from the caller too (zero in the
// reference).
#include <cstring>
#include <vector>

#include "z80_oracle.h"
#include "z80_oracle_mulopt.h"

namespace orc {

// Pool order of the workload: ADD A,A; ADD A,B; SUB B; LD B,A; SLA A; SRL A;
// RLA; RRA; RLCA; RRCA; NEG; CPL; OR A; SCF; CCF; EX AF,AF'; LD C,A;
// ADD A,C; SUB C; LD A,B; LD A,C.  kExAF marks the shadow swap.
const uint16_t kMulPool[kMulPoolSize] = {ADD_A_A, ADD_A_B, SUB_B, LD_B_A, SLA_A, SRL_A, RLA,
                                         RRA,     RLCA,    RRCA,  NEG,    CPL,   OR_A,  SCF,
                                         CCF,     kExAF,   LD_C_A, ADD_A_C, SUB_C, LD_A_B, LD_A_C};
const char* const kMulNames[kMulPoolSize] = {
    "ADD A,A", "ADD A,B", "SUB B", "LD B,A", "SLA A",    "SRL A",  "RLA",
    "RRA",     "RLCA",    "RRCA",  "NEG",    "CPL",      "OR A",   "SCF",
    "CCF",     "EX AF,AF'", "LD C,A", "ADD A,C", "SUB C", "LD A,B", "LD A,C"};

// The reference's carry-only multiply model: cmd/mulopt/main.go:55-127
// (MulState + exec) and the exec_op of cuda/z80_mulopt.cu:51-146, which is
// the same model with more instructions.  RefOp names one instruction of it.
enum RefOp { R_ADD_AA, R_ADD_AB, R_SUB_B, R_LD_BA, R_SLA_A, R_SRL_A, R_EX_AF, R_EXX,
             R_ADC_AB, R_ADC_AA, R_SBC_AB, R_SBC_AA, R_OR_A, R_NEG, R_SRA_A, R_RLA,
             R_RRA, R_RLCA, R_RRCA, R_RLC_A, R_RRC_A, R_SCF };
struct RefPool {
  int n;
  RefOp op[21];
  int cost[21];
  const char* name[21];
};
// cmd/mulopt/main.go:25-49 (iota order, opCost, opNames).
static const RefPool kPoolGo = {
    14,
    {R_ADD_AA, R_ADD_AB, R_SUB_B, R_LD_BA, R_SLA_A, R_SRL_A, R_EX_AF, R_EXX, R_ADC_AB, R_ADC_AA, R_SBC_AB,
     R_SBC_AA, R_OR_A, R_NEG},
    {4, 4, 4, 4, 8, 8, 4, 4, 4, 4, 4, 4, 4, 8},
    {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "SLA A", "SRL A", "EX AF,AF'", "EXX", "ADC A,B", "ADC A,A",
     "SBC A,B", "SBC A,A", "OR A", "NEG"}};
// cuda/z80_mulopt_fast.cu:20-51 (the 14 generated ops and their costs).
static const RefPool kPoolFast = {
    14,
    {R_ADD_AA, R_ADD_AB, R_SUB_B, R_LD_BA, R_ADC_AB, R_ADC_AA, R_SBC_AB, R_SBC_AA, R_SRL_A, R_RLA, R_RRA,
     R_RLCA, R_RRCA, R_NEG},
    {4, 4, 4, 4, 4, 4, 4, 4, 8, 4, 4, 4, 4, 8},
    {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "ADC A,B", "ADC A,A", "SBC A,B", "SBC A,A", "SRL A", "RLA",
     "RRA", "RLCA", "RRCA", "NEG"}};
// cuda/z80_mulopt.cu:19-48 (21 ops and their costs).
static const RefPool kPoolCuda = {
    21,
    {R_ADD_AA, R_ADD_AB, R_SUB_B, R_LD_BA, R_ADC_AB, R_ADC_AA, R_SBC_AB, R_SBC_AA, R_SLA_A, R_SRA_A, R_SRL_A,
     R_RLA, R_RRA, R_RLCA, R_RRCA, R_RLC_A, R_RRC_A, R_OR_A, R_NEG, R_SCF, R_EX_AF},
    {4, 4, 4, 4, 4, 4, 4, 4, 8, 8, 8, 4, 4, 4, 4, 8, 8, 4, 8, 4, 4},
    {"ADD A,A", "ADD A,B", "SUB B", "LD B,A", "ADC A,B", "ADC A,A", "SBC A,B", "SBC A,A", "SLA A", "SRA A",
     "SRL A", "RLA", "RRA", "RLCA", "RRCA", "RLC A", "RRC A", "OR A", "NEG", "SCF", "EX AF,AF'"}};

static const RefPool* refPool(int pool) {
  switch (pool) {
    case kMulPoolReference: return &kPoolGo;
    case kMulPoolFast: return &kPoolFast;
    case kMulPoolCuda: return &kPoolCuda;
    default: return nullptr;
  }
}

int MulPoolSize(int pool) {
  const RefPool* p = refPool(pool);
  return p ? p->n : (pool == kMulPoolWide ? kMulPoolSize : 0);
}

const char* MulOpName(int pool, int i) {
  const RefPool* p = refPool(pool);
  return p ? p->name[i] : kMulNames[i];
}

int MulOpTStates(int i) {
  Init();
  return kMulPool[i] == kExAF ? 4 : TStates(kMulPool[i]);
}

int MulOpTStatesPool(int pool, int i) {
  const RefPool* p = refPool(pool);
  return p ? p->cost[i] : MulOpTStates(i);
}

struct MulState {
  State s;
  uint8_t a2, f2;  // A', F'
};

static inline void mulExec(MulState& m, int i) {
  uint16_t op = kMulPool[i];
  if (op == kExAF) {
    uint8_t a = m.s.A, f = m.s.F;
    m.s.A = m.a2;
    m.s.F = m.f2;
    m.a2 = a;
    m.f2 = f;
  } else {
    Exec(m.s, op, 0);
  }
}

// The MulState of cmd/mulopt/main.go:55-61 (the CUDA tools keep the same
// fields, cuda/z80_mulopt.cu:51-53): 8-bit arithmetic with the carry as the
// only flag.
struct RefState {
  uint8_t a, b, as, bs;
  bool c, cs;
};

static inline void refExec(RefState& s, int op) {
  unsigned r;
  switch (op) {
    case R_ADD_AA: r = 2u * s.a; s.c = r > 0xFF; s.a = uint8_t(r); break;
    case R_ADD_AB: r = unsigned(s.a) + s.b; s.c = r > 0xFF; s.a = uint8_t(r); break;
    case R_SUB_B: s.c = s.a < s.b; s.a = uint8_t(s.a - s.b); break;
    case R_LD_BA: s.b = s.a; break;
    case R_SLA_A: s.c = (s.a & 0x80) != 0; s.a = uint8_t(s.a << 1); break;
    case R_SRL_A: s.c = (s.a & 0x01) != 0; s.a = uint8_t(s.a >> 1); break;
    case R_EX_AF: { uint8_t t = s.a; s.a = s.as; s.as = t; bool u = s.c; s.c = s.cs; s.cs = u; } break;
    case R_EXX: { uint8_t t = s.b; s.b = s.bs; s.bs = t; } break;
    case R_ADC_AB: r = unsigned(s.a) + s.b + (s.c ? 1u : 0u); s.c = r > 0xFF; s.a = uint8_t(r); break;
    case R_ADC_AA: r = 2u * s.a + (s.c ? 1u : 0u); s.c = r > 0xFF; s.a = uint8_t(r); break;
    case R_SBC_AB: { int d = int(s.a) - int(s.b) - (s.c ? 1 : 0); s.c = d < 0; s.a = uint8_t(d); } break;
    case R_SBC_AA: { int d = -(s.c ? 1 : 0); s.c = d < 0; s.a = uint8_t(d); } break;
    case R_OR_A: s.c = false; break;
    case R_NEG: s.c = s.a != 0; s.a = uint8_t(0u - s.a); break;
    case R_SRA_A: s.c = (s.a & 0x01) != 0; s.a = uint8_t((s.a >> 1) | (s.a & 0x80)); break;
    case R_RLA: { bool o = s.c; s.c = (s.a & 0x80) != 0; s.a = uint8_t((s.a << 1) | (o ? 1 : 0)); } break;
    case R_RRA: { bool o = s.c; s.c = (s.a & 0x01) != 0; s.a = uint8_t((s.a >> 1) | (o ? 0x80 : 0)); } break;
    case R_RLCA:
    case R_RLC_A: s.c = (s.a & 0x80) != 0; s.a = uint8_t((s.a << 1) | (s.a >> 7)); break;
    case R_RRCA:
    case R_RRC_A: s.c = (s.a & 0x01) != 0; s.a = uint8_t((s.a >> 1) | (s.a << 7)); break;
    case R_SCF: s.c = true; break;
    default: break;
  }
}

uint8_t MulRun(const int* seq, int n, uint8_t x, const MulInit& init) {
  MulState m{};
  m.s.A = x;
  m.s.B = init.b;
  m.s.C = init.c;
  m.s.F = init.f;
  for (int i = 0; i < n; i++) mulExec(m, seq[i]);
  return m.s.A;
}

uint8_t MulRunPool(int pool, const int* seq, int n, uint8_t x, const MulInit& init) {
  const RefPool* p = refPool(pool);
  if (!p) return MulRun(seq, n, x, init);
  RefState s{};
  s.a = x;
  s.b = init.b;
  s.c = (init.f & 1) != 0;
  for (int i = 0; i < n; i++) refExec(s, p->op[seq[i]]);
  return s.a;
}

// main.go:142-160
bool MulTestPool(int pool, const int* seq, int n, uint8_t k, const MulInit& init) {
  if (MulRunPool(pool, seq, n, 1, init) != k) return false;
  if (MulRunPool(pool, seq, n, 2, init) != uint8_t(2 * k)) return false;
  if (MulRunPool(pool, seq, n, 3, init) != uint8_t(3 * k)) return false;
  for (int x = 0; x < 256; x++)
    if (MulRunPool(pool, seq, n, uint8_t(x), init) != uint8_t(x * k)) return false;
  return true;
}

bool MulTest(const int* seq, int n, uint8_t k, const MulInit& init) { return MulTestPool(kMulPoolWide, seq, n, k, init); }

// main.go:186-229
bool MulFindOptimalPool(int pool, uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out) {
  Init();
  const int nops = MulPoolSize(pool);
  for (int len = minLen; len <= maxLen; len++) {
    std::vector<int> seq(size_t(len), 0), best;
    int bestCost = 999999;
    while (true) {
      if (MulTestPool(pool, seq.data(), len, k, init)) {
        int c = 0;
        for (int i = 0; i < len; i++) c += MulOpTStatesPool(pool, seq[size_t(i)]);
        if (c < bestCost) {
          bestCost = c;
          best = seq;
        }
      }
      bool carry = true;
      for (int i = len - 1; i >= 0 && carry; i--) {
        if (++seq[size_t(i)] >= nops) seq[size_t(i)] = 0;
        else carry = false;
      }
      if (carry) break;
    }
    if (!best.empty()) {
      out->k = k;
      out->length = len;
      out->tstates = bestCost;
      out->ops = best;
      return true;
    }
  }
  return false;
}

bool MulFindOptimal(uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out) {
  return MulFindOptimalPool(kMulPoolWide, k, minLen, maxLen, init, out);
}

}  // namespace orc
