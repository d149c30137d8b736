// Constant-multiply search model (oracle; test infrastructure only).
//
// Restates cmd/mulopt/main.go:186-229 (findOptimal: shortest length first,
// then minimum T-states, first sequence in odometer order wins ties) and
// main.go:142-160 (testSequence: quick reject on x = 1, 2, 3, then all 256 x)
// over a 21-op pool whose instructions follow pkg/cpu.Exec semantics, plus
// EX AF,AF' as the swap of cmd/mulopt/main.go:85-87.  The pool and the seeded
// initial B, C, F come from the workload definition; shadow A', F' start at 0.
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

int MulOpTStates(int i) {
  Init();
  return kMulPool[i] == kExAF ? 4 : TStates(kMulPool[i]);
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

uint8_t MulRun(const int* seq, int n, uint8_t x, const MulInit& init) {
  MulState m{};
  m.s.A = x;
  m.s.B = init.b;
  m.s.C = init.c;
  m.s.F = init.f;
  for (int i = 0; i < n; i++) mulExec(m, seq[i]);
  return m.s.A;
}

// main.go:142-160
bool MulTest(const int* seq, int n, uint8_t k, const MulInit& init) {
  if (MulRun(seq, n, 1, init) != k) return false;
  if (MulRun(seq, n, 2, init) != uint8_t(2 * k)) return false;
  if (MulRun(seq, n, 3, init) != uint8_t(3 * k)) return false;
  for (int x = 0; x < 256; x++)
    if (MulRun(seq, n, uint8_t(x), init) != uint8_t(x * k)) return false;
  return true;
}

// main.go:186-229
bool MulFindOptimal(uint8_t k, int minLen, int maxLen, const MulInit& init, MulResult* out) {
  Init();
  for (int len = minLen; len <= maxLen; len++) {
    std::vector<int> seq(size_t(len), 0), best;
    int bestCost = 999999;
    while (true) {
      if (MulTest(seq.data(), len, k, init)) {
        int c = 0;
        for (int i = 0; i < len; i++) c += MulOpTStates(seq[size_t(i)]);
        if (c < bestCost) {
          bestCost = c;
          best = seq;
        }
      }
      bool carry = true;
      for (int i = len - 1; i >= 0 && carry; i--) {
        if (++seq[size_t(i)] >= kMulPoolSize) seq[size_t(i)] = 0;
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

}  // namespace orc
