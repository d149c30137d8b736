// Verification / pruning / enumeration / worker restatement (oracle; test
// infrastructure only).  Follows pkg/search/verifier.go, pruner.go,
// enumerator.go, worker.go, pkg/gpu/search.go and pkg/result/output.go.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <thread>

#include "z80_oracle.h"

namespace orc {

// verifier.go:19-28
const State TestVectors[8] = {
    {0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x0000, 0x42},
    {0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFFFF, 0xBD},
    {0x01, 0x00, 0x02, 0x03, 0x04, 0x05, 0x06, 0x07, 0x1234, 0x13},
    {0x80, 0x01, 0x40, 0x20, 0x10, 0x08, 0x04, 0x02, 0x8000, 0x7E},
    {0x55, 0x00, 0xAA, 0x55, 0xAA, 0x55, 0xAA, 0x55, 0x5555, 0xA5},
    {0xAA, 0x01, 0x55, 0xAA, 0x55, 0xAA, 0x55, 0xAA, 0xAAAA, 0x5A},
    {0x0F, 0x00, 0xF0, 0x0F, 0xF0, 0x0F, 0xF0, 0x0F, 0xFFFE, 0xE1},
    {0x7F, 0x01, 0x80, 0x7F, 0x80, 0x7F, 0x80, 0x7F, 0x7FFF, 0x33},
};

// verifier.go:35-72 (first 8 equal TestVectors)
const State MidCheckVectors[32] = {
    {0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0x0000, 0x42},
    {0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFFFF, 0xBD},
    {0x01, 0x00, 0x02, 0x03, 0x04, 0x05, 0x06, 0x07, 0x1234, 0x13},
    {0x80, 0x01, 0x40, 0x20, 0x10, 0x08, 0x04, 0x02, 0x8000, 0x7E},
    {0x55, 0x00, 0xAA, 0x55, 0xAA, 0x55, 0xAA, 0x55, 0x5555, 0xA5},
    {0xAA, 0x01, 0x55, 0xAA, 0x55, 0xAA, 0x55, 0xAA, 0xAAAA, 0x5A},
    {0x0F, 0x00, 0xF0, 0x0F, 0xF0, 0x0F, 0xF0, 0x0F, 0xFFFE, 0xE1},
    {0x7F, 0x01, 0x80, 0x7F, 0x80, 0x7F, 0x80, 0x7F, 0x7FFF, 0x33},
    {0x02, 0x00, 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x0102, 0x91},
    {0x04, 0x01, 0x08, 0x10, 0x20, 0x40, 0x80, 0x01, 0x0408, 0x48},
    {0x08, 0x00, 0x10, 0x20, 0x40, 0x80, 0x01, 0x02, 0x1020, 0x24},
    {0x10, 0x01, 0x20, 0x40, 0x80, 0x01, 0x02, 0x04, 0x4080, 0xD7},
    {0x20, 0x00, 0x40, 0x80, 0x01, 0x02, 0x04, 0x08, 0x0201, 0x6B},
    {0x40, 0x01, 0x80, 0x01, 0x02, 0x04, 0x08, 0x10, 0x8040, 0xB2},
    {0x03, 0x00, 0x05, 0x09, 0x11, 0x21, 0x41, 0x81, 0x0309, 0x0F},
    {0x05, 0x01, 0x0A, 0x14, 0x28, 0x50, 0xA0, 0x41, 0x0A14, 0xF0},
    {0x11, 0x00, 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x0100, 0xC3},
    {0x22, 0x01, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x0200, 0x3C},
    {0x44, 0x00, 0x10, 0x20, 0x40, 0x80, 0x01, 0x02, 0x0400, 0x87},
    {0x88, 0x01, 0x40, 0x80, 0x01, 0x02, 0x04, 0x08, 0x0800, 0x69},
    {0x33, 0x00, 0x03, 0x0C, 0x30, 0xC0, 0x05, 0x0A, 0x3300, 0xAE},
    {0xCC, 0x01, 0x30, 0xC0, 0x03, 0x0C, 0x50, 0xA0, 0xCC00, 0x51},
    {0x66, 0x00, 0x06, 0x60, 0x09, 0x90, 0x0C, 0xC0, 0x6600, 0xDA},
    {0x99, 0x01, 0x09, 0x90, 0x06, 0x60, 0xA0, 0x0A, 0x9900, 0x25},
    {0xFE, 0x00, 0x7F, 0x80, 0x01, 0xFE, 0x55, 0xAA, 0x0001, 0x01},
    {0x81, 0x01, 0xFE, 0x01, 0x80, 0x7F, 0xAA, 0x55, 0x8001, 0xFE},
    {0x7E, 0x00, 0x81, 0x42, 0x24, 0x18, 0xE7, 0xDB, 0x7FFE, 0x80},
    {0xBF, 0x01, 0x40, 0xBF, 0x40, 0xBF, 0x40, 0xBF, 0xBF00, 0x40},
    {0xC0, 0x00, 0x3F, 0xC0, 0x3F, 0xC0, 0x3F, 0xC0, 0xC000, 0x1F},
    {0xE0, 0x01, 0x1F, 0xE0, 0x1F, 0xE0, 0x1F, 0xE0, 0xE000, 0xEF},
    {0xF0, 0x00, 0x0F, 0xF0, 0x0F, 0xF0, 0x0F, 0xF0, 0xF000, 0x55},
    {0x0E, 0x01, 0xE0, 0x0E, 0xE0, 0x0E, 0xE0, 0x0E, 0x0E0E, 0xAA},
};

// verifier.go:75-81
State ExecSeq(State s, const Instruction* seq, int n) {
  for (int i = 0; i < n; i++) Exec(s, seq[i].op, seq[i].imm);
  return s;
}

// verifier.go:615-623
bool StatesEqualMasked(const State& a, const State& b, FlagMask dead) {
  uint8_t keep = uint8_t(~dead);
  return a.A == b.A && (a.F & keep) == (b.F & keep) && a.B == b.B && a.C == b.C &&
         a.D == b.D && a.E == b.E && a.H == b.H && a.L == b.L && a.SP == b.SP && a.M == b.M;
}

bool StatesEqualMaskedRegs(const State& a, const State& b, FlagMask dead, uint8_t deadRegs) {
  const uint8_t keep = uint8_t(~dead);
  auto eq = [&](int bit, uint8_t x, uint8_t y) { return ((deadRegs >> bit) & 1) || x == y; };
  return a.A == b.A && (a.F & keep) == (b.F & keep) && eq(0, a.B, b.B) && eq(1, a.C, b.C) &&
         eq(2, a.D, b.D) && eq(3, a.E, b.E) && eq(4, a.H, b.H) && eq(5, a.L, b.L) && a.SP == b.SP && a.M == b.M;
}

bool QuickCheckMaskedRegs(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead,
                          uint8_t deadRegs) {
  for (const State& v : TestVectors)
    if (!StatesEqualMaskedRegs(ExecSeq(v, t, tn), ExecSeq(v, c, cn), dead, deadRegs)) return false;
  return true;
}

// verifier.go:85-94
bool QuickCheck(const Instruction* t, int tn, const Instruction* c, int cn) {
  for (const State& v : TestVectors)
    if (ExecSeq(v, t, tn) != ExecSeq(v, c, cn)) return false;
  return true;
}
// verifier.go:98-107
bool MidCheck(const Instruction* t, int tn, const Instruction* c, int cn) {
  for (const State& v : MidCheckVectors)
    if (ExecSeq(v, t, tn) != ExecSeq(v, c, cn)) return false;
  return true;
}
// verifier.go:111-123
bool MidCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead) {
  if (dead == DeadNone) return MidCheck(t, tn, c, cn);
  for (const State& v : MidCheckVectors)
    if (!StatesEqualMasked(ExecSeq(v, t, tn), ExecSeq(v, c, cn), dead)) return false;
  return true;
}
// verifier.go:626-638
bool QuickCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead) {
  if (dead == DeadNone) return QuickCheck(t, tn, c, cn);
  for (const State& v : TestVectors)
    if (!StatesEqualMasked(ExecSeq(v, t, tn), ExecSeq(v, c, cn), dead)) return false;
  return true;
}

// verifier.go:134-151
void Fingerprint(const Instruction* seq, int n, uint8_t out[80]) {
  for (int i = 0; i < 8; i++) {
    State o = ExecSeq(TestVectors[i], seq, n);
    uint8_t* p = out + i * 10;
    p[0] = o.A; p[1] = o.F; p[2] = o.B; p[3] = o.C; p[4] = o.D;
    p[5] = o.E; p[6] = o.H; p[7] = o.L; p[8] = uint8_t(o.SP >> 8); p[9] = uint8_t(o.SP);
  }
}

// verifier.go:658-673
FlagMask FlagDiff(const Instruction* t, int tn, const Instruction* c, int cn) {
  FlagMask diff = 0;
  for (const State& v : TestVectors) {
    State a = ExecSeq(v, t, tn), b = ExecSeq(v, c, cn);
    if (a.A != b.A || a.B != b.B || a.C != b.C || a.D != b.D || a.E != b.E || a.H != b.H ||
        a.L != b.L || a.SP != b.SP || a.M != b.M)
      return 0;
    diff |= uint8_t(a.F ^ b.F);
  }
  return diff;
}

// ------------------------------------------------------- read/write masks
// verifier.go:199-408.  Family restatement of the reference switch, including
// its omissions (e.g. ADD A,r reads only r; ADD A,n and the other
// immediate ALU forms except ADC/SBC read nothing; DAA reads only A).
static const uint16_t kR7Mask[7] = {regA, regB, regC, regD, regE, regH, regL};
static const int kAluSrcIdx[7] = {1, 2, 3, 4, 5, 6, 0};  // B,C,D,E,H,L,A
static const uint16_t kPairMask[4] = {regB | regC, regD | regE, regH | regL, regSP};

uint16_t OpReads(uint16_t op) {
  if (op < LD_A_N) {
    int d = op / 7, k = op % 7;
    return kR7Mask[d == 0 ? kAluSrcIdx[k] : k];
  }
  if (op <= LD_L_N) return 0;
  if (op < INC_A) {
    int a = (op - ADD_A_B) / 8, k = (op - ADD_A_B) % 8;
    bool carryIn = (a == 1 || a == 3);  // ADC, SBC
    if (k == 7) return carryIn ? uint16_t(regA | regF) : uint16_t(0);
    uint16_t m = kR7Mask[kAluSrcIdx[k]];
    return carryIn ? uint16_t(m | regF) : m;
  }
  if (op < RLCA) return kR7Mask[(op - INC_A) % 7];  // INC/DEC r
  switch (op) {
    case RLCA: case RRCA: case DAA: case CPL: case NEG: return regA;
    case RLA: case RRA: return regA | regF;
    case SCF: case CCF: return regF;
    case NOP: return 0;
  }
  if (op < SLL_A) {
    int k = (op - RLC_A) / 7, r = (op - RLC_A) % 7;
    bool carryIn = (k == 2 || k == 3);  // RL, RR
    return carryIn ? uint16_t(kR7Mask[r] | regF) : kR7Mask[r];
  }
  if (op <= SLL_L) return kR7Mask[op - SLL_A];
  if (op < INC_BC) return kR7Mask[(op - BIT_0_A) % 7];  // BIT/RES/SET n,r
  if (op < INC_BC + 4) return kPairMask[op - INC_BC];
  if (op < ADD_HL_BC) return kPairMask[op - DEC_BC];
  if (op < EX_DE_HL) return uint16_t(regH | regL | kPairMask[op - ADD_HL_BC]);
  if (op == EX_DE_HL) return regD | regE | regH | regL;
  if (op == LD_SP_HL) return regH | regL;
  if (op < ADC_HL_BC) return 0;  // LD rr,nn
  if (op < LD_A_HLI) {
    int p = (op - ADC_HL_BC) % 4;
    return uint16_t(regH | regL | kPairMask[p] | regF);
  }
  if (op < LD_HLI_A) return regM;
  if (op < LD_HLI_N) return kR7Mask[op - LD_HLI_A];
  if (op == LD_HLI_N) return 0;
  if (op == LD_A_BCI || op == LD_A_DEI) return regM;
  if (op == LD_BCI_A || op == LD_DEI_A) return regA;
  if (op < INC_HLI) {
    int a = op - ADD_A_HLI;
    return (a == 1 || a == 3) ? uint16_t(regA | regM | regF) : uint16_t(regA | regM);
  }
  if (op == INC_HLI || op == DEC_HLI) return regM;
  if (op < BIT_0_HLI) {
    int k = op - RLC_HLI;
    return (k == 2 || k == 3) ? uint16_t(regM | regF) : uint16_t(regM);
  }
  if (op < OpCodeCount) return regM;  // BIT/RES/SET n,(HL)
  return 0;
}

// pruner.go:66-236.  Memory ops (>= LD_A_HLI) report no writes, as in the
// reference's default case.
uint16_t OpWrites(uint16_t op) {
  if (op < LD_A_N) return kR7Mask[op / 7];
  if (op <= LD_L_N) return kR7Mask[op - LD_A_N];
  if (op < INC_A) {
    int a = (op - ADD_A_B) / 8;
    return a == 7 ? uint16_t(regF) : uint16_t(regA | regF);  // CP writes only F
  }
  if (op < RLCA) return uint16_t(kR7Mask[(op - INC_A) % 7] | regF);
  switch (op) {
    case RLCA: case RRCA: case RLA: case RRA: case DAA: case CPL: case NEG:
      return regA | regF;
    case SCF: case CCF: return regF;
    case NOP: return 0;
  }
  if (op < SLL_A) return uint16_t(kR7Mask[(op - RLC_A) % 7] | regF);
  if (op <= SLL_L) return uint16_t(kR7Mask[op - SLL_A] | regF);
  if (op < RES_0_A) return regF;                        // BIT n,r
  if (op < INC_BC) return kR7Mask[(op - RES_0_A) % 7];  // RES/SET n,r
  if (op < INC_BC + 4) return kPairMask[op - INC_BC];
  if (op < ADD_HL_BC) return kPairMask[op - DEC_BC];
  if (op < EX_DE_HL) return regH | regL | regF;
  if (op == EX_DE_HL) return regD | regE | regH | regL;
  if (op == LD_SP_HL) return regSP;
  if (op < ADC_HL_BC) return kPairMask[op - LD_BC_NN];
  if (op < LD_A_HLI) return regH | regL | regF;
  return 0;
}

uint16_t RegsRead(const Instruction* seq, int n) {
  uint16_t m = 0;
  for (int i = 0; i < n; i++) m |= OpReads(seq[i].op);
  return m;
}

// ------------------------------------------------------------ exhaustive
// verifier.go:159-612,642-853.  One implementation parameterised by the dead
// mask; with dead == 0 StatesEqualMasked equals full-state equality.
static const uint8_t kRepValues[32] = {
    0x00, 0x01, 0x02, 0x0F, 0x10, 0x1F, 0x20, 0x3F, 0x40, 0x55, 0x7E,
    0x7F, 0x80, 0x81, 0xAA, 0xBF, 0xC0, 0xD5, 0xE0, 0xEF, 0xF0, 0xF7,
    0xFE, 0xFF, 0x03, 0x07, 0x11, 0x33, 0x77, 0xBB, 0xDD, 0xEE};
static const uint16_t kRepSP[16] = {0x0000, 0x0001, 0x00FF, 0x0100, 0x7FFE, 0x7FFF,
                                    0x8000, 0x8001, 0xFFFE, 0xFFFF, 0x1234, 0x5678,
                                    0xABCD, 0xDEAD, 0xBEEF, 0xCAFE};

static void setReg(State& s, int off, uint8_t v) {
  switch (off) {
    case 2: s.B = v; break;
    case 3: s.C = v; break;
    case 4: s.D = v; break;
    case 5: s.E = v; break;
    case 6: s.H = v; break;
    case 7: s.L = v; break;
    case 10: s.M = v; break;
  }
}

// Optional CPU-time budget of the calling thread's ExhaustiveCheck sweeps
// (SetSweepBudget; used to bound a timed CPU sample, never by the parity
// tests).  Unset, every sweep runs to its end as the reference's does.
struct SweepBudget {
  double deadline = 0;  // thread CPU seconds; 0: no budget
  uint32_t tick = 0;
  bool spent = false;
};
static thread_local SweepBudget t_budget;

static double threadCpuSeconds() {
  timespec ts{};
  clock_gettime(CLOCK_THREAD_CPUTIME_ID, &ts);
  return double(ts.tv_sec) + 1e-9 * double(ts.tv_nsec);
}

void SetSweepBudget(double seconds) {
  t_budget = SweepBudget{};
  if (seconds > 0) t_budget.deadline = threadCpuSeconds() + seconds;
}
bool SweepBudgetSpent() { return t_budget.spent; }

struct Pair {
  const Instruction* t;
  int tn;
  const Instruction* c;
  int cn;
  FlagMask dead;
  uint8_t dregs;
  bool cmp(const State& s) const {
    if (t_budget.deadline > 0) {
      // every 65,536 states, look at the clock; once the budget is spent every
      // sweep of this thread stops at its next state (the caller discards
      // the target's result)
      if ((++t_budget.tick & 0xFFFFu) == 0 && threadCpuSeconds() > t_budget.deadline) t_budget.spent = true;
      if (t_budget.spent) return false;
    }
    return StatesEqualMaskedRegs(ExecSeq(s, t, tn), ExecSeq(s, c, cn), dead, dregs);
  }
};

static int extraRegs(uint16_t reads, int out[7]) {
  int n = 0;
  if (reads & regB) out[n++] = 2;
  if (reads & regC) out[n++] = 3;
  if (reads & regD) out[n++] = 4;
  if (reads & regE) out[n++] = 5;
  if (reads & regH) out[n++] = 6;
  if (reads & regL) out[n++] = 7;
  if (reads & regM) out[n++] = 10;
  return n;
}

static bool sweepAF(const Pair& p) {
  for (int a = 0; a < 256; a++)
    for (int carry = 0; carry <= 1; carry++) {
      State s{};
      s.A = uint8_t(a);
      s.F = uint8_t(carry);
      if (!p.cmp(s)) return false;
    }
  return true;
}

static bool sweepReducedRec(const Pair& p, State s, const int* regs, int n, int idx, bool sp) {
  if (idx >= n) {
    if (sp) {
      for (uint16_t v : kRepSP) {
        State s2 = s;
        s2.SP = v;
        if (!p.cmp(s2)) return false;
      }
      return true;
    }
    return p.cmp(s);
  }
  for (uint8_t v : kRepValues) {
    State s2 = s;
    setReg(s2, regs[idx], v);
    if (!sweepReducedRec(p, s2, regs, n, idx + 1, sp)) return false;
  }
  return true;
}

static bool exhaustive(const Pair& p) {
  uint16_t reads = uint16_t(RegsRead(p.t, p.tn) | RegsRead(p.c, p.cn));
  if ((reads & ~(regA | regF)) == 0) return sweepAF(p);
  int regs[7];
  int n = extraRegs(reads, regs);
  bool sp = (reads & regSP) != 0;
  if (n == 0 && !sp) return sweepAF(p);
  if (n <= 2 && !sp) {
    if (n == 1) {
      for (int a = 0; a < 256; a++)
        for (int carry = 0; carry <= 1; carry++)
          for (int r = 0; r < 256; r++) {
            State s{};
            s.A = uint8_t(a);
            s.F = uint8_t(carry);
            setReg(s, regs[0], uint8_t(r));
            if (!p.cmp(s)) return false;
          }
      return true;
    }
    for (int a = 0; a < 256; a++)
      for (int carry = 0; carry <= 1; carry++)
        for (int r1 = 0; r1 < 256; r1++)
          for (int r2 = 0; r2 < 256; r2++) {
            State s{};
            s.A = uint8_t(a);
            s.F = uint8_t(carry);
            setReg(s, regs[0], uint8_t(r1));
            setReg(s, regs[1], uint8_t(r2));
            if (!p.cmp(s)) return false;
          }
    return true;
  }
  for (int a = 0; a < 256; a++)
    for (int carry = 0; carry <= 1; carry++) {
      State s{};
      s.A = uint8_t(a);
      s.F = uint8_t(carry);
      if (!sweepReducedRec(p, s, regs, n, 0, sp)) return false;
    }
  return true;
}

bool ExhaustiveCheck(const Instruction* t, int tn, const Instruction* c, int cn) {
  return exhaustive(Pair{t, tn, c, cn, 0, 0});
}
bool ExhaustiveCheckMasked(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead) {
  return exhaustive(Pair{t, tn, c, cn, dead, 0});
}
bool ExhaustiveCheckMaskedRegs(const Instruction* t, int tn, const Instruction* c, int cn, FlagMask dead,
                               uint8_t deadRegs) {
  return exhaustive(Pair{t, tn, c, cn, dead, deadRegs});
}

uint64_t ExhaustiveStates(const Instruction* t, int tn, const Instruction* c, int cn) {
  uint16_t reads = uint16_t(RegsRead(t, tn) | RegsRead(c, cn));
  int regs[7];
  int n = extraRegs(reads, regs);
  bool sp = (reads & regSP) != 0;
  if (n == 0 && !sp) return 512;
  if (n <= 2 && !sp) return 512ull << (8 * n);
  return (512ull << (5 * n)) * (sp ? 16 : 1);
}

// ----------------------------------------------------------------- pruner
static bool isSelfLoad(uint16_t op) {
  return op == LD_A_A || op == LD_B_B || op == LD_C_C || op == LD_D_D || op == LD_E_E ||
         op == LD_H_H || op == LD_L_L;
}
static bool isDeadWrite(Instruction a, Instruction b) {
  uint16_t w = OpWrites(a.op);
  if (w == 0) return false;
  uint16_t r2 = OpReads(b.op), w2 = OpWrites(b.op);
  return (w & w2 & ~regF & ~r2 & 0xFFFF) != 0;
}
static bool areIndependent(Instruction a, Instruction b) {
  uint16_t aR = OpReads(a.op), aW = OpWrites(a.op), bR = OpReads(b.op), bW = OpWrites(b.op);
  return !((aW & bR) || (aR & bW) || (aW & bW));
}
static uint32_t instKey(Instruction i) { return (uint32_t(i.op) << 16) | i.imm; }

// pruner.go:7-35
bool ShouldPrune(const Instruction* seq, int n) {
  for (int i = 0; i < n; i++) {
    if (seq[i].op == NOP) return true;
    if (isSelfLoad(seq[i].op)) return true;
    if (i + 1 < n && isDeadWrite(seq[i], seq[i + 1])) return true;
  }
  for (int i = 0; i + 1 < n; i++)
    if (areIndependent(seq[i], seq[i + 1]) && instKey(seq[i]) > instKey(seq[i + 1])) return true;
  return false;
}

// ------------------------------------------------------------- enumerator
const std::vector<Instruction>& Instructions8() {
  static std::vector<Instruction> v = [] {
    Init();
    std::vector<Instruction> out;
    for (uint16_t op : NonImmediateOps()) out.push_back({op, 0});
    for (uint16_t op : ImmediateOps())
      for (int imm = 0; imm < 256; imm++) out.push_back({op, uint16_t(imm)});
    return out;
  }();
  return v;
}
int InstructionCount8() { return int(NonImmediateOps().size() + ImmediateOps().size() * 256); }
int InstructionCount() {
  return int(NonImmediateOps().size() + ImmediateOps().size() * 256 + Imm16Ops().size() * 65536);
}

// EnumerateSequences8 (enumerator.go:319-345): odometer over Instructions8()
// with position 0 most significant.  fn returns false to stop.
template <class Fn>
static void enumerate8(int n, Fn fn) {
  const auto& pool = Instructions8();
  const int P = int(pool.size());
  std::vector<int> idx(n, 0);
  std::vector<Instruction> seq(n);
  for (int i = 0; i < n; i++) seq[i] = pool[0];
  while (true) {
    if (!fn(seq.data())) return;
    int p = n - 1;
    while (p >= 0) {
      if (++idx[p] < P) {
        seq[p] = pool[idx[p]];
        break;
      }
      idx[p] = 0;
      seq[p] = pool[0];
      p--;
    }
    if (p < 0) return;
  }
}

// ----------------------------------------------------------------- worker
// worker.go:124-192 + 195-265
void ProcessTask(const Instruction* target, int tn, int maxCandLen, FlagMask deadFlags,
                 std::vector<Rule>& out, SearchStats* st) {
  ProcessTaskExt(target, tn, maxCandLen, deadFlags, 0, out, st);
}

void ProcessTaskExt(const Instruction* target, int tn, int maxCandLen, FlagMask deadFlags, uint8_t deadRegs,
                    std::vector<Rule>& out, SearchStats* st) {
  Init();
  const int tBytes = SeqByteSize(target, tn), tT = SeqTStates(target, tn);
  uint64_t checked = 0, found = 0;
  std::vector<Instruction> tgt(target, target + tn);
  for (int cl = 1; cl <= maxCandLen; cl++) {
    bool hit = false;
    enumerate8(cl, [&](const Instruction* c) {
      checked++;
      int cb = SeqByteSize(c, cl);
      if (cb >= tBytes) return true;
      if (ShouldPrune(c, cl)) return true;
      if (!QuickCheck(target, tn, c, cl)) return true;
      if (!ExhaustiveCheck(target, tn, c, cl)) return true;
      found++;
      Rule r;
      r.Source = tgt;
      r.Replacement.assign(c, c + cl);
      r.BytesSaved = tBytes - cb;
      r.CyclesSaved = tT - SeqTStates(c, cl);
      out.push_back(std::move(r));
      hit = true;
      return false;
    });
    if (hit) break;
  }
  if (deadFlags != DeadNone || deadRegs != 0) {
    for (int cl = 1; cl <= maxCandLen; cl++) {
      bool hit = false;
      enumerate8(cl, [&](const Instruction* c) {
        checked++;
        int cb = SeqByteSize(c, cl);
        if (cb >= tBytes) return true;
        if (ShouldPrune(c, cl)) return true;
        if (QuickCheck(target, tn, c, cl)) return true;
        if (!QuickCheckMaskedRegs(target, tn, c, cl, deadFlags, deadRegs)) return true;
        if (!ExhaustiveCheckMaskedRegs(target, tn, c, cl, deadFlags, deadRegs)) return true;
        // FlagDiff (verifier.go:658-673); with dead registers the registers
        // that differ are recorded beside the flags
        FlagMask fd = 0;
        uint8_t rd = 0;
        for (const State& v : TestVectors) {
          State a = ExecSeq(v, target, tn), b = ExecSeq(v, c, cl);
          fd |= uint8_t(a.F ^ b.F);
          rd |= uint8_t((a.B != b.B ? 1 : 0) | (a.C != b.C ? 2 : 0) | (a.D != b.D ? 4 : 0) | (a.E != b.E ? 8 : 0) |
                        (a.H != b.H ? 16 : 0) | (a.L != b.L ? 32 : 0));
        }
        if (deadRegs == 0 && rd != 0) fd = 0;  // FlagDiff is 0 when a register differs
        if (fd == 0 && rd == 0) return true;
        found++;
        Rule r;
        r.Source = tgt;
        r.Replacement.assign(c, c + cl);
        r.BytesSaved = tBytes - cb;
        r.CyclesSaved = tT - SeqTStates(c, cl);
        r.DeadFlags = fd;
        r.DeadRegs = deadRegs ? rd : 0;
        out.push_back(std::move(r));
        hit = true;
        return false;
      });
      if (hit) break;
    }
  }
  if (st) {
    st->checked += checked;
    st->found += found;
  }
}

std::vector<Rule> RunTasks(const std::vector<std::vector<Instruction>>& targets, int maxCandLen,
                           FlagMask deadFlags, int numWorkers, SearchStats* st) {
  Init();
  (void)Instructions8();
  if (numWorkers <= 0) numWorkers = int(std::thread::hardware_concurrency());
  if (numWorkers <= 0) numWorkers = 1;
  std::vector<std::vector<Rule>> per(targets.size());
  std::vector<SearchStats> stats(static_cast<size_t>(numWorkers));
  std::atomic<size_t> next{0};
  auto work = [&](int w) {
    size_t i;
    while ((i = next.fetch_add(1)) < targets.size())
      ProcessTask(targets[i].data(), int(targets[i].size()), maxCandLen, deadFlags, per[i], &stats[size_t(w)]);
  };
  std::vector<std::thread> th;
  for (int w = 0; w < numWorkers; w++) th.emplace_back(work, w);
  for (auto& t : th) t.join();
  std::vector<Rule> out;
  for (auto& v : per)
    for (auto& r : v) out.push_back(std::move(r));
  if (st)
    for (auto& s : stats) {
      st->checked += s.checked;
      st->found += s.found;
    }
  return out;
}

// ----------------------------------------------- pkg/gpu SearchGPU (one target)
// pkg/gpu/search.go:468-546: fingerprint compare (80 bytes, F masked by the
// dead flags) as the z80qc server does (cuda/z80_quickcheck.cu:666-681), then
// byte filter, prune, MidCheck[Masked], Exhaustive[Masked]; every hit kept.
void SearchGPUTarget(const Instruction* target, int tn, const std::vector<Instruction>& cands,
                     FlagMask deadFlags, std::vector<Rule>& out) {
  Init();
  uint8_t tfp[80], cfp[80];
  Fingerprint(target, tn, tfp);
  const int tBytes = SeqByteSize(target, tn), tT = SeqTStates(target, tn);
  std::vector<Instruction> tgt(target, target + tn);
  for (size_t i = 0; i < cands.size(); i++) {
    const Instruction* c = &cands[i];
    Fingerprint(c, 1, cfp);
    bool match = true;
    for (int k = 0; k < 80 && match; k++) {
      uint8_t a = cfp[k], b = tfp[k];
      if (k % 10 == 1) {
        a &= uint8_t(~deadFlags);
        b &= uint8_t(~deadFlags);
      }
      match = (a == b);
    }
    if (!match) continue;
    int cb = SeqByteSize(c, 1);
    if (cb >= tBytes) continue;
    if (ShouldPrune(c, 1)) continue;
    if (deadFlags == DeadNone) {
      if (!MidCheck(target, tn, c, 1)) continue;
      if (!ExhaustiveCheck(target, tn, c, 1)) continue;
    } else {
      if (!MidCheckMasked(target, tn, c, 1, deadFlags)) continue;
      if (!ExhaustiveCheckMasked(target, tn, c, 1, deadFlags)) continue;
    }
    Rule r;
    r.Source = tgt;
    r.Replacement.assign(c, c + 1);
    r.BytesSaved = tBytes - cb;
    r.CyclesSaved = tT - SeqTStates(c, 1);
    if (deadFlags != DeadNone) r.DeadFlags = FlagDiff(target, tn, c, 1);
    out.push_back(std::move(r));
  }
}

// ----------------------------------------------------------------- output
// output.go:93-129
std::string DeadFlagDesc(uint8_t mask) {
  if (mask == 0x00) return "";
  if (mask == 0xFF) return "all";
  if (mask == 0x28) return "undoc";
  static const char* const names[8] = {"C", "N", "P/V", "X3", "H", "X5", "Z", "S"};
  std::string s;
  for (int b = 0; b < 8; b++)
    if (mask & (1 << b)) {
      if (!s.empty()) s += ",";
      s += names[b];
    }
  return s;
}

static void jsonStr(std::string& o, const std::string& s) {
  o += '"';
  for (char ch : s) {
    unsigned char c = (unsigned char)ch;
    if (c == '"') o += "\\\"";
    else if (c == '\\') o += "\\\\";
    else if (c == '<') o += "\\u003c";
    else if (c == '>') o += "\\u003e";
    else if (c == '&') o += "\\u0026";
    else if (c < 0x20) {
      char buf[8];
      std::snprintf(buf, sizeof buf, "\\u%04x", c);
      o += buf;
    } else o += ch;
  }
  o += '"';
}

// output.go:70-90 (json.Encoder with two-space indent)
std::string WriteJSON(const std::vector<Rule>& rules) {
  if (rules.empty()) return "[]\n";
  std::string o = "[\n";
  for (size_t i = 0; i < rules.size(); i++) {
    const Rule& r = rules[i];
    o += "  {\n    \"source_asm\": ";
    jsonStr(o, DisasmSeq(r.Source));
    o += ",\n    \"replacement_asm\": ";
    jsonStr(o, DisasmSeq(r.Replacement));
    o += ",\n    \"source_bytes\": " + std::to_string(SeqByteSize(r.Source.data(), int(r.Source.size())));
    o += ",\n    \"replacement_bytes\": " +
         std::to_string(SeqByteSize(r.Replacement.data(), int(r.Replacement.size())));
    o += ",\n    \"bytes_saved\": " + std::to_string(r.BytesSaved);
    o += ",\n    \"cycles_saved\": " + std::to_string(r.CyclesSaved);
    if (r.DeadFlags != 0) {
      char buf[8];
      std::snprintf(buf, sizeof buf, "%02X", r.DeadFlags);
      o += ",\n    \"dead_flags\": ";
      jsonStr(o, buf);
      o += ",\n    \"dead_flag_desc\": ";
      jsonStr(o, DeadFlagDesc(r.DeadFlags));
    }
    o += "\n  }";
    o += (i + 1 < rules.size()) ? ",\n" : "\n";
  }
  o += "]\n";
  return o;
}

// ------------------------------------------------------------ CLI parsing
static std::string upper(std::string s) {
  for (auto& c : s) c = char(std::toupper((unsigned char)c));
  return s;
}
static std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  return s.substr(a, b - a + 1);
}

// cmd/z80opt/main.go:305-322
bool ParseDeadFlags(const std::string& in, FlagMask* out) {
  std::string s;
  for (char c : in) s += char(std::tolower((unsigned char)c));
  if (s == "none" || s.empty()) { *out = DeadNone; return true; }
  if (s == "undoc") { *out = DeadUndoc; return true; }
  if (s == "all") { *out = DeadAll; return true; }
  if (s.rfind("0x", 0) == 0) s = s.substr(2);
  // strconv.ParseUint(s, 16, 8): hex digits only, value <= 0xFF.
  if (s.empty()) return false;
  unsigned v = 0;
  for (char c : s) {
    int d = std::isdigit((unsigned char)c) ? c - '0' : (c >= 'a' && c <= 'f') ? c - 'a' + 10 : -1;
    if (d < 0) return false;
    v = v * 16 + unsigned(d);
    if (v > 0xFF) return false;
  }
  *out = FlagMask(v);
  return true;
}

// Reads an integer the way fmt.Sscanf("%x"/"%d") does: optional sign, then as
// many digits as match; at least one digit is required.
static bool scanInt(const std::string& s, int base, long* out) {
  size_t i = 0;
  bool neg = false;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) { neg = s[i] == '-'; i++; }
  long v = 0;
  size_t start = i;
  for (; i < s.size(); i++) {
    char c = s[i];
    int d = (c >= '0' && c <= '9') ? c - '0'
            : (base == 16 && c >= 'a' && c <= 'f') ? c - 'a' + 10
            : (base == 16 && c >= 'A' && c <= 'F') ? c - 'A' + 10 : -1;
    if (d < 0) break;
    v = v * base + d;
  }
  if (i == start) return false;
  *out = neg ? -v : v;
  return true;
}

// cmd/z80opt/main.go:478-504
static bool parseImmediate(std::string s, long* v) {
  s = trim(s);
  if (s.empty()) return false;
  if (s.rfind("0X", 0) == 0 || s.rfind("0x", 0) == 0) return scanInt(s.substr(2), 16, v);
  if (upper(s).back() == 'H') return scanInt(s.substr(0, s.size() - 1), 16, v);
  return scanInt(s, 10, v);
}

static bool equalFold(const std::string& a, const std::string& b) { return upper(a) == upper(b); }

// cmd/z80opt/main.go:348-397
static bool parseSingle(const std::string& in, Instruction* out) {
  std::string text = trim(in), up = upper(text);
  for (uint16_t op = 0; op < OpCodeCount; op++) {
    const std::string& m = Catalog[op].mnemonic;
    if (m.empty()) continue;
    if (!HasImmediate(op)) {
      if (equalFold(text, m)) { *out = {op, 0}; return true; }
      continue;
    }
    std::string pat = upper(m);
    size_t n = pat.rfind('N');
    if (n == std::string::npos) continue;
    std::string prefix = pat.substr(0, n), suffix = pat.substr(n + 1);
    if (up.compare(0, prefix.size(), prefix) != 0 || up.size() < prefix.size()) continue;
    if (!suffix.empty() &&
        (up.size() < suffix.size() || up.compare(up.size() - suffix.size(), suffix.size(), suffix) != 0))
      continue;
    std::string val = up.substr(prefix.size());
    if (!suffix.empty()) {
      if (val.size() < suffix.size()) continue;
      val = val.substr(0, val.size() - suffix.size());
    }
    long v;
    if (!parseImmediate(trim(val), &v)) continue;
    *out = {op, uint16_t(v)};
    return true;
  }
  return false;
}

// cmd/z80opt/main.go:325-346
bool ParseAssembly(const std::string& text, std::vector<Instruction>* out) {
  Init();
  out->clear();
  size_t start = 0;
  while (true) {
    size_t p = text.find(':', start);
    std::string part = trim(text.substr(start, p == std::string::npos ? std::string::npos : p - start));
    if (!part.empty()) {
      Instruction in;
      if (!parseSingle(part, &in)) return false;
      out->push_back(in);
    }
    if (p == std::string::npos) break;
    start = p + 1;
  }
  return !out->empty();
}

}  // namespace orc
