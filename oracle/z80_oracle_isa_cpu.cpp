// ISA catalog + emulator restatement (oracle; test infrastructure only).
//
// Follows pkg/inst/instruction.go, pkg/inst/catalog.go, pkg/cpu/flags.go and
// pkg/cpu/exec.go of the reference.  Written family-by-family from the
// reference's enum order rather than as one case per opcode; the per-opcode
// behaviour is the same as the reference switch (exec.go:8-1033) and the
// helpers (exec.go:1038-1264).
#include "z80_oracle.h"

#include <cctype>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace orc {

uint8_t Sz53Table[256], Sz53pTable[256], ParityTable[256];
// flags.go:30-33
const uint8_t HalfcarryAddTable[8] = {0, FlagH, FlagH, FlagH, 0, 0, 0, FlagH};
const uint8_t HalfcarrySubTable[8] = {0, 0, FlagH, 0, FlagH, 0, FlagH, FlagH};
const uint8_t OverflowAddTable[8] = {0, 0, 0, FlagV, FlagV, 0, 0, 0};
const uint8_t OverflowSubTable[8] = {0, FlagV, 0, 0, 0, 0, FlagV, 0};

Info Catalog[OpCodeCount];

static const char* const kOpNames[OpCodeCount] = {
#define X(n) #n,
    ORC_OPCODES
#undef X
};
const char* OpName(uint16_t op) { return op < OpCodeCount ? kOpNames[op] : "?"; }

// Register order used by most families in the enum: A,B,C,D,E,H,L.
static const char* const kR7[7] = {"A", "B", "C", "D", "E", "H", "L"};
// Z80 3-bit register field for A,B,C,D,E,H,L (catalog.go:340).
static const uint8_t kEnc7[7] = {7, 0, 1, 2, 3, 4, 5};
// Source order of the ALU/LD-A families: B,C,D,E,H,L,A (instruction.go:54-60,114-190).
static const int kAluSrc[7] = {1, 2, 3, 4, 5, 6, 0};

static void put(uint16_t op, const std::string& m, std::initializer_list<uint8_t> enc, int t) {
  Info& in = Catalog[op];
  in.mnemonic = m;
  in.nbytes = 0;
  for (uint8_t b : enc) in.bytes[in.nbytes++] = b;
  in.tstates = t;
}

// flags.go:36-53 + catalog.go:147-562
static void BuildTables() {
  for (int i = 0; i < 256; i++) {
    Sz53Table[i] = uint8_t(i) & (Flag3 | Flag5 | FlagS);
    int bits = __builtin_popcount(i);
    ParityTable[i] = (bits % 2 == 0) ? FlagP : 0;
    Sz53pTable[i] = Sz53Table[i] | ParityTable[i];
  }
  Sz53Table[0] |= FlagZ;
  Sz53pTable[0] |= FlagZ;

  // LD r,r' (ops 0..48): A-row sources B..L,A; other rows A..L.
  for (int d = 0; d < 7; d++)
    for (int k = 0; k < 7; k++) {
      int s = (d == 0) ? kAluSrc[k] : k;
      uint16_t op = uint16_t(d * 7 + k);
      put(op, std::string("LD ") + kR7[d] + ", " + kR7[s],
          {uint8_t(0x40 | (kEnc7[d] << 3) | kEnc7[s])}, 4);
    }
  for (int d = 0; d < 7; d++)
    put(uint16_t(LD_A_N + d), std::string("LD ") + kR7[d] + ", n",
        {uint8_t(0x06 | (kEnc7[d] << 3))}, 7);
  static const char* const aluReg[8] = {"ADD A, ", "ADC A, ", "SUB ", "SBC A, ",
                                        "AND ",    "XOR ",    "OR ",  "CP "};
  for (int a = 0; a < 8; a++) {
    for (int k = 0; k < 7; k++) {
      int s = kAluSrc[k];
      put(uint16_t(ADD_A_B + a * 8 + k), std::string(aluReg[a]) + kR7[s],
          {uint8_t(0x80 | (a << 3) | kEnc7[s])}, 4);
    }
    put(uint16_t(ADD_A_B + a * 8 + 7), std::string(aluReg[a]) + "n",
        {uint8_t(0xC6 | (a << 3))}, 7);
  }
  for (int r = 0; r < 7; r++) {
    put(uint16_t(INC_A + r), std::string("INC ") + kR7[r], {uint8_t(0x04 | (kEnc7[r] << 3))}, 4);
    put(uint16_t(DEC_A + r), std::string("DEC ") + kR7[r], {uint8_t(0x05 | (kEnc7[r] << 3))}, 4);
  }
  put(RLCA, "RLCA", {0x07}, 4);
  put(RRCA, "RRCA", {0x0F}, 4);
  put(RLA, "RLA", {0x17}, 4);
  put(RRA, "RRA", {0x1F}, 4);
  put(DAA, "DAA", {0x27}, 4);
  put(CPL, "CPL", {0x2F}, 4);
  put(SCF, "SCF", {0x37}, 4);
  put(CCF, "CCF", {0x3F}, 4);
  put(NEG, "NEG", {0xED, 0x44}, 8);
  put(NOP, "NOP", {0x00}, 4);
  // CB rotates/shifts: kinds RLC,RRC,RL,RR,SLA,SRA,SRL occupy 7 ops each
  // (A..L); SLL_A follows, then SLL_B..SLL_L.  CB sub-opcode kind field:
  // RLC=0 RRC=1 RL=2 RR=3 SLA=4 SRA=5 SLL=6 SRL=7.
  static const char* const cbName[7] = {"RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL"};
  static const uint8_t cbKind[7] = {0, 1, 2, 3, 4, 5, 7};
  for (int k = 0; k < 7; k++)
    for (int r = 0; r < 7; r++)
      put(uint16_t(RLC_A + k * 7 + r), std::string(cbName[k]) + " " + kR7[r],
          {0xCB, uint8_t((cbKind[k] << 3) | kEnc7[r])}, 8);
  put(SLL_A, "SLL A", {0xCB, 0x37}, 8);
  for (int r = 1; r < 7; r++)
    put(uint16_t(SLL_B + r - 1), std::string("SLL ") + kR7[r], {0xCB, uint8_t(0x30 | kEnc7[r])}, 8);
  static const char* const bitName[3] = {"BIT ", "RES ", "SET "};
  for (int f = 0; f < 3; f++)
    for (int n = 0; n < 8; n++)
      for (int r = 0; r < 7; r++)
        put(uint16_t(BIT_0_A + f * 56 + n * 7 + r),
            std::string(bitName[f]) + char('0' + n) + ", " + kR7[r],
            {0xCB, uint8_t(((f + 1) << 6) | (n << 3) | kEnc7[r])}, 8);
  // 16-bit pair ops (catalog.go:405-418)
  static const char* const rr[4] = {"BC", "DE", "HL", "SP"};
  for (int p = 0; p < 4; p++) {
    put(uint16_t(INC_BC + p), std::string("INC ") + rr[p], {uint8_t(0x03 | (p << 4))}, 6);
    put(uint16_t(DEC_BC + p), std::string("DEC ") + rr[p], {uint8_t(0x0B | (p << 4))}, 6);
    put(uint16_t(ADD_HL_BC + p), std::string("ADD HL, ") + rr[p], {uint8_t(0x09 | (p << 4))}, 11);
    put(uint16_t(LD_BC_NN + p), std::string("LD ") + rr[p] + ", nn", {uint8_t(0x01 | (p << 4))}, 10);
    put(uint16_t(ADC_HL_BC + p), std::string("ADC HL, ") + rr[p], {0xED, uint8_t(0x4A | (p << 4))}, 15);
    put(uint16_t(SBC_HL_BC + p), std::string("SBC HL, ") + rr[p], {0xED, uint8_t(0x42 | (p << 4))}, 15);
  }
  put(EX_DE_HL, "EX DE, HL", {0xEB}, 4);
  put(LD_SP_HL, "LD SP, HL", {0xF9}, 6);
  // Memory ops (catalog.go:440-561)
  for (int r = 0; r < 7; r++) {
    put(uint16_t(LD_A_HLI + r), std::string("LD ") + kR7[r] + ", (HL)",
        {uint8_t(0x46 | (kEnc7[r] << 3))}, 7);
    put(uint16_t(LD_HLI_A + r), std::string("LD (HL), ") + kR7[r], {uint8_t(0x70 | kEnc7[r])}, 7);
  }
  put(LD_HLI_N, "LD (HL), n", {0x36}, 10);
  put(LD_A_BCI, "LD A, (BC)", {0x0A}, 7);
  put(LD_A_DEI, "LD A, (DE)", {0x1A}, 7);
  put(LD_BCI_A, "LD (BC), A", {0x02}, 7);
  put(LD_DEI_A, "LD (DE), A", {0x12}, 7);
  static const char* const aluMem[8] = {"ADD A, (HL)", "ADC A, (HL)", "SUB (HL)", "SBC A, (HL)",
                                        "AND (HL)",    "XOR (HL)",    "OR (HL)",  "CP (HL)"};
  for (int a = 0; a < 8; a++) put(uint16_t(ADD_A_HLI + a), aluMem[a], {uint8_t(0x86 | (a << 3))}, 7);
  put(INC_HLI, "INC (HL)", {0x34}, 11);
  put(DEC_HLI, "DEC (HL)", {0x35}, 11);
  static const char* const cbMem[8] = {"RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL", "SLL"};
  static const uint8_t cbMemKind[8] = {0, 1, 2, 3, 4, 5, 7, 6};
  for (int k = 0; k < 8; k++)
    put(uint16_t(RLC_HLI + k), std::string(cbMem[k]) + " (HL)", {0xCB, uint8_t((cbMemKind[k] << 3) | 6)}, 15);
  for (int n = 0; n < 8; n++) {
    put(uint16_t(BIT_0_HLI + n), std::string("BIT ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0x46 | (n << 3))}, 12);
    put(uint16_t(RES_0_HLI + n), std::string("RES ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0x86 | (n << 3))}, 15);
    put(uint16_t(SET_0_HLI + n), std::string("SET ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0xC6 | (n << 3))}, 15);
  }
}

static std::once_flag g_once;
void Init() { std::call_once(g_once, BuildTables); }

// instruction.go:16-38
bool HasImm16(uint16_t op) { return op >= LD_BC_NN && op <= LD_SP_NN; }
bool HasImmediate(uint16_t op) {
  if (op >= LD_A_N && op <= LD_L_N) return true;
  switch (op) {
    case ADD_A_N: case ADC_A_N: case SUB_N: case SBC_A_N:
    case AND_N: case XOR_N: case OR_N: case CP_N: case LD_HLI_N:
      return true;
  }
  return HasImm16(op);
}
bool UsesMemory(uint16_t op) { return op >= LD_A_HLI && op < OpCodeCount; }

int TStates(uint16_t op) { return Catalog[op].tstates; }
// catalog.go:62-70
int ByteSize(uint16_t op) {
  int n = Catalog[op].nbytes;
  if (HasImm16(op)) n += 2;
  else if (HasImmediate(op)) n += 1;
  return n;
}

static void hex8(std::string& b, uint8_t v) {
  static const char* hx = "0123456789ABCDEF";
  if (v >= 0xA0) b += '0';
  b += hx[v >> 4];
  b += hx[v & 15];
  b += 'h';
}
static void hex16(std::string& b, uint16_t v) {
  static const char* hx = "0123456789ABCDEF";
  if ((v >> 12) >= 0xA) b += '0';
  b += hx[v >> 12];
  b += hx[(v >> 8) & 15];
  b += hx[(v >> 4) & 15];
  b += hx[v & 15];
  b += 'h';
}

// catalog.go:73-127
std::string Disassemble(Instruction in) {
  const std::string& m = Catalog[in.op].mnemonic;
  std::string out;
  if (HasImm16(in.op)) {
    for (size_t i = 0; i < m.size(); i++) {
      if (i + 1 < m.size() && m[i] == 'n' && m[i + 1] == 'n') {
        hex16(out, in.imm);
        i++;
      } else {
        out += m[i];
      }
    }
    return out;
  }
  if (HasImmediate(in.op)) {
    for (size_t i = 0; i < m.size(); i++) {
      if (m[i] == 'n' && (i == m.size() - 1 || m[i + 1] == ' ' || m[i + 1] == ','))
        hex8(out, uint8_t(in.imm));
      else
        out += m[i];
    }
    return out;
  }
  return m;
}

std::string DisasmSeq(const std::vector<Instruction>& seq) {
  std::string s;
  for (size_t i = 0; i < seq.size(); i++) {
    if (i) s += " : ";
    s += Disassemble(seq[i]);
  }
  return s;
}

int SeqByteSize(const Instruction* seq, int n) {
  int b = 0;
  for (int i = 0; i < n; i++) b += ByteSize(seq[i].op);
  return b;
}
int SeqTStates(const Instruction* seq, int n) {
  int t = 0;
  for (int i = 0; i < n; i++) t += TStates(seq[i].op);
  return t;
}

std::vector<uint16_t> NonImmediateOps() {
  std::vector<uint16_t> v;
  for (uint16_t i = 0; i < OpCodeCount; i++)
    if (!HasImmediate(i)) v.push_back(i);
  return v;
}
std::vector<uint16_t> ImmediateOps() {
  std::vector<uint16_t> v;
  for (uint16_t i = 0; i < OpCodeCount; i++)
    if (HasImmediate(i) && !HasImm16(i)) v.push_back(i);
  return v;
}
std::vector<uint16_t> Imm16Ops() {
  std::vector<uint16_t> v;
  for (uint16_t i = 0; i < OpCodeCount; i++)
    if (HasImm16(i)) v.push_back(i);
  return v;
}

// ---------------------------------------------------------------- emulator
// ALU helpers: exec.go:1038-1256
static inline void execAdd(State& s, uint8_t v) {
  uint16_t t = uint16_t(s.A + v);
  uint8_t lookup = uint8_t(((s.A & 0x88) >> 3) | ((v & 0x88) >> 2) | ((t & 0x88) >> 1));
  s.A = uint8_t(t);
  s.F = uint8_t(((t & 0x100) ? FlagC : 0) | HalfcarryAddTable[lookup & 7] |
                OverflowAddTable[lookup >> 4] | Sz53Table[s.A]);
}
static inline void execAdc(State& s, uint8_t v) {
  uint16_t t = uint16_t(s.A + v + (s.F & FlagC));
  uint8_t lookup = uint8_t(((s.A & 0x88) >> 3) | ((v & 0x88) >> 2) | ((t & 0x88) >> 1));
  s.A = uint8_t(t);
  s.F = uint8_t(((t & 0x100) ? FlagC : 0) | HalfcarryAddTable[lookup & 7] |
                OverflowAddTable[lookup >> 4] | Sz53Table[s.A]);
}
static inline void execSub(State& s, uint8_t v) {
  uint16_t t = uint16_t(s.A - v);
  uint8_t lookup = uint8_t(((s.A & 0x88) >> 3) | ((v & 0x88) >> 2) | ((t & 0x88) >> 1));
  s.A = uint8_t(t);
  s.F = uint8_t(((t & 0x100) ? FlagC : 0) | FlagN | HalfcarrySubTable[lookup & 7] |
                OverflowSubTable[lookup >> 4] | Sz53Table[s.A]);
}
static inline void execSbc(State& s, uint8_t v) {
  uint16_t t = uint16_t(s.A - v - (s.F & FlagC));
  uint8_t lookup = uint8_t(((s.A & 0x88) >> 3) | ((v & 0x88) >> 2) | ((t & 0x88) >> 1));
  s.A = uint8_t(t);
  s.F = uint8_t(((t & 0x100) ? FlagC : 0) | FlagN | HalfcarrySubTable[lookup & 7] |
                OverflowSubTable[lookup >> 4] | Sz53Table[s.A]);
}
static inline void execAnd(State& s, uint8_t v) { s.A &= v; s.F = FlagH | Sz53pTable[s.A]; }
static inline void execOr(State& s, uint8_t v) { s.A |= v; s.F = Sz53pTable[s.A]; }
static inline void execXor(State& s, uint8_t v) { s.A ^= v; s.F = Sz53pTable[s.A]; }
static inline void execCp(State& s, uint8_t v) {
  uint16_t t = uint16_t(s.A - v);
  uint8_t lookup = uint8_t(((s.A & 0x88) >> 3) | ((v & 0x88) >> 2) | ((t & 0x88) >> 1));
  s.F = uint8_t(((t & 0x100) ? FlagC : (t != 0 ? 0 : FlagZ)) | FlagN |
                HalfcarrySubTable[lookup & 7] | OverflowSubTable[lookup >> 4] |
                (v & (Flag3 | Flag5)) | (t & FlagS));
}
static inline void execInc(State& s, uint8_t& r) {
  r++;
  s.F = uint8_t((s.F & FlagC) | (r == 0x80 ? FlagV : 0) | ((r & 0x0F) ? 0 : FlagH) | Sz53Table[r]);
}
static inline void execDec(State& s, uint8_t& r) {
  s.F = uint8_t((s.F & FlagC) | ((r & 0x0F) ? 0 : FlagH) | FlagN);
  r--;
  s.F |= uint8_t((r == 0x7F ? FlagV : 0) | Sz53Table[r]);
}
static inline void execDaa(State& s) {
  uint8_t add = 0, carry = s.F & FlagC;
  if ((s.F & FlagH) || (s.A & 0x0F) > 9) add = 6;
  if (carry || s.A > 0x99) add |= 0x60;
  if (s.A > 0x99) carry = FlagC;
  if (s.F & FlagN) execSub(s, add);
  else execAdd(s, add);
  s.F = uint8_t((s.F & ~(FlagC | FlagP)) | carry | ParityTable[s.A]);
}
static inline uint8_t execRlc(State& s, uint8_t v) {
  v = uint8_t((v << 1) | (v >> 7));
  s.F = uint8_t((v & FlagC) | Sz53pTable[v]);
  return v;
}
static inline uint8_t execRrc(State& s, uint8_t v) {
  s.F = v & FlagC;
  v = uint8_t((v >> 1) | (v << 7));
  s.F |= Sz53pTable[v];
  return v;
}
static inline uint8_t execRl(State& s, uint8_t v) {
  uint8_t old = v;
  v = uint8_t((v << 1) | (s.F & FlagC));
  s.F = uint8_t((old >> 7) | Sz53pTable[v]);
  return v;
}
static inline uint8_t execRr(State& s, uint8_t v) {
  uint8_t old = v;
  v = uint8_t((v >> 1) | (s.F << 7));
  s.F = uint8_t((old & FlagC) | Sz53pTable[v]);
  return v;
}
static inline uint8_t execSla(State& s, uint8_t v) {
  s.F = v >> 7;
  v = uint8_t(v << 1);
  s.F |= Sz53pTable[v];
  return v;
}
static inline uint8_t execSra(State& s, uint8_t v) {
  s.F = v & FlagC;
  v = uint8_t((v & 0x80) | (v >> 1));
  s.F |= Sz53pTable[v];
  return v;
}
static inline uint8_t execSrl(State& s, uint8_t v) {
  s.F = v & FlagC;
  v = uint8_t(v >> 1);
  s.F |= Sz53pTable[v];
  return v;
}
static inline uint8_t execSll(State& s, uint8_t v) {
  s.F = v >> 7;
  v = uint8_t((v << 1) | 0x01);
  s.F |= Sz53pTable[v];
  return v;
}
static inline void execAddHL(State& s, uint16_t v) {
  uint16_t hl = uint16_t((s.H << 8) | s.L);
  uint32_t r = uint32_t(hl) + v;
  uint32_t hc = (hl & 0x0FFF) + (v & 0x0FFF);
  s.F = uint8_t((s.F & (FlagS | FlagZ | FlagP)) | ((hc & 0x1000) ? FlagH : 0) |
                ((r & 0x10000) ? FlagC : 0) | (uint8_t(r >> 8) & (Flag3 | Flag5)));
  s.H = uint8_t(r >> 8);
  s.L = uint8_t(r);
}
static inline void execAdcHL(State& s, uint16_t v) {
  uint16_t hl = uint16_t((s.H << 8) | s.L);
  uint64_t r = uint64_t(hl) + v + (s.F & FlagC);
  uint8_t lookup = uint8_t(((hl & 0x8800) >> 11) | ((v & 0x8800) >> 10) | ((r & 0x8800) >> 9));
  s.H = uint8_t(r >> 8);
  s.L = uint8_t(r);
  s.F = uint8_t(((r & 0x10000) ? FlagC : 0) | OverflowAddTable[lookup >> 4] |
                (s.H & (Flag3 | Flag5 | FlagS)) | HalfcarryAddTable[lookup & 7] |
                ((s.H | s.L) ? 0 : FlagZ));
}
static inline void execSbcHL(State& s, uint16_t v) {
  uint16_t hl = uint16_t((s.H << 8) | s.L);
  uint64_t r = uint64_t(hl) - uint64_t(v) - uint64_t(s.F & FlagC);
  uint8_t lookup = uint8_t(((hl & 0x8800) >> 11) | ((v & 0x8800) >> 10) | ((r & 0x8800) >> 9));
  s.H = uint8_t(r >> 8);
  s.L = uint8_t(r);
  s.F = uint8_t(((r & 0x10000) ? FlagC : 0) | FlagN | OverflowSubTable[lookup >> 4] |
                (s.H & (Flag3 | Flag5 | FlagS)) | HalfcarrySubTable[lookup & 7] |
                ((s.H | s.L) ? 0 : FlagZ));
}
static inline void execBit(State& s, uint8_t r, int bit) {
  s.F = uint8_t((s.F & FlagC) | FlagH | (r & (Flag3 | Flag5)));
  if ((r & (1 << bit)) == 0) s.F |= FlagP | FlagZ;
  if (bit == 7 && (r & 0x80)) s.F |= FlagS;
}

// Register by index in family order A,B,C,D,E,H,L.
static inline uint8_t& r7(State& s, int i) {
  switch (i) {
    case 0: return s.A;
    case 1: return s.B;
    case 2: return s.C;
    case 3: return s.D;
    case 4: return s.E;
    case 5: return s.H;
    default: return s.L;
  }
}
static inline uint16_t pair(State& s, int p) {
  switch (p) {
    case 0: return uint16_t((s.B << 8) | s.C);
    case 1: return uint16_t((s.D << 8) | s.E);
    case 2: return uint16_t((s.H << 8) | s.L);
    default: return s.SP;
  }
}
static inline void setPair(State& s, int p, uint16_t v) {
  switch (p) {
    case 0: s.B = uint8_t(v >> 8); s.C = uint8_t(v); break;
    case 1: s.D = uint8_t(v >> 8); s.E = uint8_t(v); break;
    case 2: s.H = uint8_t(v >> 8); s.L = uint8_t(v); break;
    default: s.SP = v; break;
  }
}

static inline void aluOp(State& s, int kind, uint8_t v) {
  switch (kind) {
    case 0: execAdd(s, v); break;
    case 1: execAdc(s, v); break;
    case 2: execSub(s, v); break;
    case 3: execSbc(s, v); break;
    case 4: execAnd(s, v); break;
    case 5: execXor(s, v); break;
    case 6: execOr(s, v); break;
    default: execCp(s, v); break;
  }
}
// CB rotate kinds in enum order RLC,RRC,RL,RR,SLA,SRA,SRL,SLL
static inline uint8_t cbOp(State& s, int kind, uint8_t v) {
  switch (kind) {
    case 0: return execRlc(s, v);
    case 1: return execRrc(s, v);
    case 2: return execRl(s, v);
    case 3: return execRr(s, v);
    case 4: return execSla(s, v);
    case 5: return execSra(s, v);
    case 6: return execSrl(s, v);
    default: return execSll(s, v);
  }
}

// exec.go:8-1034.  Returns the T-state cost.
int Exec(State& s, uint16_t op, uint16_t imm) {
  if (op < LD_A_N) {  // LD r,r'
    int d = op / 7, k = op % 7;
    int src = (d == 0) ? kAluSrc[k] : k;
    uint8_t v = r7(s, src);
    r7(s, d) = v;
  } else if (op <= LD_L_N) {
    r7(s, op - LD_A_N) = uint8_t(imm);
  } else if (op < INC_A) {  // ALU families
    int a = (op - ADD_A_B) / 8, k = (op - ADD_A_B) % 8;
    uint8_t v = (k == 7) ? uint8_t(imm) : r7(s, kAluSrc[k]);
    aluOp(s, a, v);
  } else if (op < DEC_A) {
    execInc(s, r7(s, op - INC_A));
  } else if (op < RLCA) {
    execDec(s, r7(s, op - DEC_A));
  } else if (op < RLC_A) {
    switch (op) {
      case RLCA:
        s.A = uint8_t((s.A << 1) | (s.A >> 7));
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & (FlagC | Flag3 | Flag5)));
        break;
      case RRCA:
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & FlagC));
        s.A = uint8_t((s.A >> 1) | (s.A << 7));
        s.F |= s.A & (Flag3 | Flag5);
        break;
      case RLA: {
        uint8_t old = s.A;
        s.A = uint8_t((s.A << 1) | (s.F & FlagC));
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & (Flag3 | Flag5)) | (old >> 7));
        break;
      }
      case RRA: {
        uint8_t old = s.A;
        s.A = uint8_t((s.A >> 1) | (s.F << 7));
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & (Flag3 | Flag5)) | (old & FlagC));
        break;
      }
      case DAA: execDaa(s); break;
      case CPL:
        s.A ^= 0xFF;
        s.F = uint8_t((s.F & (FlagC | FlagP | FlagZ | FlagS)) | (s.A & (Flag3 | Flag5)) | FlagN | FlagH);
        break;
      case SCF:
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & (Flag3 | Flag5)) | FlagC);
        break;
      case CCF: {
        uint8_t oldC = s.F & FlagC;
        s.F = uint8_t((s.F & (FlagP | FlagZ | FlagS)) | (s.A & (Flag3 | Flag5)));
        s.F |= oldC ? FlagH : FlagC;
        break;
      }
      case NEG: {
        uint8_t old = s.A;
        s.A = 0;
        execSub(s, old);
        break;
      }
      default: break;  // NOP
    }
  } else if (op < SLL_A) {  // RLC..SRL on A..L
    int k = (op - RLC_A) / 7, r = (op - RLC_A) % 7;
    uint8_t& reg = r7(s, r);
    reg = cbOp(s, k, reg);
  } else if (op <= SLL_L) {
    int r = op - SLL_A;  // SLL_A, SLL_B..SLL_L are contiguous A..L
    uint8_t& reg = r7(s, r);
    reg = execSll(s, reg);
  } else if (op < RES_0_A) {  // BIT n,r
    int n = (op - BIT_0_A) / 7, r = (op - BIT_0_A) % 7;
    execBit(s, r7(s, r), n);
  } else if (op < SET_0_A) {
    int n = (op - RES_0_A) / 7, r = (op - RES_0_A) % 7;
    r7(s, r) &= uint8_t(~(1u << n));
  } else if (op < INC_BC) {
    int n = (op - SET_0_A) / 7, r = (op - SET_0_A) % 7;
    r7(s, r) |= uint8_t(1u << n);
  } else if (op < INC_BC + 4) {
    int p = op - INC_BC;
    setPair(s, p, uint16_t(pair(s, p) + 1));
  } else if (op < ADD_HL_BC) {
    int p = op - DEC_BC;
    setPair(s, p, uint16_t(pair(s, p) - 1));
  } else if (op < EX_DE_HL) {
    execAddHL(s, pair(s, op - ADD_HL_BC));
  } else if (op == EX_DE_HL) {
    uint8_t d = s.D, e = s.E;
    s.D = s.H; s.E = s.L;
    s.H = d; s.L = e;
  } else if (op == LD_SP_HL) {
    s.SP = uint16_t((s.H << 8) | s.L);
  } else if (op < ADC_HL_BC) {
    setPair(s, op - LD_BC_NN, imm);
  } else if (op < SBC_HL_BC) {
    execAdcHL(s, pair(s, op - ADC_HL_BC));
  } else if (op < LD_A_HLI) {
    execSbcHL(s, pair(s, op - SBC_HL_BC));
  } else if (op < LD_HLI_A) {
    r7(s, op - LD_A_HLI) = s.M;
  } else if (op < LD_HLI_N) {
    s.M = r7(s, op - LD_HLI_A);
  } else if (op == LD_HLI_N) {
    s.M = uint8_t(imm);
  } else if (op == LD_A_BCI || op == LD_A_DEI) {
    s.A = s.M;
  } else if (op == LD_BCI_A || op == LD_DEI_A) {
    s.M = s.A;
  } else if (op < INC_HLI) {
    aluOp(s, op - ADD_A_HLI, s.M);
  } else if (op == INC_HLI) {
    execInc(s, s.M);
  } else if (op == DEC_HLI) {
    execDec(s, s.M);
  } else if (op < BIT_0_HLI) {
    // RLC,RRC,RL,RR,SLA,SRA,SRL,SLL (HL) -- same kind order as cbOp
    s.M = cbOp(s, op - RLC_HLI, s.M);
  } else if (op < RES_0_HLI) {
    execBit(s, s.M, op - BIT_0_HLI);
  } else if (op < SET_0_HLI) {
    s.M &= uint8_t(~(1u << (op - RES_0_HLI)));
  } else if (op < OpCodeCount) {
    s.M |= uint8_t(1u << (op - SET_0_HLI));
  } else {
    std::fprintf(stderr, "orc::Exec: unhandled opcode %u\n", op);
    std::abort();
  }
  return Catalog[op].tstates;
}

}  // namespace orc
