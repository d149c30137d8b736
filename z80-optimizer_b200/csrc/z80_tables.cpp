// z80_tables.cpp -- host-side catalog, masks, pruning and enumeration order.
// See z80_tables.h for the reference files each part follows.
#include "z80_tables.h"

#include "z80_exec.cuh"

#include <cctype>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace z80b {

namespace {

struct Entry {
  std::string mnem;
  uint8_t enc[2];
  int nenc;
};

// Register naming for the enum families (A,B,C,D,E,H,L) and their 3-bit
// Z80 operand field.
const char* const kName7[7] = {"A", "B", "C", "D", "E", "H", "L"};
const uint8_t kField7[7] = {7, 0, 1, 2, 3, 4, 5};
// ALU and LD-A source order B,C,D,E,H,L,A expressed as family indices.
const int kSrcOrder[7] = {1, 2, 3, 4, 5, 6, 0};
const uint16_t kMask7[7] = {kRegA, kRegB, kRegC, kRegD, kRegE, kRegH, kRegL};
const uint16_t kPair[4] = {kRegB | kRegC, kRegD | kRegE, kRegH | kRegL, kRegSP};
const char* const kPairName[4] = {"BC", "DE", "HL", "SP"};

struct Tables {
  OpInfo info[kNumOps];
  Entry cat[kNumOps];
  std::vector<uint32_t> pool;
};

void set(Tables& T, int op, std::string m, std::initializer_list<uint8_t> enc, int t, int imm,
         uint16_t rd, uint16_t wr) {
  Entry& e = T.cat[op];
  e.mnem = std::move(m);
  e.nenc = 0;
  for (uint8_t b : enc) e.enc[e.nenc++] = b;
  OpInfo& o = T.info[op];
  o.size = uint8_t(e.nenc + imm);
  o.tstates = uint8_t(t);
  o.imm = uint8_t(imm);
  o.nopish = 0;
  o.reads = rd;
  o.writes = wr;
}

void build(Tables& T) {
  int op = 0;
  // LD r,r' (catalog.go:151-187): reads the source, writes the destination.
  for (int d = 0; d < 7; d++)
    for (int k = 0; k < 7; k++, op++) {
      int s = d == 0 ? kSrcOrder[k] : k;
      set(T, op, std::string("LD ") + kName7[d] + ", " + kName7[s],
          {uint8_t(0x40 | kField7[d] << 3 | kField7[s])}, 4, 0, kMask7[s], kMask7[d]);
      if (s == d) T.info[op].nopish = 1;
    }
  for (int d = 0; d < 7; d++, op++)
    set(T, op, std::string("LD ") + kName7[d] + ", n", {uint8_t(0x06 | kField7[d] << 3)}, 7, 1, 0, kMask7[d]);
  // ALU A,src / A,n.  Reads: the source register only (the accumulator is
  // not listed), plus F for ADC/SBC; the immediate forms read nothing except
  // ADC/SBC (A|F).  Writes A|F, CP only F.
  const char* const alu[8] = {"ADD A, ", "ADC A, ", "SUB ", "SBC A, ", "AND ", "XOR ", "OR ", "CP "};
  for (int a = 0; a < 8; a++) {
    bool cin = a == 1 || a == 3;
    uint16_t wr = a == 7 ? uint16_t(kRegF) : uint16_t(kRegA | kRegF);
    for (int k = 0; k < 7; k++, op++) {
      int s = kSrcOrder[k];
      set(T, op, std::string(alu[a]) + kName7[s], {uint8_t(0x80 | a << 3 | kField7[s])}, 4, 0,
          uint16_t(kMask7[s] | (cin ? kRegF : 0)), wr);
    }
    set(T, op, std::string(alu[a]) + "n", {uint8_t(0xC6 | a << 3)}, 7, 1,
        cin ? uint16_t(kRegA | kRegF) : uint16_t(0), wr);
    op++;
  }
  for (int r = 0; r < 7; r++, op++)
    set(T, op, std::string("INC ") + kName7[r], {uint8_t(0x04 | kField7[r] << 3)}, 4, 0, kMask7[r],
        uint16_t(kMask7[r] | kRegF));
  for (int r = 0; r < 7; r++, op++)
    set(T, op, std::string("DEC ") + kName7[r], {uint8_t(0x05 | kField7[r] << 3)}, 4, 0, kMask7[r],
        uint16_t(kMask7[r] | kRegF));
  const uint16_t AF = kRegA | kRegF;
  set(T, RLCA, "RLCA", {0x07}, 4, 0, kRegA, AF);
  set(T, RRCA, "RRCA", {0x0F}, 4, 0, kRegA, AF);
  set(T, RLA, "RLA", {0x17}, 4, 0, AF, AF);
  set(T, RRA, "RRA", {0x1F}, 4, 0, AF, AF);
  set(T, DAA, "DAA", {0x27}, 4, 0, kRegA, AF);
  set(T, CPL, "CPL", {0x2F}, 4, 0, kRegA, AF);
  set(T, SCF, "SCF", {0x37}, 4, 0, kRegF, kRegF);
  set(T, CCF, "CCF", {0x3F}, 4, 0, kRegF, kRegF);
  set(T, NEG, "NEG", {0xED, 0x44}, 8, 0, kRegA, AF);
  set(T, NOP, "NOP", {0x00}, 4, 0, 0, 0);
  T.info[NOP].nopish = 1;
  op = RLC_A;
  // CB shifts: enum kinds RLC,RRC,RL,RR,SLA,SRA,SRL; CB field values.
  const char* const sh[7] = {"RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL"};
  const uint8_t shf[7] = {0, 1, 2, 3, 4, 5, 7};
  for (int k = 0; k < 7; k++)
    for (int r = 0; r < 7; r++, op++)
      set(T, op, std::string(sh[k]) + " " + kName7[r], {0xCB, uint8_t(shf[k] << 3 | kField7[r])}, 8, 0,
          uint16_t(kMask7[r] | ((k == 2 || k == 3) ? kRegF : 0)), uint16_t(kMask7[r] | kRegF));
  for (int r = 0; r < 7; r++, op++)
    set(T, op, std::string("SLL ") + kName7[r], {0xCB, uint8_t(0x30 | kField7[r])}, 8, 0, kMask7[r],
        uint16_t(kMask7[r] | kRegF));
  const char* const bn[3] = {"BIT ", "RES ", "SET "};
  for (int f = 0; f < 3; f++)
    for (int n = 0; n < 8; n++)
      for (int r = 0; r < 7; r++, op++)
        set(T, op, std::string(bn[f]) + char('0' + n) + ", " + kName7[r],
            {0xCB, uint8_t((f + 1) << 6 | n << 3 | kField7[r])}, 8, 0, kMask7[r],
            f == 0 ? uint16_t(kRegF) : kMask7[r]);
  for (int p = 0; p < 4; p++) {
    set(T, INC_BC + p, std::string("INC ") + kPairName[p], {uint8_t(0x03 | p << 4)}, 6, 0, kPair[p], kPair[p]);
    set(T, DEC_BC + p, std::string("DEC ") + kPairName[p], {uint8_t(0x0B | p << 4)}, 6, 0, kPair[p], kPair[p]);
    set(T, ADD_HL_BC + p, std::string("ADD HL, ") + kPairName[p], {uint8_t(0x09 | p << 4)}, 11, 0,
        uint16_t(kRegH | kRegL | kPair[p]), uint16_t(kRegH | kRegL | kRegF));
    set(T, LD_BC_NN + p, std::string("LD ") + kPairName[p] + ", nn", {uint8_t(0x01 | p << 4)}, 10, 2, 0, kPair[p]);
    set(T, ADC_HL_BC + p, std::string("ADC HL, ") + kPairName[p], {0xED, uint8_t(0x4A | p << 4)}, 15, 0,
        uint16_t(kRegH | kRegL | kPair[p] | kRegF), uint16_t(kRegH | kRegL | kRegF));
    set(T, SBC_HL_BC + p, std::string("SBC HL, ") + kPairName[p], {0xED, uint8_t(0x42 | p << 4)}, 15, 0,
        uint16_t(kRegH | kRegL | kPair[p] | kRegF), uint16_t(kRegH | kRegL | kRegF));
  }
  set(T, EX_DE_HL, "EX DE, HL", {0xEB}, 4, 0, kRegD | kRegE | kRegH | kRegL, kRegD | kRegE | kRegH | kRegL);
  set(T, LD_SP_HL, "LD SP, HL", {0xF9}, 6, 0, kRegH | kRegL, kRegSP);
  // Memory ops: reads as opReads lists them; writes always 0 (the
  // reference's opWrites has no memory cases).
  for (int r = 0; r < 7; r++) {
    set(T, LD_A_HLI + r, std::string("LD ") + kName7[r] + ", (HL)", {uint8_t(0x46 | kField7[r] << 3)}, 7, 0, kRegM, 0);
    set(T, LD_HLI_A + r, std::string("LD (HL), ") + kName7[r], {uint8_t(0x70 | kField7[r])}, 7, 0, kMask7[r], 0);
  }
  set(T, LD_HLI_N, "LD (HL), n", {0x36}, 10, 1, 0, 0);
  set(T, LD_A_BCI, "LD A, (BC)", {0x0A}, 7, 0, kRegM, 0);
  set(T, LD_A_DEI, "LD A, (DE)", {0x1A}, 7, 0, kRegM, 0);
  set(T, LD_BCI_A, "LD (BC), A", {0x02}, 7, 0, kRegA, 0);
  set(T, LD_DEI_A, "LD (DE), A", {0x12}, 7, 0, kRegA, 0);
  const char* const am[8] = {"ADD A, (HL)", "ADC A, (HL)", "SUB (HL)", "SBC A, (HL)",
                             "AND (HL)", "XOR (HL)", "OR (HL)", "CP (HL)"};
  for (int a = 0; a < 8; a++)
    set(T, ADD_A_HLI + a, am[a], {uint8_t(0x86 | a << 3)}, 7, 0,
        uint16_t(kRegA | kRegM | ((a == 1 || a == 3) ? kRegF : 0)), 0);
  set(T, INC_HLI, "INC (HL)", {0x34}, 11, 0, kRegM, 0);
  set(T, DEC_HLI, "DEC (HL)", {0x35}, 11, 0, kRegM, 0);
  const char* const mh[8] = {"RLC", "RRC", "RL", "RR", "SLA", "SRA", "SRL", "SLL"};
  const uint8_t mhf[8] = {0, 1, 2, 3, 4, 5, 7, 6};
  for (int k = 0; k < 8; k++)
    set(T, RLC_HLI + k, std::string(mh[k]) + " (HL)", {0xCB, uint8_t(mhf[k] << 3 | 6)}, 15, 0,
        uint16_t(kRegM | ((k == 2 || k == 3) ? kRegF : 0)), 0);
  for (int n = 0; n < 8; n++) {
    set(T, BIT_0_HLI + n, std::string("BIT ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0x46 | n << 3)}, 12, 0, kRegM, 0);
    set(T, RES_0_HLI + n, std::string("RES ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0x86 | n << 3)}, 15, 0, kRegM, 0);
    set(T, SET_0_HLI + n, std::string("SET ") + char('0' + n) + ", (HL)", {0xCB, uint8_t(0xC6 | n << 3)}, 15, 0, kRegM, 0);
  }
  // Enumeration order (enumerator.go:319-345).
  for (int o = 0; o < kNumOps; o++)
    if (T.info[o].imm == 0) T.pool.push_back(insn(uint16_t(o)));
  for (int o = 0; o < kNumOps; o++)
    if (T.info[o].imm == 1)
      for (int v = 0; v < 256; v++) T.pool.push_back(insn(uint16_t(o), uint16_t(v)));
}

Tables& tables() {
  static Tables* T = [] {
    auto* t = new Tables();
    build(*t);
    return t;
  }();
  return *T;
}

void hex2(std::string& o, unsigned v, int digits) {
  static const char* hx = "0123456789ABCDEF";
  if ((v >> (4 * (digits - 1))) >= 0xA) o += '0';
  for (int i = digits - 1; i >= 0; i--) o += hx[(v >> (4 * i)) & 15];
  o += 'h';
}

}  // namespace

const OpInfo* op_table() { return tables().info; }

namespace {
// Class of one opcode: for sampled input states (all registers, F, SP and M
// random, plus all-zero and all-one states) and several immediates, run the
// step on all 256 values of A and compare the outputs.
uint8_t classify_a(uint16_t op) {
  uint64_t x = 0x9E3779B97F4A7C15ull ^ (uint64_t(op) << 32);
  auto rnd = [&]() {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const int kind = op_table()[op].imm;
  const uint16_t imms[5] = {0x0000, 0x0001, 0x0080, 0xFFFF, 0x5A3C};
  bool pass = true, over = true;
  for (int ii = 0; ii < (kind ? 5 : 1); ii++) {
    const uint16_t imm = kind == 1 ? uint16_t(imms[ii] & 0xFFu) : imms[ii];
    for (int k = 0; k < 66; k++) {
      const uint64_t r = k == 0 ? 0 : (k == 1 ? ~0ull : rnd());
      const uint64_t r2 = k == 0 ? 0 : (k == 1 ? ~0ull : rnd());
      z80b::Z80S base{0, uint32_t(r & 0xFF), uint32_t((r >> 8) & 0xFF), uint32_t((r >> 16) & 0xFF),
                      uint32_t((r >> 24) & 0xFF), uint32_t((r >> 32) & 0xFF), uint32_t((r >> 40) & 0xFF),
                      uint32_t((r >> 48) & 0xFF), uint32_t(r2 & 0xFFFF), uint32_t((r2 >> 16) & 0xFF)};
      z80b::Z80S out0{};
      uint32_t a_first = 0;
      for (uint32_t a = 0; a < 256; a++) {
        z80b::Z80S s = base;
        s.a = a;
        z80b::z_step(s, op, imm);
        if (a == 0) {
          out0 = s;
          a_first = s.a;
        } else if (s.f != out0.f || s.b != out0.b || s.c != out0.c || s.d != out0.d || s.e != out0.e ||
                   s.h != out0.h || s.l != out0.l || s.sp != out0.sp || s.m != out0.m) {
          return kADepends;
        }
        if (s.a != a) pass = false;
        if (s.a != a_first) over = false;
      }
      if (!pass && !over) return kADepends;
    }
  }
  return pass ? kAPass : (over ? kAOverwrite : kADepends);
}
}  // namespace

const uint8_t* op_aclass() {
  static uint8_t cls[kNumOps];
  static std::once_flag once;
  std::call_once(once, [] {
    for (int op = 0; op < kNumOps; op++) cls[op] = classify_a(uint16_t(op));
  });
  return cls;
}

}  // namespace z80b

// The bit-sliced step on planes that carry dependency sets: a plane word is
// the mask of input fields it was computed from; every logic operation
// unites its operands' sets and a constant has none.
namespace z80b_dep {
using namespace z80b;
struct ZW {
  uint32_t m = 0;
  int id = -1;  // the input plane this word still is, moved only by copies; -1 once computed
  ZW() = default;
  ZW(uint32_t) {}  // a constant depends on nothing
};
inline ZW dep_join(ZW a, ZW b) {
  ZW r;
  r.m = a.m | b.m;
  return r;
}
inline ZW operator~(ZW a) {
  a.id = -1;
  return a;
}
inline ZW operator&(ZW a, ZW b) { return dep_join(a, b); }
inline ZW operator|(ZW a, ZW b) { return dep_join(a, b); }
inline ZW operator^(ZW a, ZW b) { return dep_join(a, b); }
inline ZW& operator&=(ZW& a, ZW b) { return a = dep_join(a, b); }
inline ZW& operator|=(ZW& a, ZW b) { return a = dep_join(a, b); }
inline ZW& operator^=(ZW& a, ZW b) { return a = dep_join(a, b); }
#include "z80_bits_core.cuh"
}  // namespace z80b_dep

namespace z80b {

namespace {
uint8_t g_keeps_a[kNumOps];
uint16_t g_keeps[kNumOps];
}

const uint32_t (*op_deps())[kDepFields] {
  static uint32_t T[kNumOps][kDepFields];
  static std::once_flag once;
  std::call_once(once, [] {
    for (int op = 0; op < kNumOps; op++) {
      z80b_dep::ZB z;
      for (int i = 0; i < 8; i++) {
        z.a[i].m = kRegA;
        z.a[i].id = i;
        z.b[i].id = 8 + i;
        z.c[i].id = 16 + i;
        z.d[i].id = 24 + i;
        z.e[i].id = 32 + i;
        z.h[i].id = 40 + i;
        z.l[i].id = 48 + i;
        z.m[i].id = 56 + i;
        z.f[i].m = 1u << (kDepF0 + i);
        z.b[i].m = kRegB;
        z.c[i].m = kRegC;
        z.d[i].m = kRegD;
        z.e[i].m = kRegE;
        z.h[i].m = kRegH;
        z.l[i].m = kRegL;
        z.m[i].m = kRegM;
      }
      for (int i = 0; i < 16; i++) z.sp[i].m = kRegSP;
      z80b_dep::zb_step(z, uint32_t(op), 0u);
      auto join8 = [](const z80b_dep::ZW (&r)[8]) {
        uint32_t m = 0;
        for (int i = 0; i < 8; i++) m |= r[i].m;
        return m;
      };
      uint32_t* d = T[op];
      for (int g = 0; g < kDepFields; g++) d[g] = 0;
      d[0] = join8(z.a);
      d[2] = join8(z.b);
      d[3] = join8(z.c);
      d[4] = join8(z.d);
      d[5] = join8(z.e);
      d[6] = join8(z.h);
      d[7] = join8(z.l);
      uint32_t sp = 0;
      for (int i = 0; i < 16; i++) sp |= z.sp[i].m;
      d[8] = sp;
      d[9] = join8(z.m);
      for (int k = 0; k < 8; k++) d[kDepF0 + k] = z.f[k].m;
      bool ka = true, kb = true, kc = true, kd = true, ke = true, kh = true, kl = true, km = true;
      for (int i = 0; i < 8; i++) {
        ka = ka && z.a[i].id == i;
        kb = kb && z.b[i].id == 8 + i;
        kc = kc && z.c[i].id == 16 + i;
        kd = kd && z.d[i].id == 24 + i;
        ke = ke && z.e[i].id == 32 + i;
        kh = kh && z.h[i].id == 40 + i;
        kl = kl && z.l[i].id == 48 + i;
        km = km && z.m[i].id == 56 + i;
      }
      g_keeps_a[op] = ka ? 1 : 0;
      g_keeps[op] = uint16_t((ka ? kRegA : 0) | (kb ? kRegB : 0) | (kc ? kRegC : 0) | (kd ? kRegD : 0) |
                             (ke ? kRegE : 0) | (kh ? kRegH : 0) | (kl ? kRegL : 0) | (km ? kRegM : 0));
    }
  });
  return T;
}

const uint8_t* op_keeps_a() {
  (void)op_deps();
  return g_keeps_a;
}

const uint16_t* op_keeps() {
  (void)op_deps();
  return g_keeps;
}

uint32_t seq_keeps(const uint32_t* s, int n) {
  uint32_t k = 0xFFFFu;
  for (int i = 0; i < n; i++) k &= op_keeps()[insn_op(s[i])];
  return k;
}

uint32_t pair_kept_out(const uint32_t* t, int tn, const uint32_t* c, int cn, uint32_t cmp, uint32_t swept) {
  const uint32_t both = seq_keeps(t, tn) & seq_keeps(c, cn) & swept & ~uint32_t(kRegA);
  uint32_t out = 0;
  for (uint32_t b = both; b; b &= b - 1) {
    const uint32_t r = b & (0u - b);
    if (!((seq_relevant(t, tn, cmp & ~r) | seq_relevant(c, cn, cmp & ~r)) & r)) out |= r;
  }
  return out;
}

bool seq_keeps_a(const uint32_t* s, int n) {
  const uint8_t* k = op_keeps_a();
  for (int i = 0; i < n; i++)
    if (!k[insn_op(s[i])]) return false;
  return true;
}

bool pair_a_free(const uint32_t* t, int tn, const uint32_t* c, int cn, uint32_t cmp) {
  const uint32_t rest = seq_relevant(t, tn, cmp & ~uint32_t(kRegA)) | seq_relevant(c, cn, cmp & ~uint32_t(kRegA));
  if (rest & kRegA) return false;
  const bool t_ok = !(seq_relevant(t, tn, kRegA) & kRegA) || seq_keeps_a(t, tn);
  const bool c_ok = !(seq_relevant(c, cn, kRegA) & kRegA) || seq_keeps_a(c, cn);
  return t_ok && c_ok;
}

uint32_t seq_relevant(const uint32_t* s, int n, uint32_t out) {
  const uint32_t (*D)[kDepFields] = op_deps();
  for (int i = n - 1; i >= 0; i--) {
    const uint32_t* d = D[insn_op(s[i])];
    uint32_t in = 0;
    for (uint32_t o = out; o; o &= o - 1) in |= d[__builtin_ctz(o)];
    out = in;
  }
  return out;
}

uint32_t seq_aflow(const uint32_t* s, int n) {
  const uint8_t* c = op_aclass();
  bool a_is_x = true;
  for (int i = 0; i < n; i++) {
    const uint8_t k = c[insn_op(s[i])];
    if (k == kADepends && a_is_x) return 0;
    if (k == kAOverwrite) a_is_x = false;
  }
  return a_is_x ? 3u : 1u;
}
const char* op_mnemonic(uint16_t op) { return tables().cat[op].mnem.c_str(); }

uint8_t op_regs(uint16_t op) {
  static const char* kRegs = "BCDEHL";
  const std::string& m = tables().cat[op].mnem;
  uint8_t r = 0;
  int depth = 0;
  for (size_t i = 0; i < m.size(); i++) {
    const char ch = m[i];
    if (ch == '(') {
      depth++;
      r |= 0x40;  // a memory operand
      continue;
    }
    if (ch == ')') {
      depth--;
      continue;
    }
    const bool word_start = i == 0 || m[i - 1] == ' ' || m[i - 1] == ',';
    if (depth != 0 || !word_start) continue;
    size_t j = i;
    while (j < m.size() && m[j] != ',' && m[j] != ' ') j++;
    const std::string w = m.substr(i, j - i);
    if (w == "SP") r |= 0x80;
    else if (w == "BC") r |= 0x03;
    else if (w == "DE") r |= 0x0C;
    else if (w == "HL") r |= 0x30;
    else if (w.size() == 1 && std::strchr(kRegs, w[0])) r |= uint8_t(1u << (std::strchr(kRegs, w[0]) - kRegs));
  }
  return r;
}

bool compact_map(const uint32_t* t, int tn, const uint32_t* c, int cn, uint8_t (&map)[6], uint32_t* tw,
                 uint32_t* cw) {
  uint8_t fp = 0;
  for (int i = 0; i < tn; i++) fp |= op_regs(insn_op(t[i]));
  for (int i = 0; i < cn; i++) fp |= op_regs(insn_op(c[i]));
  if (fp & 0xC0) return false;  // SP or the memory byte
  if (__builtin_popcount(fp) > 2) return false;
  // a register pair that an instruction uses as one has both halves in the
  // set; they land on B and C in order, so the pair becomes BC
  compact_set_map(fp, map);
  for (int i = 0; i < tn; i++) {
    const int o = op_rename(insn_op(t[i]), map);
    if (o < 0) return false;
    tw[i] = insn(uint16_t(o), insn_imm(t[i]));
  }
  for (int i = 0; i < cn; i++) {
    const int o = op_rename(insn_op(c[i]), map);
    if (o < 0) return false;
    cw[i] = insn(uint16_t(o), insn_imm(c[i]));
  }
  return true;
}

void compact_set_map(uint8_t set, uint8_t (&map)[6]) {
  int target[6] = {-1, -1, -1, -1, -1, -1};
  if ((set & 0x03u) == set) {
    for (int r = 0; r < 6; r++) target[r] = r;  // already in B, C
  } else {
    int k = 0;
    for (int r = 0; r < 6; r++)
      if (set & (1u << r)) target[r] = k++;  // in order onto B, C (a pair's halves onto B, C)
  }
  bool used[6] = {false, false, false, false, false, false};
  for (int r = 0; r < 6; r++)
    if (target[r] >= 0) used[target[r]] = true;
  for (int r = 0; r < 6; r++)
    if (target[r] < 0)
      for (int d = 0; d < 6; d++)
        if (!used[d]) {
          target[r] = d;
          used[d] = true;
          break;
        }
  for (int r = 0; r < 6; r++) map[r] = uint8_t(target[r]);
}

const CompactTables& compact_tables() {
  static CompactTables T;
  static std::once_flag once;
  std::call_once(once, [] {
    std::memset(T.id_of_set, 0, sizeof T.id_of_set);
    int e = 0;
    for (uint32_t set = 0; set < 64; set++) {
      if (__builtin_popcount(set) > 2) continue;
      T.id_of_set[set] = uint8_t(e + 1);
      uint8_t map[6];
      compact_set_map(uint8_t(set), map);
      for (int op = 0; op < kNumOps; op++) T.ren[e][op] = int16_t(op_rename(uint16_t(op), map));
      for (int slot = 0; slot < 2; slot++) {
        T.orig[e][slot] = -1;
        for (int r = 0; r < 6; r++)
          if ((set & (1u << r)) && map[r] == slot) T.orig[e][slot] = int8_t(r);
      }
      e++;
    }
    for (int op = 0; op < kNumOps; op++) T.opregs[op] = op_regs(uint16_t(op));
  });
  return T;
}

void wide_set_map(uint8_t set, uint8_t (&map)[6]) {
  // places B, C, H, L (0, 1, 4, 5); pairs BC, DE, HL are groups 0, 1, 2
  int target[6] = {-1, -1, -1, -1, -1, -1};
  bool used[6] = {false, false, false, false, false, false};
  auto full = [&](int g) { return ((set >> (2 * g)) & 3u) == 3u; };
  // register pairs (both halves named) onto BC or HL, their own first
  for (int g : {0, 2, 1}) {
    if (!full(g)) continue;
    int slot = -1;
    if (g != 1 && !used[2 * g]) slot = 2 * g;
    else if (!used[0]) slot = 0;
    else if (!used[4]) slot = 4;
    if (slot < 0) continue;  // three pairs: more than four registers
    target[2 * g] = slot;
    target[2 * g + 1] = slot + 1;
    used[slot] = used[slot + 1] = true;
  }
  // single registers: their own place if it is B, C, H or L and free, else
  // the first free of those
  static const int kPlaces[4] = {0, 1, 4, 5};
  for (int r = 0; r < 6; r++) {
    if (!(set & (1u << r)) || target[r] >= 0) continue;
    if ((r < 2 || r > 3) && !used[r]) {
      target[r] = r;
      used[r] = true;
      continue;
    }
    for (int p : kPlaces)
      if (!used[p]) {
        target[r] = p;
        used[p] = true;
        break;
      }
  }
  // the registers outside the set take the places left, in order
  for (int r = 0; r < 6; r++)
    if (target[r] < 0)
      for (int d = 0; d < 6; d++)
        if (!used[d]) {
          target[r] = d;
          used[d] = true;
          break;
        }
  for (int r = 0; r < 6; r++) map[r] = uint8_t(target[r]);
}

bool wide_map(const uint32_t* t, int tn, const uint32_t* c, int cn, uint8_t (&map)[6], uint32_t* tw, uint32_t* cw) {
  uint8_t fp = 0;
  for (int i = 0; i < tn; i++) fp |= op_regs(insn_op(t[i]));
  for (int i = 0; i < cn; i++) fp |= op_regs(insn_op(c[i]));
  if (fp & 0x80) return false;  // SP
  if (__builtin_popcount(fp & 0x3Fu) > 4) return false;
  wide_set_map(uint8_t(fp & 0x3Fu), map);
  for (int i = 0; i < tn; i++) {
    const int o = op_rename(insn_op(t[i]), map);
    if (o < 0) return false;
    tw[i] = insn(uint16_t(o), insn_imm(t[i]));
  }
  for (int i = 0; i < cn; i++) {
    const int o = op_rename(insn_op(c[i]), map);
    if (o < 0) return false;
    cw[i] = insn(uint16_t(o), insn_imm(c[i]));
  }
  return true;
}

const WideTables& wide_tables() {
  static WideTables T;
  static std::once_flag once;
  std::call_once(once, [] {
    std::memset(T.id_of_set, 0, sizeof T.id_of_set);
    static const int kPlaces[4] = {0, 1, 4, 5};
    int e = 0;
    for (uint32_t set = 0; set < 64; set++) {
      if (__builtin_popcount(set) > 4) continue;
      T.id_of_set[set] = uint8_t(e + 1);
      uint8_t map[6];
      wide_set_map(uint8_t(set), map);
      for (int op = 0; op < kNumOps; op++) T.ren[e][op] = int16_t(op_rename(uint16_t(op), map));
      for (int s = 0; s < 4; s++) {
        T.orig[e][s] = -1;
        for (int r = 0; r < 6; r++)
          if ((set & (1u << r)) && map[r] == kPlaces[s]) T.orig[e][s] = int8_t(r);
      }
      e++;
    }
  });
  return T;
}

int op_rename(uint16_t op, const uint8_t (&map)[6]) {
  static const char* kRegs = "BCDEHL";
  static const char* kPairs[3] = {"BC", "DE", "HL"};
  const std::string& m = tables().cat[op].mnem;
  std::string out;
  int depth = 0;
  for (size_t i = 0; i < m.size(); i++) {
    const char ch = m[i];
    if (ch == '(') depth++;
    if (ch == ')') depth--;
    const bool word_start = i == 0 || m[i - 1] == ' ' || m[i - 1] == ',';
    if (depth == 0 && word_start) {
      // a register pair operand
      bool done = false;
      for (int p = 0; p < 3 && !done; p++) {
        if (m.compare(i, 2, kPairs[p]) == 0 && (i + 2 == m.size() || m[i + 2] == ',' || m[i + 2] == ' ')) {
          const uint8_t hi = map[2 * p], lo = map[2 * p + 1];
          if (hi % 2 != 0 || lo != hi + 1) return -1;  // not onto a pair in order
          out += kPairs[hi / 2];
          i += 1;
          done = true;
        }
      }
      if (done) continue;
      // an 8-bit register operand (mnemonic words like "SLA" are longer)
      const char* r = std::strchr(kRegs, ch);
      if (r && *r && (i + 1 == m.size() || m[i + 1] == ',' || m[i + 1] == ' ')) {
        out += kRegs[map[r - kRegs]];
        continue;
      }
    }
    out += ch;
  }
  if (out == m) return op;
  for (int o = 0; o < kNumOps; o++)
    if (tables().cat[o].mnem == out && op_table()[o].imm == op_table()[op].imm) return o;
  return -1;
}
const uint8_t* op_encoding(uint16_t op, int* n) {
  *n = tables().cat[op].nenc;
  return tables().cat[op].enc;
}
const std::vector<uint32_t>& pool8() { return tables().pool; }

std::vector<uint32_t> first_op_pool() {
  std::vector<uint32_t> v = pool8();
  for (int o = 0; o < kNumOps; o++)
    if (op_table()[o].imm == 2)
      for (int x = 0; x < 65536; x++) v.push_back(insn(uint16_t(o), uint16_t(x)));
  return v;
}

std::string disassemble(uint32_t w) {
  uint16_t op = insn_op(w), imm = insn_imm(w);
  const std::string& m = tables().cat[op].mnem;
  const int kind = op_table()[op].imm;
  if (kind == 0) return m;
  std::string out;
  for (size_t i = 0; i < m.size(); i++) {
    if (kind == 2 && i + 1 < m.size() && m[i] == 'n' && m[i + 1] == 'n') {
      hex2(out, imm, 4);
      i++;
    } else if (kind == 1 && m[i] == 'n' && (i + 1 == m.size() || m[i + 1] == ' ' || m[i + 1] == ',')) {
      hex2(out, imm & 0xFFu, 2);
    } else {
      out += m[i];
    }
  }
  return out;
}

std::string disasm_seq(const uint32_t* seq, int n) {
  std::string s;
  for (int i = 0; i < n; i++) {
    if (i) s += " : ";
    s += disassemble(seq[i]);
  }
  return s;
}

bool should_prune(const uint32_t* seq, int n) {
  const OpInfo* T = op_table();
  for (int i = 0; i < n; i++) {
    if (T[insn_op(seq[i])].nopish) return true;  // NOP and LD r,r
    if (i + 1 < n) {
      const OpInfo& x = T[insn_op(seq[i])];
      const OpInfo& y = T[insn_op(seq[i + 1])];
      // dead write: written by both, not read by the second, flags excluded
      if (x.writes && (x.writes & y.writes & ~kRegF & ~y.reads)) return true;
    }
  }
  for (int i = 0; i + 1 < n; i++) {
    const OpInfo& x = T[insn_op(seq[i])];
    const OpInfo& y = T[insn_op(seq[i + 1])];
    bool indep = !((x.writes & y.reads) || (x.reads & y.writes) || (x.writes & y.writes));
    // canonical order key op<<16|imm (pruner.go:254-256) -- the packed word
    // with its halves swapped
    uint32_t kx = (uint32_t(insn_op(seq[i])) << 16) | insn_imm(seq[i]);
    uint32_t ky = (uint32_t(insn_op(seq[i + 1])) << 16) | insn_imm(seq[i + 1]);
    if (indep && kx > ky) return true;
  }
  return false;
}

uint16_t seq_reads(const uint32_t* s, int n) {
  uint16_t m = 0;
  for (int i = 0; i < n; i++) m |= op_table()[insn_op(s[i])].reads;
  return m;
}

Sweep sweep_for(uint16_t reads) {
  Sweep w{};
  const uint16_t order[7] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM};
  for (int i = 0; i < 7; i++)
    if (reads & order[i]) w.regs[w.nextra++] = uint8_t(i);
  w.sp = (reads & kRegSP) != 0;
  if (w.nextra == 0 && !w.sp) {
    w.kind = 0;
    w.states = 512;
  } else if (w.nextra <= 2 && !w.sp) {
    w.kind = 1;
    w.states = 512ull << (8 * w.nextra);
  } else {
    w.kind = 2;
    w.states = (512ull << (5 * w.nextra)) * (w.sp ? 16 : 1);
  }
  if (w.kind != 2) w.sp = false;
  return w;
}

std::string dead_flag_desc(uint8_t mask) {
  if (mask == 0) return "";
  if (mask == 0xFF) return "all";
  if (mask == 0x28) return "undoc";
  static const char* const nm[8] = {"C", "N", "P/V", "X3", "H", "X5", "Z", "S"};
  std::string s;
  for (int b = 0; b < 8; b++)
    if (mask >> b & 1) {
      if (!s.empty()) s += ',';
      s += nm[b];
    }
  return s;
}

namespace {
std::string up(std::string s) {
  for (auto& c : s) c = char(std::toupper((unsigned char)c));
  return s;
}
std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}
// fmt.Sscanf-style integer: optional sign, longest digit run, >= 1 digit.
bool scan(const std::string& s, int base, long* v) {
  size_t i = 0;
  bool neg = false;
  if (i < s.size() && (s[i] == '-' || s[i] == '+')) neg = s[i++] == '-';
  size_t st = i;
  long x = 0;
  for (; i < s.size(); i++) {
    int d = std::isdigit((unsigned char)s[i]) ? s[i] - '0'
            : (base == 16 && std::isxdigit((unsigned char)s[i])) ? (std::toupper((unsigned char)s[i]) - 'A' + 10)
            : -1;
    if (d < 0) break;
    x = x * base + d;
  }
  if (i == st) return false;
  *v = neg ? -x : x;
  return true;
}
bool parse_imm(std::string s, long* v) {
  s = trim(s);
  if (s.empty()) return false;
  if (s.size() >= 2 && s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) return scan(s.substr(2), 16, v);
  if (std::toupper((unsigned char)s.back()) == 'H') return scan(s.substr(0, s.size() - 1), 16, v);
  return scan(s, 10, v);
}
bool parse_one(const std::string& text0, uint32_t* out) {
  std::string text = trim(text0), U = up(text);
  for (int op = 0; op < kNumOps; op++) {
    const std::string& m = tables().cat[op].mnem;
    if (op_table()[op].imm == 0) {
      if (up(m) == U) {
        *out = insn(uint16_t(op));
        return true;
      }
      continue;
    }
    std::string pat = up(m);
    size_t n = pat.rfind('N');
    std::string pre = pat.substr(0, n), suf = pat.substr(n + 1);
    if (U.size() < pre.size() || U.compare(0, pre.size(), pre) != 0) continue;
    if (!suf.empty() && (U.size() < suf.size() || U.compare(U.size() - suf.size(), suf.size(), suf) != 0)) continue;
    std::string val = U.substr(pre.size());
    if (!suf.empty()) {
      if (val.size() < suf.size()) continue;
      val.resize(val.size() - suf.size());
    }
    long v;
    if (!parse_imm(val, &v)) continue;
    *out = insn(uint16_t(op), uint16_t(v));
    return true;
  }
  return false;
}
}  // namespace

bool parse_dead_flags(const std::string& in, uint8_t* out) {
  std::string s;
  for (char c : in) s += char(std::tolower((unsigned char)c));
  if (s.empty() || s == "none") { *out = 0x00; return true; }
  if (s == "undoc") { *out = 0x28; return true; }
  if (s == "all") { *out = 0xFF; return true; }
  if (s.compare(0, 2, "0x") == 0) s = s.substr(2);
  if (s.empty()) return false;
  unsigned v = 0;
  for (char c : s) {
    if (!std::isxdigit((unsigned char)c)) return false;
    v = v * 16 + unsigned(std::isdigit((unsigned char)c) ? c - '0' : c - 'a' + 10);
    if (v > 0xFF) return false;
  }
  *out = uint8_t(v);
  return true;
}

bool parse_assembly(const std::string& text, std::vector<uint32_t>* out) {
  out->clear();
  size_t st = 0;
  for (;;) {
    size_t p = text.find(':', st);
    std::string part = trim(text.substr(st, p == std::string::npos ? std::string::npos : p - st));
    if (!part.empty()) {
      uint32_t w;
      if (!parse_one(part, &w)) return false;
      out->push_back(w);
    }
    if (p == std::string::npos) break;
    st = p + 1;
  }
  return !out->empty();
}

}  // namespace z80b

namespace z80b {
namespace {
struct V {
  uint8_t a, f, b, c, d, e, h, l;
  uint16_t sp;
  uint8_t m;
};
// verifier.go:35-72; the first 8 rows are the QuickCheck vectors (19-28).
const V kVec[32] = {
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
uint32_t g_vec[32][3];
const uint8_t kRep[32] = {0x00, 0x01, 0x02, 0x0F, 0x10, 0x1F, 0x20, 0x3F, 0x40, 0x55, 0x7E,
                          0x7F, 0x80, 0x81, 0xAA, 0xBF, 0xC0, 0xD5, 0xE0, 0xEF, 0xF0, 0xF7,
                          0xFE, 0xFF, 0x03, 0x07, 0x11, 0x33, 0x77, 0xBB, 0xDD, 0xEE};
const uint16_t kRepSP[16] = {0x0000, 0x0001, 0x00FF, 0x0100, 0x7FFE, 0x7FFF, 0x8000, 0x8001,
                             0xFFFE, 0xFFFF, 0x1234, 0x5678, 0xABCD, 0xDEAD, 0xBEEF, 0xCAFE};
std::once_flag g_vec_once;
void pack_vectors() {
  for (int i = 0; i < 32; i++) {
    const V& v = kVec[i];
    g_vec[i][0] = uint32_t(v.a) | uint32_t(v.f) << 8 | uint32_t(v.b) << 16 | uint32_t(v.c) << 24;
    g_vec[i][1] = uint32_t(v.d) | uint32_t(v.e) << 8 | uint32_t(v.h) << 16 | uint32_t(v.l) << 24;
    g_vec[i][2] = uint32_t(v.sp) | uint32_t(v.m) << 16;
  }
}
}  // namespace

const uint32_t (*qc_vectors())[3] {
  std::call_once(g_vec_once, pack_vectors);
  return g_vec;
}
const uint32_t (*mid_vectors())[3] {
  std::call_once(g_vec_once, pack_vectors);
  return g_vec;
}
const uint8_t* rep_values() { return kRep; }
const uint16_t* rep_sp() { return kRepSP; }

}  // namespace z80b
