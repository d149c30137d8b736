// Host check of the compact-state mapping (op_regs, compact_map in
// z80_tables.cpp).  (1) op_regs is sound: a register or the memory byte an
// instruction does not name keeps its value and changes no other output,
// for every opcode, every value of that field and sampled states and
// immediates (oracle's Exec).  (2) For random pairs that compact_map
// accepts, running the renamed programs on the renamed states over the
// reference's whole ExhaustiveCheck sweep, comparing A, F (under the dead
// flags) and the registers B, C only, gives the oracle's verdict for the
// original pair.  (3) The bit-sliced step on the compact states (ZBc: A, F,
// B, C and shared scratch; ZB4: A, F, B, C with its own step zb4_step)
// gives the full state's A, F, B and C for every opcode that names no
// register but B and C.  (4) The device's tables
// (compact_tables) accept, rename and place registers as compact_map does.
// (5), (6) The compact kernel's sweep units (A-dependent pairs, and
// A-independent pairs at A = 0 and 1 with 32 blocks per state word),
// restated with their plane layouts and their dead-flag and dead-register
// compares, give the oracle's verdicts.  Built
// and run by tests/test_tables.py.
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_bits.cuh"
#include "../../z80-optimizer_b200/csrc/z80_exec.cuh"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

using namespace z80b;

static uint8_t* field(orc::State& s, int i) {
  switch (i) {
    case 0: return &s.B;
    case 1: return &s.C;
    case 2: return &s.D;
    case 3: return &s.E;
    case 4: return &s.H;
    case 5: return &s.L;
    default: return &s.M;
  }
}

// the reference sweep's states of a read mask, in block order, all A values
struct Shape {
  bool spw, reduced;
  int nx, fw, slot[7];
  uint64_t nblocks;
};
static Shape shape_of(uint16_t reads) {
  Shape s{};
  const uint32_t bits[7] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM};
  int k = 0;
  for (int r = 0; r < 7; r++) s.slot[r] = (reads & bits[r]) ? k++ : -1;
  s.nx = k;
  s.spw = (reads & kRegSP) != 0;
  s.reduced = s.spw || s.nx > 2;
  s.fw = s.reduced ? 5 : 8;
  s.nblocks = sweep_for(reads).states / 256;
  return s;
}
static Z80S decode(uint64_t ab, const Shape& s) {
  const uint8_t* rep = rep_values();
  const uint16_t* repsp = rep_sp();
  uint64_t rest = ab;
  uint32_t sp = 0;
  if (s.spw) {
    sp = repsp[rest & 15];
    rest >>= 4;
  }
  uint32_t fv[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int f = 6; f >= 0; f--)
    if (f < s.nx) {
      const uint32_t x = uint32_t(rest) & (s.reduced ? 31u : 255u);
      fv[f] = s.reduced ? rep[x] : x;
      rest >>= s.fw;
    }
  uint32_t rv[7];
  for (int r = 0; r < 7; r++) rv[r] = s.slot[r] >= 0 ? fv[s.slot[r]] : 0;
  return Z80S{0, uint32_t(rest & 1), rv[0], rv[1], rv[2], rv[3], rv[4], rv[5], sp, rv[6]};
}
static uint32_t* zreg(Z80S& s, int r) {
  switch (r) {
    case 0: return &s.b;
    case 1: return &s.c;
    case 2: return &s.d;
    case 3: return &s.e;
    case 4: return &s.h;
    default: return &s.l;
  }
}

int main() {
  orc::Init();
  std::mt19937_64 rng(31);
  // (1) soundness of op_regs
  for (int op = 0; op < orc::OpCodeCount; op++) {
    const uint8_t named = op_regs(uint16_t(op));
    const bool imm16 = orc::HasImm16(uint16_t(op));
    for (int fld = 0; fld < 8; fld++) {  // B..L, M (6), SP (7)
      const uint8_t bit = fld < 6 ? uint8_t(1u << fld) : (fld == 6 ? 0x40 : 0x80);
      if (named & bit) continue;
      for (int k = 0; k < 24; k++) {
        const uint64_t r = rng(), r2 = rng();
        orc::State s{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                     uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2), uint8_t(r2 >> 16)};
        const uint16_t imm = imm16 ? uint16_t(rng()) : uint16_t(rng() & 0xFF);
        orc::State base = s;
        orc::Exec(base, uint16_t(op), imm);
        for (int v = 0; v < 256; v++) {
          orc::State t = s;
          if (fld == 7) t.SP = uint16_t((rng() & 0xFF00) | v);
          else *field(t, fld) = uint8_t(v);
          const orc::State in = t;
          orc::Exec(t, uint16_t(op), imm);
          // the field keeps its value and the others match the base run
          orc::State u = t, b2 = base;
          if (fld == 7) {
            if (t.SP != in.SP) goto bad;
            u.SP = b2.SP = 0;
          } else {
            if (*field(t, fld) != *field(const_cast<orc::State&>(in), fld)) goto bad;
            *field(u, fld) = *field(b2, fld) = 0;
          }
          if (u != b2) goto bad;
          continue;
        bad:
          std::printf("op %d (%s) uses field %d that it does not name\n", op, op_mnemonic(uint16_t(op)), fld);
          return 1;
        }
      }
    }
  }
  // (2) verdicts of compact pairs over the reference sweep
  const auto& I = orc::Instructions8();
  int pairs = 0, equal = 0, renamed = 0;
  for (int trial = 0; trial < 2000000 && pairs < 600; trial++) {
    const int tn = 1 + int(rng() % 2);
    int cn = 1 + int(rng() % 2);
    orc::Instruction ti[2], ci[2];
    uint32_t tw[2], cw[2], tr[2], cr[2];
    for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
    for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
    if (rng() % 3 == 0) {  // the target itself or swapped: equivalences
      cn = tn;
      ci[0] = ti[tn == 2 && (rng() & 1) ? 1 : 0];
      if (tn == 2) ci[1] = ti[ci[0].op == ti[0].op && ci[0].imm == ti[0].imm ? 1 : 0];
    }
    for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
    for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
    uint8_t map[6];
    if (!compact_map(tw, tn, cw, cn, map, tr, cr)) continue;
    const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn));
    const Shape s = shape_of(reads);
    if (s.nblocks > 512) continue;
    pairs++;
    bool moved = false;
    for (int r = 0; r < 6; r++) moved = moved || map[r] != r;
    renamed += moved ? 1 : 0;
    for (uint8_t dead : {uint8_t(0x00), uint8_t(0xFF)}) {
      bool eq = true;
      for (uint64_t b = 0; b < s.nblocks && eq; b++) {
        const Z80S x = decode(b, s);
        for (uint32_t a = 0; a < 256 && eq; a++) {
          Z80S y = x;
          y.a = a;
          Z80S p = y;  // renamed state: register r's value in register map[r]
          for (int r = 0; r < 6; r++) *zreg(p, map[r]) = *zreg(y, r);
          Z80S pt = p, pc = p;
          for (int i = 0; i < tn; i++) z_step(pt, insn_op(tr[i]), insn_imm(tr[i]));
          for (int i = 0; i < cn; i++) z_step(pc, insn_op(cr[i]), insn_imm(cr[i]));
          const uint32_t keepF = uint8_t(~dead);
          eq = pt.a == pc.a && ((pt.f ^ pc.f) & keepF) == 0 && pt.b == pc.b && pt.c == pc.c;
        }
      }
      const bool want = dead ? orc::ExhaustiveCheckMasked(ti, tn, ci, cn, dead) : orc::ExhaustiveCheck(ti, tn, ci, cn);
      if (want != eq) {
        std::printf("compact verdict differs: target %08x %08x (%d) candidate %08x %08x (%d) dead %02x oracle %d\n",
                    tw[0], tn > 1 ? tw[1] : 0, tn, cw[0], cn > 1 ? cw[1] : 0, cn, dead, want ? 1 : 0);
        return 1;
      }
      equal += want ? 1 : 0;
    }
  }
  // (3) the compact bit-sliced step
  int compact_ops = 0;
  for (uint32_t op = 0; op < uint32_t(kNumOps); op++) {
    if (op_regs(uint16_t(op)) & ~0x03u) continue;
    compact_ops++;
    for (int rep = 0; rep < 32; rep++) {
      Z80S st[32];
      for (int j = 0; j < 32; j++) {
        const uint64_t r = rng();
        st[j] = Z80S{uint32_t(r & 0xFF), uint32_t((r >> 8) & 0xFF), uint32_t((r >> 16) & 0xFF),
                     uint32_t((r >> 24) & 0xFF), 0, 0, 0, 0, 0, 0};
      }
      const uint32_t imm = uint32_t(rng() & 0xFFFF);
      ZB full;
      zb_from(full, st);
      ZBc cz;
      for (int i = 0; i < 8; i++) {
        cz.a[i] = full.a[i];
        cz.f[i] = full.f[i];
        cz.b[i] = full.b[i];
        cz.c[i] = full.c[i];
        cz.x[i] = 0;
      }
      for (int i = 0; i < 16; i++) cz.sp[i] = 0;
      ZB4 z4;
      for (int i = 0; i < 8; i++) {
        z4.a[i] = full.a[i];
        z4.f[i] = full.f[i];
        z4.b[i] = full.b[i];
        z4.c[i] = full.c[i];
      }
      zb_step(full, op, imm);
      zb_step(cz, op, imm);
      zb4_step(z4, op, imm);
      for (int i = 0; i < 8; i++)
        if (cz.a[i] != full.a[i] || cz.f[i] != full.f[i] || cz.b[i] != full.b[i] || cz.c[i] != full.c[i]) {
          std::printf("compact step differs on op %u (%s)\n", op, op_mnemonic(uint16_t(op)));
          return 1;
        }
      for (int i = 0; i < 8; i++)
        if (z4.a[i] != full.a[i] || z4.f[i] != full.f[i] || z4.b[i] != full.b[i] || z4.c[i] != full.c[i]) {
          std::printf("A/F/B/C step differs on op %u (%s)\n", op, op_mnemonic(uint16_t(op)));
          return 1;
        }
    }
  }
  // (4) the device's tables (compact_tables) decide and rename as
  // compact_map does
  {
    const CompactTables& T = compact_tables();
    int agreed = 0;
    for (int trial = 0; trial < 200000; trial++) {
      const int tn = 1 + int(rng() % 3), cn = 1 + int(rng() % 2);
      uint32_t tw[3], cw[2], tr[3], cr[2];
      for (int i = 0; i < tn; i++) {
        const auto& x = I[rng() % I.size()];
        tw[i] = uint32_t(x.op) | uint32_t(x.imm) << 16;
      }
      for (int i = 0; i < cn; i++) {
        const auto& x = I[rng() % I.size()];
        cw[i] = uint32_t(x.op) | uint32_t(x.imm) << 16;
      }
      uint8_t map[6];
      const bool by_map = compact_map(tw, tn, cw, cn, map, tr, cr);
      uint8_t fp = 0;
      for (int i = 0; i < tn; i++) fp |= T.opregs[insn_op(tw[i])];
      for (int i = 0; i < cn; i++) fp |= T.opregs[insn_op(cw[i])];
      const int id = (fp & 0xC0) ? 0 : T.id_of_set[fp & 0x3F];
      bool by_table = id != 0;
      for (int i = 0; i < tn && by_table; i++) by_table = T.ren[id - 1][insn_op(tw[i])] >= 0;
      for (int i = 0; i < cn && by_table; i++) by_table = T.ren[id - 1][insn_op(cw[i])] >= 0;
      if (by_map != by_table) {
        std::printf("compact tables disagree with compact_map (%d vs %d)\n", by_table, by_map);
        return 1;
      }
      if (!by_map) continue;
      agreed++;
      for (int i = 0; i < tn; i++)
        if (uint32_t(T.ren[id - 1][insn_op(tw[i])]) != insn_op(tr[i])) {
          std::printf("compact table renames differently\n");
          return 1;
        }
      for (int i = 0; i < cn; i++)
        if (uint32_t(T.ren[id - 1][insn_op(cw[i])]) != insn_op(cr[i])) {
          std::printf("compact table renames differently\n");
          return 1;
        }
      for (int slot = 0; slot < 2; slot++) {
        int want = -1;
        for (int r = 0; r < 6; r++)
          if ((fp & (1u << r)) && map[r] == slot) want = r;
        if (T.orig[id - 1][slot] != want) {
          std::printf("compact table origin differs\n");
          return 1;
        }
      }
    }
    if (agreed < 1000) {
      std::printf("too few compact pairs for the table check (%d)\n", agreed);
      return 1;
    }
  }
  // (5) the compact kernel's unit restated (cbits_unit in z80b_kernels.cu):
  // per block and 32 values of A, the compact planes from the decoded state
  // (B, C from the registers they stand for, 0 where none), renamed
  // programs, A / F under the dead flags / B, C under the dead registers of
  // the registers they stand for; against the oracle with dead registers
  {
    const CompactTables& T = compact_tables();
    int cp = 0, ceq = 0;
    for (int trial = 0; trial < 2000000 && cp < 400; trial++) {
      const int tn = 1 + int(rng() % 2);
      int cn = 1 + int(rng() % 2);
      orc::Instruction ti[2], ci[2];
      uint32_t tw[2], cw[2];
      for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
      for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
      if (rng() % 3 == 0) {
        ci[0] = ti[0];
        cn = 1;
      }
      for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
      for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
      if (seq_aflow(tw, tn) && seq_aflow(cw, cn)) continue;  // the compact class takes A-dependent pairs
      uint8_t fp = 0;
      for (int i = 0; i < tn; i++) fp |= T.opregs[insn_op(tw[i])];
      for (int i = 0; i < cn; i++) fp |= T.opregs[insn_op(cw[i])];
      const int id = (fp & 0xC0) ? 0 : T.id_of_set[fp & 0x3F];
      bool ok = id != 0;
      for (int i = 0; i < tn && ok; i++) ok = T.ren[id - 1][insn_op(tw[i])] >= 0;
      for (int i = 0; i < cn && ok; i++) ok = T.ren[id - 1][insn_op(cw[i])] >= 0;
      if (!ok) continue;
      const Shape s = shape_of(uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn)));
      if (s.nblocks > 512) continue;
      cp++;
      uint32_t tr[2], cr[2];
      for (int i = 0; i < tn; i++) tr[i] = uint32_t(uint16_t(T.ren[id - 1][insn_op(tw[i])])) | (tw[i] & 0xFFFF0000u);
      for (int i = 0; i < cn; i++) cr[i] = uint32_t(uint16_t(T.ren[id - 1][insn_op(cw[i])])) | (cw[i] & 0xFFFF0000u);
      const int o0 = T.orig[id - 1][0], o1 = T.orig[id - 1][1];
      const uint8_t dead = uint8_t(rng() & 0xFF), dregs = uint8_t(rng() & 0x3F);
      const uint32_t keepF = uint8_t(~dead), keepR = ~uint32_t(dregs) & 0x3Fu;
      const bool cmp_b = o0 >= 0 && ((keepR >> o0) & 1u), cmp_c = o1 >= 0 && ((keepR >> o1) & 1u);
      bool bad = false;
      const CDec dec = cdec_make(s.nx, s.slot, o0, o1);
      for (uint64_t b = 0; b < s.nblocks && !bad; b++) {
        const Z80S x = decode(b, s);
        const uint32_t regs[6] = {x.b, x.c, x.d, x.e, x.h, x.l};
        {
          // the kernel's shift-and-mask decoding of B, C and the carry
          uint32_t vb, vc, carry;
          cdec_vals(dec, b, vb, vc, carry);
          if (vb != (o0 >= 0 ? regs[o0] : 0u) || vc != (o1 >= 0 ? regs[o1] : 0u) || carry != x.f) {
            std::printf("compact block decoding differs at block %llu\n", (unsigned long long)b);
            return 1;
          }
        }
        for (uint32_t a0 = 0; a0 < 256 && !bad; a0 += 32) {
          ZB4 z;
          z.a[0] = 0xAAAAAAAAu;
          z.a[1] = 0xCCCCCCCCu;
          z.a[2] = 0xF0F0F0F0u;
          z.a[3] = 0xFF00FF00u;
          z.a[4] = 0xFFFF0000u;
          for (int i = 5; i < 8; i++) z.a[i] = ((a0 >> i) & 1u) ? kZBOnes : 0u;
          zb_set8(z.f, x.f);
          zb_set8(z.b, o0 >= 0 ? regs[o0] : 0u);
          zb_set8(z.c, o1 >= 0 ? regs[o1] : 0u);
          ZB4 zc = z, zt = z;
          for (int i = 0; i < cn; i++) zb4_step(zc, insn_op(cr[i]), insn_imm(cr[i]));
          for (int i = 0; i < tn; i++) zb4_step(zt, insn_op(tr[i]), insn_imm(tr[i]));
          uint32_t d = 0;
          for (int i = 0; i < 8; i++) {
            d |= zc.a[i] ^ zt.a[i];
            if ((keepF >> i) & 1u) d |= zc.f[i] ^ zt.f[i];
            if (cmp_b) d |= zc.b[i] ^ zt.b[i];
            if (cmp_c) d |= zc.c[i] ^ zt.c[i];
          }
          bad = d != 0;
        }
      }
      const bool want = orc::ExhaustiveCheckMaskedRegs(ti, tn, ci, cn, dead, dregs);
      if (want == bad) {
        std::printf("compact unit verdict differs: target %08x %08x (%d) candidate %08x %08x (%d) dead %02x regs %02x\n",
                    tw[0], tn > 1 ? tw[1] : 0, tn, cw[0], cn > 1 ? cw[1] : 0, cn, dead, dregs);
        return 1;
      }
      ceq += want ? 1 : 0;
    }
    if (cp < 200 || ceq < 30) {
      std::printf("too few compact A-dependent pairs (%d) or equivalences (%d)\n", cp, ceq);
      return 1;
    }
  }
  // (6) the compact kernel's A-independent unit restated (cxbits_unit in
  // z80b_kernels.cu): per aligned group of 32 blocks one state word (block j
  // in bit j), the moving field -- the last swept register, renamed onto B
  // or C, or the carry -- as counting planes plus the group's high bits,
  // every other field the group's decoded value; A at 0 and then 1; lanes
  // past the sweep's end masked out; against the oracle with dead registers
  {
    const CompactTables& T = compact_tables();
    int cp = 0, ceq = 0;
    for (int trial = 0; trial < 4000000 && cp < 400; trial++) {
      const int tn = 1 + int(rng() % 2);
      int cn = 1 + int(rng() % 2);
      orc::Instruction ti[2], ci[2];
      uint32_t tw[2], cw[2];
      for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
      for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
      if (rng() % 3 == 0) {
        ci[0] = ti[tn - 1];
        cn = 1;
      }
      for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
      for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
      if (!(seq_aflow(tw, tn) && seq_aflow(cw, cn))) continue;  // A-independent pairs only
      uint8_t fp = 0;
      for (int i = 0; i < tn; i++) fp |= T.opregs[insn_op(tw[i])];
      for (int i = 0; i < cn; i++) fp |= T.opregs[insn_op(cw[i])];
      const int id = (fp & 0xC0) ? 0 : T.id_of_set[fp & 0x3F];
      bool ok = id != 0;
      for (int i = 0; i < tn && ok; i++) ok = T.ren[id - 1][insn_op(tw[i])] >= 0;
      for (int i = 0; i < cn && ok; i++) ok = T.ren[id - 1][insn_op(cw[i])] >= 0;
      if (!ok) continue;
      const Shape s = shape_of(uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn)));
      if (s.spw || s.reduced) {
        std::printf("a compact pair with a reduced or SP sweep\n");
        return 1;
      }
      cp++;
      uint32_t tr[2], cr[2];
      for (int i = 0; i < tn; i++) tr[i] = uint32_t(uint16_t(T.ren[id - 1][insn_op(tw[i])])) | (tw[i] & 0xFFFF0000u);
      for (int i = 0; i < cn; i++) cr[i] = uint32_t(uint16_t(T.ren[id - 1][insn_op(cw[i])])) | (cw[i] & 0xFFFF0000u);
      const int o0 = T.orig[id - 1][0], o1 = T.orig[id - 1][1];
      int rlast = -1;
      for (int r = 0; r < 7; r++)
        if (s.slot[r] == s.nx - 1) rlast = r;
      if (s.nx > 0 && rlast != o0 && rlast != o1) {
        std::printf("the last swept register is neither renamed register\n");
        return 1;
      }
      const uint8_t dead = uint8_t(rng() & 0xFF), dregs = uint8_t(rng() & 0x3F);
      const uint32_t keepF = uint8_t(~dead), keepR = ~uint32_t(dregs) & 0x3Fu;
      const bool cmp_b = o0 >= 0 && ((keepR >> o0) & 1u), cmp_c = o1 >= 0 && ((keepR >> o1) & 1u);
      bool bad = false;
      const CDec dec = cdec_make(s.nx, s.slot, o0, o1);
      for (uint64_t g0 = 0; g0 < s.nblocks && !bad; g0 += 32) {
        const uint32_t valid = s.nblocks - g0 >= 32 ? 0xFFFFFFFFu : ((1u << uint32_t(s.nblocks - g0)) - 1u);
        const Z80S x = decode(g0, s);
        const uint32_t regs[6] = {x.b, x.c, x.d, x.e, x.h, x.l};
        const uint32_t vb = o0 >= 0 ? regs[o0] : 0u, vc = o1 >= 0 ? regs[o1] : 0u;
        {
          uint32_t db, dc, dcarry;
          cdec_vals(dec, g0, db, dc, dcarry);
          if (db != vb || dc != vc || dcarry != x.f) {
            std::printf("compact group decoding differs at block %llu\n", (unsigned long long)g0);
            return 1;
          }
        }
        const uint32_t v = rlast == o0 ? vb : vc;
        uint32_t vp[8] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u, 0, 0, 0};
        for (int i = 5; i < 8; i++) vp[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
        for (uint32_t abit = 0; abit < 2 && !bad; abit++) {
          ZB4 z;
          zb_set8(z.a, abit);
          zb_set8(z.f, x.f);
          zb_set8(z.b, vb);
          zb_set8(z.c, vc);
          if (s.nx == 0) z.f[0] = 0xAAAAAAAAu;
          else if (rlast == o0) zb_copy8(z.b, vp);
          else zb_copy8(z.c, vp);
          ZB4 zc = z, zt = z;
          for (int i = 0; i < cn; i++) zb4_step(zc, insn_op(cr[i]), insn_imm(cr[i]));
          for (int i = 0; i < tn; i++) zb4_step(zt, insn_op(tr[i]), insn_imm(tr[i]));
          uint32_t d = 0;
          for (int i = 0; i < 8; i++) {
            d |= zc.a[i] ^ zt.a[i];
            if ((keepF >> i) & 1u) d |= zc.f[i] ^ zt.f[i];
            if (cmp_b) d |= zc.b[i] ^ zt.b[i];
            if (cmp_c) d |= zc.c[i] ^ zt.c[i];
          }
          bad = (d & valid) != 0;
        }
      }
      const bool want = orc::ExhaustiveCheckMaskedRegs(ti, tn, ci, cn, dead, dregs);
      if (want == bad) {
        std::printf("compact A-independent unit verdict differs: target %08x %08x (%d) candidate %08x %08x (%d) "
                    "dead %02x regs %02x\n",
                    tw[0], tn > 1 ? tw[1] : 0, tn, cw[0], cn > 1 ? cw[1] : 0, cn, dead, dregs);
        return 1;
      }
      ceq += want ? 1 : 0;
    }
    if (cp < 200 || ceq < 30) {
      std::printf("too few compact A-independent pairs (%d) or equivalences (%d)\n", cp, ceq);
      return 1;
    }
  }
  if (compact_ops < 150) {
    std::printf("too few compact opcodes (%d)\n", compact_ops);
    return 1;
  }
  if (pairs < 300 || equal < 50 || renamed < 50) {
    std::printf("too few pairs (%d), equivalences (%d) or renamed pairs (%d)\n", pairs, equal, renamed);
    return 1;
  }
  std::printf("OK %d compact pairs (%d renamed), %d equivalent verdicts, %d opcodes on the compact step\n", pairs,
              renamed, equal, compact_ops);
  return 0;
}
