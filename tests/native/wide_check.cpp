// Host check of the wide compact state (wide_map, wide_tables in
// z80_tables.cpp; ZBW, zbw_step, WDec in z80_bits.cuh).  (1) Every register
// an instruction reads is one it names, so a wide pair's swept registers all
// have a field in the wide state.  (2) zbw_step gives the full bit-sliced
// step's A, F, B, C, H, L and M for every opcode that names no register but
// B, C, H, L and not SP.  (3) The device's tables (wide_tables) accept,
// rename and place registers as wide_map does.  (4) The wide kernel's sweep
// unit (wbits_unit in z80b_kernels.cu), restated with its block decoding
// (WDec), plane layout and dead-flag and dead-register compares, gives the
// oracle's ExhaustiveCheck verdict with dead registers for A-dependent pairs
// that the compact state does not take.  (5), (6) The register state (ZB6:
// A, F, B..L): zb6_step against the full step, and the register-state unit
// (rbits_unit) restated against the oracle for pairs naming neither SP nor
// the memory byte that no compact state takes.  Built and run by
// tests/test_tables.py.
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_bits.cuh"
#include "../../z80-optimizer_b200/csrc/z80_exec.cuh"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

using namespace z80b;

// the reference sweep's shape for a read mask and its block decoding
// (verifier.go:428-612)
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

int main() {
  orc::Init();
  std::mt19937_64 rng(47);
  // (1) registers read are named
  for (int op = 0; op < orc::OpCodeCount; op++) {
    const uint16_t rd = orc::OpReads(uint16_t(op));
    const uint8_t named = op_regs(uint16_t(op));
    const uint16_t bits[6] = {orc::regB, orc::regC, orc::regD, orc::regE, orc::regH, orc::regL};
    for (int r = 0; r < 6; r++)
      if ((rd & bits[r]) && !(named & (1u << r))) {
        std::printf("op %d (%s) reads register %d that it does not name\n", op, op_mnemonic(uint16_t(op)), r);
        return 1;
      }
    if ((rd & orc::regSP) && !(named & 0x80u)) {
      std::printf("op %d (%s) reads SP without naming it\n", op, op_mnemonic(uint16_t(op)));
      return 1;
    }
  }
  // (2) the wide bit-sliced step
  int wide_ops = 0;
  for (uint32_t op = 0; op < uint32_t(kNumOps); op++) {
    if (op_regs(uint16_t(op)) & ~0x73u) continue;  // B, C, H, L and the memory byte
    wide_ops++;
    for (int rep = 0; rep < 32; rep++) {
      Z80S st[32];
      for (int j = 0; j < 32; j++) {
        const uint64_t r = rng(), r2 = rng();
        st[j] = Z80S{uint32_t(r & 0xFF), uint32_t((r >> 8) & 0xFF), uint32_t((r >> 16) & 0xFF),
                     uint32_t((r >> 24) & 0xFF), 0, 0, uint32_t((r >> 32) & 0xFF), uint32_t((r >> 40) & 0xFF),
                     0, uint32_t(r2 & 0xFF)};
      }
      const uint32_t imm = uint32_t(rng() & 0xFFFF);
      ZB full;
      zb_from(full, st);
      ZBW w;
      for (int i = 0; i < 8; i++) {
        w.a[i] = full.a[i];
        w.f[i] = full.f[i];
        w.b[i] = full.b[i];
        w.c[i] = full.c[i];
        w.h[i] = full.h[i];
        w.l[i] = full.l[i];
        w.m[i] = full.m[i];
      }
      zb_step(full, op, imm);
      zbw_step(w, op, imm);
      for (int i = 0; i < 8; i++)
        if (w.a[i] != full.a[i] || w.f[i] != full.f[i] || w.b[i] != full.b[i] || w.c[i] != full.c[i] ||
            w.h[i] != full.h[i] || w.l[i] != full.l[i] || w.m[i] != full.m[i]) {
          std::printf("wide step differs on op %u (%s)\n", op, op_mnemonic(uint16_t(op)));
          return 1;
        }
    }
  }
  if (wide_ops < 250) {
    std::printf("too few wide opcodes (%d)\n", wide_ops);
    return 1;
  }
  const auto& I = orc::Instructions8();
  const WideTables& W = wide_tables();
  const CompactTables& C = compact_tables();
  auto pick = [&](uint32_t* w, int n) {
    for (int i = 0; i < n; i++) {
      const auto& x = I[rng() % I.size()];
      w[i] = uint32_t(x.op) | uint32_t(x.imm) << 16;
    }
  };
  auto wide_id = [&](const uint32_t* tw, int tn, const uint32_t* cw, int cn) {
    uint8_t fp = 0;
    for (int i = 0; i < tn; i++) fp |= C.opregs[insn_op(tw[i])];
    for (int i = 0; i < cn; i++) fp |= C.opregs[insn_op(cw[i])];
    int id = (fp & 0x80) ? 0 : W.id_of_set[fp & 0x3F];
    for (int i = 0; i < tn && id; i++)
      if (W.ren[id - 1][insn_op(tw[i])] < 0) id = 0;
    for (int i = 0; i < cn && id; i++)
      if (W.ren[id - 1][insn_op(cw[i])] < 0) id = 0;
    return id;
  };
  auto compact_id = [&](const uint32_t* tw, int tn, const uint32_t* cw, int cn) {
    uint8_t fp = 0;
    for (int i = 0; i < tn; i++) fp |= C.opregs[insn_op(tw[i])];
    for (int i = 0; i < cn; i++) fp |= C.opregs[insn_op(cw[i])];
    int id = (fp & 0xC0) ? 0 : C.id_of_set[fp & 0x3F];
    for (int i = 0; i < tn && id; i++)
      if (C.ren[id - 1][insn_op(tw[i])] < 0) id = 0;
    for (int i = 0; i < cn && id; i++)
      if (C.ren[id - 1][insn_op(cw[i])] < 0) id = 0;
    return id;
  };
  // (3) the device's tables decide and rename as wide_map does
  {
    static const int kPlaces[4] = {0, 1, 4, 5};
    int agreed = 0, beyond = 0;
    for (int trial = 0; trial < 300000; trial++) {
      const int tn = 1 + int(rng() % 3), cn = 1 + int(rng() % 2);
      uint32_t tw[3], cw[2], tr[3], cr[2];
      pick(tw, tn);
      pick(cw, cn);
      uint8_t map[6];
      const bool by_map = wide_map(tw, tn, cw, cn, map, tr, cr);
      const int id = wide_id(tw, tn, cw, cn);
      if (by_map != (id != 0)) {
        std::printf("wide tables disagree with wide_map (%d vs %d)\n", id != 0, by_map);
        return 1;
      }
      if (!by_map) continue;
      agreed++;
      if (!compact_id(tw, tn, cw, cn)) beyond++;
      for (int i = 0; i < tn; i++)
        if (uint32_t(W.ren[id - 1][insn_op(tw[i])]) != insn_op(tr[i])) {
          std::printf("wide table renames differently\n");
          return 1;
        }
      for (int i = 0; i < cn; i++)
        if (uint32_t(W.ren[id - 1][insn_op(cw[i])]) != insn_op(cr[i])) {
          std::printf("wide table renames differently\n");
          return 1;
        }
      uint8_t fp = 0;
      for (int i = 0; i < tn; i++) fp |= op_regs(insn_op(tw[i]));
      for (int i = 0; i < cn; i++) fp |= op_regs(insn_op(cw[i]));
      for (int s = 0; s < 4; s++) {
        int want = -1;
        for (int r = 0; r < 6; r++)
          if ((fp & (1u << r)) && map[r] == kPlaces[s]) want = r;
        if (W.orig[id - 1][s] != want) {
          std::printf("wide table origin differs\n");
          return 1;
        }
      }
      // renamed programs name no register outside B, C, H, L
      for (int i = 0; i < tn; i++)
        if (op_regs(insn_op(tr[i])) & 0x8Cu) {
          std::printf("a renamed program names D, E or SP\n");
          return 1;
        }
      for (int i = 0; i < cn; i++)
        if (op_regs(insn_op(cr[i])) & 0x8Cu) {
          std::printf("a renamed program names D, E or SP\n");
          return 1;
        }
    }
    if (agreed < 1000 || beyond < 200) {
      std::printf("too few wide pairs for the table check (%d, %d beyond the compact state)\n", agreed, beyond);
      return 1;
    }
  }
  // (4) the wide unit restated: per block and 32 values of A, the five wide
  // fields and the carry from WDec, renamed programs, A and M always
  // compared, F under the dead flags, B, C, H, L under the dead registers of
  // the registers they stand for; against the oracle with dead registers
  {
    int wp = 0, weq = 0, mem = 0, many = 0;
    for (int trial = 0; trial < 40000000 && (wp - many < 476 || many < 24); trial++) {
      const int tn = 1 + int(rng() % 3);
      int cn = 1 + int(rng() % 2);
      orc::Instruction ti[3], ci[2];
      uint32_t tw[3], cw[2];
      for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
      for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
      const uint64_t how = rng() % 3;
      if (how == 1) {  // a candidate that keeps part of the target: more equivalences
        ci[0] = ti[rng() % tn];
        if (cn == 2) ci[1] = ti[rng() % tn];
      } else if (how == 2 && tn >= 2) {  // the target less one instruction
        const int drop = int(rng() % tn);
        cn = 0;
        for (int i = 0; i < tn; i++)
          if (i != drop) ci[cn++] = ti[i];
      }
      for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
      for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
      if (seq_aflow(tw, tn) && seq_aflow(cw, cn)) continue;  // the wide class takes A-dependent pairs
      if (compact_id(tw, tn, cw, cn)) continue;              // ... the compact one does not take
      const int id = wide_id(tw, tn, cw, cn);
      if (!id) continue;
      const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn));
      const Shape s = shape_of(reads);
      if (s.spw) {
        std::printf("a wide pair with an SP sweep\n");
        return 1;
      }
      // full sweeps up to 4,096 blocks; reduced ones (65,536 blocks and
      // more) for a bounded number of pairs
      if (s.reduced ? (s.nblocks > 65536 || many >= 24) : (s.nblocks > 4096 || wp - many >= 476)) continue;
      wp++;
      mem += (reads & kRegM) ? 1 : 0;
      many += s.reduced ? 1 : 0;
      uint32_t tr[3], cr[2];
      for (int i = 0; i < tn; i++) tr[i] = uint32_t(uint16_t(W.ren[id - 1][insn_op(tw[i])])) | (tw[i] & 0xFFFF0000u);
      for (int i = 0; i < cn; i++) cr[i] = uint32_t(uint16_t(W.ren[id - 1][insn_op(cw[i])])) | (cw[i] & 0xFFFF0000u);
      int o[4];
      for (int f = 0; f < 4; f++) o[f] = W.orig[id - 1][f];
      const uint8_t dead = uint8_t(rng() & 0xFF), dregs = uint8_t(rng() % 4 == 0 ? 0 : rng() & 0x3F);
      const uint32_t keepF = uint8_t(~dead), keepR = ~uint32_t(dregs) & 0x3Fu;
      uint32_t cmp = 0;
      for (int f = 0; f < 4; f++)
        if (o[f] >= 0 && ((keepR >> o[f]) & 1u)) cmp |= 1u << f;
      const WDec dec = wdec_make(s.nx, s.reduced, s.slot, o);
      bool bad = false;
      for (uint64_t b = 0; b < s.nblocks && !bad; b++) {
        const Z80S x = decode(b, s);
        const uint32_t regs[6] = {x.b, x.c, x.d, x.e, x.h, x.l};
        uint32_t v[5], carry;
        wdec_vals(dec, uint32_t(b), rep_values(), v, carry);
        for (int f = 0; f < 4; f++)
          if (v[f] != (o[f] >= 0 ? regs[o[f]] : 0u)) {
            std::printf("wide block decoding differs at block %llu field %d\n", (unsigned long long)b, f);
            return 1;
          }
        if (v[4] != x.m || carry != x.f) {
          std::printf("wide block decoding differs at block %llu (M or carry)\n", (unsigned long long)b);
          return 1;
        }
        for (uint32_t a0 = 0; a0 < 256 && !bad; a0 += 32) {
          ZBW z;
          z.a[0] = 0xAAAAAAAAu;
          z.a[1] = 0xCCCCCCCCu;
          z.a[2] = 0xF0F0F0F0u;
          z.a[3] = 0xFF00FF00u;
          z.a[4] = 0xFFFF0000u;
          for (int i = 5; i < 8; i++) z.a[i] = ((a0 >> i) & 1u) ? kZBOnes : 0u;
          zb_set8(z.f, carry);
          zb_set8(z.b, v[0]);
          zb_set8(z.c, v[1]);
          zb_set8(z.h, v[2]);
          zb_set8(z.l, v[3]);
          zb_set8(z.m, v[4]);
          ZBW zc = z, zt = z;
          for (int i = 0; i < cn; i++) zbw_step(zc, insn_op(cr[i]), insn_imm(cr[i]));
          for (int i = 0; i < tn; i++) zbw_step(zt, insn_op(tr[i]), insn_imm(tr[i]));
          uint32_t d = 0;
          for (int i = 0; i < 8; i++) {
            d |= zc.a[i] ^ zt.a[i];
            if ((keepF >> i) & 1u) d |= zc.f[i] ^ zt.f[i];
            if (cmp & 1u) d |= zc.b[i] ^ zt.b[i];
            if (cmp & 2u) d |= zc.c[i] ^ zt.c[i];
            if (cmp & 4u) d |= zc.h[i] ^ zt.h[i];
            if (cmp & 8u) d |= zc.l[i] ^ zt.l[i];
            d |= zc.m[i] ^ zt.m[i];
          }
          bad = d != 0;
        }
      }
      const bool want = orc::ExhaustiveCheckMaskedRegs(ti, tn, ci, cn, dead, dregs);
      if (want == bad) {
        std::printf("wide unit verdict differs: target %08x %08x %08x (%d) candidate %08x %08x (%d) dead %02x regs %02x\n",
                    tw[0], tn > 1 ? tw[1] : 0, tn > 2 ? tw[2] : 0, tn, cw[0], cn > 1 ? cw[1] : 0, cn, dead, dregs);
        return 1;
      }
      weq += want ? 1 : 0;
    }
    if (wp < 300 || weq < 20 || mem < 50 || many < 20) {
      std::printf("too few wide pairs (%d), equivalences (%d), memory pairs (%d) or reduced sweeps (%d)\n", wp,
                  weq, mem, many);
      return 1;
    }
    std::printf("OK wide: %d opcodes, %d pairs (%d equivalent, %d with memory, %d reduced sweeps)\n", wide_ops, wp,
                weq, mem, many);
  }
  // (5) the register state (ZB6: A, F, B..L): zb6_step gives the full step's
  // planes for every opcode naming neither SP nor the memory byte
  int reg_ops = 0;
  for (uint32_t op = 0; op < uint32_t(kNumOps); op++) {
    if (op_regs(uint16_t(op)) & 0xC0u) continue;
    reg_ops++;
    for (int rep = 0; rep < 32; rep++) {
      Z80S st[32];
      for (int j = 0; j < 32; j++) {
        const uint64_t r = rng();
        st[j] = Z80S{uint32_t(r & 0xFF), uint32_t((r >> 8) & 0xFF), uint32_t((r >> 16) & 0xFF),
                     uint32_t((r >> 24) & 0xFF), uint32_t((r >> 32) & 0xFF), uint32_t((r >> 40) & 0xFF),
                     uint32_t((r >> 48) & 0xFF), uint32_t((r >> 56) & 0xFF), 0, 0};
      }
      const uint32_t imm = uint32_t(rng() & 0xFFFF);
      ZB full;
      zb_from(full, st);
      ZB6 z6;
      for (int i = 0; i < 8; i++) {
        z6.a[i] = full.a[i];
        z6.f[i] = full.f[i];
        z6.b[i] = full.b[i];
        z6.c[i] = full.c[i];
        z6.d[i] = full.d[i];
        z6.e[i] = full.e[i];
        z6.h[i] = full.h[i];
        z6.l[i] = full.l[i];
      }
      zb_step(full, op, imm);
      zb6_step(z6, op, imm);
      for (int i = 0; i < 8; i++)
        if (z6.a[i] != full.a[i] || z6.f[i] != full.f[i] || z6.b[i] != full.b[i] || z6.c[i] != full.c[i] ||
            z6.d[i] != full.d[i] || z6.e[i] != full.e[i] || z6.h[i] != full.h[i] || z6.l[i] != full.l[i]) {
          std::printf("register-state step differs on op %u (%s)\n", op, op_mnemonic(uint16_t(op)));
          return 1;
        }
    }
  }
  // (6) the register-state unit (rbits_unit in z80b_kernels.cu) restated:
  // per block and 32 values of A, the planes of the decoded state, A always
  // compared, F under the dead flags, B..L under the dead registers; against
  // the oracle with dead registers, for A-dependent pairs naming neither SP
  // nor the memory byte that no compact state takes
  {
    int rp = 0, req = 0, five = 0;
    for (int trial = 0; trial < 40000000 && rp < 400; trial++) {
      int tn = 1 + int(rng() % 3);
      int cn = 1 + int(rng() % 2);
      orc::Instruction ti[3], ci[2];
      uint32_t tw[3], cw[2];
      for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
      for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
      const uint64_t how = rng() % 4;
      uint8_t dropped_regs = 0;  // registers the dropped instruction names: made dead below
      if (how == 3) {
        // the candidate with one more instruction put in that writes no A:
        // equivalent when what it writes is dead and nothing after reads it
        orc::Instruction j;
        do j = I[rng() % I.size()];
        while (orc::OpWrites(j.op) & orc::regA);
        cn = 1 + int(rng() % 2);
        tn = cn + 1;
        const int at = (rng() & 1) ? tn - 1 : int(rng() % tn);  // last: nothing after it reads what it writes
        for (int k = 0, m = 0; k < tn; k++) ti[k] = k == at ? j : ci[m++];
        dropped_regs = uint8_t(op_regs(j.op) & 0x3Fu);
      } else if (how == 1) {
        ci[0] = ti[rng() % tn];
        if (cn == 2) ci[1] = ti[rng() % tn];
      } else if (how == 2 && tn >= 2) {
        const int drop = int(rng() % tn);
        dropped_regs = uint8_t(op_regs(ti[drop].op) & 0x3Fu);
        cn = 0;
        for (int i = 0; i < tn; i++)
          if (i != drop) ci[cn++] = ti[i];
      }
      for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
      for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
      if (seq_aflow(tw, tn) && seq_aflow(cw, cn)) continue;
      if (compact_id(tw, tn, cw, cn) || wide_id(tw, tn, cw, cn)) continue;
      uint8_t fp = 0;
      for (int i = 0; i < tn; i++) fp |= op_regs(insn_op(tw[i]));
      for (int i = 0; i < cn; i++) fp |= op_regs(insn_op(cw[i]));
      if (fp & 0xC0u) continue;
      const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn));
      const Shape s = shape_of(reads);
      if (s.nblocks > 65536) continue;
      rp++;
      five += __builtin_popcount(fp & 0x3Fu) >= 5 ? 1 : 0;
      const bool drop_dead = dropped_regs && (how == 3 || (rng() & 1));
      const uint8_t dead = drop_dead ? uint8_t(0xFF) : uint8_t(rng() & 0xFF);
      const uint8_t dregs = drop_dead ? uint8_t(dropped_regs | (rng() & 0x3F))
                                      : uint8_t(rng() % 4 == 0 ? 0 : rng() & 0x3F);
      const uint32_t keepF = uint8_t(~dead), keepR = ~uint32_t(dregs) & 0x3Fu;
      bool bad = false;
      for (uint64_t b = 0; b < s.nblocks && !bad; b++) {
        const Z80S x = decode(b, s);
        for (uint32_t a0 = 0; a0 < 256 && !bad; a0 += 32) {
          ZB6 z;
          z.a[0] = 0xAAAAAAAAu;
          z.a[1] = 0xCCCCCCCCu;
          z.a[2] = 0xF0F0F0F0u;
          z.a[3] = 0xFF00FF00u;
          z.a[4] = 0xFFFF0000u;
          for (int i = 5; i < 8; i++) z.a[i] = ((a0 >> i) & 1u) ? kZBOnes : 0u;
          zb_set8(z.f, x.f);
          zb_set8(z.b, x.b);
          zb_set8(z.c, x.c);
          zb_set8(z.d, x.d);
          zb_set8(z.e, x.e);
          zb_set8(z.h, x.h);
          zb_set8(z.l, x.l);
          ZB6 zc = z, zt = z;
          for (int i = 0; i < cn; i++) zb6_step(zc, insn_op(cw[i]), insn_imm(cw[i]));
          for (int i = 0; i < tn; i++) zb6_step(zt, insn_op(tw[i]), insn_imm(tw[i]));
          uint32_t d = 0;
          for (int i = 0; i < 8; i++) {
            d |= zc.a[i] ^ zt.a[i];
            if ((keepF >> i) & 1u) d |= zc.f[i] ^ zt.f[i];
            if (keepR & 1u) d |= zc.b[i] ^ zt.b[i];
            if (keepR & 2u) d |= zc.c[i] ^ zt.c[i];
            if (keepR & 4u) d |= zc.d[i] ^ zt.d[i];
            if (keepR & 8u) d |= zc.e[i] ^ zt.e[i];
            if (keepR & 16u) d |= zc.h[i] ^ zt.h[i];
            if (keepR & 32u) d |= zc.l[i] ^ zt.l[i];
          }
          bad = d != 0;
        }
      }
      const bool want = orc::ExhaustiveCheckMaskedRegs(ti, tn, ci, cn, dead, dregs);
      if (want == bad) {
        std::printf("register-state unit verdict differs: target %08x %08x %08x (%d) candidate %08x %08x (%d)\n",
                    tw[0], tn > 1 ? tw[1] : 0, tn > 2 ? tw[2] : 0, tn, cw[0], cn > 1 ? cw[1] : 0, cn);
        return 1;
      }
      req += want ? 1 : 0;
    }
    if (reg_ops < 380 || rp < 300 || req < 2 || five < 20) {
      std::printf("too few register-state opcodes (%d), pairs (%d), equivalences (%d) or five-register pairs (%d)\n",
                  reg_ops, rp, req, five);
      return 1;
    }
    std::printf("register state: %d opcodes, %d pairs (%d equivalent, %d naming five or six registers)\n", reg_ops, rp,
                req, five);
  }
  return 0;
}
