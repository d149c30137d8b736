// Host check of the dependency sets (op_deps, seq_relevant in
// z80_tables.cpp) and of leaving irrelevant swept registers out of a sweep
// (put_pair in z80b_kernels.cu).  (1) Soundness against the oracle's Exec:
// for every opcode, every input field (A, each flag bit, B..L, SP, the
// memory byte) and sampled states and immediates, changing that field
// leaves every output field whose set does not hold it unchanged.  (2) For
// random pairs, many with dead flags and registers and an inserted write of
// a dead register, a sweep that drops the swept registers no compared output
// depends on, or that both programs keep exactly and no other compared
// output depends on (the others keeping the reference's values: a reduced sweep
// stays reduced), keeps only carry 0 when no compared output depends on the
// carry, and only A = 0, 1 when no compared output but A depends on A and
// each program keeps A or computes it from other inputs (pair_a_free), gives
// the oracle's ExhaustiveCheck verdict.  (1b) The instructions said to keep
// A leave it unchanged under the oracle's Exec.  Built and run
// by tests/test_tables.py.
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_bits.cuh"
#include "../../z80-optimizer_b200/csrc/z80_exec.cuh"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

using namespace z80b;

// field g of a state in the op_deps layout
static uint32_t get_field(const orc::State& s, int g) {
  switch (g) {
    case 0: return s.A;
    case 2: return s.B;
    case 3: return s.C;
    case 4: return s.D;
    case 5: return s.E;
    case 6: return s.H;
    case 7: return s.L;
    case 8: return s.SP;
    case 9: return s.M;
    default: return (s.F >> (g - kDepF0)) & 1u;
  }
}
static void set_field(orc::State& s, int g, uint32_t v) {
  switch (g) {
    case 0: s.A = uint8_t(v); break;
    case 2: s.B = uint8_t(v); break;
    case 3: s.C = uint8_t(v); break;
    case 4: s.D = uint8_t(v); break;
    case 5: s.E = uint8_t(v); break;
    case 6: s.H = uint8_t(v); break;
    case 7: s.L = uint8_t(v); break;
    case 8: s.SP = uint16_t(v); break;
    case 9: s.M = uint8_t(v); break;
    default: s.F = uint8_t((s.F & ~(1u << (g - kDepF0))) | ((v & 1u) << (g - kDepF0))); break;
  }
}
static const int kFields[] = {0, 2, 3, 4, 5, 6, 7, 8, 9, 16, 17, 18, 19, 20, 21, 22, 23};

// the reference sweep's block decoding for a read mask (verifier.go:428-612),
// with `reduced` forced when the reference's sweep of the pair is reduced
struct Shape {
  bool spw, reduced;
  int nx, fw, slot[7];
  uint64_t nblocks;
};
static Shape shape_of(uint16_t reads, bool force_reduced) {
  Shape s{};
  const uint32_t bits[7] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM};
  int k = 0;
  for (int r = 0; r < 7; r++) s.slot[r] = (reads & bits[r]) ? k++ : -1;
  s.nx = k;
  s.spw = (reads & kRegSP) != 0;
  s.reduced = s.spw || s.nx > 2 || force_reduced;
  s.fw = s.reduced ? 5 : 8;
  s.nblocks = s.reduced ? (2ull << (5 * s.nx)) * (s.spw ? 16 : 1) : (2ull << (8 * s.nx));
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
  std::mt19937_64 rng(53);
  const uint32_t (*D)[kDepFields] = op_deps();
  // (1) soundness of every dependency set against the oracle's Exec
  long checks = 0;
  for (int op = 0; op < orc::OpCodeCount; op++) {
    for (int k = 0; k < 48; k++) {
      const uint64_t r = rng(), r2 = rng();
      orc::State s{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                   uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2), uint8_t(r2 >> 16)};
      const uint16_t imm = uint16_t(rng());
      orc::State base = s;
      orc::Exec(base, uint16_t(op), imm);
      for (int f : kFields) {
        for (int v = 0; v < 4; v++) {
          orc::State t = s;
          const uint32_t old = get_field(s, f);
          const uint32_t nv = f >= kDepF0 ? (old ^ 1u) : (f == 8 ? uint32_t(rng() & 0xFFFF) : uint32_t(rng() & 0xFF));
          set_field(t, f, nv);
          orc::Exec(t, uint16_t(op), imm);
          for (int g : kFields) {
            if (D[op][g] & (1u << f)) continue;
            checks++;
            if (get_field(t, g) != get_field(base, g)) {
              std::printf("op %d (%s): output field %d changes with input field %d outside its set\n", op,
                          op_mnemonic(uint16_t(op)), g, f);
              return 1;
            }
          }
        }
      }
    }
  }
  // (1b) instructions said to keep A (or any register, or the memory byte)
  // leave it exactly as it was
  int keepers = 0;
  for (int op = 0; op < orc::OpCodeCount; op++) {
    const uint16_t kept = op_keeps()[op];
    if (bool(kept & kRegA) != bool(op_keeps_a()[op])) {
      std::printf("op %d (%s): the two keeps-A tables disagree\n", op, op_mnemonic(uint16_t(op)));
      return 1;
    }
    for (int k = 0; k < 64; k++) {
      const uint64_t r = rng(), r2 = rng();
      orc::State st{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                    uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2), uint8_t(r2 >> 16)};
      const orc::State in = st;
      orc::Exec(st, uint16_t(op), uint16_t(rng()));
      const int fields[7] = {2, 3, 4, 5, 6, 7, 9};
      for (int g : fields)
        if ((kept & (1u << g)) && get_field(st, g) != get_field(in, g)) {
          std::printf("op %d (%s) is said to keep field %d but changes it\n", op, op_mnemonic(uint16_t(op)), g);
          return 1;
        }
    }
    if (!op_keeps_a()[op]) continue;
    keepers++;
    for (int k = 0; k < 256; k++) {
      const uint64_t r = rng(), r2 = rng();
      orc::State st{uint8_t(k), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                    uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2), uint8_t(r2 >> 16)};
      orc::Exec(st, uint16_t(op), uint16_t(rng()));
      if (st.A != uint8_t(k)) {
        std::printf("op %d (%s) is said to keep A but changes it\n", op, op_mnemonic(uint16_t(op)));
        return 1;
      }
    }
  }
  if (keepers < 200) {
    std::printf("too few instructions keep A (%d)\n", keepers);
    return 1;
  }
  // (2) sweeps without the irrelevant registers give the oracle's verdicts
  const auto& I = orc::Instructions8();
  int pairs = 0, equal = 0, dropped = 0, carries = 0, carry_only = 0, a_free = 0;
  for (int trial = 0; trial < 40000000 && (pairs < 400 || a_free < 40); trial++) {
    int tn = 1 + int(rng() % 3), cn = 1 + int(rng() % 2);
    orc::Instruction ti[3], ci[2];
    for (int i = 0; i < tn; i++) ti[i] = I[rng() % I.size()];
    for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
    uint8_t extra_dead = 0;
    if (rng() % 2) {
      // the candidate with one more instruction put in the target, whose
      // named registers are made dead below
      cn = 1 + int(rng() % 2);
      tn = cn + 1;
      const orc::Instruction j = I[rng() % I.size()];
      const int at = int(rng() % tn);
      for (int k = 0, m = 0; k < tn; k++) ti[k] = k == at ? j : ci[m++];
      extra_dead = uint8_t(op_regs(j.op) & 0x3Fu);
    }
    uint32_t tw[3], cw[2];
    for (int i = 0; i < tn; i++) tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
    for (int i = 0; i < cn; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
    const uint8_t dead = (rng() & 1) ? uint8_t(0xFF) : uint8_t(rng());
    const uint8_t dregs = uint8_t((extra_dead | (rng() % 3 == 0 ? rng() : 0)) & 0x3Fu);
    const uint32_t keepF = uint8_t(~dead), keepR = ~uint32_t(dregs) & 0x3Fu;
    const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cn));
    const uint32_t ext = reads & (kRegB | kRegC | kRegD | kRegE | kRegH | kRegL | kRegM);
    const uint32_t cmp = kRegA | kRegSP | kRegM | (keepR << 2) | (keepF << kDepF0);
    const uint32_t rel = seq_relevant(tw, tn, cmp) | seq_relevant(cw, cn, cmp);
    const uint32_t drop = (ext & ~rel) | pair_kept_out(tw, tn, cw, cn, cmp, ext);
    const bool carry_out = (rel & (1u << kDepF0)) == 0;
    const bool a_out = pair_a_free(tw, tn, cw, cn, cmp);
    if (!drop && !carry_out && !a_out) continue;
    if (pairs >= 400 && !a_out) continue;  // past 400: A-free pairs only
    if (sweep_for(reads).states > (1ull << 23)) continue;
    const int n_ext = __builtin_popcount(ext);
    const bool ref_reduced = (reads & kRegSP) != 0 || n_ext > 2;
    Shape s = shape_of(uint16_t(reads & ~drop), ref_reduced);
    if (carry_out) s.nblocks >>= 1;  // the carry is the block index's top field: carry 0 only
    if (s.nblocks > 4096) continue;
    if (!drop && carry_only >= 150) continue;
    pairs++;
    a_free += a_out ? 1 : 0;
    carry_only += drop ? 0 : 1;
    carries += carry_out ? 1 : 0;
    dropped += __builtin_popcount(drop);
    bool bad = false;
    for (uint64_t b = 0; b < s.nblocks && !bad; b++) {
      const Z80S x = decode(b, s);
      // a pair whose compared outputs other than A do not depend on A, and
      // whose programs keep A or compute it from other inputs: A = 0 and 1
      // decide, as in the A-independent sweeps the pair is then given to
      for (uint32_t a0 = 0; a0 < (a_out ? 32u : 256u) && !bad; a0 += 32) {
        Z80S st[32];
        for (int j = 0; j < 32; j++) {
          st[j] = x;
          st[j].a = a0 + uint32_t(j);
        }
        ZB z;
        zb_from(z, st);
        ZB zc = z, zt = z;
        for (int i = 0; i < cn; i++) zb_step(zc, insn_op(cw[i]), insn_imm(cw[i]));
        for (int i = 0; i < tn; i++) zb_step(zt, insn_op(tw[i]), insn_imm(tw[i]));
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
          d |= zc.m[i] ^ zt.m[i];
        }
        for (int i = 0; i < 16; i++) d |= zc.sp[i] ^ zt.sp[i];
        if (a_out) d &= 3u;
        bad = d != 0;
      }
    }
    const bool want = orc::ExhaustiveCheckMaskedRegs(ti, tn, ci, cn, dead, dregs);
    if (want == bad) {
      std::printf("verdict without the irrelevant registers differs: %s -> %s dead %02x regs %02x (dropped %03x)\n",
                  disasm_seq(tw, tn).c_str(), disasm_seq(cw, cn).c_str(), dead, dregs, drop);
      return 1;
    }
    equal += want ? 1 : 0;
  }
  if (pairs < 300 || equal < 20 || carries < 100 || pairs - carry_only < 150 || a_free < 30) {
    std::printf("too few pairs (%d), equivalences (%d), pairs without the carry (%d), with registers left out (%d) "
                "or at A = 0, 1 (%d)\n", pairs, equal, carries, pairs - carry_only, a_free);
    return 1;
  }
  std::printf("OK deps: %ld independence checks; %d pairs: %d registers left out, %d without the carry, %d at A = 0, 1 "
              "(%d equivalent)\n", checks, pairs, dropped, carries, a_free, equal);
  return 0;
}
