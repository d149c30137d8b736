// Host check of the A-dependence classes that the sweep kernel relies on
// (op_aclass in z80_tables.cpp, derived from the device step function):
// every claim is re-checked with the CPU oracle's Exec on states and
// immediates other than those the classification sampled, and the
// two-values-of-A rule is checked on random A-independent pairs against a
// sweep of all 256 values.  Built and run by tests/test_tables.py.
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

int main() {
  orc::Init();
  const uint8_t* cls = z80b::op_aclass();
  std::mt19937_64 rng(777);
  long long n = 0;
  for (int op = 0; op < orc::OpCodeCount; op++) {
    const bool imm = orc::HasImmediate(uint16_t(op));
    for (int t = 0; t < 300; t++) {
      const uint64_t r = rng(), r2 = rng();
      const uint16_t iv = imm ? uint16_t(rng()) : 0;
      orc::State base{0, uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                      uint8_t(r >> 40), uint8_t(r >> 48), uint16_t(r2), uint8_t(r2 >> 16)};
      orc::State o0{};
      for (int a = 0; a < 256; a++) {
        orc::State s = base;
        s.A = uint8_t(a);
        orc::Exec(s, uint16_t(op), orc::HasImm16(uint16_t(op)) ? iv : uint16_t(iv & 0xFF));
        if (a == 0) o0 = s;
        n++;
        const bool others = s.F == o0.F && s.B == o0.B && s.C == o0.C && s.D == o0.D && s.E == o0.E &&
                            s.H == o0.H && s.L == o0.L && s.SP == o0.SP && s.M == o0.M;
        if (cls[op] == z80b::kAPass && (!others || s.A != a)) {
          std::printf("op %d claimed pass-through fails at A=%d\n", op, a);
          return 1;
        }
        if (cls[op] == z80b::kAOverwrite && (!others || s.A != o0.A)) {
          std::printf("op %d claimed overwrite fails at A=%d\n", op, a);
          return 1;
        }
      }
    }
  }
  // two values of A decide: random pairs (target of 1..3, candidate of 1..2
  // instructions from the 8-bit list) whose sequences are both A-independent
  const auto& pool = orc::Instructions8();
  long long pairs = 0;
  for (int t = 0; t < 200000 && pairs < 20000; t++) {
    orc::Instruction tg[3], cd[2];
    uint32_t tw[3], cw[2];
    const int tn = 1 + int(rng() % 3), cn = 1 + int(rng() % 2);
    for (int i = 0; i < tn; i++) {
      tg[i] = pool[rng() % pool.size()];
      tw[i] = uint32_t(tg[i].op) | uint32_t(tg[i].imm) << 16;
    }
    for (int i = 0; i < cn; i++) {
      cd[i] = pool[rng() % pool.size()];
      cw[i] = uint32_t(cd[i].op) | uint32_t(cd[i].imm) << 16;
    }
    if (!z80b::seq_aflow(tw, tn) || !z80b::seq_aflow(cw, cn)) continue;
    pairs++;
    for (int s = 0; s < 8; s++) {
      const uint64_t r = rng();
      orc::State base{0, uint8_t(r & 1), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                      uint8_t(r >> 40), uint8_t(r >> 48), uint16_t(rng()), uint8_t(rng())};
      bool two = true, all = true;
      for (int a = 0; a < 256; a++) {
        orc::State x = base;
        x.A = uint8_t(a);
        const bool eq = orc::ExecSeq(x, tg, tn) == orc::ExecSeq(x, cd, cn);
        if (a < 2) two = two && eq;
        all = all && eq;
      }
      if (two != all) {
        std::printf("two-value rule fails: target %u,%u,%u candidate %u,%u\n", tw[0], tn > 1 ? tw[1] : 0,
                    tn > 2 ? tw[2] : 0, cw[0], cn > 1 ? cw[1] : 0);
        return 1;
      }
    }
  }
  std::printf("OK %lld steps, %lld pairs\n", n, pairs);
  return 0;
}
