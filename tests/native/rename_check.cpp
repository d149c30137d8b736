// Host check of op_rename (z80_tables.cpp), the register renaming that maps a
// pair's registers onto other ones: for every opcode and every permutation
// of B, C, D, E, H, L, when a renamed opcode exists, executing it on the
// permuted state gives the permuted result of the original under the CPU
// oracle's Exec; and every instruction whose only register operands are
// 8-bit ones has a renamed form under every permutation.  Built and run by
// tests/test_tables.py.
#include <algorithm>
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

static uint8_t* reg(orc::State& s, int r) {
  switch (r) {
    case 0: return &s.B;
    case 1: return &s.C;
    case 2: return &s.D;
    case 3: return &s.E;
    case 4: return &s.H;
    default: return &s.L;
  }
}

// register r's value moves to register map[r]
static orc::State permute(const orc::State& s, const uint8_t (&map)[6]) {
  orc::State t = s, src = s;
  for (int r = 0; r < 6; r++) *reg(t, map[r]) = *reg(src, r);
  return t;
}

int main() {
  orc::Init();
  std::mt19937_64 rng(99);
  uint8_t map[6] = {0, 1, 2, 3, 4, 5};
  long long renamed = 0, checks = 0;
  int perms = 0;
  do {
    perms++;
    for (int op = 0; op < orc::OpCodeCount; op++) {
      const int o2 = z80b::op_rename(uint16_t(op), map);
      const std::string m = z80b::op_mnemonic(uint16_t(op));
      const bool pairs_used = m.find("BC") != std::string::npos || m.find("DE") != std::string::npos ||
                              (m.find("HL") != std::string::npos && m.find("(HL)") == std::string::npos);
      if (o2 < 0) {
        if (!pairs_used) {
          std::printf("op %d (%s) has no renamed form\n", op, m.c_str());
          return 1;
        }
        continue;
      }
      renamed++;
      const bool imm16 = orc::HasImm16(uint16_t(op));
      for (int k = 0; k < 6; k++) {
        const uint64_t r = rng(), r2 = rng();
        const orc::State s{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                           uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2), uint8_t(r2 >> 16)};
        const uint16_t imm = imm16 ? uint16_t(rng()) : uint16_t(rng() & 0xFF);
        orc::State a = s;
        orc::Exec(a, uint16_t(op), imm);
        orc::State b = permute(s, map);
        orc::Exec(b, uint16_t(o2), imm);
        checks++;
        if (b != permute(a, map)) {
          std::printf("op %d (%s) -> %d (%s) breaks the renaming\n", op, m.c_str(), o2, z80b::op_mnemonic(uint16_t(o2)));
          return 1;
        }
      }
    }
  } while (std::next_permutation(map, map + 6));
  std::printf("OK %d permutations, %lld renamed opcodes, %lld checks\n", perms, renamed, checks);
  return 0;
}
