// Host check of the write masks that the bit-sliced sweep relies on (op_wmask
// in z80_tables.cpp, sampled from the device step function): a field outside
// an opcode's mask never changes under the CPU oracle's Exec.  Every 16-bit
// pair of fields (AF, BC, DE, HL, SP, and M with A) is swept over all 65,536
// values on random backgrounds, for every immediate of the 8-bit-immediate
// opcodes and sampled 16-bit immediates.  Built and run by tests/test_tables.py.
#include <cstdio>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

static uint16_t changed(const orc::State& a, const orc::State& b) {
  uint16_t m = 0;
  if (a.A != b.A) m |= z80b::kWA;
  if (a.F != b.F) m |= z80b::kWF;
  if (a.B != b.B) m |= z80b::kWB;
  if (a.C != b.C) m |= z80b::kWC;
  if (a.D != b.D) m |= z80b::kWD;
  if (a.E != b.E) m |= z80b::kWE;
  if (a.H != b.H) m |= z80b::kWH;
  if (a.L != b.L) m |= z80b::kWL;
  if (a.SP != b.SP) m |= z80b::kWSP;
  if (a.M != b.M) m |= z80b::kWM;
  return m;
}

static void set_pair(orc::State& s, int p, uint16_t v) {
  const uint8_t hi = uint8_t(v >> 8), lo = uint8_t(v);
  switch (p) {
    case 0: s.A = hi; s.F = lo; break;
    case 1: s.B = hi; s.C = lo; break;
    case 2: s.D = hi; s.E = lo; break;
    case 3: s.H = hi; s.L = lo; break;
    case 4: s.SP = v; break;
    default: s.M = hi; s.A = lo; break;
  }
}

int main() {
  orc::Init();
  const uint16_t* wm = z80b::op_wmask();
  std::mt19937_64 rng(4242);
  long long n = 0;
  for (int op = 0; op < orc::OpCodeCount; op++) {
    const bool imm = orc::HasImmediate(uint16_t(op));
    const bool imm16 = orc::HasImm16(uint16_t(op));
    // immediates: none, every 8-bit value, or 256 sampled 16-bit values
    const int nimm = imm ? 256 : 1;
    // values of each pair per immediate: all of them without an immediate,
    // a 1/64 stride (with a random offset) otherwise
    const int step = imm ? 64 : 1;
    for (int k = 0; k < nimm; k++) {
      const uint16_t iv = !imm ? 0 : imm16 ? (k < 2 ? uint16_t(k ? 0xFFFF : 0) : uint16_t(rng())) : uint16_t(k);
      for (int bg = 0; bg < 2; bg++) {
        const uint64_t r = rng(), r2 = rng();
        const orc::State base{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                              uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(r2),
                              uint8_t(r2 >> 16)};
        for (int p = 0; p < 6; p++) {
          const int off = step > 1 ? int(rng() % step) : 0;
          for (int v = off; v < 65536; v += step) {
            orc::State s = base;
            set_pair(s, p, uint16_t(v));
            const orc::State in = s;
            orc::Exec(s, uint16_t(op), iv);
            const uint16_t c = changed(in, s);
            n++;
            if (c & ~wm[op]) {
              std::printf("op %d imm %u changes fields %03x outside its mask %03x\n", op, iv, c, wm[op]);
              return 1;
            }
          }
        }
      }
    }
  }
  std::printf("OK %lld executions\n", n);
  return 0;
}
