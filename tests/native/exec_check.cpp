// Host-side comparison of the device step function (z80_exec.cuh compiled
// as plain C++) with the CPU oracle, opcode by opcode.  Built and run by
// tests/test_exec_host.py; exits non-zero on the first mismatch.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_exec.cuh"

static bool same(const orc::State& a, const z80b::Z80S& b) {
  return a.A == b.a && a.F == b.f && a.B == b.b && a.C == b.c && a.D == b.d && a.E == b.e &&
         a.H == b.h && a.L == b.l && a.SP == b.sp && a.M == b.m;
}

int main() {
  orc::Init();
  std::mt19937_64 rng(12345);
  long long checked = 0;
  for (int op = 0; op < orc::OpCodeCount; op++) {
    bool imm = orc::HasImmediate(uint16_t(op)), imm16 = orc::HasImm16(uint16_t(op));
    // all (A, F) pairs with random other registers; imm ops add 64 immediates
    int nimm = imm ? (imm16 ? 64 : 256) : 1;
    for (int ii = 0; ii < nimm; ii++) {
      uint16_t iv = imm16 ? uint16_t(rng()) : uint16_t(ii);
      int fstep = imm ? 17 : 1;  // F sweep thinned for the immediate forms
      for (int a = 0; a < 256; a++)
        for (int f = (imm ? int(rng() % 17) : 0); f < 256; f += fstep) {
          uint64_t r = rng();
          orc::State s{uint8_t(a), uint8_t(f), uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16),
                       uint8_t(r >> 24), uint8_t(r >> 32), uint8_t(r >> 40), uint16_t(r >> 48),
                       uint8_t(rng())};
          if ((r & 7) == 0) { s.H = s.L = 0; s.B = 0; s.C = 0; }
          z80b::Z80S d{s.A, s.F, s.B, s.C, s.D, s.E, s.H, s.L, s.SP, s.M};
          orc::Exec(s, uint16_t(op), iv);
          z80b::z_step(d, uint32_t(op), iv);
          checked++;
          if (!same(s, d)) {
            std::printf("MISMATCH op=%d (%s) imm=%u a=%d f=%d: oracle A=%02X F=%02X B=%02X C=%02X D=%02X E=%02X "
                        "H=%02X L=%02X SP=%04X M=%02X  device A=%02X F=%02X B=%02X C=%02X D=%02X E=%02X H=%02X "
                        "L=%02X SP=%04X M=%02X\n",
                        op, orc::OpName(uint16_t(op)), iv, a, f, s.A, s.F, s.B, s.C, s.D, s.E, s.H, s.L, s.SP, s.M,
                        d.a, d.f, d.b, d.c, d.d, d.e, d.h, d.l, d.sp, d.m);
            return 1;
          }
        }
    }
  }
  // 16-bit arithmetic: random HL/rr/SP with both carries
  for (int op : {orc::ADD_HL_BC, orc::ADD_HL_DE, orc::ADD_HL_HL, orc::ADD_HL_SP, orc::ADC_HL_BC,
                 orc::ADC_HL_DE, orc::ADC_HL_HL, orc::ADC_HL_SP, orc::SBC_HL_BC, orc::SBC_HL_DE,
                 orc::SBC_HL_HL, orc::SBC_HL_SP, orc::INC_BC, orc::DEC_DE, orc::INC_SP, orc::DEC_SP}) {
    for (int i = 0; i < 400000; i++) {
      uint64_t r = rng();
      orc::State s{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                   uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(rng()), uint8_t(rng())};
      z80b::Z80S d{s.A, s.F, s.B, s.C, s.D, s.E, s.H, s.L, s.SP, s.M};
      orc::Exec(s, uint16_t(op), 0);
      z80b::z_step(d, uint32_t(op), 0);
      checked++;
      if (!same(s, d)) {
        std::printf("MISMATCH16 op=%d (%s)\n", op, orc::OpName(uint16_t(op)));
        return 1;
      }
    }
  }
  // z_stepK with several states per dispatch (the sweep kernel's form)
  for (int op = 0; op < orc::OpCodeCount; op++) {
    for (int i = 0; i < 2000; i++) {
      orc::State o[3];
      z80b::Z80S d[3];
      uint16_t iv = uint16_t(rng());
      for (int k = 0; k < 3; k++) {
        uint64_t r = rng();
        o[k] = orc::State{uint8_t(r), uint8_t(r >> 8), uint8_t(r >> 16), uint8_t(r >> 24), uint8_t(r >> 32),
                          uint8_t(r >> 40), uint8_t(r >> 48), uint8_t(r >> 56), uint16_t(rng()), uint8_t(rng())};
        d[k] = z80b::Z80S{o[k].A, o[k].F, o[k].B, o[k].C, o[k].D, o[k].E, o[k].H, o[k].L, o[k].SP, o[k].M};
        orc::Exec(o[k], uint16_t(op), iv);
      }
      z80b::z_stepK<3>(d, uint32_t(op), iv);
      for (int k = 0; k < 3; k++) {
        checked++;
        if (!same(o[k], d[k])) {
          std::printf("MISMATCH K=3 op=%d (%s) state %d\n", op, orc::OpName(uint16_t(op)), k);
          return 1;
        }
      }
    }
  }
  std::printf("OK %lld states\n", checked);
  return 0;
}
