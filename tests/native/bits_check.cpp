// Host check of the bit-sliced step (z80_bits.cuh) against the scalar step
// function (z80_exec.cuh, itself checked against the oracle): every opcode,
// several immediates, random full states (F included) and all 256 values of
// A with the other registers fixed, 32 states per bit-sliced step.  Built and
// run by tests/test_exec_host.py; exits non-zero on the first mismatch.
#include <cstdio>
#include <random>

#include "../../z80-optimizer_b200/csrc/z80_bits.cuh"

using namespace z80b;

static bool same(const Z80S& x, const Z80S& y) {
  return x.a == y.a && x.f == y.f && x.b == y.b && x.c == y.c && x.d == y.d && x.e == y.e && x.h == y.h &&
         x.l == y.l && x.sp == y.sp && x.m == y.m;
}

int main() {
  std::mt19937_64 rng(4242);
  long long n = 0;
  for (uint32_t op = 0; op < uint32_t(kNumOps); op++) {
    for (int rep = 0; rep < 64; rep++) {
      const uint32_t imm = uint32_t(rng() & 0xFFFF);
      Z80S s[32];
      const bool sweepA = rep < 8;  // 8 x 32 consecutive A values, other registers fixed
      const uint64_t base = rng();
      for (int j = 0; j < 32; j++) {
        const uint64_t r = sweepA ? base : rng();
        s[j] = Z80S{uint32_t(sweepA ? (rep * 32 + j) : (r & 0xFF)), uint32_t((r >> 8) & 0xFF),
                    uint32_t((r >> 16) & 0xFF), uint32_t((r >> 24) & 0xFF), uint32_t((r >> 32) & 0xFF),
                    uint32_t((r >> 40) & 0xFF), uint32_t((r >> 48) & 0xFF), uint32_t((r >> 56) & 0xFF),
                    uint32_t(rng() & 0xFFFF), uint32_t(rng() & 0xFF)};
      }
      ZB z;
      zb_from(z, s);
      zb_step(z, op, imm);
      for (int j = 0; j < 32; j++) {
        Z80S want = s[j];
        z_step(want, op, imm);
        const Z80S got = zb_get(z, j);
        n++;
        if (!same(want, got)) {
          std::printf("MISMATCH op %u (%u) imm %04X state %d: want A=%02X F=%02X B=%02X C=%02X D=%02X E=%02X "
                      "H=%02X L=%02X SP=%04X M=%02X got A=%02X F=%02X B=%02X C=%02X D=%02X E=%02X H=%02X "
                      "L=%02X SP=%04X M=%02X\n",
                      op, op, imm, j, want.a, want.f, want.b, want.c, want.d, want.e, want.h, want.l, want.sp,
                      want.m, got.a, got.f, got.b, got.c, got.d, got.e, got.h, got.l, got.sp, got.m);
          return 1;
        }
      }
    }
  }
  std::printf("OK %lld\n", n);
  return 0;
}
