// Host check of the layouts behind the two bit-sliced sweeps
// (z80b_kernels.cu).  A-independent pairs (xbits_unit): for every sweep
// shape, the state planes the kernel builds for an aligned group of 32
// A-blocks (the moving field's planes from counting patterns, transposed
// representative tables or constants) hold, in bit j, exactly the initial
// state of block g0 + j as the block decoder defines it, and sweeping random
// A-independent pairs this way at A = 0 and 1 gives the CPU oracle's
// ExhaustiveCheck[Masked] verdict.  A-dependent pairs (bits_unit): lane l of
// a unit takes block 4u + l/8 and A = 32(l % 8) .. +31, and sweeping random
// A-dependent pairs that way gives the oracle's verdict too.  The decoder
// and the plane construction are restated here from the kernel (warp ballots
// become loops over j).  Built and run by tests/test_exec_host.py.
#include <cstdio>
#include <random>
#include <vector>

#include "../../oracle/z80_oracle.h"
#include "../../z80-optimizer_b200/csrc/z80_bits.cuh"
#include "../../z80-optimizer_b200/csrc/z80_tables.h"

using namespace z80b;

namespace {

struct Shape {
  bool spw, reduced;
  int nx, fw;
  int slot[7];
  int rlast;
  uint64_t nblocks;
};

Shape shape_of(uint16_t reads) {
  Shape s{};
  const uint32_t bits[7] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM};
  int k = 0;
  for (int r = 0; r < 7; r++) s.slot[r] = (reads & bits[r]) ? k++ : -1;
  s.nx = k;
  s.spw = (reads & kRegSP) != 0;
  s.reduced = s.spw || s.nx > 2;
  s.fw = s.reduced ? 5 : 8;
  s.rlast = -1;
  for (int r = 0; r < 7; r++)
    if (s.slot[r] == s.nx - 1) s.rlast = r;
  s.nblocks = sweep_for(reads).states / 256;
  return s;
}

// the kernel's block decoder: SP fastest, then the fields last to first,
// then the carry
Z80S decode(uint64_t ab, const Shape& s) {
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

// The kernels' shift-and-mask block decoder (bdec_make / bdec_state in
// z80_bits.cuh) against the decoder above, for every combination of swept
// registers and SP; returns false on a difference.
bool check_bdec() {
  std::mt19937_64 rng(99);
  int n = 0;
  for (uint32_t m = 0; m < 256; m++) {
    uint16_t reads = uint16_t(kRegA);
    const uint32_t bits[8] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM, kRegSP};
    for (int i = 0; i < 8; i++)
      if ((m >> i) & 1u) reads |= uint16_t(bits[i]);
    const Shape s = shape_of(reads);
    const BDec d = bdec_make(s.spw, s.reduced, s.nx, s.fw, s.slot);
    for (int t = 0; t < 600; t++) {
      const uint64_t ab = t < 64 ? (t < 32 ? uint64_t(t) : s.nblocks - 1 - uint64_t(t - 32) % s.nblocks)
                                 : rng() % s.nblocks;
      const Z80S a = decode(ab, s), b = bdec_state(d, ab, rep_values(), rep_sp());
      if (a.a != b.a || a.f != b.f || a.b != b.b || a.c != b.c || a.d != b.d || a.e != b.e || a.h != b.h ||
          a.l != b.l || a.sp != b.sp || a.m != b.m) {
        std::printf("block decoder differs: reads %03x block %llu\n", reads, (unsigned long long)ab);
        return false;
      }
      n++;
    }
  }
  return n > 0;
}

uint32_t* reg_planes(ZB& z, int r) {
  switch (r) {
    case 0: return z.b;
    case 1: return z.c;
    case 2: return z.d;
    case 3: return z.e;
    case 4: return z.h;
    case 5: return z.l;
    default: return z.m;
  }
}

// the kernel's planes for the group starting at block g0, A = abit
ZB group_planes(uint64_t g0, const Shape& s, uint32_t abit) {
  const uint8_t* rep = rep_values();
  const uint16_t* repsp = rep_sp();
  const Z80S x = decode(g0 < s.nblocks ? g0 : 0, s);
  uint32_t vp[8] = {0, 0, 0, 0, 0, 0, 0, 0}, spp[16] = {0};
  uint32_t fp0 = 0;
  if (s.spw) {
    for (int i = 0; i < 16; i++)
      for (int j = 0; j < 32; j++) spp[i] |= ((repsp[j & 15] >> i) & 1u) << j;
    const uint32_t x0 = uint32_t(g0 >> 4) & 31u;
    const uint32_t lo = rep[x0], hi = rep[(x0 + 1) & 31];
    for (int i = 0; i < 8; i++) vp[i] = (((lo >> i) & 1) ? 0x0000FFFFu : 0u) | (((hi >> i) & 1) ? 0xFFFF0000u : 0u);
    fp0 = 0xFFFF0000u;
  } else if (s.reduced) {
    for (int i = 0; i < 8; i++)
      for (int j = 0; j < 32; j++) vp[i] |= ((rep[j] >> i) & 1u) << j;
  } else {
    uint32_t v = 0;
    const uint32_t vals[7] = {x.b, x.c, x.d, x.e, x.h, x.l, x.m};
    if (s.rlast >= 0) v = vals[s.rlast];
    const uint32_t pat[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
    for (int i = 0; i < 5; i++) vp[i] = pat[i];
    for (int i = 5; i < 8; i++) vp[i] = ((v >> i) & 1u) ? kZBOnes : 0u;
    fp0 = 0xAAAAAAAAu;
  }
  ZB z;
  zb_set8(z.a, abit);
  zb_set8(z.f, x.f);
  zb_set8(z.b, x.b);
  zb_set8(z.c, x.c);
  zb_set8(z.d, x.d);
  zb_set8(z.e, x.e);
  zb_set8(z.h, x.h);
  zb_set8(z.l, x.l);
  zb_set8(z.m, x.m);
  for (int i = 0; i < 16; i++) z.sp[i] = s.spw ? spp[i] : (((x.sp >> i) & 1u) ? kZBOnes : 0u);
  if (s.nx >= 1) {
    uint32_t* p = reg_planes(z, s.rlast);
    for (int i = 0; i < 8; i++) p[i] = vp[i];
  } else {
    z.f[0] = fp0;
  }
  return z;
}

bool same(const Z80S& a, const Z80S& b) {
  return a.a == b.a && a.f == b.f && a.b == b.b && a.c == b.c && a.d == b.d && a.e == b.e && a.h == b.h &&
         a.l == b.l && a.sp == b.sp && a.m == b.m;
}

uint32_t diff_mask(const ZB& x, const ZB& y, uint32_t keepF) {
  uint32_t d = 0;
  for (int i = 0; i < 8; i++) {
    d |= x.a[i] ^ y.a[i];
    if ((keepF >> i) & 1u) d |= x.f[i] ^ y.f[i];
    d |= (x.b[i] ^ y.b[i]) | (x.c[i] ^ y.c[i]) | (x.d[i] ^ y.d[i]) | (x.e[i] ^ y.e[i]) | (x.h[i] ^ y.h[i]) |
         (x.l[i] ^ y.l[i]) | (x.m[i] ^ y.m[i]);
  }
  for (int i = 0; i < 16; i++) d |= x.sp[i] ^ y.sp[i];
  return d;
}

}  // namespace

int main() {
  orc::Init();
  if (!check_bdec()) return 1;
  std::mt19937_64 rng(2027);
  // 1. layout: every read mask over B..L, M, SP (A and F do not shape the
  // sweep), sampled groups of each shape
  long long checked = 0;
  for (uint32_t m = 0; m < 256; m++) {
    uint16_t reads = 0;
    const uint16_t bits[8] = {kRegB, kRegC, kRegD, kRegE, kRegH, kRegL, kRegM, kRegSP};
    for (int b = 0; b < 8; b++)
      if ((m >> b) & 1) reads |= bits[b];
    const Shape s = shape_of(reads);
    const uint64_t ngroups = (s.nblocks + 31) / 32;
    for (int t = 0; t < 24; t++) {
      const uint64_t g = t == 0 ? 0 : (t == 1 ? ngroups - 1 : rng() % ngroups);
      const uint64_t g0 = g * 32;
      for (uint32_t abit = 0; abit < 2; abit++) {
        const ZB z = group_planes(g0, s, abit);
        for (uint64_t j = 0; j < 32 && g0 + j < s.nblocks; j++) {
          Z80S want = decode(g0 + j, s);
          want.a = abit;
          if (!same(zb_get(z, int(j)), want)) {
            std::printf("layout mismatch: reads %03x group %llu state %llu\n", reads, (unsigned long long)g,
                        (unsigned long long)j);
            return 1;
          }
          checked++;
        }
      }
    }
  }
  // 2. verdicts: random A-independent pairs with sweeps of at most 2^15
  // blocks, swept group by group at A = 0 and 1, against the oracle
  const auto& I = orc::Instructions8();
  int pairs = 0, equal = 0;
  for (int trial = 0; trial < 400000 && pairs < 3000; trial++) {
    const int tn = 1 + int(rng() % 2), cn = 1 + int(rng() % 2);
    uint32_t tw[2], cw[2];
    orc::Instruction ti[2], ci[2];
    for (int i = 0; i < tn; i++) {
      ti[i] = I[rng() % I.size()];
      tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
    }
    const int mode = int(rng() % 3);  // 0: random candidate, 1: the target, 2: the target swapped
    for (int i = 0; i < cn; i++) ci[i] = I[rng() % I.size()];
    if (mode == 1 || (mode == 2 && tn == 2)) {
      ci[0] = ti[mode == 2 ? 1 : 0];
      ci[1] = ti[mode == 2 ? 0 : 1];
    }
    const int cl = mode == 0 ? cn : tn;
    for (int i = 0; i < cl; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
    if (!seq_aflow(tw, tn) || !seq_aflow(cw, cl)) continue;
    const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cl));
    const Shape s = shape_of(reads);
    if (s.nblocks > (1u << 15)) continue;
    pairs++;
    for (uint8_t dead : {uint8_t(0x00), uint8_t(0xFF)}) {
      const uint32_t keepF = uint8_t(~dead);
      bool bad = false;
      for (uint64_t g0 = 0; g0 < s.nblocks && !bad; g0 += 32) {
        const uint32_t valid = s.nblocks - g0 >= 32 ? 0xFFFFFFFFu : ((1u << uint32_t(s.nblocks - g0)) - 1u);
        for (uint32_t abit = 0; abit < 2 && !bad; abit++) {
          ZB zc = group_planes(g0, s, abit), zt = zc;
          for (int i = 0; i < cl; i++) zb_step(zc, cw[i] & 0xFFFFu, cw[i] >> 16);
          for (int i = 0; i < tn; i++) zb_step(zt, tw[i] & 0xFFFFu, tw[i] >> 16);
          bad = (diff_mask(zc, zt, keepF) & valid) != 0;
        }
      }
      const bool want = dead ? orc::ExhaustiveCheckMasked(ti, tn, ci, cl, dead) : orc::ExhaustiveCheck(ti, tn, ci, cl);
      if (want != !bad) {
        std::printf("verdict mismatch: target %08x %08x (%d) candidate %08x %08x (%d) dead %02x: oracle %d\n", tw[0],
                    tn > 1 ? tw[1] : 0, tn, cw[0], cl > 1 ? cw[1] : 0, cl, dead, want ? 1 : 0);
        return 1;
      }
      equal += want ? 1 : 0;
    }
  }
  if (pairs < 1000 || equal < 100) {
    std::printf("too few pairs (%d) or equivalences (%d)\n", pairs, equal);
    return 1;
  }
  // 3. A-dependent pairs: every block at all 256 values of A, 32 per word
  // (lane l of a unit: block 4u + l/8, A from 32(l % 8)), against the oracle
  int dpairs = 0, dequal = 0;
  for (int trial = 0; trial < 400000 && dpairs < 1500; trial++) {
    const int tn = 1 + int(rng() % 2);
    uint32_t tw[2], cw[2];
    orc::Instruction ti[2], ci[2];
    for (int i = 0; i < tn; i++) {
      ti[i] = I[rng() % I.size()];
      tw[i] = uint32_t(ti[i].op) | uint32_t(ti[i].imm) << 16;
    }
    const int mode = int(rng() % 3);
    int cl = 1 + int(rng() % 2);
    for (int i = 0; i < cl; i++) ci[i] = I[rng() % I.size()];
    if (mode == 1 || (mode == 2 && tn == 2)) {
      cl = tn;
      ci[0] = ti[mode == 2 ? 1 : 0];
      ci[1] = ti[mode == 2 ? 0 : 1];
    }
    for (int i = 0; i < cl; i++) cw[i] = uint32_t(ci[i].op) | uint32_t(ci[i].imm) << 16;
    if (seq_aflow(tw, tn) && seq_aflow(cw, cl)) continue;  // A-dependent pairs only
    const uint16_t reads = uint16_t(seq_reads(tw, tn) | seq_reads(cw, cl));
    const Shape s = shape_of(reads);
    if (s.nblocks > (1u << 12)) continue;
    dpairs++;
    for (uint8_t dead : {uint8_t(0x00), uint8_t(0xFF)}) {
      const uint32_t keepF = uint8_t(~dead);
      bool bad = false;
      for (uint64_t blk = 0; blk < s.nblocks && !bad; blk++) {
        const Z80S x = decode(blk, s);
        for (uint32_t a0 = 0; a0 < 256 && !bad; a0 += 32) {
          ZB z;
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
          zb_set8(z.m, x.m);
          for (int i = 0; i < 16; i++) z.sp[i] = ((x.sp >> i) & 1u) ? kZBOnes : 0u;
          for (int j = 0; j < 32; j++) {
            Z80S want = x;
            want.a = a0 + uint32_t(j);
            if (!same(zb_get(z, j), want)) {
              std::printf("A-dependent layout mismatch: block %llu A %u\n", (unsigned long long)blk, a0 + j);
              return 1;
            }
          }
          ZB zc = z, zt = z;
          for (int i = 0; i < cl; i++) zb_step(zc, cw[i] & 0xFFFFu, cw[i] >> 16);
          for (int i = 0; i < tn; i++) zb_step(zt, tw[i] & 0xFFFFu, tw[i] >> 16);
          bad = diff_mask(zc, zt, keepF) != 0;
        }
      }
      const bool want = dead ? orc::ExhaustiveCheckMasked(ti, tn, ci, cl, dead) : orc::ExhaustiveCheck(ti, tn, ci, cl);
      if (want != !bad) {
        std::printf("A-dependent verdict mismatch: target %08x %08x (%d) candidate %08x %08x (%d) dead %02x\n", tw[0],
                    tn > 1 ? tw[1] : 0, tn, cw[0], cl > 1 ? cw[1] : 0, cl, dead);
        return 1;
      }
      dequal += want ? 1 : 0;
    }
  }
  if (dpairs < 500 || dequal < 50) {
    std::printf("too few A-dependent pairs (%d) or equivalences (%d)\n", dpairs, dequal);
    return 1;
  }
  std::printf("OK %lld states, %d A-independent pairs (%d equivalent verdicts), %d A-dependent pairs (%d)\n", checked,
              pairs, equal, dpairs, dequal);
  return 0;
}
