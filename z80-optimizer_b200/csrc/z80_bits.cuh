// z80_bits.cuh -- bit-sliced Z80 step: 32 states at once, one 32-bit word
// per register bit ("plane"), bit j of every plane belonging to state j.
//
// Every instruction becomes word-wide logic on planes: an 8-bit add is a
// ripple of 8 majority/xor steps for all 32 states, a register move is a
// copy of 8 words, a flag is one plane.  The results follow the scalar step
// function of z80_exec.cuh bit for bit (pkg/cpu/exec.go semantics, flag
// formulas included); the host tests compare the two on every opcode.  The
// ExhaustiveCheck sweep uses it for A-blocks: a lane holds 32 consecutive
// values of A with the other registers equal across them.
#pragma once
#include <cstdint>

#include "z80_exec.cuh"

namespace z80b {

using ZW = uint32_t;  // a plane word: bit j belongs to state j
#include "z80_bits_core.cuh"

// A compact state for pairs whose instructions name no register but B and C
// (after renaming) and neither SP nor the memory byte: D, E, H, L and M
// share one scratch array that such instructions never touch, SP another.
// The step functions below are templates over the state type.
struct ZBc {
  uint32_t a[8], f[8], b[8], c[8];
  union {
    uint32_t x[8], d[8], e[8], h[8], l[8], m[8];
  };
  uint32_t sp[16];
};

// The A, F, B, C state of a compact sweep.  A compact program (a pair's
// instructions renamed by compact_map) names no register but A, F, B and C
// and neither SP nor the memory byte, so nothing else needs to be held.
struct ZB4 {
  uint32_t a[8], f[8], b[8], c[8];
};
#define ZB4_R(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c)
#define ZB4_S(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 6, a)

// The step on ZB4: the cases of zb_step for every instruction that names no
// register but A, F, B and C (the only ones a compact program holds); any
// other opcode leaves the state unchanged and must not occur.
Z80_HD void zb4_step(ZB4& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZB4_S(ZB_LDA, LD_A_B)
    ZB4_R(ZB_LDB, LD_B_A)
    ZB4_R(ZB_LDC, LD_C_A)
    ZB4_R(ZB_LDN, LD_A_N)
    ZB4_S(ZB_ADD, ADD_A_B)
    case ADD_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, 0u); break;
    ZB4_S(ZB_ADC, ADC_A_B)
    case ADC_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, z.f[0]); break;
    ZB4_S(ZB_SUB, SUB_B)
    case SUB_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, 0u); break;
    ZB4_S(ZB_SBC, SBC_A_B)
    case SBC_A_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, z.f[0]); break;
    ZB4_S(ZB_AND, AND_B)
    case AND_N: zb_set8(t8, imm & 0xFFu); zb_and(z, t8); break;
    ZB4_S(ZB_XOR, XOR_B)
    case XOR_N: zb_set8(t8, imm & 0xFFu); zb_xor(z, t8); break;
    ZB4_S(ZB_OR, OR_B)
    case OR_N: zb_set8(t8, imm & 0xFFu); zb_or(z, t8); break;
    ZB4_S(ZB_CP, CP_B)
    case CP_N: zb_set8(t8, imm & 0xFFu); zb_cp(z, t8); break;
    ZB4_R(ZB_INC, INC_A)
    ZB4_R(ZB_DEC, DEC_A)
    ZB4_R(ZB_RLC, RLC_A)
    ZB4_R(ZB_RRC, RRC_A)
    ZB4_R(ZB_RL, RL_A)
    ZB4_R(ZB_RR, RR_A)
    ZB4_R(ZB_SLA, SLA_A)
    ZB4_R(ZB_SRA, SRA_A)
    ZB4_R(ZB_SRL, SRL_A)
    ZB4_R(ZB_SLL, SLL_A)
    ZB4_R(ZB_BIT, BIT_0_A) ZB4_R(ZB_BIT, BIT_1_A) ZB4_R(ZB_BIT, BIT_2_A) ZB4_R(ZB_BIT, BIT_3_A)
    ZB4_R(ZB_BIT, BIT_4_A) ZB4_R(ZB_BIT, BIT_5_A) ZB4_R(ZB_BIT, BIT_6_A) ZB4_R(ZB_BIT, BIT_7_A)
    ZB4_R(ZB_RES, RES_0_A) ZB4_R(ZB_RES, RES_1_A) ZB4_R(ZB_RES, RES_2_A) ZB4_R(ZB_RES, RES_3_A)
    ZB4_R(ZB_RES, RES_4_A) ZB4_R(ZB_RES, RES_5_A) ZB4_R(ZB_RES, RES_6_A) ZB4_R(ZB_RES, RES_7_A)
    ZB4_R(ZB_SET, SET_0_A) ZB4_R(ZB_SET, SET_1_A) ZB4_R(ZB_SET, SET_2_A) ZB4_R(ZB_SET, SET_3_A)
    ZB4_R(ZB_SET, SET_4_A) ZB4_R(ZB_SET, SET_5_A) ZB4_R(ZB_SET, SET_6_A) ZB4_R(ZB_SET, SET_7_A)
    case INC_BC: zb_inc16(z.b, z.c, false); break;
    case DEC_BC: zb_inc16(z.b, z.c, true); break;
    case LD_BC_NN: zb_set8(z.b, (imm >> 8) & 0xFFu); zb_set8(z.c, imm & 0xFFu); break;
    default: zb_acc_step(z, op); break;
  }
}

// The register state: A, F and B..L, for pairs whose programs name neither
// SP nor the memory byte (no renaming: all six registers are held).
struct ZB6 {
  uint32_t a[8], f[8], b[8], c[8], d[8], e[8], h[8], l[8];
};
// The step on ZB6: the cases of zb_step for every instruction that names
// neither SP nor the memory byte; any other opcode leaves the state
// unchanged and must not occur.
Z80_HD void zb6_step(ZB6& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZB_REG_CASES
    default: zb_acc_step(z, op); break;
  }
}

// The wide compact state: A, F, the register pairs BC and HL and the memory
// byte.  A wide program (a pair's instructions renamed by wide_map) names no
// register but B, C, H and L and never SP; it may use the memory byte.
struct ZBW {
  uint32_t a[8], f[8], b[8], c[8], h[8], l[8], m[8];
};
#define ZBW_R(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c) M((base) + 5, h) M((base) + 6, l)
#define ZBW_S(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 4, h) M((base) + 5, l) M((base) + 6, a)

// The step on ZBW: the cases of zb_step for every instruction that names no
// register but A, F, B, C, H, L (and possibly the memory byte) and not SP;
// any other opcode leaves the state unchanged and must not occur.
Z80_HD void zbw_step(ZBW& z, uint32_t op, uint32_t imm) {
  uint32_t t8[8];
  switch (op) {
    ZBW_S(ZB_LDA, LD_A_B)
    ZBW_R(ZB_LDB, LD_B_A)
    ZBW_R(ZB_LDC, LD_C_A)
    ZBW_R(ZB_LDH, LD_H_A)
    ZBW_R(ZB_LDL, LD_L_A)
    ZBW_R(ZB_LDN, LD_A_N)
    ZBW_S(ZB_ADD, ADD_A_B)
    case ADD_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, 0u); break;
    ZBW_S(ZB_ADC, ADC_A_B)
    case ADC_A_N: zb_set8(t8, imm & 0xFFu); zb_add(z, t8, z.f[0]); break;
    ZBW_S(ZB_SUB, SUB_B)
    case SUB_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, 0u); break;
    ZBW_S(ZB_SBC, SBC_A_B)
    case SBC_A_N: zb_set8(t8, imm & 0xFFu); zb_sub(z, t8, z.f[0]); break;
    ZBW_S(ZB_AND, AND_B)
    case AND_N: zb_set8(t8, imm & 0xFFu); zb_and(z, t8); break;
    ZBW_S(ZB_XOR, XOR_B)
    case XOR_N: zb_set8(t8, imm & 0xFFu); zb_xor(z, t8); break;
    ZBW_S(ZB_OR, OR_B)
    case OR_N: zb_set8(t8, imm & 0xFFu); zb_or(z, t8); break;
    ZBW_S(ZB_CP, CP_B)
    case CP_N: zb_set8(t8, imm & 0xFFu); zb_cp(z, t8); break;
    ZBW_R(ZB_INC, INC_A)
    ZBW_R(ZB_DEC, DEC_A)
    ZBW_R(ZB_RLC, RLC_A)
    ZBW_R(ZB_RRC, RRC_A)
    ZBW_R(ZB_RL, RL_A)
    ZBW_R(ZB_RR, RR_A)
    ZBW_R(ZB_SLA, SLA_A)
    ZBW_R(ZB_SRA, SRA_A)
    ZBW_R(ZB_SRL, SRL_A)
    ZBW_R(ZB_SLL, SLL_A)
    ZBW_R(ZB_BIT, BIT_0_A) ZBW_R(ZB_BIT, BIT_1_A) ZBW_R(ZB_BIT, BIT_2_A) ZBW_R(ZB_BIT, BIT_3_A)
    ZBW_R(ZB_BIT, BIT_4_A) ZBW_R(ZB_BIT, BIT_5_A) ZBW_R(ZB_BIT, BIT_6_A) ZBW_R(ZB_BIT, BIT_7_A)
    ZBW_R(ZB_RES, RES_0_A) ZBW_R(ZB_RES, RES_1_A) ZBW_R(ZB_RES, RES_2_A) ZBW_R(ZB_RES, RES_3_A)
    ZBW_R(ZB_RES, RES_4_A) ZBW_R(ZB_RES, RES_5_A) ZBW_R(ZB_RES, RES_6_A) ZBW_R(ZB_RES, RES_7_A)
    ZBW_R(ZB_SET, SET_0_A) ZBW_R(ZB_SET, SET_1_A) ZBW_R(ZB_SET, SET_2_A) ZBW_R(ZB_SET, SET_3_A)
    ZBW_R(ZB_SET, SET_4_A) ZBW_R(ZB_SET, SET_5_A) ZBW_R(ZB_SET, SET_6_A) ZBW_R(ZB_SET, SET_7_A)
    case INC_BC: zb_inc16(z.b, z.c, false); break;
    case INC_HL: zb_inc16(z.h, z.l, false); break;
    case DEC_BC: zb_inc16(z.b, z.c, true); break;
    case DEC_HL: zb_inc16(z.h, z.l, true); break;
    case ADD_HL_BC: zb_hl16(z, z.c, z.b, 0); break;
    case ADD_HL_HL: zb_hl16(z, z.l, z.h, 0); break;
    case LD_BC_NN: zb_set8(z.b, (imm >> 8) & 0xFFu); zb_set8(z.c, imm & 0xFFu); break;
    case LD_HL_NN: zb_set8(z.h, (imm >> 8) & 0xFFu); zb_set8(z.l, imm & 0xFFu); break;
    case ADC_HL_BC: zb_hl16(z, z.c, z.b, 1); break;
    case ADC_HL_HL: zb_hl16(z, z.l, z.h, 1); break;
    case SBC_HL_BC: zb_hl16(z, z.c, z.b, 2); break;
    case SBC_HL_HL: zb_hl16(z, z.l, z.h, 2); break;
    case LD_A_HLI: zb_copy8(z.a, z.m); break;
    case LD_B_HLI: zb_copy8(z.b, z.m); break;
    case LD_C_HLI: zb_copy8(z.c, z.m); break;
    case LD_H_HLI: zb_copy8(z.h, z.m); break;
    case LD_L_HLI: zb_copy8(z.l, z.m); break;
    case LD_HLI_A: zb_copy8(z.m, z.a); break;
    case LD_HLI_B: zb_copy8(z.m, z.b); break;
    case LD_HLI_C: zb_copy8(z.m, z.c); break;
    case LD_HLI_H: zb_copy8(z.m, z.h); break;
    case LD_HLI_L: zb_copy8(z.m, z.l); break;
    case LD_HLI_N: zb_set8(z.m, imm & 0xFFu); break;
    case LD_A_BCI: case LD_A_DEI: zb_copy8(z.a, z.m); break;
    case LD_BCI_A: case LD_DEI_A: zb_copy8(z.m, z.a); break;
    case ADD_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, 0u); break;
    case ADC_A_HLI: zb_copy8(t8, z.m); zb_add(z, t8, z.f[0]); break;
    case SUB_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, 0u); break;
    case SBC_A_HLI: zb_copy8(t8, z.m); zb_sub(z, t8, z.f[0]); break;
    case AND_HLI: zb_copy8(t8, z.m); zb_and(z, t8); break;
    case XOR_HLI: zb_copy8(t8, z.m); zb_xor(z, t8); break;
    case OR_HLI: zb_copy8(t8, z.m); zb_or(z, t8); break;
    case CP_HLI: zb_copy8(t8, z.m); zb_cp(z, t8); break;
    case INC_HLI: zb_inc(z, z.m); break;
    case DEC_HLI: zb_dec(z, z.m); break;
    case RLC_HLI: zb_rot(z, z.m, 0); break;
    case RRC_HLI: zb_rot(z, z.m, 1); break;
    case RL_HLI: zb_rot(z, z.m, 2); break;
    case RR_HLI: zb_rot(z, z.m, 3); break;
    case SLA_HLI: zb_rot(z, z.m, 4); break;
    case SRA_HLI: zb_rot(z, z.m, 5); break;
    case SRL_HLI: zb_rot(z, z.m, 6); break;
    case SLL_HLI: zb_rot(z, z.m, 7); break;
    case BIT_0_HLI: zb_bit(z, z.m, 0); break;
    case BIT_1_HLI: zb_bit(z, z.m, 1); break;
    case BIT_2_HLI: zb_bit(z, z.m, 2); break;
    case BIT_3_HLI: zb_bit(z, z.m, 3); break;
    case BIT_4_HLI: zb_bit(z, z.m, 4); break;
    case BIT_5_HLI: zb_bit(z, z.m, 5); break;
    case BIT_6_HLI: zb_bit(z, z.m, 6); break;
    case BIT_7_HLI: zb_bit(z, z.m, 7); break;
    case RES_0_HLI: z.m[0] = 0u; break;
    case RES_1_HLI: z.m[1] = 0u; break;
    case RES_2_HLI: z.m[2] = 0u; break;
    case RES_3_HLI: z.m[3] = 0u; break;
    case RES_4_HLI: z.m[4] = 0u; break;
    case RES_5_HLI: z.m[5] = 0u; break;
    case RES_6_HLI: z.m[6] = 0u; break;
    case RES_7_HLI: z.m[7] = 0u; break;
    case SET_0_HLI: z.m[0] = kZBOnes; break;
    case SET_1_HLI: z.m[1] = kZBOnes; break;
    case SET_2_HLI: z.m[2] = kZBOnes; break;
    case SET_3_HLI: z.m[3] = kZBOnes; break;
    case SET_4_HLI: z.m[4] = kZBOnes; break;
    case SET_5_HLI: z.m[5] = kZBOnes; break;
    case SET_6_HLI: z.m[6] = kZBOnes; break;
    case SET_7_HLI: z.m[7] = kZBOnes; break;
    default: zb_acc_step(z, op); break;
  }
}

// Block decoding of an ExhaustiveCheck sweep (pkg/search/verifier.go:
// 428-612), set up once per pair.  Block index fields, fastest first: SP (4
// bits, reduced sweeps that read SP), the swept registers from the last to
// the first (8 bits each in a full sweep, 5 bits indexing the representative
// values in a reduced one), carry.  Packed into two words so that it costs
// the sweep kernels two registers: register r's field position (6 bits, r =
// B, C, D, E, H, L, M; five in lo, two in hi), then in hi the swept
// registers (bit r), the SP field, the reduced sweep and the carry's
// position.  Unswept registers start at 0.
struct BDec {
  uint32_t lo, hi;
};
Z80_HD BDec bdec_make(bool spw, bool reduced, int nx, int fw, const int (&slot)[7]) {
  const int base = spw ? 4 : 0;
  uint32_t sh[7] = {0, 0, 0, 0, 0, 0, 0}, on = 0;
  for (int r = 0; r < 7; r++) {
    if (slot[r] < 0) continue;
    sh[r] = uint32_t(base + (nx - 1 - slot[r]) * fw);
    on |= 1u << r;
  }
  BDec d;
  d.lo = sh[0] | sh[1] << 6 | sh[2] << 12 | sh[3] << 18 | sh[4] << 24;
  d.hi = sh[5] | sh[6] << 6 | on << 12 | (spw ? 1u : 0u) << 19 | (reduced ? 1u : 0u) << 20 |
         uint32_t(base + nx * fw) << 21;
  return d;
}
// The initial state of block ab (A = 0); rep / repsp: the 32 representative
// register values and the 16 SP values.
Z80_HD Z80S bdec_state(const BDec& d, unsigned long long ab, const uint8_t* rep, const uint16_t* repsp) {
  const bool reduced = (d.hi >> 20) & 1u;
  uint32_t v[7];
  for (int r = 0; r < 7; r++) {
    v[r] = 0u;
    if ((d.hi >> (12 + r)) & 1u) {
      const uint32_t sh = (r < 5 ? d.lo >> (6 * r) : d.hi >> (6 * (r - 5))) & 63u;
      const uint32_t x = uint32_t(ab >> sh) & (reduced ? 31u : 255u);
      v[r] = reduced ? uint32_t(rep[x]) : x;
    }
  }
  Z80S s;
  s.a = 0;
  s.f = uint32_t(ab >> (d.hi >> 21)) & 1u;
  s.b = v[0];
  s.c = v[1];
  s.d = v[2];
  s.e = v[3];
  s.h = v[4];
  s.l = v[5];
  s.m = v[6];
  s.sp = ((d.hi >> 19) & 1u) ? uint32_t(repsp[uint32_t(ab) & 15u]) : 0u;
  return s;
}

// Block decoding for compact pairs.  A compact pair reads at most two
// registers and neither SP nor the memory byte, so its sweep is a full one:
// block index = carry above nx 8-bit fields, the last swept register in the
// lowest byte.  The initial values of the renamed B and C (the registers o0
// and o1 stand for) and the carry are then shifts and masks of the block
// index, set up once per pair: slot[r] is register r's field (-1: not
// swept; a register that is named but not read starts at 0).
struct CDec {
  uint32_t shb, mb, shc, mc, shf;
};
Z80_HD CDec cdec_make(int nx, const int (&slot)[7], int o0, int o1) {
  CDec d{0u, 0u, 0u, 0u, uint32_t(8 * nx)};
  if (o0 >= 0 && slot[o0] >= 0) {
    d.shb = uint32_t(8 * (nx - 1 - slot[o0]));
    d.mb = 0xFFu;
  }
  if (o1 >= 0 && slot[o1] >= 0) {
    d.shc = uint32_t(8 * (nx - 1 - slot[o1]));
    d.mc = 0xFFu;
  }
  return d;
}
// B, C and the carry of block ab.
Z80_HD void cdec_vals(const CDec& d, unsigned long long ab, uint32_t& vb, uint32_t& vc, uint32_t& carry) {
  const uint32_t lo = uint32_t(ab);
  vb = (lo >> d.shb) & d.mb;
  vc = (lo >> d.shc) & d.mc;
  carry = (lo >> d.shf) & 1u;
}

// Block decoding for wide compact pairs.  A wide pair reads at most four
// registers and the memory byte, never SP, so its block index (below 2^26)
// is the carry above at most five fields, 8 bits each in a full sweep and
// 5 bits indexing the representative values in a reduced one.  The initial
// values of the five wide fields (B, C, H, L as renamed, then M) are shifts
// and masks of the index: lo packs the five fields' shifts (6 bits each),
// hi the fields that are swept (bits 0..4), the reduced flag (bit 5) and the
// carry's shift (bits 6..11).  o[s]: the original register (0..5) that
// field s stands for, or -1; slot[r]: register r's sweep field (-1: not
// swept; a named register that is not read starts at 0).
struct WDec {
  uint32_t lo, hi;
};
Z80_HD WDec wdec_make(int nx, bool reduced, const int (&slot)[7], const int (&o)[4]) {
  const int fw = reduced ? 5 : 8;
  uint32_t lo = 0, on = 0;
  for (int s = 0; s < 5; s++) {
    const int r = s < 4 ? o[s] : 6;
    if (r < 0 || slot[r] < 0) continue;
    lo |= uint32_t((nx - 1 - slot[r]) * fw) << (6 * s);
    on |= 1u << s;
  }
  return WDec{lo, on | (reduced ? 32u : 0u) | uint32_t(nx * fw) << 6};
}
// The five fields and the carry of block ab.
Z80_HD void wdec_vals(const WDec& d, uint32_t ab, const uint8_t* rep, uint32_t (&v)[5], uint32_t& carry) {
  const bool reduced = (d.hi >> 5) & 1u;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int s = 0; s < 5; s++) {
    const uint32_t x = (ab >> ((d.lo >> (6 * s)) & 63u)) & (reduced ? 31u : 255u);
    v[s] = ((d.hi >> s) & 1u) ? (reduced ? uint32_t(rep[x]) : x) : 0u;
  }
  carry = (ab >> ((d.hi >> 6) & 63u)) & 1u;
}

// Planes <-> scalar states (host tests; the sweep builds planes directly).
template <class ZT>
Z80_HD void zb_from(ZT& z, const Z80S (&s)[32]) {
  for (int i = 0; i < 8; i++) {
    z.a[i] = z.f[i] = z.b[i] = z.c[i] = z.d[i] = z.e[i] = z.h[i] = z.l[i] = z.m[i] = 0;
  }
  for (int i = 0; i < 16; i++) z.sp[i] = 0;
  for (int j = 0; j < 32; j++) {
    const uint32_t bit = 1u << j;
    for (int i = 0; i < 8; i++) {
      if ((s[j].a >> i) & 1u) z.a[i] |= bit;
      if ((s[j].f >> i) & 1u) z.f[i] |= bit;
      if ((s[j].b >> i) & 1u) z.b[i] |= bit;
      if ((s[j].c >> i) & 1u) z.c[i] |= bit;
      if ((s[j].d >> i) & 1u) z.d[i] |= bit;
      if ((s[j].e >> i) & 1u) z.e[i] |= bit;
      if ((s[j].h >> i) & 1u) z.h[i] |= bit;
      if ((s[j].l >> i) & 1u) z.l[i] |= bit;
      if ((s[j].m >> i) & 1u) z.m[i] |= bit;
    }
    for (int i = 0; i < 16; i++)
      if ((s[j].sp >> i) & 1u) z.sp[i] |= bit;
  }
}
template <class ZT>
Z80_HD Z80S zb_get(const ZT& z, int j) {
  Z80S s{};
  for (int i = 0; i < 8; i++) {
    s.a |= ((z.a[i] >> j) & 1u) << i;
    s.f |= ((z.f[i] >> j) & 1u) << i;
    s.b |= ((z.b[i] >> j) & 1u) << i;
    s.c |= ((z.c[i] >> j) & 1u) << i;
    s.d |= ((z.d[i] >> j) & 1u) << i;
    s.e |= ((z.e[i] >> j) & 1u) << i;
    s.h |= ((z.h[i] >> j) & 1u) << i;
    s.l |= ((z.l[i] >> j) & 1u) << i;
    s.m |= ((z.m[i] >> j) & 1u) << i;
  }
  for (int i = 0; i < 16; i++) s.sp |= ((z.sp[i] >> j) & 1u) << i;
  return s;
}

}  // namespace z80b
