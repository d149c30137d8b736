// z80_exec.cuh -- the Z80 step function shared by every kernel.
//
// One instruction of the reference emulator (pkg/cpu/exec.go:8-1034, helpers
// exec.go:1038-1264) over register-resident states.  Each Z80 register
// lives in its own 32-bit register (8-bit values, SP 16-bit), so the opcode
// switch's cases touch named registers only; z_stepK applies one dispatch to
// K states, which amortizes the dispatch over the K states a lane carries
// through a sweep.  Inside a warp every lane runs the same opcode, so the
// dispatch never diverges.
//
// The flag lookups of pkg/cpu/flags.go are computed instead of loaded:
//   Sz53Table[v]   = (v & 0xA8) | (v == 0 ? Z : 0)
//   ParityTable[v] = popcount(v) even ? P : 0
//   HalfcarryAdd/SubTable[idx from bit 3 of a, v, result] = bit 4 of a^v^r
//     (carry resp. borrow out of bit 3; bit 12 for the 16-bit forms)
//   OverflowAddTable = (a ^ r) & (v ^ r) & 0x80,
//   OverflowSubTable = (a ^ v) & (a ^ r) & 0x80 (bit 15 for 16-bit forms).
// The header also compiles as plain C++ so the host tests can compare it with
// the CPU oracle opcode by opcode.
#pragma once
#include <cstdint>

#include "z80_isa.h"

#if defined(__CUDACC__)
#define Z80_HD __host__ __device__ __forceinline__
#else
#define Z80_HD inline
#endif

namespace z80b {

struct Z80S {
  uint32_t a, f, b, c, d, e, h, l, sp, m;
};

Z80_HD uint32_t z_popc(uint32_t v) {
#if defined(__CUDA_ARCH__)
  return uint32_t(__popc(v));
#else
  return uint32_t(__builtin_popcount(v));
#endif
}
Z80_HD uint32_t z_sz53(uint32_t v) { return (v & 0xA8u) | (v ? 0u : 0x40u); }
Z80_HD uint32_t z_par(uint32_t v) { return (z_popc(v) & 1u) ? 0u : 0x04u; }
Z80_HD uint32_t z_sz53p(uint32_t v) { return z_sz53(v) | z_par(v); }

// ---- 8-bit ALU (exec.go:1038-1102)
Z80_HD void z_add(Z80S& s, uint32_t v) {
  uint32_t t = s.a + v;
  s.f = (t >> 8) | ((s.a ^ v ^ t) & 0x10u) | (((s.a ^ t) & (v ^ t) & 0x80u) >> 5) | z_sz53(t & 0xFFu);
  s.a = t & 0xFFu;
}
Z80_HD void z_adc(Z80S& s, uint32_t v) {
  uint32_t t = s.a + v + (s.f & 1u);
  s.f = (t >> 8) | ((s.a ^ v ^ t) & 0x10u) | (((s.a ^ t) & (v ^ t) & 0x80u) >> 5) | z_sz53(t & 0xFFu);
  s.a = t & 0xFFu;
}
Z80_HD void z_sub(Z80S& s, uint32_t v) {
  uint32_t t = s.a - v;
  s.f = ((t >> 8) & 1u) | 0x02u | ((s.a ^ v ^ t) & 0x10u) | (((s.a ^ v) & (s.a ^ t) & 0x80u) >> 5) |
        z_sz53(t & 0xFFu);
  s.a = t & 0xFFu;
}
Z80_HD void z_sbc(Z80S& s, uint32_t v) {
  uint32_t t = s.a - v - (s.f & 1u);
  s.f = ((t >> 8) & 1u) | 0x02u | ((s.a ^ v ^ t) & 0x10u) | (((s.a ^ v) & (s.a ^ t) & 0x80u) >> 5) |
        z_sz53(t & 0xFFu);
  s.a = t & 0xFFu;
}
Z80_HD void z_and(Z80S& s, uint32_t v) { s.a &= v; s.f = 0x10u | z_sz53p(s.a); }
Z80_HD void z_xor(Z80S& s, uint32_t v) { s.a ^= v; s.f = z_sz53p(s.a); }
Z80_HD void z_or(Z80S& s, uint32_t v) { s.a |= v; s.f = z_sz53p(s.a); }
Z80_HD void z_cp(Z80S& s, uint32_t v) {
  uint32_t t = s.a - v;
  uint32_t borrow = (t >> 8) & 1u;
  s.f = (borrow ? 1u : (s.a == v ? 0x40u : 0u)) | 0x02u | ((s.a ^ v ^ t) & 0x10u) |
        (((s.a ^ v) & (s.a ^ t) & 0x80u) >> 5) | (v & 0x28u) | (t & 0x80u);
}
// exec.go:1104-1116
Z80_HD void z_inc(Z80S& s, uint32_t& r) {
  r = (r + 1u) & 0xFFu;
  s.f = (s.f & 1u) | (r == 0x80u ? 0x04u : 0u) | ((r & 0x0Fu) ? 0u : 0x10u) | z_sz53(r);
}
Z80_HD void z_dec(Z80S& s, uint32_t& r) {
  uint32_t f = (s.f & 1u) | ((r & 0x0Fu) ? 0u : 0x10u) | 0x02u;
  r = (r - 1u) & 0xFFu;
  s.f = f | (r == 0x7Fu ? 0x04u : 0u) | z_sz53(r);
}
// exec.go:1118-1136
Z80_HD void z_daa(Z80S& s) {
  uint32_t add = 0, carry = s.f & 1u;
  if ((s.f & 0x10u) || (s.a & 0x0Fu) > 9u) add = 6u;
  if (carry || s.a > 0x99u) add |= 0x60u;
  if (s.a > 0x99u) carry = 1u;
  if (s.f & 0x02u) z_sub(s, add);
  else z_add(s, add);
  s.f = (s.f & ~0x05u & 0xFFu) | carry | z_par(s.a);
}
// ---- CB rotates/shifts (exec.go:1139-1185,1251-1256); return the new value
Z80_HD uint32_t z_rlc(Z80S& s, uint32_t v) {
  v = ((v << 1) | (v >> 7)) & 0xFFu;
  s.f = (v & 1u) | z_sz53p(v);
  return v;
}
Z80_HD uint32_t z_rrc(Z80S& s, uint32_t v) {
  uint32_t c = v & 1u;
  v = ((v >> 1) | (v << 7)) & 0xFFu;
  s.f = c | z_sz53p(v);
  return v;
}
Z80_HD uint32_t z_rl(Z80S& s, uint32_t v) {
  uint32_t n = ((v << 1) | (s.f & 1u)) & 0xFFu;
  s.f = (v >> 7) | z_sz53p(n);
  return n;
}
Z80_HD uint32_t z_rr(Z80S& s, uint32_t v) {
  uint32_t n = (v >> 1) | ((s.f & 1u) << 7);
  s.f = (v & 1u) | z_sz53p(n);
  return n;
}
Z80_HD uint32_t z_sla(Z80S& s, uint32_t v) {
  uint32_t n = (v << 1) & 0xFFu;
  s.f = (v >> 7) | z_sz53p(n);
  return n;
}
Z80_HD uint32_t z_sra(Z80S& s, uint32_t v) {
  uint32_t n = (v & 0x80u) | (v >> 1);
  s.f = (v & 1u) | z_sz53p(n);
  return n;
}
Z80_HD uint32_t z_srl(Z80S& s, uint32_t v) {
  uint32_t n = v >> 1;
  s.f = (v & 1u) | z_sz53p(n);
  return n;
}
Z80_HD uint32_t z_sll(Z80S& s, uint32_t v) {
  uint32_t n = ((v << 1) | 1u) & 0xFFu;
  s.f = (v >> 7) | z_sz53p(n);
  return n;
}
// exec.go:1240-1248
Z80_HD void z_bit(Z80S& s, uint32_t r, uint32_t bit) {
  uint32_t f = (s.f & 1u) | 0x10u | (r & 0x28u);
  if (!(r & (1u << bit))) f |= 0x44u;
  if (bit == 7u && (r & 0x80u)) f |= 0x80u;
  s.f = f;
}
// ---- 16-bit arithmetic (exec.go:1189-1236)
Z80_HD void z_addhl(Z80S& s, uint32_t v) {
  uint32_t hl = (s.h << 8) | s.l;
  uint32_t r = hl + v;
  uint32_t hc = (hl & 0x0FFFu) + (v & 0x0FFFu);
  s.f = (s.f & 0xC4u) | ((hc >> 8) & 0x10u) | (r >> 16) | ((r >> 8) & 0x28u);
  s.h = (r >> 8) & 0xFFu;
  s.l = r & 0xFFu;
}
Z80_HD void z_adchl(Z80S& s, uint32_t v) {
  uint32_t hl = (s.h << 8) | s.l;
  uint32_t r = hl + v + (s.f & 1u);
  s.h = (r >> 8) & 0xFFu;
  s.l = r & 0xFFu;
  s.f = (r >> 16) | (((hl ^ r) & (v ^ r) & 0x8000u) >> 13) | (s.h & 0xA8u) |
        (((hl ^ v ^ r) >> 8) & 0x10u) | ((r & 0xFFFFu) ? 0u : 0x40u);
}
Z80_HD void z_sbchl(Z80S& s, uint32_t v) {
  uint32_t hl = (s.h << 8) | s.l;
  uint32_t r = hl - v - (s.f & 1u);
  s.h = (r >> 8) & 0xFFu;
  s.l = r & 0xFFu;
  s.f = ((r >> 16) & 1u) | 0x02u | (((hl ^ v) & (hl ^ r) & 0x8000u) >> 13) | (s.h & 0xA8u) |
        (((hl ^ v ^ r) >> 8) & 0x10u) | ((r & 0xFFFFu) ? 0u : 0x40u);
}

// Register lists in the enum's family orders.
#define Z80B_R7(M, base) M((base) + 0, a) M((base) + 1, b) M((base) + 2, c) M((base) + 3, d) \
  M((base) + 4, e) M((base) + 5, h) M((base) + 6, l)
#define Z80B_S7(M, base) M((base) + 0, b) M((base) + 1, c) M((base) + 2, d) M((base) + 3, e) \
  M((base) + 4, h) M((base) + 5, l) M((base) + 6, a)

// Applies a statement to every state S[0..K) (named s inside).
#if defined(__CUDA_ARCH__)  // device pass only: host compilers do not know the pragma
#define Z80B_UNROLL _Pragma("unroll")
#else
#define Z80B_UNROLL
#endif
#define Z80B_EACH(...)                 \
  Z80B_UNROLL for (int k_ = 0; k_ < K; k_++) { \
    Z80S& s = S[k_];                   \
    __VA_ARGS__;                       \
  }

#define Z_LDA(o, r) case (o): Z80B_EACH(s.a = s.r); break;
#define Z_LDB(o, r) case (o): Z80B_EACH(s.b = s.r); break;
#define Z_LDC(o, r) case (o): Z80B_EACH(s.c = s.r); break;
#define Z_LDD(o, r) case (o): Z80B_EACH(s.d = s.r); break;
#define Z_LDE(o, r) case (o): Z80B_EACH(s.e = s.r); break;
#define Z_LDH(o, r) case (o): Z80B_EACH(s.h = s.r); break;
#define Z_LDL(o, r) case (o): Z80B_EACH(s.l = s.r); break;
#define Z_LDN(o, r) case (o): Z80B_EACH(s.r = imm & 0xFFu); break;
#define Z_ADD(o, r) case (o): Z80B_EACH(z_add(s, s.r)); break;
#define Z_ADC(o, r) case (o): Z80B_EACH(z_adc(s, s.r)); break;
#define Z_SUB(o, r) case (o): Z80B_EACH(z_sub(s, s.r)); break;
#define Z_SBC(o, r) case (o): Z80B_EACH(z_sbc(s, s.r)); break;
#define Z_AND(o, r) case (o): Z80B_EACH(z_and(s, s.r)); break;
#define Z_XOR(o, r) case (o): Z80B_EACH(z_xor(s, s.r)); break;
#define Z_OR(o, r) case (o): Z80B_EACH(z_or(s, s.r)); break;
#define Z_CP(o, r) case (o): Z80B_EACH(z_cp(s, s.r)); break;
#define Z_INC(o, r) case (o): Z80B_EACH(z_inc(s, s.r)); break;
#define Z_DEC(o, r) case (o): Z80B_EACH(z_dec(s, s.r)); break;
#define Z_RLC(o, r) case (o): Z80B_EACH(s.r = z_rlc(s, s.r)); break;
#define Z_RRC(o, r) case (o): Z80B_EACH(s.r = z_rrc(s, s.r)); break;
#define Z_RL(o, r) case (o): Z80B_EACH(s.r = z_rl(s, s.r)); break;
#define Z_RR(o, r) case (o): Z80B_EACH(s.r = z_rr(s, s.r)); break;
#define Z_SLA(o, r) case (o): Z80B_EACH(s.r = z_sla(s, s.r)); break;
#define Z_SRA(o, r) case (o): Z80B_EACH(s.r = z_sra(s, s.r)); break;
#define Z_SRL(o, r) case (o): Z80B_EACH(s.r = z_srl(s, s.r)); break;
#define Z_SLL(o, r) case (o): Z80B_EACH(s.r = z_sll(s, s.r)); break;
#define Z_BIT(o, r) case (o): Z80B_EACH(z_bit(s, s.r, uint32_t(((o) - BIT_0_A) / 7))); break;
#define Z_RES(o, r) case (o): Z80B_EACH(s.r &= ~(1u << (((o) - RES_0_A) / 7))); break;
#define Z_SET(o, r) case (o): Z80B_EACH(s.r |= 1u << (((o) - SET_0_A) / 7)); break;

// Executes one instruction on K states at once: one dispatch on the opcode,
// then the case body for each state (the "vectors per lane" of a sweep).
// Opcodes outside 0..454 leave the states alone (the host rejects them
// before any launch).
template <int K>
Z80_HD void z_stepK(Z80S (&S)[K], uint32_t op, uint32_t imm) {
  switch (op) {
    Z80B_S7(Z_LDA, LD_A_B)
    Z80B_R7(Z_LDB, LD_B_A)
    Z80B_R7(Z_LDC, LD_C_A)
    Z80B_R7(Z_LDD, LD_D_A)
    Z80B_R7(Z_LDE, LD_E_A)
    Z80B_R7(Z_LDH, LD_H_A)
    Z80B_R7(Z_LDL, LD_L_A)
    Z80B_R7(Z_LDN, LD_A_N)
    Z80B_S7(Z_ADD, ADD_A_B)
    case ADD_A_N: Z80B_EACH(z_add(s, imm & 0xFFu)); break;
    Z80B_S7(Z_ADC, ADC_A_B)
    case ADC_A_N: Z80B_EACH(z_adc(s, imm & 0xFFu)); break;
    Z80B_S7(Z_SUB, SUB_B)
    case SUB_N: Z80B_EACH(z_sub(s, imm & 0xFFu)); break;
    Z80B_S7(Z_SBC, SBC_A_B)
    case SBC_A_N: Z80B_EACH(z_sbc(s, imm & 0xFFu)); break;
    Z80B_S7(Z_AND, AND_B)
    case AND_N: Z80B_EACH(z_and(s, imm & 0xFFu)); break;
    Z80B_S7(Z_XOR, XOR_B)
    case XOR_N: Z80B_EACH(z_xor(s, imm & 0xFFu)); break;
    Z80B_S7(Z_OR, OR_B)
    case OR_N: Z80B_EACH(z_or(s, imm & 0xFFu)); break;
    Z80B_S7(Z_CP, CP_B)
    case CP_N: Z80B_EACH(z_cp(s, imm & 0xFFu)); break;
    Z80B_R7(Z_INC, INC_A)
    Z80B_R7(Z_DEC, DEC_A)
    case RLCA:
      Z80B_EACH(s.a = ((s.a << 1) | (s.a >> 7)) & 0xFFu; s.f = (s.f & 0xC4u) | (s.a & 0x29u));
      break;
    case RRCA:
      Z80B_EACH(const uint32_t c = s.a & 1u; s.a = ((s.a >> 1) | (s.a << 7)) & 0xFFu;
                s.f = (s.f & 0xC4u) | c | (s.a & 0x28u));
      break;
    case RLA:
      Z80B_EACH(const uint32_t old = s.a; s.a = ((s.a << 1) | (s.f & 1u)) & 0xFFu;
                s.f = (s.f & 0xC4u) | (s.a & 0x28u) | (old >> 7));
      break;
    case RRA:
      Z80B_EACH(const uint32_t old = s.a; s.a = (s.a >> 1) | ((s.f & 1u) << 7);
                s.f = (s.f & 0xC4u) | (s.a & 0x28u) | (old & 1u));
      break;
    case DAA: Z80B_EACH(z_daa(s)); break;
    case CPL: Z80B_EACH(s.a ^= 0xFFu; s.f = (s.f & 0xC5u) | (s.a & 0x28u) | 0x12u); break;
    case SCF: Z80B_EACH(s.f = (s.f & 0xC4u) | (s.a & 0x28u) | 1u); break;
    case CCF: Z80B_EACH(s.f = (s.f & 0xC4u) | (s.a & 0x28u) | ((s.f & 1u) ? 0x10u : 1u)); break;
    case NEG: Z80B_EACH(const uint32_t v = s.a; s.a = 0; z_sub(s, v)); break;
    case NOP: break;
    Z80B_R7(Z_RLC, RLC_A)
    Z80B_R7(Z_RRC, RRC_A)
    Z80B_R7(Z_RL, RL_A)
    Z80B_R7(Z_RR, RR_A)
    Z80B_R7(Z_SLA, SLA_A)
    Z80B_R7(Z_SRA, SRA_A)
    Z80B_R7(Z_SRL, SRL_A)
    Z80B_R7(Z_SLL, SLL_A)
    Z80B_R7(Z_BIT, BIT_0_A) Z80B_R7(Z_BIT, BIT_1_A) Z80B_R7(Z_BIT, BIT_2_A) Z80B_R7(Z_BIT, BIT_3_A)
    Z80B_R7(Z_BIT, BIT_4_A) Z80B_R7(Z_BIT, BIT_5_A) Z80B_R7(Z_BIT, BIT_6_A) Z80B_R7(Z_BIT, BIT_7_A)
    Z80B_R7(Z_RES, RES_0_A) Z80B_R7(Z_RES, RES_1_A) Z80B_R7(Z_RES, RES_2_A) Z80B_R7(Z_RES, RES_3_A)
    Z80B_R7(Z_RES, RES_4_A) Z80B_R7(Z_RES, RES_5_A) Z80B_R7(Z_RES, RES_6_A) Z80B_R7(Z_RES, RES_7_A)
    Z80B_R7(Z_SET, SET_0_A) Z80B_R7(Z_SET, SET_1_A) Z80B_R7(Z_SET, SET_2_A) Z80B_R7(Z_SET, SET_3_A)
    Z80B_R7(Z_SET, SET_4_A) Z80B_R7(Z_SET, SET_5_A) Z80B_R7(Z_SET, SET_6_A) Z80B_R7(Z_SET, SET_7_A)
    case INC_BC: Z80B_EACH(const uint32_t v = (((s.b << 8) | s.c) + 1u) & 0xFFFFu; s.b = v >> 8; s.c = v & 0xFFu); break;
    case INC_DE: Z80B_EACH(const uint32_t v = (((s.d << 8) | s.e) + 1u) & 0xFFFFu; s.d = v >> 8; s.e = v & 0xFFu); break;
    case INC_HL: Z80B_EACH(const uint32_t v = (((s.h << 8) | s.l) + 1u) & 0xFFFFu; s.h = v >> 8; s.l = v & 0xFFu); break;
    case INC_SP: Z80B_EACH(s.sp = (s.sp + 1u) & 0xFFFFu); break;
    case DEC_BC: Z80B_EACH(const uint32_t v = (((s.b << 8) | s.c) - 1u) & 0xFFFFu; s.b = v >> 8; s.c = v & 0xFFu); break;
    case DEC_DE: Z80B_EACH(const uint32_t v = (((s.d << 8) | s.e) - 1u) & 0xFFFFu; s.d = v >> 8; s.e = v & 0xFFu); break;
    case DEC_HL: Z80B_EACH(const uint32_t v = (((s.h << 8) | s.l) - 1u) & 0xFFFFu; s.h = v >> 8; s.l = v & 0xFFu); break;
    case DEC_SP: Z80B_EACH(s.sp = (s.sp - 1u) & 0xFFFFu); break;
    case ADD_HL_BC: Z80B_EACH(z_addhl(s, (s.b << 8) | s.c)); break;
    case ADD_HL_DE: Z80B_EACH(z_addhl(s, (s.d << 8) | s.e)); break;
    case ADD_HL_HL: Z80B_EACH(z_addhl(s, (s.h << 8) | s.l)); break;
    case ADD_HL_SP: Z80B_EACH(z_addhl(s, s.sp)); break;
    case EX_DE_HL:
      Z80B_EACH(const uint32_t d = s.d; const uint32_t e = s.e; s.d = s.h; s.e = s.l; s.h = d; s.l = e);
      break;
    case LD_SP_HL: Z80B_EACH(s.sp = (s.h << 8) | s.l); break;
    case LD_BC_NN: Z80B_EACH(s.b = (imm >> 8) & 0xFFu; s.c = imm & 0xFFu); break;
    case LD_DE_NN: Z80B_EACH(s.d = (imm >> 8) & 0xFFu; s.e = imm & 0xFFu); break;
    case LD_HL_NN: Z80B_EACH(s.h = (imm >> 8) & 0xFFu; s.l = imm & 0xFFu); break;
    case LD_SP_NN: Z80B_EACH(s.sp = imm & 0xFFFFu); break;
    case ADC_HL_BC: Z80B_EACH(z_adchl(s, (s.b << 8) | s.c)); break;
    case ADC_HL_DE: Z80B_EACH(z_adchl(s, (s.d << 8) | s.e)); break;
    case ADC_HL_HL: Z80B_EACH(z_adchl(s, (s.h << 8) | s.l)); break;
    case ADC_HL_SP: Z80B_EACH(z_adchl(s, s.sp)); break;
    case SBC_HL_BC: Z80B_EACH(z_sbchl(s, (s.b << 8) | s.c)); break;
    case SBC_HL_DE: Z80B_EACH(z_sbchl(s, (s.d << 8) | s.e)); break;
    case SBC_HL_HL: Z80B_EACH(z_sbchl(s, (s.h << 8) | s.l)); break;
    case SBC_HL_SP: Z80B_EACH(z_sbchl(s, s.sp)); break;
    // memory ops on the single byte M (exec.go:883-1028)
    case LD_A_HLI: Z80B_EACH(s.a = s.m); break;
    case LD_B_HLI: Z80B_EACH(s.b = s.m); break;
    case LD_C_HLI: Z80B_EACH(s.c = s.m); break;
    case LD_D_HLI: Z80B_EACH(s.d = s.m); break;
    case LD_E_HLI: Z80B_EACH(s.e = s.m); break;
    case LD_H_HLI: Z80B_EACH(s.h = s.m); break;
    case LD_L_HLI: Z80B_EACH(s.l = s.m); break;
    case LD_HLI_A: Z80B_EACH(s.m = s.a); break;
    case LD_HLI_B: Z80B_EACH(s.m = s.b); break;
    case LD_HLI_C: Z80B_EACH(s.m = s.c); break;
    case LD_HLI_D: Z80B_EACH(s.m = s.d); break;
    case LD_HLI_E: Z80B_EACH(s.m = s.e); break;
    case LD_HLI_H: Z80B_EACH(s.m = s.h); break;
    case LD_HLI_L: Z80B_EACH(s.m = s.l); break;
    case LD_HLI_N: Z80B_EACH(s.m = imm & 0xFFu); break;
    case LD_A_BCI: case LD_A_DEI: Z80B_EACH(s.a = s.m); break;
    case LD_BCI_A: case LD_DEI_A: Z80B_EACH(s.m = s.a); break;
    case ADD_A_HLI: Z80B_EACH(z_add(s, s.m)); break;
    case ADC_A_HLI: Z80B_EACH(z_adc(s, s.m)); break;
    case SUB_HLI: Z80B_EACH(z_sub(s, s.m)); break;
    case SBC_A_HLI: Z80B_EACH(z_sbc(s, s.m)); break;
    case AND_HLI: Z80B_EACH(z_and(s, s.m)); break;
    case XOR_HLI: Z80B_EACH(z_xor(s, s.m)); break;
    case OR_HLI: Z80B_EACH(z_or(s, s.m)); break;
    case CP_HLI: Z80B_EACH(z_cp(s, s.m)); break;
    case INC_HLI: Z80B_EACH(z_inc(s, s.m)); break;
    case DEC_HLI: Z80B_EACH(z_dec(s, s.m)); break;
    case RLC_HLI: Z80B_EACH(s.m = z_rlc(s, s.m)); break;
    case RRC_HLI: Z80B_EACH(s.m = z_rrc(s, s.m)); break;
    case RL_HLI: Z80B_EACH(s.m = z_rl(s, s.m)); break;
    case RR_HLI: Z80B_EACH(s.m = z_rr(s, s.m)); break;
    case SLA_HLI: Z80B_EACH(s.m = z_sla(s, s.m)); break;
    case SRA_HLI: Z80B_EACH(s.m = z_sra(s, s.m)); break;
    case SRL_HLI: Z80B_EACH(s.m = z_srl(s, s.m)); break;
    case SLL_HLI: Z80B_EACH(s.m = z_sll(s, s.m)); break;
    case BIT_0_HLI: case BIT_1_HLI: case BIT_2_HLI: case BIT_3_HLI:
    case BIT_4_HLI: case BIT_5_HLI: case BIT_6_HLI: case BIT_7_HLI:
      Z80B_EACH(z_bit(s, s.m, op - BIT_0_HLI));
      break;
    case RES_0_HLI: case RES_1_HLI: case RES_2_HLI: case RES_3_HLI:
    case RES_4_HLI: case RES_5_HLI: case RES_6_HLI: case RES_7_HLI:
      Z80B_EACH(s.m &= ~(1u << (op - RES_0_HLI)));
      break;
    case SET_0_HLI: case SET_1_HLI: case SET_2_HLI: case SET_3_HLI:
    case SET_4_HLI: case SET_5_HLI: case SET_6_HLI: case SET_7_HLI:
      Z80B_EACH(s.m |= 1u << (op - SET_0_HLI));
      break;
    default: break;
  }
}

Z80_HD void z_step(Z80S& s, uint32_t op, uint32_t imm) {
  Z80S S[1] = {s};
  z_stepK<1>(S, op, imm);
  s = S[0];
}

Z80_HD void z_run(Z80S& s, const uint32_t* prog, int n) {
  for (int i = 0; i < n; i++) z_step(s, prog[i] & 0xFFFFu, prog[i] >> 16);
}

// Equality of two states with the flag bits in `dead` ignored
// (pkg/search/verifier.go:615-623; dead == 0 gives plain equality).
Z80_HD bool z_equal(const Z80S& x, const Z80S& y, uint32_t keepF) {
  uint32_t d = (x.a ^ y.a) | ((x.f ^ y.f) & keepF) | (x.b ^ y.b) | (x.c ^ y.c) | (x.d ^ y.d) |
               (x.e ^ y.e) | (x.h ^ y.h) | (x.l ^ y.l) | (x.sp ^ y.sp) | (x.m ^ y.m);
  return d == 0;
}

// Packs a state into three words: A|F<<8|B<<16|C<<24, D|E<<8|H<<16|L<<24, SP|M<<16.
Z80_HD void z_pack(const Z80S& s, uint32_t w[3]) {
  w[0] = s.a | (s.f << 8) | (s.b << 16) | (s.c << 24);
  w[1] = s.d | (s.e << 8) | (s.h << 16) | (s.l << 24);
  w[2] = s.sp | (s.m << 16);
}
Z80_HD Z80S z_unpack(uint32_t w0, uint32_t w1, uint32_t w2) {
  Z80S s;
  s.a = w0 & 0xFFu; s.f = (w0 >> 8) & 0xFFu; s.b = (w0 >> 16) & 0xFFu; s.c = w0 >> 24;
  s.d = w1 & 0xFFu; s.e = (w1 >> 8) & 0xFFu; s.h = (w1 >> 16) & 0xFFu; s.l = w1 >> 24;
  s.sp = w2 & 0xFFFFu; s.m = (w2 >> 16) & 0xFFu;
  return s;
}

}  // namespace z80b
